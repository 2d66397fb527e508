// Seeded initial state built on the device (cs_init_problem): the same
// construction as init_problem_host (init.cpp, after the reference's
// INIT_PATCH_CUBE_SPHERE, 820init_patch_cube_sphere.f:319-689) with one
// thread per zone or face:
//   * zone averages of the conserved variables: 27-point isoparametric
//     volume quadrature of the point state (20-node element, midside nodes
//     of the angular edges on the sphere of their radius);
//   * the entropy variable p / rho^(gamma-1) of the zone average;
//   * face B: circulation of A = a Psi r-hat around the face (midpoint rule
//     per edge, arcs as r * angle, each edge integrated in a canonical
//     direction so the two faces sharing it use the same number) over the
//     face area, so div B is zero to round-off.
// The seeded harmonic sums are drawn on the host (init_harmonics) and
// copied to the device; the results agree with the host construction to
// the last bits (FMA contraction and CUDA's sqrt / acos / pow).
#include <cmath>
#include <mutex>

#include "cs_solve.h"

namespace cs {
namespace {

__constant__ double c_vol[2187];  // vol_rule_pack: N, dx, dy, dz [27][20], w [27]

struct HarmDev {
  const int8_t* e;  // exponents a, b, c per term
  const double* w;
  int n, deg;
  double scale;
};

struct InitDev {
  int kind;
  double gamma, rho_amp, a_amp, v_amp, p0, gm, ob8pi, rhofloor, prsfloor, smallnum;
  HarmDev Y, Psi;
};

__device__ void powers(double x, int deg, double* p) {
  p[0] = 1.0;
  for (int e = 1; e <= deg; ++e) p[e] = p[e - 1] * x;
}

__device__ double harm_value(const HarmDev& h, double u, double v, double t) {
  double pu[16], pv[16], pt[16];
  powers(u, h.deg, pu);
  powers(v, h.deg, pv);
  powers(t, h.deg, pt);
  double s = 0.0;
  for (int n = 0; n < h.n; ++n) s += h.w[n] * pu[h.e[3 * n]] * pv[h.e[3 * n + 1]] * pt[h.e[3 * n + 2]];
  return s * h.scale;
}

__device__ void harm_grad(const HarmDev& h, double u, double v, double t, double g[3]) {
  double pu[16], pv[16], pt[16];
  powers(u, h.deg, pu);
  powers(v, h.deg, pv);
  powers(t, h.deg, pt);
  g[0] = g[1] = g[2] = 0.0;
  for (int n = 0; n < h.n; ++n) {
    const int a = h.e[3 * n], b = h.e[3 * n + 1], c = h.e[3 * n + 2];
    if (a > 0) g[0] += h.w[n] * a * pu[a - 1] * pv[b] * pt[c];
    if (b > 0) g[1] += h.w[n] * b * pu[a] * pv[b - 1] * pt[c];
    if (c > 0) g[2] += h.w[n] * c * pu[a] * pv[b] * pt[c - 1];
  }
  for (int q = 0; q < 3; ++q) g[q] *= h.scale;
}

// Point conserved state at (x, y, z) of the seeded problem.
__device__ void point_state(const InitDev& P, double x, double y, double z, double U[8]) {
  const double r = sqrt(x * x + y * y + z * z);
  const double u = x / r, v = y / r, t = z / r;
  double rho, p, vx, vy, vz;
  if (P.kind == 0) {
    rho = 1.0 + P.rho_amp * harm_value(P.Y, u, v, t);
    p = P.p0;
    vx = -P.v_amp * y;
    vy = P.v_amp * x;
    vz = 0.0;
  } else {
    rho = (1.0 / (r * r)) * (1.0 + P.rho_amp * harm_value(P.Y, u, v, t));
    p = P.gm / (3.0 * r * r * r) + P.p0;
    vx = vy = vz = 0.0;
  }
  double g[3];
  harm_grad(P.Psi, u, v, t, g);
  const double bx = (P.a_amp / r) * (g[1] * t - g[2] * v);
  const double by = (P.a_amp / r) * (g[2] * u - g[0] * t);
  const double bz = (P.a_amp / r) * (g[0] * v - g[1] * u);
  U[0] = rho;
  U[1] = rho * vx;
  U[2] = rho * vy;
  U[3] = rho * vz;
  U[4] = p / (P.gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + P.ob8pi * (bx * bx + by * by + bz * bz);
  U[5] = bx;
  U[6] = by;
  U[7] = bz;
}

__device__ void vert3(const DGeom& g, const Dims& d, int p, int i, int j, int k, double* o) {
  o[0] = geo(g, d, CS_G_VERT, 0, p, i, j, k);
  o[1] = geo(g, d, CS_G_VERT, 1, p, i, j, k);
  o[2] = geo(g, d, CS_G_VERT, 2, p, i, j, k);
}

__device__ void onto_radius(const double* a, const double* b, double r, double smallnum, double* o) {
  double m[3] = {(a[0] + b[0]) * 0.5, (a[1] + b[1]) * 0.5, (a[2] + b[2]) * 0.5};
  const double t = fmax(smallnum, sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]));
  for (int q = 0; q < 3; ++q) o[q] = m[q] * (r / t);
}

template <typename R>
__global__ void k_init_zones(Dims d, DGeom g, InitDev P, DStateT<R> s, Range3 rg) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < rg.count();
       t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    rg.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    double v[20][3];
    vert3(g, d, p, i - 1, j - 1, k - 1, v[0]);
    vert3(g, d, p, i, j - 1, k - 1, v[1]);
    vert3(g, d, p, i, j, k - 1, v[2]);
    vert3(g, d, p, i - 1, j, k - 1, v[3]);
    vert3(g, d, p, i - 1, j - 1, k, v[4]);
    vert3(g, d, p, i, j - 1, k, v[5]);
    vert3(g, d, p, i, j, k, v[6]);
    vert3(g, d, p, i - 1, j, k, v[7]);
    const double r1 = sqrt(v[0][0] * v[0][0] + v[0][1] * v[0][1] + v[0][2] * v[0][2]);
    const double r2 = sqrt(v[4][0] * v[4][0] + v[4][1] * v[4][1] + v[4][2] * v[4][2]);
    onto_radius(v[0], v[1], r1, P.smallnum, v[8]);
    onto_radius(v[2], v[3], r1, P.smallnum, v[9]);
    onto_radius(v[6], v[7], r2, P.smallnum, v[10]);
    onto_radius(v[4], v[5], r2, P.smallnum, v[11]);
    onto_radius(v[0], v[3], r1, P.smallnum, v[12]);
    onto_radius(v[1], v[2], r1, P.smallnum, v[15]);
    onto_radius(v[4], v[7], r2, P.smallnum, v[13]);
    onto_radius(v[5], v[6], r2, P.smallnum, v[14]);
    for (int q = 0; q < 3; ++q) {
      v[16][q] = (v[0][q] + v[4][q]) * 0.5;
      v[17][q] = (v[1][q] + v[5][q]) * 0.5;
      v[18][q] = (v[2][q] + v[6][q]) * 0.5;
      v[19][q] = (v[3][q] + v[7][q]) * 0.5;
    }
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0}, vol = 0.0;
    for (int q27 = 0; q27 < 27; ++q27) {
      double x[3] = {0, 0, 0}, A[3] = {0, 0, 0}, B[3] = {0, 0, 0}, C[3] = {0, 0, 0};
      for (int n = 0; n < 20; ++n) {
        const double sn = c_vol[q27 * 20 + n], sx = c_vol[540 + q27 * 20 + n], sy = c_vol[1080 + q27 * 20 + n],
                     sz = c_vol[1620 + q27 * 20 + n];
        for (int c = 0; c < 3; ++c) {
          x[c] = x[c] + v[n][c] * sn;
          A[c] = A[c] + v[n][c] * sx;
          B[c] = B[c] + v[n][c] * sy;
          C[c] = C[c] + v[n][c] * sz;
        }
      }
      const double D0 = A[1] * B[2] - A[2] * B[1], D1 = A[2] * B[0] - A[0] * B[2], D2 = A[0] * B[1] - A[1] * B[0];
      const double w = c_vol[2160 + q27] * fabs(C[0] * D0 + C[1] * D1 + C[2] * D2);
      vol += w;
      double Up[8];
      point_state(P, x[0], x[1], x[2], Up);
      for (int q = 0; q < 8; ++q) acc[q] = acc[q] + Up[q] * w;
    }
    vol = fmax(P.smallnum, vol);
    for (int q = 0; q < 8; ++q) acc[q] = acc[q] / vol;
    for (int q = 0; q < 8; ++q) s.U[d.at(q, p, i, j, k)] = (R)acc[q];
    const double rho = fmax(acc[0], P.rhofloor);
    const double v0 = rho / (rho * rho + P.rhofloor * P.rhofloor);
    const double vx = acc[1] * v0, vy = acc[2] * v0, vz = acc[3] * v0;
    double prs = (P.gamma - 1.0) * (acc[4] - 0.5 * rho * (vx * vx + vy * vy + vz * vz) -
                                    (acc[5] * acc[5] + acc[6] * acc[6] + acc[7] * acc[7]) * P.ob8pi);
    prs = fmax(prs, P.prsfloor);
    s.ent[d.at(0, p, i, j, k)] = (R)(prs / pow(rho, P.gamma - 1.0));
  }
}

// A . dl from a to b (midpoint rule; an arc's midpoint is put on the radius
// of a and dl is r * angle along the chord).
__device__ double a_dot_dl(const InitDev& P, const double* pa, const double* pb, bool arc) {
  double m[3], dl[3];
  for (int q = 0; q < 3; ++q) {
    m[q] = 0.5 * (pa[q] + pb[q]);
    dl[q] = pb[q] - pa[q];
  }
  if (arc) {
    const double ra = sqrt(pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]);
    const double rb = sqrt(pb[0] * pb[0] + pb[1] * pb[1] + pb[2] * pb[2]);
    const double rm = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    for (int q = 0; q < 3; ++q) m[q] *= ra / rm;
    double cosang = (pa[0] * pb[0] + pa[1] * pb[1] + pa[2] * pb[2]) / (ra * rb);
    cosang = fmax(-1.0, fmin(1.0, cosang));
    const double ang = acos(cosang);
    const double dn = sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
    for (int q = 0; q < 3; ++q) dl[q] = ra * ang * dl[q] / dn;
  }
  const double r = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  const double psi = harm_value(P.Psi, m[0] / r, m[1] / r, m[2] / r);
  const double ar = P.a_amp * psi / r;
  return ar * (m[0] * dl[0] + m[1] * dl[1] + m[2] * dl[2]);
}

struct Corner {
  int i, j, k;
};

__device__ double edge_circ(const DGeom& g, const Dims& d, const InitDev& P, int p, Corner a, Corner b, bool arc) {
  double pa[3], pb[3];
  vert3(g, d, p, a.i, a.j, a.k, pa);
  vert3(g, d, p, b.i, b.j, b.k, pb);
  const bool swap = (a.k > b.k) || (a.k == b.k && (a.j > b.j || (a.j == b.j && a.i > b.i)));
  return swap ? -a_dot_dl(P, pb, pa, arc) : a_dot_dl(P, pa, pb, arc);
}

__device__ bool nonzero(const DGeom& g, const Dims& d, int p, Corner c) {
  double v[3];
  vert3(g, d, p, c.i, c.j, c.k, v);
  return (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) > 0.0;
}

// Face B of direction dir from the circulation around the face, in the
// loop orders of init_problem_host (positive about +x, +y, +radial).
template <typename R>
__global__ void k_init_faces(Dims d, DGeom g, InitDev P, DStateT<R> s, Range3 rg, int dir) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < rg.count();
       t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    rg.decode(t, p, i, j, k);
    Corner c0, c1, c2, c3;
    bool arc0, arc1, arc2, arc3;
    if (dir == 0) {
      c0 = {i, j - 1, k - 1}, c1 = {i, j, k - 1}, c2 = {i, j, k}, c3 = {i, j - 1, k};
      arc0 = true, arc1 = false, arc2 = true, arc3 = false;
    } else if (dir == 1) {
      c0 = {i - 1, j, k - 1}, c1 = {i - 1, j, k}, c2 = {i, j, k}, c3 = {i, j, k - 1};
      arc0 = false, arc1 = true, arc2 = false, arc3 = true;
    } else {
      c0 = {i - 1, j - 1, k}, c1 = {i, j - 1, k}, c2 = {i, j, k}, c3 = {i - 1, j, k};
      arc0 = arc1 = arc2 = arc3 = true;
    }
    if (!(nonzero(g, d, p, c0) && nonzero(g, d, p, c1) && nonzero(g, d, p, c2) && nonzero(g, d, p, c3))) continue;
    const double c = edge_circ(g, d, P, p, c0, c1, arc0) + edge_circ(g, d, P, p, c1, c2, arc1) +
                     edge_circ(g, d, P, p, c2, c3, arc2) + edge_circ(g, d, P, p, c3, c0, arc3);
    const int AREA = dir == 0 ? CS_G_XF_AREA : (dir == 1 ? CS_G_YF_AREA : CS_G_ZF_AREA);
    double* B = dir == 0 ? s.Bxf : (dir == 1 ? s.Byf : s.Bzf);
    B[d.at(0, p, i, j, k)] = c / geo(g, d, AREA, 0, p, i, j, k);
  }
}

std::once_flag g_vol_once[64];

template <typename R>
int init_device_t(Solve& sv, DStateT<R>& st, const InitDev& P) {
  const Dims& d = sv.d;
  const size_t S6 = (size_t)6 * d.S;
  cudaError_t e = cudaMemsetAsync(st.U, 0, NVAR * S6 * sizeof(R), sv.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(st.ent, 0, S6 * sizeof(R), sv.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(st.Bxf, 0, S6 * sizeof(double), sv.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(st.Byf, 0, S6 * sizeof(double), sv.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(st.Bzf, 0, S6 * sizeof(double), sv.stream);
  if (e != cudaSuccess) return cuda_fail(sv, e, "cudaMemsetAsync(initial state)");
  const int G = d.G, N = d.N, nr = d.nr;
  const Range3 z = {1 - G, N + G, 1 - G, N + G, 1 - G, nr + G};
  k_init_zones<R><<<blocks_for(z.count(), 128, grid_sms(sv)), 128, 0, sv.stream>>>(d, sv.g, P, st, z);
  mark(sv, "k_init_zones");
  const Range3 fr[3] = {{-G, N + G, 1 - G, N + G, 1 - G, nr + G},
                        {1 - G, N + G, -G, N + G, 1 - G, nr + G},
                        {1 - G, N + G, 1 - G, N + G, -G, nr + G}};
  for (int dir = 0; dir < 3; ++dir) {
    k_init_faces<R><<<blocks_for(fr[dir].count(), 128, grid_sms(sv)), 128, 0, sv.stream>>>(d, sv.g, P, st,
                                                                                             fr[dir], dir);
    mark(sv, "k_init_faces");
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(sv, e, "initial-state launch");
  return CS_OK;
}

}  // namespace

int init_problem_device(Solve& sv, const cs_init_desc& desc) {
  InitHarmonics Y, Psi;
  std::string why = init_harmonics(desc, Y, Psi);
  if (!why.empty()) return fail(sv, CS_ERR_ARG, why);
  cudaError_t e = cudaSuccess;
  std::call_once(g_vol_once[sv.device & 63], [&] {
    double tab[2187];
    vol_rule_pack(tab);
    e = cudaMemcpyToSymbol(c_vol, tab, sizeof tab);
  });
  if (e != cudaSuccess) return cuda_fail(sv, e, "cudaMemcpyToSymbol(volume rule)");
  // harmonic terms: exponents (3 bytes each) and weights, Y then Psi
  const int ny = (int)Y.w.size(), np = (int)Psi.w.size();
  std::vector<int8_t> ex(3 * (ny + np));
  std::vector<double> w(ny + np);
  for (int q = 0; q < 2; ++q) {
    const InitHarmonics& h = q ? Psi : Y;
    const int o = q ? ny : 0;
    for (size_t n = 0; n < h.w.size(); ++n) {
      ex[3 * (o + n)] = (int8_t)h.a[n];
      ex[3 * (o + n) + 1] = (int8_t)h.b[n];
      ex[3 * (o + n) + 2] = (int8_t)h.c[n];
      w[o + n] = h.w[n];
    }
  }
  const size_t wb = w.size() * sizeof(double), eb = ex.size();
  if (sv.init_buf_bytes < wb + eb + 16) {
    sv.init_buf = (unsigned char*)solve_alloc(sv, wb + eb + 16, e);
    if (!sv.init_buf) return cuda_fail(sv, e, "cudaMalloc(initial-state terms)");
    sv.init_buf_bytes = wb + eb + 16;
  }
  e = cudaMemcpyAsync(sv.init_buf, w.data(), wb, cudaMemcpyHostToDevice, sv.stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sv.init_buf + wb, ex.data(), eb, cudaMemcpyHostToDevice, sv.stream);
  if (e != cudaSuccess) return cuda_fail(sv, e, "cudaMemcpyAsync(initial-state terms)");
  InitDev P;
  P.kind = desc.kind;
  P.gamma = sv.p.gamma;
  P.rho_amp = desc.rho_amp;
  P.a_amp = desc.a_amp;
  P.v_amp = desc.v_amp;
  P.p0 = desc.p0;
  P.gm = sv.p.gm;
  P.ob8pi = 1.0 / (8.0 * (4.0 * std::atan(1.0)));
  P.rhofloor = sv.p.rhofloor;
  P.prsfloor = sv.p.prsfloor;
  P.smallnum = sv.p.smallnum;
  const double* wd = (const double*)sv.init_buf;
  const int8_t* ed = (const int8_t*)(sv.init_buf + wb);
  P.Y = {ed, wd, ny, Y.deg, Y.scale};
  P.Psi = {ed + 3 * ny, wd + ny, np, Psi.deg, Psi.scale};
  int rc = sv.fp32 ? init_device_t(sv, sv.stF, P) : init_device_t(sv, sv.st, P);
  if (rc) return rc;
  e = cudaStreamSynchronize(sv.stream);  // the host term arrays go out of scope
  if (e != cudaSuccess) return cuda_fail(sv, e, "initial state");
  return CS_OK;
}

}  // namespace cs
