// Edge electric fields for the constrained-transport update: three-point
// Simpson rule along every edge, four-state multidimensional HLL solver
// with the symmetrised (LLF) speeds, and the three-state solver on the
// radial edges at the four cube corners of each panel.
//
// Follows MAKE_EDGE_EFIELDS_P1 with USE_2D_LLF_RS_FOR_EZ = 1
// (pkg/inc/cubesphere/400riemann_integrate/460make_edge_fields_p1.f:335-7037),
// Two_D_RS_Ez_4State_HLL (620riemann_2d/630...:10-372) and
// Two_D_RS_Ez_3State_HLL (620riemann_2d/631...:9-338).  One thread per edge.
#include "cs_solve.h"

namespace cs {

namespace {

constexpr int TPB = 128;

template <typename R>
__device__ __forceinline__ double E1(const DStateT<R>& s, const Dims& d, int q, int p, int i, int j, int k) {
  return s.E[d.at(q, p, i, j, k)];
}
template <typename T>
__device__ __forceinline__ double Sg(const T* a, const Dims& d, int p, int i, int j, int k) {
  return a[d.at(0, p, i, j, k)];
}
template <typename R>
__device__ __forceinline__ double Bqa(const DStateT<R>& s, const Dims& d, int dir, int q, int p, int i, int j, int k) {
  return s.Bq[dir][d.at(q, p, i, j, k)];
}

// Simpson point jq on the edge between vertices a and b.
__device__ __forceinline__ void edge_point(const DGeom& g, const Dims& d, int p, int jq, int ax, int ay, int az, int bx,
                                           int by, int bz, bool rescale, double* e) {
  if (jq == 0) {
    double va[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      va[q] = geo(g, d, CS_G_VERT, q, p, ax, ay, az);
      e[q] = 0.5 * (va[q] + geo(g, d, CS_G_VERT, q, p, bx, by, bz));
    }
    if (rescale) {
      const double t = sqrt(va[0] * va[0] + va[1] * va[1] + va[2] * va[2]) / sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
#pragma unroll
      for (int q = 0; q < 3; ++q) e[q] = e[q] * t;
    }
  } else if (jq == 1) {
#pragma unroll
    for (int q = 0; q < 3; ++q) e[q] = geo(g, d, CS_G_VERT, q, p, ax, ay, az);
  } else {
#pragma unroll
    for (int q = 0; q < 3; ++q) e[q] = geo(g, d, CS_G_VERT, q, p, bx, by, bz);
  }
}
__device__ __forceinline__ void unit3(double* v) {
  const double t = 1.0 / sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  v[0] = v[0] * t;
  v[1] = v[1] * t;
  v[2] = v[2] * t;
}
__device__ __forceinline__ void orth3(double* v, const double* n) {
  const double t = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
  v[0] = v[0] - t * n[0];
  v[1] = v[1] - t * n[1];
  v[2] = v[2] - t * n[2];
  unit3(v);
}
__device__ __forceinline__ void llf4(double& SR, double& SL, double& SU, double& SD) {
  const double t = fmax(fmax(fabs(SR), fabs(SL)), fmax(fabs(SU), fabs(SD)));
  SR = t;
  SL = -t;
  SU = t;
  SD = -t;
}

// x-edges (460:393-1493): i in 1..N, j in 0..N, k in 0..nr.
template <typename R>
__global__ void k_edges_x(Dims d, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const double Ex = (E1(s, d, 0, p, i, j, k) + E1(s, d, 0, p, i, j + 1, k) + E1(s, d, 0, p, i, j + 1, k + 1) + E1(s, d, 0, p, i, j, k + 1)) * 0.25;
    const double Ey = (E1(s, d, 1, p, i, j, k) + E1(s, d, 1, p, i, j + 1, k) + E1(s, d, 1, p, i, j + 1, k + 1) + E1(s, d, 1, p, i, j, k + 1)) * 0.25;
    const double Ez = (E1(s, d, 2, p, i, j, k) + E1(s, d, 2, p, i, j + 1, k) + E1(s, d, 2, p, i, j + 1, k + 1) + E1(s, d, 2, p, i, j, k + 1)) * 0.25;
    const double ByR = Bqa(s, d, 2, 4, p, i, j + 1, k), ByL = Bqa(s, d, 2, 3, p, i, j, k);
    const double BnU = Bqa(s, d, 1, 2, p, i, j, k + 1), BnD = Bqa(s, d, 1, 1, p, i, j, k);
    double SR = fmax(Sg(s.S[3], d, p, i, j, k + 1), Sg(s.S[3], d, p, i, j, k));
    double SL = fmin(Sg(s.S[2], d, p, i, j, k + 1), Sg(s.S[2], d, p, i, j, k));
    double SU = fmax(Sg(s.S[5], d, p, i, j + 1, k), Sg(s.S[5], d, p, i, j, k));
    double SD = fmin(Sg(s.S[4], d, p, i, j + 1, k), Sg(s.S[4], d, p, i, j, k));
    llf4(SR, SL, SU, SD);
    double acc = 0.0;
    for (int jq = 0; jq < 3; ++jq) {
      const double wt = jq == 0 ? 4.0 / 6.0 : 1.0 / 6.0;
      double n2[3], n3[3];
      edge_point(g, d, p, jq, i, j, k, i - 1, j, k, true, n2);
      unit3(n2);
#pragma unroll
      for (int q = 0; q < 3; ++q) n3[q] = geo(g, d, CS_G_VERT, q, p, i, j, k) - geo(g, d, CS_G_VERT, q, p, i - 1, j, k);
      orth3(n3, n2);
      const double Ezl = Ex * n3[0] + Ey * n3[1] + Ez * n3[2];
      acc = acc + wt * d_rs4(SR, SL, SU, SD, 0.0, 1.0, Ezl, BnU, BnD, ByR, ByL);
    }
    s.Ef[0][d.at(0, p, i, j, k)] = acc;
  }
}

// y-edges (460:1497-2587): i in 0..N, j in 1..N, k in 0..nr.
template <typename R>
__global__ void k_edges_y(Dims d, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const double Ex = (E1(s, d, 0, p, i, j, k) + E1(s, d, 0, p, i, j, k + 1) + E1(s, d, 0, p, i + 1, j, k + 1) + E1(s, d, 0, p, i + 1, j, k)) * 0.25;
    const double Ey = (E1(s, d, 1, p, i, j, k) + E1(s, d, 1, p, i, j, k + 1) + E1(s, d, 1, p, i + 1, j, k + 1) + E1(s, d, 1, p, i + 1, j, k)) * 0.25;
    const double Ez = (E1(s, d, 2, p, i, j, k) + E1(s, d, 2, p, i, j, k + 1) + E1(s, d, 2, p, i + 1, j, k + 1) + E1(s, d, 2, p, i + 1, j, k)) * 0.25;
    const double ByR = Bqa(s, d, 0, 4, p, i, j, k + 1), ByL = Bqa(s, d, 0, 3, p, i, j, k);
    const double BnU = Bqa(s, d, 2, 2, p, i + 1, j, k), BnD = Bqa(s, d, 2, 1, p, i, j, k);
    double SR = fmax(Sg(s.S[5], d, p, i + 1, j, k), Sg(s.S[5], d, p, i, j, k));
    double SL = fmin(Sg(s.S[4], d, p, i + 1, j, k), Sg(s.S[4], d, p, i, j, k));
    double SU = fmax(Sg(s.S[1], d, p, i, j, k), Sg(s.S[1], d, p, i, j, k + 1));
    double SD = fmin(Sg(s.S[0], d, p, i, j, k), Sg(s.S[0], d, p, i, j, k + 1));
    llf4(SR, SL, SU, SD);
    double acc = 0.0;
    for (int jq = 0; jq < 3; ++jq) {
      const double wt = jq == 0 ? 4.0 / 6.0 : 1.0 / 6.0;
      double n1[3], n3[3];
      edge_point(g, d, p, jq, i, j, k, i, j - 1, k, true, n1);
      unit3(n1);
#pragma unroll
      for (int q = 0; q < 3; ++q) n3[q] = geo(g, d, CS_G_VERT, q, p, i, j, k) - geo(g, d, CS_G_VERT, q, p, i, j - 1, k);
      orth3(n3, n1);
      const double Ezl = Ex * n3[0] + Ey * n3[1] + Ez * n3[2];
      acc = acc + wt * d_rs4(SR, SL, SU, SD, 0.0, 1.0, Ezl, BnU, BnD, ByR, ByL);
    }
    s.Ef[1][d.at(0, p, i, j, k)] = acc;
  }
}

// z-edges (460:2591-3721): i, j in 0..N, k in 1..nr, skipped where a
// neighbour is masked; the four cube corners (460:3725-7037) use the
// three-state solver.
template <typename R>
__global__ void k_edges_z(Dims d, DGeom g, DStateT<R> s, Range3 r) {
  const int N = d.N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const bool corner = (i == 0 || i == N) && (j == 0 || j == N);
    double acc = 0.0;
    if (!corner) {
      if (mask_at(g, d, p, i, j) == 0 || mask_at(g, d, p, i + 1, j) == 0 || mask_at(g, d, p, i + 1, j + 1) == 0 ||
          mask_at(g, d, p, i, j + 1) == 0) {
        s.Ef[2][d.at(0, p, i, j, k)] = 0.0;
        continue;
      }
      const double Ex = (E1(s, d, 0, p, i, j, k) + E1(s, d, 0, p, i + 1, j, k) + E1(s, d, 0, p, i + 1, j + 1, k) + E1(s, d, 0, p, i, j + 1, k)) * 0.25;
      const double Ey = (E1(s, d, 1, p, i, j, k) + E1(s, d, 1, p, i + 1, j, k) + E1(s, d, 1, p, i + 1, j + 1, k) + E1(s, d, 1, p, i, j + 1, k)) * 0.25;
      const double Ez = (E1(s, d, 2, p, i, j, k) + E1(s, d, 2, p, i + 1, j, k) + E1(s, d, 2, p, i + 1, j + 1, k) + E1(s, d, 2, p, i, j + 1, k)) * 0.25;
      const double ByR = Bqa(s, d, 1, 4, p, i + 1, j, k), ByL = Bqa(s, d, 1, 3, p, i, j, k);
      const double BnU = Bqa(s, d, 0, 2, p, i, j + 1, k), BnD = Bqa(s, d, 0, 1, p, i, j, k);
      double SR = fmax(Sg(s.S[1], d, p, i, j + 1, k), Sg(s.S[1], d, p, i, j, k));
      double SL = fmin(Sg(s.S[0], d, p, i, j + 1, k), Sg(s.S[0], d, p, i, j, k));
      double SU = fmax(Sg(s.S[3], d, p, i + 1, j, k), Sg(s.S[3], d, p, i, j, k));
      double SD = fmin(Sg(s.S[2], d, p, i + 1, j, k), Sg(s.S[2], d, p, i, j, k));
      llf4(SR, SL, SU, SD);
      for (int jq = 0; jq < 3; ++jq) {
        const double wt = jq == 0 ? 4.0 / 6.0 : 1.0 / 6.0;
        double n3[3], n1[3], tau[3];
        edge_point(g, d, p, jq, i, j, k, i, j, k - 1, false, n3);
        unit3(n3);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          n1[q] = geo(g, d, CS_G_VERT, q, p, i + 1, j, k) - geo(g, d, CS_G_VERT, q, p, i - 1, j, k);
          tau[q] = geo(g, d, CS_G_VERT, q, p, i, j + 1, k) - geo(g, d, CS_G_VERT, q, p, i, j - 1, k);
        }
        orth3(n1, n3);
        orth3(tau, n3);
        const double cos_t = tau[0] * n1[0] + tau[1] * n1[1] + tau[2] * n1[2];
        const double sin_t = sqrt(1.0 - cos_t * cos_t);
        const double Ezl = Ex * n3[0] + Ey * n3[1] + Ez * n3[2];
        acc = acc + wt * d_rs4(SR, SL, SU, SD, cos_t, sin_t, Ezl, BnU, BnD, ByR, ByL);
      }
    } else {
      const int c = (i == 0 && j == 0) ? 0 : (i == N && j == 0) ? 1 : (i == N && j == N) ? 2 : 3;
      int z1x, z1y, z2x, z2y, z3x, z3y;
      if (c == 0) { z1x = i + 1; z1y = j + 1; z2x = i; z2y = j + 1; z3x = i + 1; z3y = j; }
      else if (c == 1) { z1x = i + 1; z1y = j + 1; z2x = i; z2y = j + 1; z3x = i; z3y = j; }
      else if (c == 2) { z1x = i; z1y = j + 1; z2x = i; z2y = j; z3x = i + 1; z3y = j; }
      else { z1x = i + 1; z1y = j + 1; z2x = i; z2y = j; z3x = i + 1; z3y = j; }
      const double ob3 = 1.0 / 3.0;
      const double Ex = (E1(s, d, 0, p, z1x, z1y, k) + E1(s, d, 0, p, z2x, z2y, k) + E1(s, d, 0, p, z3x, z3y, k)) * ob3;
      const double Ey = (E1(s, d, 1, p, z1x, z1y, k) + E1(s, d, 1, p, z2x, z2y, k) + E1(s, d, 1, p, z3x, z3y, k)) * ob3;
      const double Ez = (E1(s, d, 2, p, z1x, z1y, k) + E1(s, d, 2, p, z2x, z2y, k) + E1(s, d, 2, p, z3x, z3y, k)) * ob3;
      double Bn1, Bn2, Bn3, SR1, SL1, SR2, SL2, SR3, SL3;
      if (c == 0) {
        Bn1 = -Bqa(s, d, 1, 4, p, z3x, z3y, k); Bn2 = Bqa(s, d, 0, 2, p, z2x, z2y, k); Bn3 = Bqa(s, d, 1, 3, p, z2x, z2y - 1, k);
        SR1 = -Sg(s.S[2], d, p, z3x, z3y, k); SL1 = -Sg(s.S[3], d, p, z3x, z3y, k);
        SR2 = Sg(s.S[1], d, p, z2x, z2y, k); SL2 = Sg(s.S[0], d, p, z2x, z2y, k);
        SR3 = Sg(s.S[3], d, p, z2x, z2y - 1, k); SL3 = Sg(s.S[2], d, p, z2x, z2y - 1, k);
      } else if (c == 1) {
        Bn1 = -Bqa(s, d, 1, 4, p, z1x, z1y - 1, k); Bn2 = Bqa(s, d, 0, 2, p, z2x, z2y, k); Bn3 = Bqa(s, d, 1, 3, p, z3x, z3y, k);
        SR1 = -Sg(s.S[0], d, p, z3x, z3y, k); SL1 = -Sg(s.S[1], d, p, z3x, z3y, k);
        SR2 = Sg(s.S[1], d, p, z2x, z2y, k); SL2 = Sg(s.S[0], d, p, z2x, z2y, k);
        SR3 = Sg(s.S[3], d, p, z3x, z3y, k); SL3 = Sg(s.S[2], d, p, z3x, z3y, k);
      } else if (c == 2) {
        Bn1 = Bqa(s, d, 0, 2, p, z1x, z1y, k); Bn2 = Bqa(s, d, 1, 3, p, z2x, z2y, k); Bn3 = -Bqa(s, d, 0, 1, p, z2x, z2y, k);
        SR1 = Sg(s.S[1], d, p, z1x, z1y, k); SL1 = Sg(s.S[0], d, p, z1x, z1y, k);
        SR2 = Sg(s.S[3], d, p, z2x, z2y, k); SL2 = Sg(s.S[2], d, p, z2x, z2y, k);
        SR3 = -Sg(s.S[0], d, p, z2x, z2y, k); SL3 = -Sg(s.S[1], d, p, z2x, z2y, k);
      } else {
        Bn1 = -Bqa(s, d, 1, 4, p, z3x, z3y, k); Bn2 = Bqa(s, d, 1, 3, p, z2x, z2y, k); Bn3 = -Bqa(s, d, 0, 1, p, z2x, z2y, k);
        SR1 = -Sg(s.S[2], d, p, z3x, z3y, k); SL1 = -Sg(s.S[3], d, p, z3x, z3y, k);
        SR2 = Sg(s.S[3], d, p, z2x, z2y, k); SL2 = Sg(s.S[2], d, p, z2x, z2y, k);
        SR3 = -Sg(s.S[0], d, p, z2x, z2y, k); SL3 = -Sg(s.S[1], d, p, z2x, z2y, k);
      }
      const double tm = fmax(fmax(fmax(fabs(SR1), fabs(SL1)), fmax(fabs(SR2), fabs(SL2))), fmax(fabs(SR3), fabs(SL3)));
      for (int jq = 0; jq < 3; ++jq) {
        const double wt = jq == 0 ? 4.0 / 6.0 : 1.0 / 6.0;
        double n3[3];
        edge_point(g, d, p, jq, i, j, k, i, j, k - 1, false, n3);
        unit3(n3);
        const double Ezl = Ex * n3[0] + Ey * n3[1] + Ez * n3[2];
        acc = acc + wt * d_rs3(tm, -tm, tm, -tm, tm, -tm, Ezl, Bn1, Bn2, Bn3);
      }
    }
    s.Ef[2][d.at(0, p, i, j, k)] = acc;
  }
}

// Panel-edge ownership for the EMFs: a non-owner copy of a shared edge
// takes the owner's value, negated where the two panels run the edge in
// opposite directions.
template <typename R>
__global__ void k_sync_emf(DStateT<R> s, PanelSync ps) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ps.ne; t += (long long)gridDim.x * blockDim.x)
    s.Ef[ps.e_df[t]][ps.e_dst[t]] = (double)ps.e_sign[t] * s.Ef[ps.e_sf[t]][ps.e_src[t]];
}

// The reference's rule for a shared edge (CS_FLAG_PANEL_AVERAGE): all
// copies take the average of the panels' EMFs, signed where a panel runs the
// edge the other way; two copies (own + other) * 0.5, the three of a
// cube-corner radial edge their sum / 3 (334fetch_buffers_fill_in_flux_x.f:
// 341-395, 335fetch_buffers_fill_in_flux_y.f:761-795).  One thread an edge:
// its owner's copy, then the one or two entries from e_cls[q].
template <typename R>
__global__ void k_avg_emf(DStateT<R> s, PanelSync ps) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ps.ncls; q += (long long)gridDim.x * blockDim.x) {
    const int h = ps.e_cls[q], n = ps.e_cls[q + 1] - h;
    double* own = s.Ef[ps.e_sf[h]] + ps.e_src[h];
    double sum = *own;
    for (int m = h; m < h + n; ++m) sum += (double)ps.e_sign[m] * s.Ef[ps.e_df[m]][ps.e_dst[m]];
    const double avg = n == 1 ? sum * 0.5 : sum / 3.0;
    *own = avg;
    for (int m = h; m < h + n; ++m) s.Ef[ps.e_df[m]][ps.e_dst[m]] = (double)ps.e_sign[m] * avg;
  }
}

}  // namespace

template <typename R>
void launch_edges_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  const int N = d.N, nr = d.nr;
  Range3 ex = {1, N, 0, N, 0, nr};
  Range3 ey = {0, N, 1, N, 0, nr};
  Range3 ez = {0, N, 0, N, 1, nr};
  k_edges_x<R><<<blocks_for(ex.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, ex);
  mark(sv, "k_edges_x");
  k_edges_y<R><<<blocks_for(ey.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, ey);
  mark(sv, "k_edges_y");
  k_edges_z<R><<<blocks_for(ez.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, ez);
  mark(sv, "k_edges_z");
  if (sv.psync.ncls > 0 && (sv.p.flags & CS_FLAG_PANEL_AVERAGE)) {
    k_avg_emf<R><<<blocks_for(sv.psync.ncls, 128, grid_sms(sv)), 128, 0, sv.stream>>>(st, sv.psync);
    mark(sv, "k_avg_emf");
  } else if (sv.psync.ne > 0) {
    k_sync_emf<R><<<blocks_for(sv.psync.ne, 128, grid_sms(sv)), 128, 0, sv.stream>>>(st, sv.psync);
    mark(sv, "k_sync_emf");
  }
}

void launch_edges(Solve& sv) {
  if (sv.fp32)
    launch_edges_t(sv, sv.stF);
  else
    launch_edges_t(sv, sv.st);
}

}  // namespace cs

// Known-answer access to the two multidimensional Riemann solvers: one
// thread per case evaluates the device function the edge kernels call.
namespace {
__global__ void k_twod_rs_ez(int n, int kind, const double* in, double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (kind == 4) {
    const double* a = in + (long long)t * 11;
    out[t] = cs::d_rs4(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10]);
  } else {
    const double* a = in + (long long)t * 10;
    out[t] = cs::d_rs3(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9]);
  }
}
}  // namespace

extern "C" int cs_twod_rs_ez(int32_t kind, int32_t n, const double* in, double* out) {
  if ((kind != 3 && kind != 4) || n < 0 || (n > 0 && (!in || !out))) return CS_ERR_ARG;
  if (n == 0) return CS_OK;
  const size_t nin = (size_t)n * (kind == 4 ? 11 : 10);
  double *din = nullptr, *dout = nullptr;
  if (cudaMalloc(&din, nin * sizeof(double)) != cudaSuccess) return CS_ERR_CUDA;
  if (cudaMalloc(&dout, (size_t)n * sizeof(double)) != cudaSuccess) {
    cudaFree(din);
    return CS_ERR_CUDA;
  }
  cudaError_t e = cudaMemcpy(din, in, nin * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_twod_rs_ez<<<(n + 127) / 128, 128>>>(n, kind, din, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(din);
  cudaFree(dout);
  return e == cudaSuccess ? CS_OK : CS_ERR_CUDA;
}
