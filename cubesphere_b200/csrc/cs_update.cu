// Ghost exchange across the panel edges, radial padding, the RK stage
// combine, the conservative update with the constrained-transport face-B
// update, the post-update clean-up and the CFL reduction.
//
// Follows FETCH_BUFFERS_FILL_IN_UX / _UY (300riemann_module/330-332),
// PAD_BOUNDARY_R (800applications_cs/826pad_boundary_r.f:190-420),
// UPDATE_IMEX_RK_STEP_P1 (400riemann_integrate/484update_imex_rk_step_p1.f:212-906),
// CLEANUP_AFTER_UPDATE (485cleanup_after_update.f:383-1273),
// EVALUATE_TIMESTEP (490evaluate_timestep.f:121-286) and the RK combine of
// the driver (_I/_1000riemann_geomesh_cs_mhd/1000riemann_geomesh_cs_mhd.f:2661-2773).
#include "cs_solve.h"

namespace cs {

namespace {

constexpr int TPB = 128;

// Fields the ghost exchange moves: 0 U, 1 entropy (the state's type R),
// 2..4 face B (always FP64).  Values travel as doubles.
template <typename R>
__device__ __forceinline__ double fill_load(const DStateT<R>& s, int f, int32_t at) {
  switch (f) {
    case 0: return (double)s.U[at];
    case 1: return (double)s.ent[at];
    case 2: return s.Bxf[at];
    case 3: return s.Byf[at];
    default: return s.Bzf[at];
  }
}
template <typename R>
__device__ __forceinline__ void fill_store(const DStateT<R>& s, int f, int32_t at, double v) {
  switch (f) {
    case 0: s.U[at] = (R)v; break;
    case 1: s.ent[at] = (R)v; break;
    case 2: s.Bxf[at] = v; break;
    case 3: s.Byf[at] = v; break;
    default: s.Bzf[at] = v;
  }
}

// Phase 1 of the exchange: every destination value is computed from the
// pre-exchange arrays (the reference reads all sources from buffers packed
// before any ghost is written).
template <typename R>
__global__ void k_fill_gather(DStateT<R> s, const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                              const uint8_t* __restrict__ meta, double* __restrict__ tmp, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int m = meta[t];
    double v = fill_load(s, (m >> 5) & 7, src[t]);
    if (m & 8) v = -v;
    if (m & 16) v = (fill_load(s, m & 7, dst[t]) + v) * 0.5;
    tmp[t] = v;
  }
}

template <typename R>
__global__ void k_fill_scatter(DStateT<R> s, const int32_t* __restrict__ dst, const uint8_t* __restrict__ meta,
                               const double* __restrict__ tmp, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    fill_store(s, meta[t] & 7, dst[t], tmp[t]);
}

// Radial outflow padding below k = 1 and above k = nr (826:190-420).  Two
// columns that share an x- or y-face copy the same value into it.
template <typename R>
__global__ void k_pad_radial(Dims d, DGeom g, DStateT<R> s, int bc_lower, int bc_upper) {
  const int n1 = d.N + 2 * d.G;
  const long long n = 6LL * n1 * n1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % n1) + 1 - d.G;
    const int j = (int)((t / n1) % n1) + 1 - d.G;
    const int p = (int)(t / ((long long)n1 * n1));
    if (mask_at(g, d, p, i, j) != 1) continue;
    if (bc_lower == 2) {
      for (int kk = 1; kk <= d.G; ++kk) {
        const int l = 1 - kk, r = 1;
        for (int q = 0; q < NVAR; ++q) s.U[d.at(q, p, i, j, l)] = s.U[d.at(q, p, i, j, r)];
        s.Bxf[d.at(0, p, i, j, l)] = s.Bxf[d.at(0, p, i, j, r)];
        s.Bxf[d.at(0, p, i - 1, j, l)] = s.Bxf[d.at(0, p, i - 1, j, r)];
        s.Byf[d.at(0, p, i, j, l)] = s.Byf[d.at(0, p, i, j, r)];
        s.Byf[d.at(0, p, i, j - 1, l)] = s.Byf[d.at(0, p, i, j - 1, r)];
        s.Bzf[d.at(0, p, i, j, l - 1)] = s.Bzf[d.at(0, p, i, j, r - 1)];
      }
    }
    if (bc_upper == 2) {
      const int r = d.nr;
      for (int kk = 1; kk <= d.G; ++kk) {
        const int l = d.nr + kk;
        const double vr = geo(g, d, CS_G_V_VOL, 0, p, i, j, r), vl = geo(g, d, CS_G_V_VOL, 0, p, i, j, l);
        for (int q = 0; q < NVAR; ++q) s.U[d.at(q, p, i, j, l)] = s.U[d.at(q, p, i, j, r)] * vr / vl;
        s.Bzf[d.at(0, p, i, j, l)] =
            s.Bzf[d.at(0, p, i, j, r)] * geo(g, d, CS_G_ZF_AREA, 0, p, i, j, r) / geo(g, d, CS_G_ZF_AREA, 0, p, i, j, l);
        s.Bxf[d.at(0, p, i, j, l)] =
            s.Bxf[d.at(0, p, i, j, r)] * geo(g, d, CS_G_XF_AREA, 0, p, i, j, r) / geo(g, d, CS_G_XF_AREA, 0, p, i, j, l);
        s.Byf[d.at(0, p, i, j, l)] =
            s.Byf[d.at(0, p, i, j, r)] * geo(g, d, CS_G_YF_AREA, 0, p, i, j, r) / geo(g, d, CS_G_YF_AREA, 0, p, i, j, l);
        s.Bxf[d.at(0, p, i - 1, j, l)] = s.Bxf[d.at(0, p, i - 1, j, r)] * geo(g, d, CS_G_XF_AREA, 0, p, i - 1, j, r) /
                                          geo(g, d, CS_G_XF_AREA, 0, p, i - 1, j, l);
        s.Byf[d.at(0, p, i, j - 1, l)] = s.Byf[d.at(0, p, i, j - 1, r)] * geo(g, d, CS_G_YF_AREA, 0, p, i, j - 1, r) /
                                          geo(g, d, CS_G_YF_AREA, 0, p, i, j - 1, l);
      }
    }
  }
}

// RK stage combine on the whole box: kind 0 is the two-stage average
// (x + x0) / 2, kind 1 the Shu-Osher form a0 x0 + (1 - a0) x.  Segments
// 0..1 (U, entropy) hold the state's type R, 2..4 (face B) FP64.
template <typename R>
struct CombineSeg {
  R* x[2];
  const R* x0[2];
  double* b[3];
  const double* b0[3];
  long long n[5];
};
template <typename R>
__global__ void k_combine(CombineSeg<R> sg, long long total, double a0, int kind) {
  const double a1 = 1.0 - a0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    long long u = t;
    int q = 0;
    while (q < 4 && u >= sg.n[q]) {
      u -= sg.n[q];
      ++q;
    }
    if (q < 2) {
      const double x = sg.x[q][u], x0 = sg.x0[q][u];
      sg.x[q][u] = (R)(kind == 1 ? a0 * x0 + a1 * x : (x + x0) * 0.5);
    } else {
      const double x = sg.b[q - 2][u], x0 = sg.b0[q - 2][u];
      sg.b[q - 2][u] = kind == 1 ? a0 * x0 + a1 * x : (x + x0) * 0.5;
    }
  }
}

// Zone update (484:212-372): U += dt dU/dt on every zone, then on the
// interior the entropy update and the conserved->primitive repair.  The
// time step is scale times the device-resident step of the solve.
template <typename R>
__global__ void k_update_zones(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r, double scale) {
  const R dt = (R)(scale * *s.dt);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    R U[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) U[q] = s.U[d.at(q, p, i, j, k)] + dt * s.dUdt[d.at(q, p, i, j, k)];
    if (i >= 1 && i <= d.N && j >= 1 && j <= d.N && k >= 1 && k <= d.nr) {
      const R div = geoR<R>(g, d, CS_G_XF_AREA, 0, p, i, j, k) * s.EF[0][d.at(0, p, i, j, k)] -
                         geoR<R>(g, d, CS_G_XF_AREA, 0, p, i - 1, j, k) * s.EF[0][d.at(0, p, i - 1, j, k)] +
                         geoR<R>(g, d, CS_G_YF_AREA, 0, p, i, j, k) * s.EF[1][d.at(0, p, i, j, k)] -
                         geoR<R>(g, d, CS_G_YF_AREA, 0, p, i, j - 1, k) * s.EF[1][d.at(0, p, i, j - 1, k)] +
                         geoR<R>(g, d, CS_G_ZF_AREA, 0, p, i, j, k) * s.EF[2][d.at(0, p, i, j, k)] -
                         geoR<R>(g, d, CS_G_ZF_AREA, 0, p, i, j, k - 1) * s.EF[2][d.at(0, p, i, j, k - 1)];
      R en = s.ent[d.at(0, p, i, j, k)] - dt * div / geoR<R>(g, d, CS_G_V_VOL, 0, p, i, j, k);
      R V[8];
      d_cons_to_prim(ph, en, U, V);
      s.ent[d.at(0, p, i, j, k)] = en;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) s.U[d.at(q, p, i, j, k)] = U[q];
  }
}

__device__ __forceinline__ double vrad(const DGeom& g, const Dims& d, int p, int i, int j, int k) {
  const double x = geo(g, d, CS_G_VERT, 0, p, i, j, k), y = geo(g, d, CS_G_VERT, 1, p, i, j, k),
               z = geo(g, d, CS_G_VERT, 2, p, i, j, k);
  return sqrt(x * x + y * y + z * z);
}
// Angle between the vertices a and b on the sphere of radius 1/inv.
__device__ __forceinline__ double vang(const DGeom& g, const Dims& d, int p, int ax, int ay, int bx, int by, int k,
                                       double inv) {
  const double c = (geo(g, d, CS_G_VERT, 0, p, ax, ay, k) * inv) * (geo(g, d, CS_G_VERT, 0, p, bx, by, k) * inv) +
                   (geo(g, d, CS_G_VERT, 1, p, ax, ay, k) * inv) * (geo(g, d, CS_G_VERT, 1, p, bx, by, k) * inv) +
                   (geo(g, d, CS_G_VERT, 2, p, ax, ay, k) * inv) * (geo(g, d, CS_G_VERT, 2, p, bx, by, k) * inv);
  return acos(c);
}

// Constrained-transport face update (484:376-906): Stokes circulation of
// the edge EMFs with spherical arc lengths for the angular edges.
template <typename R>
__global__ void k_ct(Dims d, DGeom g, DStateT<R> s, Range3 r, int dir, double scale) {
  const double dt = scale * *s.dt;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const double* Ex = s.Ef[0];
    const double* Ey = s.Ef[1];
    const double* Ez = s.Ef[2];
    if (dir == 0) {
      const double rout = vrad(g, d, p, i, j, k), rin = vrad(g, d, p, i, j, k - 1), dr = rout - rin;
      const double th = vang(g, d, p, i, j, i, j - 1, k, 1.0 / rout);
      const double lin = rin * th, lout = rout * th;
      const double c = dr * Ez[d.at(0, p, i, j, k)] - dr * Ez[d.at(0, p, i, j - 1, k)] - lout * Ey[d.at(0, p, i, j, k)] +
                       lin * Ey[d.at(0, p, i, j, k - 1)];
      double& b = s.Bxf[d.at(0, p, i, j, k)];
      b = b - dt * c / geo(g, d, CS_G_XF_AREA, 0, p, i, j, k);
    } else if (dir == 1) {
      const double rout = vrad(g, d, p, i, j, k), rin = vrad(g, d, p, i, j, k - 1), dr = rout - rin;
      const double th = vang(g, d, p, i, j, i - 1, j, k, 1.0 / rout);
      const double lin = rin * th, lout = rout * th;
      const double c = -dr * Ez[d.at(0, p, i, j, k)] + dr * Ez[d.at(0, p, i - 1, j, k)] + lout * Ex[d.at(0, p, i, j, k)] -
                       lin * Ex[d.at(0, p, i, j, k - 1)];
      double& b = s.Byf[d.at(0, p, i, j, k)];
      b = b - dt * c / geo(g, d, CS_G_YF_AREA, 0, p, i, j, k);
    } else {
      const double rout = vrad(g, d, p, i, j, k), inv = 1.0 / rout;
      const double lxp = rout * vang(g, d, p, i, j, i - 1, j, k, inv);
      const double lxm = rout * vang(g, d, p, i, j - 1, i - 1, j - 1, k, inv);
      const double lyp = rout * vang(g, d, p, i, j, i, j - 1, k, inv);
      const double lym = rout * vang(g, d, p, i - 1, j, i - 1, j - 1, k, inv);
      const double c = lyp * Ey[d.at(0, p, i, j, k)] - lym * Ey[d.at(0, p, i - 1, j, k)] - lxp * Ex[d.at(0, p, i, j, k)] +
                       lxm * Ex[d.at(0, p, i, j - 1, k)];
      double& b = s.Bzf[d.at(0, p, i, j, k)];
      b = b - dt * c / geo(g, d, CS_G_ZF_AREA, 0, p, i, j, k);
    }
  }
}

// Clean-up zone pass (485:688-1273): least-squares zone-centred B from the
// six face values on active zones with the matching total-energy fix, then
// the conserved->primitive repair on every zone.
template <typename R>
__global__ void k_cleanup_zones(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    double U[8], V[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) U[q] = s.U[d.at(q, p, i, j, k)];
    if (mask_at(g, d, p, i, j) == 1) {
      double nv[3] = {geo(g, d, CS_G_ZF_CEN, 0, p, i, j, k), geo(g, d, CS_G_ZF_CEN, 1, p, i, j, k),
                      geo(g, d, CS_G_ZF_CEN, 2, p, i, j, k)};
      const double a = 1.0 / fmax(ph.smallnum, sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]));
      nv[0] = nv[0] * a;
      nv[1] = nv[1] * a;
      nv[2] = nv[2] * a;
      double Am[6][3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        Am[0][q] = geo(g, d, CS_G_XF_N, q, p, i, j, k);
        Am[1][q] = geo(g, d, CS_G_XF_N, q, p, i - 1, j, k);
        Am[2][q] = geo(g, d, CS_G_YF_N, q, p, i, j, k);
        Am[3][q] = geo(g, d, CS_G_YF_N, q, p, i, j - 1, k);
        Am[4][q] = nv[q];
        Am[5][q] = nv[q];
      }
      const double Rm[6] = {s.Bxf[d.at(0, p, i, j, k)], s.Bxf[d.at(0, p, i - 1, j, k)], s.Byf[d.at(0, p, i, j, k)],
                            s.Byf[d.at(0, p, i, j - 1, k)], s.Bzf[d.at(0, p, i, j, k)], s.Bzf[d.at(0, p, i, j, k - 1)]};
      double M[3][3], rhs[3];
#pragma unroll
      for (int a1 = 0; a1 < 3; ++a1) {
#pragma unroll
        for (int a2 = 0; a2 < 3; ++a2) {
          double sm = 0.0;
#pragma unroll
          for (int q = 0; q < 6; ++q) sm = sm + Am[q][a1] * Am[q][a2];
          M[a1][a2] = sm;
        }
        double sm = 0.0;
#pragma unroll
        for (int q = 0; q < 6; ++q) sm = sm + Am[q][a1] * Rm[q];
        rhs[a1] = sm;
      }
      const double a11 = M[0][0], a12 = M[0][1], a13 = M[0][2], a21 = M[1][0], a22 = M[1][1], a23 = M[1][2],
                   a31 = M[2][0], a32 = M[2][1], a33 = M[2][2];
      const double det = a11 * (a22 * a33 - a32 * a23) - a12 * (a21 * a33 - a31 * a23) + a13 * (a21 * a32 - a31 * a22);
      const double ob = copysign(1.0, det) / fmax(1.0e-32, fabs(det));
      const double b11 = (a22 * a33 - a23 * a32) * ob, b12 = (a13 * a32 - a12 * a33) * ob, b13 = (a12 * a23 - a22 * a13) * ob;
      const double b21 = (a23 * a31 - a21 * a33) * ob, b22 = (a11 * a33 - a13 * a31) * ob, b23 = (a13 * a21 - a11 * a23) * ob;
      const double b31 = (a21 * a32 - a22 * a31) * ob, b32 = (a12 * a31 - a11 * a32) * ob, b33 = (a11 * a22 - a12 * a21) * ob;
      const double nb0 = b11 * rhs[0] + b12 * rhs[1] + b13 * rhs[2];
      const double nb1 = b21 * rhs[0] + b22 * rhs[1] + b23 * rhs[2];
      const double nb2 = b31 * rhs[0] + b32 * rhs[1] + b33 * rhs[2];
      const double Bx = U[5], By = U[6], Bz = U[7];
      U[5] = nb0;
      U[6] = nb1;
      U[7] = nb2;
      U[4] = U[4] - (Bx * Bx + By * By + Bz * Bz) * ph.ob8pi + (nb0 * nb0 + nb1 * nb1 + nb2 * nb2) * ph.ob8pi;
    }
    double en = s.ent[d.at(0, p, i, j, k)];
    d_cons_to_prim(ph, en, U, V);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      s.U[d.at(q, p, i, j, k)] = U[q];
      s.V[d.at(q, p, i, j, k)] = V[q];
    }
    s.ent[d.at(0, p, i, j, k)] = en;
  }
}

__global__ void k_set_f64(double* p, double v) { *p = v; }

// The CFL reduction starts from 1.1 times the current step (490:121-286);
// its result becomes the solve's next step.
__global__ void k_dt_start(const double* dt, unsigned long long* dtmin) {
  *dtmin = (unsigned long long)__double_as_longlong(1.1 * *dt);
}
__global__ void k_dt_commit(const unsigned long long* dtmin, double* dt) { *dt = __longlong_as_double((long long)*dtmin); }

// CFL limit over the active interior zones; the minimum positive double is
// found with an integer atomicMin on its bit pattern (positive IEEE doubles
// order like their bit patterns).
template <typename R>
__global__ void k_timestep(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  double dtl = 1.0e300;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) == 0) continue;
    double U[8], V[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) U[q] = s.U[d.at(q, p, i, j, k)];
    double en = s.ent[d.at(0, p, i, j, k)];
    d_cons_to_prim(ph, en, U, V);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      s.U[d.at(q, p, i, j, k)] = U[q];
      s.V[d.at(q, p, i, j, k)] = V[q];
    }
    s.ent[d.at(0, p, i, j, k)] = en;
    const double b2 = V[5] * V[5] + V[6] * V[6] + V[7] * V[7];
    const double ms = sqrt((ph.gamma * V[4] + ph.ob4pi * b2) / V[0]);
    s.msonic[d.at(0, p, i, j, k)] = ms;
    const double a21 = sqrt(V[1] * V[1] + V[2] * V[2] + V[3] * V[3]) + ms;
    dtl = fmin(dtl, ph.cfl * geo(g, d, CS_G_V_SCALE, 0, p, i, j, k) / a21);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_down_sync(0xffffffffu, dtl, o));
  if ((threadIdx.x & 31) == 0 && dtl < 1.0e300 && dtl > 0.0)
    atomicMin(s.dtmin, (unsigned long long)__double_as_longlong(dtl));
}

inline Range3 zones_all(const Dims& d) { return {1 - d.G, d.N + d.G, 1 - d.G, d.N + d.G, 1 - d.G, d.nr + d.G}; }

}  // namespace

template <typename R>
void launch_fill_ghosts_t(Solve& sv, const DStateT<R>& st) {
  const FillMap& f = sv.fill;
  if (f.n > 0) {
    const int nb = blocks_for(f.n, 256, grid_sms(sv));
    k_fill_gather<R><<<nb, 256, 0, sv.stream>>>(st, f.d_src, f.d_dst, f.d_meta, f.d_tmp, f.n);
    mark(sv, "k_fill_gather");
    k_fill_scatter<R><<<nb, 256, 0, sv.stream>>>(st, f.d_dst, f.d_meta, f.d_tmp, f.n);
    mark(sv, "k_fill_scatter");
  }
  const int n1 = sv.d.N + 2 * sv.d.G;
  k_pad_radial<R><<<blocks_for(6LL * n1 * n1, TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(sv.d, sv.g, st, sv.p.bc_lower,
                                                                                      sv.p.bc_upper);
  mark(sv, "k_pad_radial");
}
void launch_fill_ghosts(Solve& sv) {
  if (sv.fp32)
    launch_fill_ghosts_t(sv, sv.stF);
  else
    launch_fill_ghosts_t(sv, sv.st);
}

template <typename R>
void launch_save_stage0_t(Solve& sv, const DStateT<R>& st) {
  const size_t S6 = (size_t)6 * sv.d.S;
  cudaMemcpyAsync(st.U0, st.U, NVAR * S6 * sizeof(R), cudaMemcpyDeviceToDevice, sv.stream);
  cudaMemcpyAsync(st.ent0, st.ent, S6 * sizeof(R), cudaMemcpyDeviceToDevice, sv.stream);
  cudaMemcpyAsync(st.B0[0], st.Bxf, S6 * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream);
  cudaMemcpyAsync(st.B0[1], st.Byf, S6 * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream);
  cudaMemcpyAsync(st.B0[2], st.Bzf, S6 * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream);
  mark(sv, "copy_stage0", false);
}
void launch_save_stage0(Solve& sv) {
  if (sv.fp32)
    launch_save_stage0_t(sv, sv.stF);
  else
    launch_save_stage0_t(sv, sv.st);
}

template <typename R>
void launch_combine_t(Solve& sv, const DStateT<R>& st, double a0, int kind) {
  const long long S6 = 6LL * sv.d.S;
  CombineSeg<R> sg;
  sg.x[0] = st.U;     sg.x0[0] = st.U0;    sg.n[0] = NVAR * S6;
  sg.x[1] = st.ent;   sg.x0[1] = st.ent0;  sg.n[1] = S6;
  sg.b[0] = st.Bxf;   sg.b0[0] = st.B0[0]; sg.n[2] = S6;
  sg.b[1] = st.Byf;   sg.b0[1] = st.B0[1]; sg.n[3] = S6;
  sg.b[2] = st.Bzf;   sg.b0[2] = st.B0[2]; sg.n[4] = S6;
  const long long total = (NVAR + 4) * S6;
  k_combine<R><<<blocks_for(total, 256, grid_sms(sv)), 256, 0, sv.stream>>>(sg, total, a0, kind);
  mark(sv, "k_combine");
}
void launch_combine(Solve& sv, double a0, int kind) {
  if (sv.fp32)
    launch_combine_t(sv, sv.stF, a0, kind);
  else
    launch_combine_t(sv, sv.st, a0, kind);
}

template <typename R>
void launch_update_with(Solve& sv, const DStateT<R>& st, double scale) {
  const Dims& d = sv.d;
  Range3 z = zones_all(d);
  k_update_zones<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, z, scale);
  mark(sv, "k_update_zones");
  const int N = d.N, nr = d.nr;
  Range3 fx = {0, N, 1, N, 1, nr}, fy = {1, N, 0, N, 1, nr}, fz = {1, N, 1, N, 0, nr};
  k_ct<R><<<blocks_for(fx.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, fx, 0, scale);
  mark(sv, "k_ct");
  k_ct<R><<<blocks_for(fy.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, fy, 1, scale);
  mark(sv, "k_ct");
  k_ct<R><<<blocks_for(fz.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, fz, 2, scale);
  mark(sv, "k_ct");
}
template void launch_update_with<double>(Solve&, const DStateT<double>&, double);
template void launch_update_with<float>(Solve&, const DStateT<float>&, double);

void launch_update(Solve& sv, double scale) {
  if (sv.fp32)
    launch_update_with(sv, sv.stF, scale);
  else
    launch_update_with(sv, sv.st, scale);
}

// ---- IMEX-RK2: ARS(2,2,2) with the point-mass gravity implicit ----
// Gravity S(U) = (0, -rho g, -m . g), g = GM x / r^3, on the active zones
// 0..N+1 (the zones of BUILD_NON_STIFF_SOURCES).  rho is unchanged by it,
// so the implicit stage U = U* + a S(U) has the closed form
// m = m* - a rho g, E = E* - a m . g.
template <typename R>
__global__ void k_gravity_implicit(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r, double scale) {
  const R a = (R)(scale * *s.dt);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const R x = geoR<R>(g, d, CS_G_V_CEN, 0, p, i, j, k), y = geoR<R>(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 z = geoR<R>(g, d, CS_G_V_CEN, 2, p, i, j, k);
    const R rad = sqrt(x * x + y * y + z * z);
    const R gmb = R(ph.gm) * (R(1.0) / (rad * rad * rad));
    const R gx = gmb * x, gy = gmb * y, gz = gmb * z;
    const R rho = s.U[d.at(0, p, i, j, k)];
    R& m1 = s.U[d.at(1, p, i, j, k)];
    R& m2 = s.U[d.at(2, p, i, j, k)];
    R& m3 = s.U[d.at(3, p, i, j, k)];
    m1 = m1 - a * (gx * rho);
    m2 = m2 - a * (gy * rho);
    m3 = m3 - a * (gz * rho);
    R& e = s.U[d.at(4, p, i, j, k)];
    e = e - a * (gx * m1 + gy * m2 + gz * m3);
  }
}

// dUdt += c S(U) with the gravity of the current state (explicit use of
// the previous stage's source).
template <typename R>
__global__ void k_add_gravity(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r, R c) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const R x = geoR<R>(g, d, CS_G_V_CEN, 0, p, i, j, k), y = geoR<R>(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 z = geoR<R>(g, d, CS_G_V_CEN, 2, p, i, j, k);
    const R rad = sqrt(x * x + y * y + z * z);
    const R gmb = R(ph.gm) * (R(1.0) / (rad * rad * rad));
    const R gx = gmb * x, gy = gmb * y, gz = gmb * z;
    const R rho = s.U[d.at(0, p, i, j, k)];
    const R m1 = s.U[d.at(1, p, i, j, k)], m2 = s.U[d.at(2, p, i, j, k)], m3 = s.U[d.at(3, p, i, j, k)];
    s.dUdt[d.at(1, p, i, j, k)] += c * (-(gx * rho));
    s.dUdt[d.at(2, p, i, j, k)] += c * (-(gy * rho));
    s.dUdt[d.at(3, p, i, j, k)] += c * (-(gz * rho));
    s.dUdt[d.at(4, p, i, j, k)] += c * (-(gx * m1 + gy * m2 + gz * m3));
  }
}

template <typename R>
void launch_gravity_implicit_t(Solve& sv, const DStateT<R>& st, double scale) {
  Range3 z = {0, sv.d.N + 1, 0, sv.d.N + 1, 0, sv.d.nr + 1};
  k_gravity_implicit<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(sv.d, sv.ph, sv.g, st, z,
                                                                                        scale);
  mark(sv, "k_gravity_implicit");
}
void launch_gravity_implicit(Solve& sv, double scale) {
  if (!(sv.ph.gm > sv.p.smallnum)) return;
  if (sv.fp32)
    launch_gravity_implicit_t(sv, sv.stF, scale);
  else
    launch_gravity_implicit_t(sv, sv.st, scale);
}

template <typename R>
void launch_add_gravity_t(Solve& sv, const DStateT<R>& st, double c) {
  Range3 z = {0, sv.d.N + 1, 0, sv.d.N + 1, 0, sv.d.nr + 1};
  k_add_gravity<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(sv.d, sv.ph, sv.g, st, z, c);
  mark(sv, "k_add_gravity");
}
void launch_add_gravity(Solve& sv, double c) {
  if (!(sv.ph.gm > sv.p.smallnum)) return;
  if (sv.fp32)
    launch_add_gravity_t(sv, sv.stF, c);
  else
    launch_add_gravity_t(sv, sv.st, c);
}

// Copies of the first stage's flux divergence, entropy fluxes and EMFs,
// and the restore of the step's initial state.
template <typename R>
void launch_save_stage1_rates_t(Solve& sv, const DStateT<R>& st) {
  const size_t S6 = (size_t)6 * sv.d.S;
  cudaMemcpyAsync(st.K1, st.dUdt, NVAR * S6 * sizeof(R), cudaMemcpyDeviceToDevice, sv.stream);
  for (int q = 0; q < 3; ++q) {
    cudaMemcpyAsync(st.EF1[q], st.EF[q], S6 * sizeof(R), cudaMemcpyDeviceToDevice, sv.stream);
    cudaMemcpyAsync(st.Ef1[q], st.Ef[q], S6 * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream);
  }
  mark(sv, "copy_stage1_rates", false);
}
void launch_save_stage1_rates(Solve& sv) {
  if (sv.fp32)
    launch_save_stage1_rates_t(sv, sv.stF);
  else
    launch_save_stage1_rates_t(sv, sv.st);
}

template <typename R>
void launch_restore_stage0_t(Solve& sv, const DStateT<R>& st) {
  const size_t S6 = (size_t)6 * sv.d.S;
  cudaMemcpyAsync(st.U, st.U0, NVAR * S6 * sizeof(R), cudaMemcpyDeviceToDevice, sv.stream);
  cudaMemcpyAsync(st.ent, st.ent0, S6 * sizeof(R), cudaMemcpyDeviceToDevice, sv.stream);
  cudaMemcpyAsync(st.Bxf, st.B0[0], S6 * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream);
  cudaMemcpyAsync(st.Byf, st.B0[1], S6 * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream);
  cudaMemcpyAsync(st.Bzf, st.B0[2], S6 * sizeof(double), cudaMemcpyDeviceToDevice, sv.stream);
  mark(sv, "copy_restore", false);
}
void launch_restore_stage0(Solve& sv) {
  if (sv.fp32)
    launch_restore_stage0_t(sv, sv.stF);
  else
    launch_restore_stage0_t(sv, sv.st);
}

template <typename R>
void launch_cleanup_t(Solve& sv, const DStateT<R>& st) {
  Range3 z = zones_all(sv.d);
  k_cleanup_zones<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(sv.d, sv.ph, sv.g, st, z);
  mark(sv, "k_cleanup_zones");
}
void launch_cleanup(Solve& sv) {
  launch_face_masks(sv);
  if (sv.fp32)
    launch_cleanup_t(sv, sv.stF);
  else
    launch_cleanup_t(sv, sv.st);
}

template <typename R>
void launch_timestep_t(Solve& sv, const DStateT<R>& st) {
  k_dt_start<<<1, 1, 0, sv.stream>>>(st.dt, st.dtmin);
  mark(sv, "k_dt_start");
  Range3 r = {1, sv.d.N, 1, sv.d.N, 1, sv.d.nr};
  k_timestep<R><<<blocks_for(r.count(), 256, grid_sms(sv)), 256, 0, sv.stream>>>(sv.d, sv.ph, sv.g, st, r);
  mark(sv, "k_timestep");
  k_dt_commit<<<1, 1, 0, sv.stream>>>(st.dtmin, st.dt);
  mark(sv, "k_dt_commit");
}
void launch_timestep(Solve& sv) {
  if (sv.fp32)
    launch_timestep_t(sv, sv.stF);
  else
    launch_timestep_t(sv, sv.st);
}

// Conservation diagnostics over the interior zones (FP64): volume-weighted
// sums of rho and of the total energy, and the largest |div B| (face-area
// weighted circulation of the face B over the zone volume).  A fixed grid
// of DIAG_BLOCKS blocks writes partial sums that one block then adds in a
// fixed order, so the result does not depend on launch shapes or timing.
constexpr int DIAG_BLOCKS = 512, DIAG_TPB = 256;
template <typename R>
__global__ void __launch_bounds__(DIAG_TPB) k_diag_partial(Dims d, DGeom g, DStateT<R> s, Range3 r, double* part) {
  double m = 0.0, e = 0.0, dv = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const double vol = geo(g, d, CS_G_V_VOL, 0, p, i, j, k);
    m += (double)s.U[d.at(0, p, i, j, k)] * vol;
    e += (double)s.U[d.at(4, p, i, j, k)] * vol;
    const double flux = geo(g, d, CS_G_XF_AREA, 0, p, i, j, k) * s.Bxf[d.at(0, p, i, j, k)] -
                        geo(g, d, CS_G_XF_AREA, 0, p, i - 1, j, k) * s.Bxf[d.at(0, p, i - 1, j, k)] +
                        geo(g, d, CS_G_YF_AREA, 0, p, i, j, k) * s.Byf[d.at(0, p, i, j, k)] -
                        geo(g, d, CS_G_YF_AREA, 0, p, i, j - 1, k) * s.Byf[d.at(0, p, i, j - 1, k)] +
                        geo(g, d, CS_G_ZF_AREA, 0, p, i, j, k) * s.Bzf[d.at(0, p, i, j, k)] -
                        geo(g, d, CS_G_ZF_AREA, 0, p, i, j, k - 1) * s.Bzf[d.at(0, p, i, j, k - 1)];
    dv = fmax(dv, fabs(flux) / vol);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m += __shfl_down_sync(0xffffffffu, m, o);
    e += __shfl_down_sync(0xffffffffu, e, o);
    dv = fmax(dv, __shfl_down_sync(0xffffffffu, dv, o));
  }
  __shared__ double red[3][DIAG_TPB / 32];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = m;
    red[1][w] = e;
    red[2][w] = dv;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int q = 0; q < DIAG_TPB / 32; ++q) {
      a += red[0][q];
      b += red[1][q];
      c = fmax(c, red[2][q]);
    }
    part[3 * blockIdx.x] = a;
    part[3 * blockIdx.x + 1] = b;
    part[3 * blockIdx.x + 2] = c;
  }
}
__global__ void k_diag_final(const double* part, int n, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int q = 0; q < n; ++q) {
      a += part[3 * q];
      b += part[3 * q + 1];
      c = fmax(c, part[3 * q + 2]);
    }
    out[0] = a;
    out[1] = b;
    out[2] = c;
  }
}

template <typename R>
void launch_diag_t(Solve& sv, const DStateT<R>& st, double* part, double* out) {
  const Range3 r = {1, sv.d.N, 1, sv.d.N, 1, sv.d.nr};
  k_diag_partial<R><<<DIAG_BLOCKS, DIAG_TPB, 0, sv.stream>>>(sv.d, sv.g, st, r, part);
  mark(sv, "k_diag_partial");
  k_diag_final<<<1, 32, 0, sv.stream>>>(part, DIAG_BLOCKS, out);
  mark(sv, "k_diag_final");
}
void launch_diag(Solve& sv, double* part, double* out) {
  if (sv.fp32)
    launch_diag_t(sv, sv.stF, part, out);
  else
    launch_diag_t(sv, sv.st, part, out);
}
size_t diag_scratch_doubles() { return 3 * DIAG_BLOCKS + 4; }

void launch_set_dt(Solve& sv, double dt) {
  k_set_f64<<<1, 1, 0, sv.stream>>>(sv.fp32 ? sv.stF.dt : sv.st.dt, dt);
  mark(sv, "k_set_dt");
}

}  // namespace cs
