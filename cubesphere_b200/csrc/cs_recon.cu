// Reconstruction kernels of the stage: primitive variables, flattener,
// WENO-AO / MRWENO (P12) slopes, positivity limiting, face-B quadrature
// values, the ADP constrained least-squares magnetic reconstruction and the
// zone-centred electric field with its WENO limiting.
//
// Follows LIMIT_ALL_SLOPES_P12
// (pkg/inc/cubesphere/400riemann_integrate/421limit_all_slopes_p12.f) and
// ENFORCE_PRESSURE_POSITIVITY_PRIM (440enforce_pressure_positivity_prim.f);
// each kernel names the reference step it implements.  One thread per zone
// or face; the ADP solve uses one warp per zone with the 36x36 KKT system
// in shared memory.
#include <algorithm>

#include <utility>

#include "cs_solve.h"

namespace cs {

namespace {

constexpr int TPB = 128;

template <typename R>
__device__ __forceinline__ R& Vat(const DStateT<R>& s, const Dims& d, int comp, int mode, int p, int i, int j, int k) {
  return s.V[d.at(mode * NVAR + comp, p, i, j, k)];
}

// STEP 2 (zone part, 421:597-635) and STEP 5 (421:1497-1628).
template <typename R>
__global__ void k_prim(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const int m = mask_at(g, d, p, i, j);
    R U[8], V[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) U[c] = s.U[d.at(c, p, i, j, k)];
    if (m == 0) {
#pragma unroll
      for (int c = 0; c < 8; ++c) U[c] = R(0.0);
      U[0] = R(ph.rhofloor);
      U[4] = R(ph.prsfloor) / (R(ph.gamma) - R(1.0));
    }
    R en = s.ent[d.at(0, p, i, j, k)];
    d_cons_to_prim(ph, en, U, V);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      s.U[d.at(c, p, i, j, k)] = U[c];
      s.V[d.at(c, p, i, j, k)] = V[c];
    }
    s.ent[d.at(0, p, i, j, k)] = en;
    s.ent[d.at(1, p, i, j, k)] = R(0.0);
    s.ent[d.at(2, p, i, j, k)] = R(0.0);
    s.ent[d.at(3, p, i, j, k)] = R(0.0);
    // Modes 2..10 stay zero wherever the P12 steps do not write them.
    const int lo = 3 - d.G, hx = d.N + d.G - 2, hz = d.nr + d.G - 2;
    const bool full = m == 1 && i >= lo && i <= hx && j >= lo && j <= hx && k >= lo && k <= hz;
    if (!full)
      for (int q = NVAR; q < NVAR * NMODE; ++q) s.V[d.at(q, p, i, j, k)] = R(0.0);
    const R a12 = (V[5] * V[5] + V[6] * V[6] + V[7] * V[7]) * R(ph.ob4pi);
    s.msonic[d.at(0, p, i, j, k)] = sqrt((R(ph.gamma) * V[4] + a12) / V[0]);
  }
}

// Masked-face zeroing (421:658-759; 485:383-484).
template <typename R>
__global__ void k_zero_masked_faces(Dims d, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const int lo = 1 - d.G, hi = d.N + d.G;
    if (k >= lo && j >= lo && mask_at(g, d, p, max(i, lo), j) == 0 && mask_at(g, d, p, min(i + 1, hi), j) == 0)
      s.Bxf[d.at(0, p, i, j, k)] = 0.0;
    if (k >= lo && i >= lo && mask_at(g, d, p, i, max(j, lo)) == 0 && mask_at(g, d, p, i, min(j + 1, hi)) == 0)
      s.Byf[d.at(0, p, i, j, k)] = 0.0;
    if (i >= lo && j >= lo && mask_at(g, d, p, i, j) == 0) s.Bzf[d.at(0, p, i, j, k)] = 0.0;
  }
}

// Tri-corner face-B synchronisation (421:779-962; 485:504-687).  One
// thread per (panel, corner, ghost column, k).
template <typename R>
__global__ void k_tricorner(Dims d, DGeom g, DStateT<R> s) {
  const long long n = 6LL * 4 * d.G * (d.NK - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    long long u = t;
    const int k = (int)(u % (d.NK - 1)) + 1 - d.G;
    u /= (d.NK - 1);
    const int col = (int)(u % d.G);
    u /= d.G;
    const int corner = (int)(u % 4);
    const int p = (int)(u / 4);
    const int N = d.N;
    if (corner == 0) {  // LD
      const int i = 1 - d.G + col;
      const int xd = sten(g, d, p, i, 1, 3, 0), yd = sten(g, d, p, i, 1, 3, 1);
      double& a = s.Byf[d.at(0, p, i, 0, k)];
      double& b = s.Bxf[d.at(0, p, xd - 1, yd, k)];
      const double a11 = 0.5 * (a - b);
      a = a11;
      b = -a11;
    } else if (corner == 1) {  // RD
      const int i = N + 1 + col;
      const int xd = sten(g, d, p, i, 1, 3, 0), yd = sten(g, d, p, i, 1, 3, 1);
      double& a = s.Byf[d.at(0, p, i, 0, k)];
      double& b = s.Bxf[d.at(0, p, xd, yd, k)];
      const double a11 = 0.5 * (a + b);
      a = a11;
      b = a11;
    } else if (corner == 2) {  // RU
      const int i = N + 1 + col;
      const int xu = sten(g, d, p, i, N, 2, 0), yu = sten(g, d, p, i, N, 2, 1);
      double& a = s.Byf[d.at(0, p, i, N, k)];
      double& b = s.Bxf[d.at(0, p, xu, yu, k)];
      const double a11 = 0.5 * (a - b);
      a = a11;
      b = -a11;
    } else {  // LU
      const int i = 1 - d.G + col;
      const int xu = sten(g, d, p, i, N, 2, 0), yu = sten(g, d, p, i, N, 2, 1);
      double& a = s.Byf[d.at(0, p, i, N, k)];
      double& b = s.Bxf[d.at(0, p, xu - 1, yu, k)];
      const double a11 = 0.5 * (a + b);
      a = a11;
      b = a11;
    }
  }
}

// STEP 6.a (421:1837-2131): velocity divergence and the divergence flattener.
template <typename R>
__global__ void k_flat_a(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const int lo = 2 - d.G, hx = d.N + d.G - 1, hz = d.nr + d.G - 1;
    R fl = R(0.0);
    if (i >= lo && i <= hx && j >= lo && j <= hx && k >= lo && k <= hz) {
      const int xr = sten(g, d, p, i, j, 0, 0), yr = sten(g, d, p, i, j, 0, 1);
      const int xl = sten(g, d, p, i, j, 1, 0), yl = sten(g, d, p, i, j, 1, 1);
      const int xu = sten(g, d, p, i, j, 2, 0), yu = sten(g, d, p, i, j, 2, 1);
      const int xd = sten(g, d, p, i, j, 3, 0), yd = sten(g, d, p, i, j, 3, 1);
      const R obl0 = R(1.0) / fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, p, i, j, k), R(ph.smallnum));
      const R* ms = s.msonic;
      R w = ms[d.at(0, p, i, j, k)];
      w = fmin(w, ms[d.at(0, p, xr, yr, k)]);
      w = fmin(w, ms[d.at(0, p, xl, yl, k)]);
      w = fmin(w, ms[d.at(0, p, xu, yu, k)]);
      w = fmin(w, ms[d.at(0, p, xd, yd, k)]);
      w = fmin(w, ms[d.at(0, p, i, j, k + 1)]);
      w = fmin(w, ms[d.at(0, p, i, j, k - 1)]);
      R dv = R(0.0);
      auto term = [&](int ax, int ay, int az, int bx, int by, int bz, R nx, R ny, R nz) {
        const R x = (geoR<R>(g, d, CS_G_V_CEN, 0, p, bx, by, bz) - geoR<R>(g, d, CS_G_V_CEN, 0, p, ax, ay, az)) * obl0;
        const R y = (geoR<R>(g, d, CS_G_V_CEN, 1, p, bx, by, bz) - geoR<R>(g, d, CS_G_V_CEN, 1, p, ax, ay, az)) * obl0;
        const R z = (geoR<R>(g, d, CS_G_V_CEN, 2, p, bx, by, bz) - geoR<R>(g, d, CS_G_V_CEN, 2, p, ax, ay, az)) * obl0;
        const R a11 = R(0.5) / fmax(sqrt(x * x + y * y + z * z), R(ph.smallnum));
        dv = dv + nx * a11 * (Vat(s, d, 1, 0, p, bx, by, bz) - Vat(s, d, 1, 0, p, ax, ay, az)) +
             ny * a11 * (Vat(s, d, 2, 0, p, bx, by, bz) - Vat(s, d, 2, 0, p, ax, ay, az)) +
             nz * a11 * (Vat(s, d, 3, 0, p, bx, by, bz) - Vat(s, d, 3, 0, p, ax, ay, az));
      };
      term(i, j, k, xr, yr, k, geoR<R>(g, d, CS_G_XF_N, 0, p, i, j, k), geoR<R>(g, d, CS_G_XF_N, 1, p, i, j, k),
           geoR<R>(g, d, CS_G_XF_N, 2, p, i, j, k));
      term(xl, yl, k, i, j, k, geoR<R>(g, d, CS_G_XF_N, 0, p, i - 1, j, k), geoR<R>(g, d, CS_G_XF_N, 1, p, i - 1, j, k),
           geoR<R>(g, d, CS_G_XF_N, 2, p, i - 1, j, k));
      term(i, j, k, xu, yu, k, geoR<R>(g, d, CS_G_YF_N, 0, p, i, j, k), geoR<R>(g, d, CS_G_YF_N, 1, p, i, j, k),
           geoR<R>(g, d, CS_G_YF_N, 2, p, i, j, k));
      term(xd, yd, k, i, j, k, geoR<R>(g, d, CS_G_YF_N, 0, p, i, j - 1, k), geoR<R>(g, d, CS_G_YF_N, 1, p, i, j - 1, k),
           geoR<R>(g, d, CS_G_YF_N, 2, p, i, j - 1, k));
      R nx = geoR<R>(g, d, CS_G_ZF_CEN, 0, p, i, j, k), ny = geoR<R>(g, d, CS_G_ZF_CEN, 1, p, i, j, k),
             nz = geoR<R>(g, d, CS_G_ZF_CEN, 2, p, i, j, k);
      const R a12 = R(1.0) / fmax(sqrt(nx * nx + ny * ny + nz * nz), R(ph.smallnum));
      nx = nx * a12;
      ny = ny * a12;
      nz = nz * a12;
      term(i, j, k, i, j, k + 1, nx, ny, nz);
      term(i, j, k - 1, i, j, k, nx, ny, nz);
      R a13 = fabs(dv) / (R(ph.flatten_coef) * w);
      a13 = a13 - R(1.0);
      fl = (a13 <= R(0.0)) ? R(0.0) : fmin(R(1.0), a13);
      if (mask_at(g, d, p, i, j) != 1) fl = R(0.0);
    }
    s.flatA[d.at(0, p, i, j, k)] = fl;
  }
}

// STEP 6.b (pressure-ratio raise, pass 0) and 6.c (upwinding, pass 1),
// 421:2150-2458: dst(self) = max over the six neighbours of src.
template <typename R>
__global__ void k_flat_bc(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r, const R* src, R* dst, int pass) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const int lo = 2 - d.G, hx = d.N + d.G - 1, hz = d.nr + d.G - 1;
    R fl = src[d.at(0, p, i, j, k)];
    if (i >= lo && i <= hx && j >= lo && j <= hx && k >= lo && k <= hz) {
      int xs[6], ys[6];
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        xs[w] = sten(g, d, p, i, j, w, 0);
        ys[w] = sten(g, d, p, i, j, w, 1);
      }
      xs[4] = xs[5] = i;
      ys[4] = ys[5] = j;
      const int zs[6] = {k, k, k, k, k + 1, k - 1};
      const R p0 = Vat(s, d, 4, 0, p, i, j, k);
#pragma unroll
      for (int w = 0; w < 6; ++w) {
        const bool take = pass == 1 || (Vat(s, d, 4, 0, p, xs[w], ys[w], zs[w]) > R(ph.prs_flatten_coef) * p0);
        if (take) fl = fmax(fl, src[d.at(0, p, xs[w], ys[w], zs[w])]);
      }
    }
    dst[d.at(0, p, i, j, k)] = fl;
  }
}

// Stencils of STEP 7.a: (neighbour in plane, neighbour in plane, dz).
__constant__ int c_st8[8][3] = {{0, 2, 1}, {0, 2, -1}, {1, 2, 1}, {1, 2, -1}, {0, 3, 1}, {0, 3, -1}, {1, 3, 1}, {1, 3, -1}};
// Central 18-zone stencil of STEP 7.b / 9.c: (neighbour w or -1 for self, dz).
__constant__ int c_n18[18][2] = {{0, 0},  {1, 0},  {2, 0},  {3, 0},  {-1, 1}, {-1, -1}, {8, 0}, {9, 0},  {10, 0},
                                 {11, 0}, {0, 1},  {1, 1},  {0, -1}, {1, -1}, {2, 1},   {3, 1}, {2, -1}, {3, -1}};

struct Nbr12 {
  int x[12], y[12];
};
__device__ __forceinline__ Nbr12 load_nbr(const DGeom& g, const Dims& d, int p, int i, int j) {
  Nbr12 n;
#pragma unroll
  for (int w = 0; w < 12; ++w) {
    n.x[w] = sten(g, d, p, i, j, w, 0);
    n.y[w] = sten(g, d, p, i, j, w, 1);
  }
  return n;
}

// ---- bulk asynchronous copies (cp.async.bulk) and mbarriers ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n selp.u32 %0, 1, 0, P;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Bounded wait on an mbarrier phase: after 2^23 polls (seconds, far beyond
// any copy) it records an error in *err and returns, so no wait can hang.
__device__ __noinline__ void mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
  for (int it = 0; it < (1 << 23); ++it)
    if (mbar_try_wait(bar, parity)) return;
  atomicOr(err, 1);
}

// STEP 7.a (kE false) and STEP 9.b (kE true, the WENO-AO slopes of the
// three E components, 421:6840-8400) with the work of a zone spread over
// three threads: a block takes 32 zones; warp w first forms stencils w,
// w + 3, w + 6 of each zone's eight one-sided 3x3 stencils (two in-plane
// neighbours and one radial, 421:2561-3110) as closed-form inverses of the
// scaled centroid offsets into shared memory; then, for variables w, w + 3,
// w + 6 (STEP 7.a: primitives 0-7, 8 = entropy; STEP 9.b: E component w),
// it forms the eight stencil gradients and their mean and combines them
// with the WENO weights (IS + eps)^-4, central weight 100 (421:3116-3432),
// so no thread keeps the 72 inverse entries in registers.  kEnt: the
// entropy only (LIMIT_ALL_SLOPES_P2's STEP 7.a limits the entropy this way,
// 420:5396-6306, and the primitives with k_p2).
constexpr int W7A_ZT = 32;
template <bool kE, typename R, bool kEnt = false>
__global__ void __launch_bounds__(W7A_ZT * 3, sizeof(R) == 4 ? 8 : 6) k_weno_ao_split(Dims d, PhysC ph, DGeom g,
                                                                                        DStateT<R> s, Range3 r) {
  __shared__ R ai[72][W7A_ZT];  // [stencil * 9 + entry][zone]
  // c_st8 as a compile-time table, so that the unrolled stencil loop
  // indexes the neighbour list with constants (registers, not local memory)
  constexpr int st8[8][3] = {{0, 2, 1}, {0, 2, -1}, {1, 2, 1}, {1, 2, -1}, {0, 3, 1}, {0, 3, -1}, {1, 3, 1}, {1, 3, -1}};
  const int zl = threadIdx.x % W7A_ZT, w = threadIdx.x / W7A_ZT;
  const long long nz = r.count(), ntile = (nz + W7A_ZT - 1) / W7A_ZT;
  for (long long T = blockIdx.x; T < ntile; T += gridDim.x) {
    const long long t = T * W7A_ZT + zl;
    int p = 0, i = 0, j = 0, k = 0;
    bool act = t < nz;
    if (act) {
      r.decode(t, p, i, j, k);
      act = mask_at(g, d, p, i, j) == 1;
    }
    Nbr12 n;
    if (act) {
      n = load_nbr(g, d, p, i, j);
      const R obl0 = R(1.0) / fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, p, i, j, k), R(ph.smallnum));
      const R cx = geoR<R>(g, d, CS_G_V_CEN, 0, p, i, j, k), cy = geoR<R>(g, d, CS_G_V_CEN, 1, p, i, j, k),
              cz = geoR<R>(g, d, CS_G_V_CEN, 2, p, i, j, k);
#pragma unroll 1
      for (int st = w; st < 8; st += 3) {
        const int w1 = c_st8[st][0], w2 = c_st8[st][1], dz = c_st8[st][2];
        const R a11 = (geoR<R>(g, d, CS_G_V_CEN, 0, p, n.x[w1], n.y[w1], k) - cx) * obl0;
        const R a12 = (geoR<R>(g, d, CS_G_V_CEN, 1, p, n.x[w1], n.y[w1], k) - cy) * obl0;
        const R a13 = (geoR<R>(g, d, CS_G_V_CEN, 2, p, n.x[w1], n.y[w1], k) - cz) * obl0;
        const R a21 = (geoR<R>(g, d, CS_G_V_CEN, 0, p, n.x[w2], n.y[w2], k) - cx) * obl0;
        const R a22 = (geoR<R>(g, d, CS_G_V_CEN, 1, p, n.x[w2], n.y[w2], k) - cy) * obl0;
        const R a23 = (geoR<R>(g, d, CS_G_V_CEN, 2, p, n.x[w2], n.y[w2], k) - cz) * obl0;
        const R a31 = (geoR<R>(g, d, CS_G_V_CEN, 0, p, i, j, k + dz) - cx) * obl0;
        const R a32 = (geoR<R>(g, d, CS_G_V_CEN, 1, p, i, j, k + dz) - cy) * obl0;
        const R a33 = (geoR<R>(g, d, CS_G_V_CEN, 2, p, i, j, k + dz) - cz) * obl0;
        R ob = (-a13 * a22 * a31 + a12 * a23 * a31 + a13 * a21 * a32 - a11 * a23 * a32 - a12 * a21 * a33 + a11 * a22 * a33);
        ob = copysign(R(1.0), ob) / fmax(R(1.0e-32), fabs(ob));
        ai[st * 9 + 0][zl] = (-a23 * a32 + a22 * a33) * ob;
        ai[st * 9 + 1][zl] = (a13 * a32 - a12 * a33) * ob;
        ai[st * 9 + 2][zl] = (-a13 * a22 + a12 * a23) * ob;
        ai[st * 9 + 3][zl] = (a23 * a31 - a21 * a33) * ob;
        ai[st * 9 + 4][zl] = (-a13 * a31 + a11 * a33) * ob;
        ai[st * 9 + 5][zl] = (a13 * a21 - a11 * a23) * ob;
        ai[st * 9 + 6][zl] = (-a22 * a31 + a21 * a32) * ob;
        ai[st * 9 + 7][zl] = (a12 * a31 - a11 * a32) * ob;
        ai[st * 9 + 8][zl] = (-a12 * a21 + a11 * a22) * ob;
      }
    }
    __syncthreads();
    if (act) {
#pragma unroll 1
      for (int q = kEnt ? (w == 2 ? 8 : 9) : w; q < (kE ? 3 : 9); q += 3) {
        const R* f = kE ? s.Esnap + ((long long)q * NPANEL + p) * d.S
                        : (q < 8 ? s.V + ((long long)q * NPANEL + p) * d.S : s.ent + (long long)p * d.S);
        const R f0 = f[d.idx(i, j, k)];
        R X[3][9];
#pragma unroll
        for (int st = 0; st < 8; ++st) {
          const int w1 = st8[st][0], w2 = st8[st][1], dz = st8[st][2];
          const R R0 = f[d.idx(n.x[w1], n.y[w1], k)] - f0;
          const R R1 = f[d.idx(n.x[w2], n.y[w2], k)] - f0;
          const R R2 = f[d.idx(i, j, k + dz)] - f0;
#pragma unroll
          for (int rr = 0; rr < 3; ++rr)
            X[rr][st] = ai[st * 9 + rr * 3 + 0][zl] * R0 + ai[st * 9 + rr * 3 + 1][zl] * R1 + ai[st * 9 + rr * 3 + 2][zl] * R2;
        }
#pragma unroll
        for (int rr = 0; rr < 3; ++rr)
          X[rr][8] = R(0.125) * (X[rr][0] + X[rr][1] + X[rr][2] + X[rr][3] + X[rr][4] + X[rr][5] + X[rr][6] + X[rr][7]);
        // The nonlinear weights (IS + eps)^-4 span far more than the FP32
        // range, so they are formed in FP64 in every form.
        double W[9];
#pragma unroll
        for (int st = 0; st < 9; ++st) {
          const double x0 = X[0][st], x1 = X[1][st], x2 = X[2][st];
          const double IS = x0 * x0 + x1 * x1 + x2 * x2;
          const double tt = IS + ph.smallnum;
          const double t2 = tt * tt;
          W[st] = (st < 8 ? 1.0 : 100.0) / (t2 * t2);
        }
        const double a11 = 1.0 / (W[0] + W[1] + W[2] + W[3] + W[4] + W[5] + W[6] + W[7] + W[8]);
#pragma unroll
        for (int st = 0; st < 9; ++st) W[st] = W[st] * a11;
        R gr[3];
#pragma unroll
        for (int rr = 0; rr < 3; ++rr) {
          double tt = W[0] * (double)X[rr][0];
#pragma unroll
          for (int st = 1; st < 9; ++st) tt = tt + W[st] * (double)X[rr][st];
          gr[rr] = (R)tt;
        }
        if (kE) {
          s.E[d.at(3 + q, p, i, j, k)] = gr[0];
          s.E[d.at(6 + q, p, i, j, k)] = gr[1];
          s.E[d.at(9 + q, p, i, j, k)] = gr[2];
        } else if (q < 8) {
          Vat(s, d, q, 1, p, i, j, k) = gr[0];
          Vat(s, d, q, 2, p, i, j, k) = gr[1];
          Vat(s, d, q, 3, p, i, j, k) = gr[2];
        } else {
          const R om = R(1.0) - s.flatA[d.at(0, p, i, j, k)];
          s.ent[d.at(1, p, i, j, k)] = gr[0] * om;
          s.ent[d.at(2, p, i, j, k)] = gr[1] * om;
          s.ent[d.at(3, p, i, j, k)] = gr[2] * om;
        }
      }
    }
    __syncthreads();
  }
}

template <typename R>
__device__ __forceinline__ void coef10(const DGeom& g, const Dims& d, int p, int i, int j, int k, R* c) {
#pragma unroll
  for (int t = 0; t < 10; ++t) c[t] = geoR<R>(g, d, CS_G_COEF, t, p, i, j, k);
}

// Row rr of the 18 x 9 least-squares matrix of STEP 7.b (421:3869-4001)
// for zone (i,j,k): neighbour centroid offsets scaled by l0, quadratic
// modes corrected by the neighbour's own moments.
template <typename R>
__device__ __forceinline__ void w7b_row(const Dims& d, const PhysC& ph, const DGeom& g, int p, int i, int j, int k,
                                        const Nbr12& n, int rr, R cx, R cy, R cz, R l0, R obl0,
                                        const R* c0, R* A, long long& off) {
  const int w = c_n18[rr][0], dz = c_n18[rr][1];
  const int zx = w < 0 ? i : n.x[w], zy = w < 0 ? j : n.y[w], zz = k + dz;
  off = d.idx(zx, zy, zz);
  const R x = (geoR<R>(g, d, CS_G_V_CEN, 0, p, zx, zy, zz) - cx) * obl0;
  const R y = (geoR<R>(g, d, CS_G_V_CEN, 1, p, zx, zy, zz) - cy) * obl0;
  const R z = (geoR<R>(g, d, CS_G_V_CEN, 2, p, zx, zy, zz) - cz) * obl0;
  const R lj = fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, p, zx, zy, zz), R(ph.smallnum));
  const R rt = lj / l0, r2 = rt * rt;
  A[0] = x;
  A[1] = y;
  A[2] = z;
  A[3] = x * x - c0[4] + geoR<R>(g, d, CS_G_COEF, 4, p, zx, zy, zz) * r2;
  A[4] = y * y - c0[5] + geoR<R>(g, d, CS_G_COEF, 5, p, zx, zy, zz) * r2;
  A[5] = z * z - c0[6] + geoR<R>(g, d, CS_G_COEF, 6, p, zx, zy, zz) * r2;
  A[6] = x * y - c0[7] + geoR<R>(g, d, CS_G_COEF, 7, p, zx, zy, zz) * r2;
  A[7] = y * z - c0[8] + geoR<R>(g, d, CS_G_COEF, 8, p, zx, zy, zz) * r2;
  A[8] = x * z - c0[9] + geoR<R>(g, d, CS_G_COEF, 9, p, zx, zy, zz) * r2;
}

// Inverse of the 9 x 9 normal matrix A^T A of STEP 7.b for one zone.
template <typename R>
__device__ __forceinline__ void w7b_minv(const Dims& d, const PhysC& ph, const DGeom& g, int p, int i, int j, int k,
                                         const Nbr12& n, R cx, R cy, R cz, R l0, R obl0,
                                         const R* c0, R* Minv) {
  R M[81];
#pragma unroll
  for (int t = 0; t < 81; ++t) M[t] = R(0.0);
  for (int rr = 0; rr < 18; ++rr) {
    R A[9];
    long long off;
    w7b_row(d, ph, g, p, i, j, k, n, rr, cx, cy, cz, l0, obl0, c0, A, off);
#pragma unroll
    for (int a = 0; a < 9; ++a)
#pragma unroll
      for (int b = a; b < 9; ++b) M[a * 9 + b] = M[a * 9 + b] + A[a] * A[b];
  }
#pragma unroll
  for (int a = 0; a < 9; ++a)
#pragma unroll
    for (int b = 0; b < a; ++b) M[a * 9 + b] = M[b * 9 + a];
  d_matinv<9>(M, Minv);
}

// Zones of a least-squares range in the order a stage visits them.  With
// the row weights shared by the panels (kShared), iteration it covers tile
// it / 6 of panel it % 6, so the six blocks that read one tile's weights run
// side by side and five of them find the weights in L2; otherwise the plain
// grid-stride order.  t indexes the range, tw the stored weights (panel 1's
// zone when shared); nw is their stride.
template <bool kShared>
struct LsqOrder {
  long long nr, npp, nw, nit;
  __device__ explicit LsqOrder(const Range3& r) {
    nr = r.count();
    npp = nr / 6;
    nw = kShared ? npp : nr;
    nit = kShared ? 6 * ((npp + blockDim.x - 1) / blockDim.x) : nr;
  }
  __device__ long long begin() const {
    return kShared ? (long long)blockIdx.x : blockIdx.x * (long long)blockDim.x + threadIdx.x;
  }
  __device__ long long stride() const { return kShared ? (long long)gridDim.x : (long long)gridDim.x * blockDim.x; }
  __device__ bool zone(long long it, long long& t, long long& tw) const {
    if (!kShared) {
      t = tw = it;
      return true;
    }
    tw = (it / 6) * blockDim.x + threadIdx.x;
    t = (it % 6) * npp + tw;
    return tw < npp;
  }
};

// Mode mm of panel p's least-squares solution from the sums Y over panel
// 1's row weights: sign x Y at panel 1's mode (src >> 4mm) & 15, which lies
// in mm's group (the constant, x y z, xx yy zz, xy yz xz), so the choice is
// a select among three registers.  Y holds modes M0.. (M0 = 0 with the
// constant, 1 without).
template <int M0, typename R>
__device__ __forceinline__ R lsq_rotated(const R* Y, int mm, unsigned long long src, unsigned int neg) {
  const int mu = (int)((src >> (4 * mm)) & 15);
  R v;
  if (mm == 0) {
    v = Y[0 - M0];
  } else {
    const int g0 = 1 + 3 * ((mm - 1) / 3);
    v = mu == g0 ? Y[g0 - M0] : (mu == g0 + 1 ? Y[g0 + 1 - M0] : Y[g0 + 2 - M0]);
  }
  return ((neg >> mm) & 1u) ? -v : v;
}

// STEP 7.b (421:3869-4551): 18-zone quadratic least squares hybridised
// with the linear WENO slopes (MRWENO weights, flattener damping).  With
// kCached the inverse normal matrix (geometry only) comes from the
// operator cache built at mesh build; the result is the same either way.
constexpr int W7B_QG = NVAR;
template <bool kCached, bool kShared, typename R>
__global__ void __launch_bounds__(TPB) k_weno7b(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  const R ob12 = R(1.0) / R(12.0), ob180 = R(1.0) / R(180.0), ob144 = R(1.0) / R(144.0);
  const LsqOrder<kShared> ord(r);
  for (long long it = ord.begin(); it < ord.nit; it += ord.stride()) {
    long long t, tw;
    if (!ord.zone(it, t, tw)) continue;
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const Nbr12 n = load_nbr(g, d, p, i, j);
    const R l0 = fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, p, i, j, k), R(ph.smallnum)), obl0 = R(1.0) / l0;
    R c0[10];
    coef10(g, d, p, i, j, k, c0);
    const R cx = geoR<R>(g, d, CS_G_V_CEN, 0, p, i, j, k), cy = geoR<R>(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 cz = geoR<R>(g, d, CS_G_V_CEN, 2, p, i, j, k);
    // kCached: the least-squares solution operator comes from the cache as
    // W_rr = Minv A_rr^T, one 9-vector per stencil row (geometry only), so
    // the slopes are X = sum_rr W_rr (V_rr - V_0) with no row rebuild and
    // no neighbour geometry; without the cache the rows are rebuilt and the
    // inverse applied to their sums.
    R Minv[kCached ? 1 : 81];
    if (!kCached) {
      // formed in FP64 in every form, like the cached row weights; the
      // precision form rounds the inverse once
      double c0d[10], Md[81];
      coef10(g, d, p, i, j, k, c0d);
      const double l0d = fmax(geo(g, d, CS_G_V_SCALE, 0, p, i, j, k), ph.smallnum);
      w7b_minv<double>(d, ph, g, p, i, j, k, n, geo(g, d, CS_G_V_CEN, 0, p, i, j, k), geo(g, d, CS_G_V_CEN, 1, p, i, j, k),
                       geo(g, d, CS_G_V_CEN, 2, p, i, j, k), l0d, 1.0 / l0d, c0d, Md);
#pragma unroll
      for (int e = 0; e < 81; ++e) Minv[e] = (R)Md[e];
    }
    // kShared: panel 1's row weights; the sums are rotated at the end
    const R* wc = s.op_m9 + tw;
    auto MI = [&](int e) { return Minv[kCached ? 0 : e]; };
    const R f = s.flatA[d.at(0, p, i, j, k)];
    const R betalo = f + (R(1.0) - f) * R(2.0);
    const R ghi = f * R(0.6) + (R(1.0) - f) * R(0.95), glo = R(1.0) - ghi, obghi = R(1.0) / ghi, grat = glo / ghi;
    // The primitives go in groups of W7B_QG, each group rebuilding the
    // matrix rows; on B200 one group of all eight is faster than smaller
    // groups (the row rebuild costs more than the extra live sums).  Every
    // component's sums run over the rows in the same order either way.
#pragma unroll 1
    for (int q0 = 0; q0 < NVAR; q0 += W7B_QG) {
      R v0[W7B_QG];
#pragma unroll
      for (int qq = 0; qq < W7B_QG; ++qq) v0[qq] = s.V[((long long)(q0 + qq) * NPANEL + p) * d.S + d.idx(i, j, k)];
      R Y[W7B_QG][9];
#pragma unroll
      for (int qq = 0; qq < W7B_QG; ++qq)
#pragma unroll
        for (int a = 0; a < 9; ++a) Y[qq][a] = R(0.0);
#pragma unroll 1
      for (int rr = 0; rr < 18; ++rr) {
        R A[9];
        long long off;
        if (kCached) {
          const int w = c_n18[rr][0];
          off = d.idx(w < 0 ? i : n.x[w], w < 0 ? j : n.y[w], k + c_n18[rr][1]);
#pragma unroll
          for (int a = 0; a < 9; ++a) A[a] = __ldg(wc + (long long)(rr * 9 + a) * m9_stride(ord.nw));
        } else {
          w7b_row(d, ph, g, p, i, j, k, n, rr, cx, cy, cz, l0, obl0, c0, A, off);
        }
#pragma unroll
        for (int qq = 0; qq < W7B_QG; ++qq) {
          const R Rv = s.V[((long long)(q0 + qq) * NPANEL + p) * d.S + off] - v0[qq];
#pragma unroll
          for (int a = 0; a < 9; ++a) Y[qq][a] = Y[qq][a] + A[a] * Rv;
        }
      }
      const unsigned long long qsrc = kShared ? s.lsq_map9[p].src : LSQ_IDENTITY_SRC;
      const unsigned int qneg = kShared ? s.lsq_map9[p].neg : 0u;
#pragma unroll
      for (int qq = 0; qq < W7B_QG; ++qq) {
        const int q = q0 + qq;
        R X[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) {
          if (kCached) {
            X[a] = kShared ? lsq_rotated<1>(Y[qq], a + 1, qsrc, qneg) : Y[qq][a];
          } else {
            R sacc = R(0.0);
#pragma unroll
            for (int b = 0; b < 9; ++b) sacc = sacc + MI(a * 9 + b) * Y[qq][b];
            X[a] = sacc;
          }
        }
        const R v2 = Vat(s, d, q, 1, p, i, j, k), v3 = Vat(s, d, q, 2, p, i, j, k), v4 = Vat(s, d, q, 3, p, i, j, k);
        const R ISlo = betalo * (v2 * v2 + v3 * v3 + v4 * v4) * ob12;
        R Phi[9];
        Phi[0] = X[0] * obghi - v2 * grat;
        Phi[1] = X[1] * obghi - v3 * grat;
        Phi[2] = X[2] * obghi - v4 * grat;
#pragma unroll
        for (int a = 3; a < 9; ++a) Phi[a] = X[a] * obghi;
        const R IShi = (Phi[0] * Phi[0] + Phi[1] * Phi[1] + Phi[2] * Phi[2]) * ob12 +
                            (Phi[3] * Phi[3]) * (sqr(c0[4] - ob12) + ob180) + (Phi[4] * Phi[4]) * (sqr(c0[5] - ob12) + ob180) +
                            (Phi[5] * Phi[5]) * (sqr(c0[6] - ob12) + ob180) + (Phi[6] * Phi[6]) * (c0[7] * c0[7] + ob144) +
                            (Phi[7] * Phi[7]) * (c0[8] * c0[8] + ob144) + (Phi[8] * Phi[8]) * (c0[9] * c0[9] + ob144);
        const R tau = fabs(IShi - ISlo);
        R Wlo = glo * (R(1.0) + tau / (ISlo + R(ph.smallnum))), Whi = ghi * (R(1.0) + tau / (IShi + R(ph.smallnum)));
        const R aa = R(1.0) / (Wlo + Whi);
        Wlo = Wlo * aa;
        Whi = Whi * aa;
        const R x = R(1.0) - f;
        Vat(s, d, q, 1, p, i, j, k) = (Whi * Phi[0] + Wlo * v2) * x;
        Vat(s, d, q, 2, p, i, j, k) = (Whi * Phi[1] + Wlo * v3) * x;
        Vat(s, d, q, 3, p, i, j, k) = (Whi * Phi[2] + Wlo * v4) * x;
#pragma unroll
        for (int m = 4; m < 10; ++m) Vat(s, d, q, m, p, i, j, k) = (Whi * Phi[m - 1]) * x;
      }
    }
  }
}

template <typename R>
__global__ void k_ops_m9(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  // shared by the panels: panel 1's zones only (the first sixth of the range)
  const long long nr_ = s.lsq_map9 ? r.count() / 6 : r.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nr_; t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const Nbr12 n = load_nbr(g, d, p, i, j);
    const double l0 = fmax(geo(g, d, CS_G_V_SCALE, 0, p, i, j, k), ph.smallnum), obl0 = 1.0 / l0;
    double c0[10];
    coef10(g, d, p, i, j, k, c0);
    const double cx = geo(g, d, CS_G_V_CEN, 0, p, i, j, k), cy = geo(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 cz = geo(g, d, CS_G_V_CEN, 2, p, i, j, k);
    double Minv[81];
    w7b_minv(d, ph, g, p, i, j, k, n, cx, cy, cz, l0, obl0, c0, Minv);
    // W_rr = Minv A_rr^T for the 18 stencil rows, [rr * 9 + a][zones]
    for (int rr = 0; rr < 18; ++rr) {
      double A[9];
      long long off;
      w7b_row(d, ph, g, p, i, j, k, n, rr, cx, cy, cz, l0, obl0, c0, A, off);
      for (int a = 0; a < 9; ++a) {
        double w = 0.0;
        for (int b = 0; b < 9; ++b) w = w + Minv[a * 9 + b] * A[b];
        s.op_m9[(long long)(rr * 9 + a) * m9_stride(nr_) + t] = (R)w;
      }
    }
  }
}

// Node a of the 27 positivity nodes of zone (i,j,k), as its offset from the
// centroid vc scaled by obl0: 0-7 the vertices (bit 0: +x side, bit 1: +y,
// bit 2: +z), 8-13 the face centroids (+x, -x, +y, -y, +z, -z), 14-25 the
// edge midpoints, 26 the centroid.  Read from the geometry where it is
// used, so no thread keeps the 81 coordinates.
__device__ __forceinline__ void pos_vertex(const DGeom& g, const Dims& d, int p, int i, int j, int k, int v,
                                           double* c) {
  const int vi = i - 1 + (v & 1), vj = j - 1 + ((v >> 1) & 1), vk = k - 1 + (v >> 2);
#pragma unroll
  for (int q = 0; q < 3; ++q) c[q] = geo(g, d, CS_G_VERT, q, p, vi, vj, vk);
}

__device__ __forceinline__ void pos_node(const DGeom& g, const Dims& d, int p, int i, int j, int k, int a,
                                         const double* vc, double obl0, double& x, double& y, double& z) {
  double c[3];
  if (a < 8) {
    pos_vertex(g, d, p, i, j, k, a, c);
  } else if (a < 14) {
    const int f = a - 8, dir = f >> 1, lo = f & 1;
    const int F = dir == 0 ? CS_G_XF_CEN : (dir == 1 ? CS_G_YF_CEN : CS_G_ZF_CEN);
    const int fi = i - (dir == 0 ? lo : 0), fj = j - (dir == 1 ? lo : 0), fk = k - (dir == 2 ? lo : 0);
#pragma unroll
    for (int q = 0; q < 3; ++q) c[q] = geo(g, d, F, q, p, fi, fj, fk);
  } else if (a < 26) {
    // vertex pairs along x (0-3), y (4-7), z (8-11)
    const int e = a - 14, ax = e >> 2, w = e & 3;
    int v0;
    if (ax == 0) v0 = 2 * w;
    else if (ax == 1) v0 = (w & 1) | ((w >> 1) << 2);
    else v0 = w;
    const int v1 = v0 | (1 << ax);
    double c0[3], c1[3];
    pos_vertex(g, d, p, i, j, k, v0, c0);
    pos_vertex(g, d, p, i, j, k, v1, c1);
#pragma unroll
    for (int q = 0; q < 3; ++q) c[q] = (c0[q] + c1[q]) * 0.5;
  } else {
#pragma unroll
    for (int q = 0; q < 3; ++q) c[q] = vc[q];
  }
  x = (c[0] - vc[0]) * obl0;
  y = (c[1] - vc[1]) * obl0;
  z = (c[2] - vc[2]) * obl0;
}

// STEP 7.c (440:204-829): shrink the higher modes until the 27 nodal
// values of density, pressure and entropy lie in the expanded local range.
// Four blocks per SM (measured).
template <typename R>
__global__ void __launch_bounds__(TPB, 4) k_positivity(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    const int lo = 2 - d.G, hx = d.N + d.G - 1, hz = d.nr + d.G - 1;
    if (!(i >= lo && i <= hx && j >= lo && j <= hx && k >= lo && k <= hz)) {
      s.giveup[d.at(0, p, i, j, k)] = 0;
      continue;
    }
    const Nbr12 n = load_nbr(g, d, p, i, j);
    const int px[9] = {i, n.x[0], n.x[1], n.x[2], n.x[3], n.x[8], n.x[9], n.x[10], n.x[11]};
    const int py[9] = {j, n.y[0], n.y[1], n.y[2], n.y[3], n.y[8], n.y[9], n.y[10], n.y[11]};
    double mn0 = 1e300, mx0 = -1e300, mn4 = 1e300, mx4 = -1e300, emin = 1e300, emax = -1e300;
    for (int a = 0; a < 9; ++a)
      for (int dz = -1; dz <= 1; ++dz) {
        const long long o = d.idx(px[a], py[a], k + dz);
        const double v0 = s.V[((long long)0 * NPANEL + p) * d.S + o], v4 = s.V[((long long)4 * NPANEL + p) * d.S + o];
        const double e = s.ent[(long long)p * d.S + o];
        mn0 = fmin(mn0, v0);
        mx0 = fmax(mx0, v0);
        mn4 = fmin(mn4, v4);
        mx4 = fmax(mx4, v4);
        emin = fmin(emin, e);
        emax = fmax(emax, e);
      }
    const double ef = 0.2;
    const double ff = fmax(fmin((s.flatA[d.at(0, p, i, j, k)] - 0.1) / 0.4, 1.0), 0.0), omff = 1.0 - ff;
    mn0 = fmax(mn0 * (1.0 - ef * omff), ph.rhofloor);
    mx0 = fmax(mx0 * (1.0 + ef * omff), ph.rhofloor);
    mn4 = fmax(mn4 * (1.0 - ef * omff), ph.prsfloor);
    mx4 = fmax(mx4 * (1.0 + ef * omff), ph.prsfloor);
    emin = emin * (1.0 - ef * omff);
    emax = emax * (1.0 + ef * omff);
    const double obl0 = 1.0 / fmax(geo(g, d, CS_G_V_SCALE, 0, p, i, j, k), ph.smallnum);
    const double vc[3] = {geo(g, d, CS_G_V_CEN, 0, p, i, j, k), geo(g, d, CS_G_V_CEN, 1, p, i, j, k),
                          geo(g, d, CS_G_V_CEN, 2, p, i, j, k)};
    double c0[10];
    coef10(g, d, p, i, j, k, c0);
    double vr[10], vp[10], ep[4];
#pragma unroll
    for (int m = 0; m < 10; ++m) {
      vr[m] = Vat(s, d, 0, m, p, i, j, k);
      vp[m] = Vat(s, d, 4, m, p, i, j, k);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) ep[m] = s.ent[d.at(m, p, i, j, k)];
    const int niter = 15;
    const double ratio = pow(0.10, 1.0 / (double)niter);
    double scale = 1.0;  // cumulative shrink of the higher modes
    int gave_up = 0;
    for (int iter = 1; iter <= niter + 1; ++iter) {
      if (iter == niter + 1) {
        gave_up = 1;
        break;
      }
      bool pass = true;
      for (int a = 0; a < 27 && pass; ++a) {
        double x, y, z;
        pos_node(g, d, p, i, j, k, a, vc, obl0, x, y, z);
        const double v1 = d_poly10(vr, c0, x, y, z), v5 = d_poly10(vp, c0, x, y, z);
        const double en = ep[0] + ep[1] * x + ep[2] * y + ep[3] * z;
        if (v1 < mn0 || v1 > mx0 || v5 < mn4 || v5 > mx4 || en < emin || en > emax) pass = false;
      }
      if (pass) break;
#pragma unroll
      for (int m = 1; m < 10; ++m) {
        vr[m] = ratio * vr[m];
        vp[m] = ratio * vp[m];
      }
#pragma unroll
      for (int m = 1; m < 4; ++m) ep[m] = ratio * ep[m];
      scale = scale + 1.0;  // counts the shrinks applied
    }
    const int nshrink = (int)(scale - 1.0);
    if (gave_up || nshrink > 0) {
      for (int q = 0; q < NVAR; ++q)
        for (int m = 1; m < 10; ++m) {
          double v = Vat(s, d, q, m, p, i, j, k);
          if (gave_up) {
            v = 0.0;
          } else {
            for (int it = 0; it < nshrink; ++it) v = ratio * v;
          }
          Vat(s, d, q, m, p, i, j, k) = v;
        }
      for (int m = 1; m < 4; ++m) s.ent[d.at(m, p, i, j, k)] = gave_up ? 0.0 : ep[m];
    }
    // bit 0: gave up; bits 1-4: shrink passes applied
    s.giveup[d.at(0, p, i, j, k)] = gave_up | (nshrink << 1);
  }
}

// A zone that exhausted the shrink passes also zeroes its entropy value
// (440:569-575); applied after every zone has read its neighbours.
template <typename R>
__global__ void k_apply_giveup(Dims d, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (s.giveup[d.at(0, p, i, j, k)] & 1) s.ent[d.at(0, p, i, j, k)] = 0.0;
  }
}

// STEP 8.a-c (421:4686-5567): B at the five quadrature points of each face,
// averaged from both sides and shifted to the facial mean.
template <typename R>
__global__ void __launch_bounds__(TPB) k_faceB(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r, int dir) {
  const int QP = dir == 0 ? CS_G_XF_QP : (dir == 1 ? CS_G_YF_QP : CS_G_ZF_QP);
  const int BW = dir == 0 ? CS_G_XB_QW : (dir == 1 ? CS_G_YB_QW : CS_G_ZB_QW);
  const int NF = dir == 0 ? CS_G_XF_N : (dir == 1 ? CS_G_YF_N : CS_G_ZF_N);
  double* Bq = s.Bq[dir];
  const double* Bf = dir == 0 ? s.Bxf : (dir == 1 ? s.Byf : s.Bzf);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    int lx = i, ly = j, lz = k, rx = i, ry = j, rz = k;
    bool skip = false;
    if (dir == 0) {
      const int mL = mask_at(g, d, p, i, j), mR = mask_at(g, d, p, i + 1, j);
      rx = i + 1;
      if (mL == 0 && mR == 1) { lx = sten(g, d, p, rx, ry, 1, 0); ly = sten(g, d, p, rx, ry, 1, 1); }
      else if (mL == 1 && mR == 0) { rx = sten(g, d, p, lx, ly, 0, 0); ry = sten(g, d, p, lx, ly, 0, 1); }
      else if (mL == 0 && mR == 0) skip = true;
    } else if (dir == 1) {
      const int mL = mask_at(g, d, p, i, j), mR = mask_at(g, d, p, i, j + 1);
      ry = j + 1;
      if (mL == 0 && mR == 1) { lx = sten(g, d, p, rx, ry, 3, 0); ly = sten(g, d, p, rx, ry, 3, 1); }
      else if (mL == 1 && mR == 0) { rx = sten(g, d, p, lx, ly, 2, 0); ry = sten(g, d, p, lx, ly, 2, 1); }
      else if (mL == 0 && mR == 0) skip = true;
    } else {
      if (mask_at(g, d, p, i, j) == 0) skip = true;
      rz = k + 1;
    }
    // the two sides' values in the state's type; the shift to the facial
    // mean in FP64, so the values average to the FP64 face B exactly
    R bq[5] = {R(0), R(0), R(0), R(0), R(0)};
    if (!skip) {
      const R obl0 = R(1.0) / fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, p, lx, ly, lz), R(ph.smallnum));
      const R obl02 = R(1.0) / fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, p, rx, ry, rz), R(ph.smallnum));
      R cL[10], cR[10], vL[3][10], vR[3][10];
      coef10(g, d, p, lx, ly, lz, cL);
      coef10(g, d, p, rx, ry, rz, cR);
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int m = 0; m < 10; ++m) {
          vL[b][m] = Vat(s, d, 5 + b, m, p, lx, ly, lz);
          vR[b][m] = Vat(s, d, 5 + b, m, p, rx, ry, rz);
        }
      const R lcx = geoR<R>(g, d, CS_G_V_CEN, 0, p, lx, ly, lz), lcy = geoR<R>(g, d, CS_G_V_CEN, 1, p, lx, ly, lz),
              lcz = geoR<R>(g, d, CS_G_V_CEN, 2, p, lx, ly, lz);
      const R rcx = geoR<R>(g, d, CS_G_V_CEN, 0, p, rx, ry, rz), rcy = geoR<R>(g, d, CS_G_V_CEN, 1, p, rx, ry, rz),
              rcz = geoR<R>(g, d, CS_G_V_CEN, 2, p, rx, ry, rz);
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        const int nq = dir == 2 ? q : 0, ns = dir == 2 ? 5 : 1;
        const R nx = geoR<R>(g, d, NF, 0 * ns + nq, p, i, j, k), ny = geoR<R>(g, d, NF, 1 * ns + nq, p, i, j, k),
                nz = geoR<R>(g, d, NF, 2 * ns + nq, p, i, j, k);
        const R px = geoR<R>(g, d, QP, q, p, i, j, k), py = geoR<R>(g, d, QP, 5 + q, p, i, j, k),
                pz = geoR<R>(g, d, QP, 10 + q, p, i, j, k);
        const R x = (px - lcx) * obl0, y = (py - lcy) * obl0, z = (pz - lcz) * obl0;
        const R x2 = (px - rcx) * obl02, y2 = (py - rcy) * obl02, z2 = (pz - rcz) * obl02;
        const R bx = d_poly10(vL[0], cL, x, y, z), by = d_poly10(vL[1], cL, x, y, z), bz = d_poly10(vL[2], cL, x, y, z);
        const R bx2 = d_poly10(vR[0], cR, x2, y2, z2), by2 = d_poly10(vR[1], cR, x2, y2, z2),
                bz2 = d_poly10(vR[2], cR, x2, y2, z2);
        bq[q] = R(0.5) * (nx * (bx + bx2) + ny * (by + by2) + nz * (bz + bz2));
      }
    }
    double bd = Bf[d.at(0, p, i, j, k)];
#pragma unroll
    for (int q = 0; q < 5; ++q) bd = bd - geo(g, d, BW, q, p, i, j, k) * (double)bq[q];
#pragma unroll
    for (int q = 0; q < 5; ++q) Bq[d.at(q, p, i, j, k)] = (double)bq[q] + bd;
  }
}

// STEP 8.d ADP (421:5617-6677): constrained least squares for the 30
// quadratic B modes matching the 6 face means exactly, solved per zone as
// the 36x36 KKT system by one warp with Gaussian elimination (scaled
// partial pivoting) in shared memory.
constexpr int ADP_WARPS = 4;
// Resident ADP factors are stored as one stream per block of ADP_ZB zones
// (zone fastest), in the order the substitution consumes them: the strict
// lower triangle row by row (630), then for rows 35..0 the entries right of
// the diagonal followed by the diagonal (666).
constexpr int ADP_ZB = 128;
__host__ __device__ constexpr int adp_stream_pos(int a, int b) {
  return b < a ? a * (a - 1) / 2 + b : 630 + (35 - a) * (36 - a) / 2 + (b == a ? 35 - a : b - a - 1);
}
// Factor stream of the panel-shared cache: blocks of ADP6_ZB zones; the
// strict lower triangle column by column (630: column b, rows b+1..35),
// then for rows 35..0 the entries right of the diagonal followed by the
// diagonal (666).  Column order lets the forward pass update 35 - b rows
// independently per column; each row still receives its terms in
// ascending column order, so the arithmetic is that of the row order.
constexpr int ADP6_ZB = 32;
__host__ __device__ constexpr int adp6_stream_pos(int a, int b) {
  return b < a ? b * 35 - b * (b - 1) / 2 + (a - b - 1)
               : 630 + (35 - a) * (36 - a) / 2 + (b == a ? 35 - a : b - a - 1);
}
struct AdpSmem {
  double K[36][37];
  double Q[30][31];
  double bq[30], wt[30], C[6][30], D[6], rhs[36], sol[36], sc[36], vB[30];
  int piv[36];
};

// kFactorOnly: assemble and factor the geometry-only KKT matrix and store
// the factors and the row permutation for k_adp_solve (once per mesh).
// tmax: zones of the range handled (all of it, or panel 1's share when the
// factors are shared by the six panels); zb: zones per factor block.
template <bool kFactorOnly, typename R>
__global__ void __launch_bounds__(32 * ADP_WARPS) k_adp(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r,
                                                        long long tmax, int zb) {
  extern __shared__ unsigned char smem_raw[];
  AdpSmem& S = reinterpret_cast<AdpSmem*>(smem_raw)[threadIdx.x / 32];
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * ADP_WARPS;
  for (long long t = blockIdx.x * (long long)ADP_WARPS + threadIdx.x / 32; t < tmax; t += nw) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) == 0) continue;
    const double obl0 = 1.0 / fmax(geo(g, d, CS_G_V_SCALE, 0, p, i, j, k), ph.smallnum);
    const double vc0 = geo(g, d, CS_G_V_CEN, 0, p, i, j, k), vc1 = geo(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 vc2 = geo(g, d, CS_G_V_CEN, 2, p, i, j, k);
    double c0[10];
    coef10(g, d, p, i, j, k, c0);
    // 1. the 30 quadrature rows, one per lane
    if (lane < 30) {
      const int f = lane / 5, q = lane % 5, dir = f / 2;
      const int fx = (f == 1) ? i - 1 : i, fy = (f == 3) ? j - 1 : j, fz = (f == 5) ? k - 1 : k;
      const int QP = dir == 0 ? CS_G_XF_QP : (dir == 1 ? CS_G_YF_QP : CS_G_ZF_QP);
      const int BW = dir == 0 ? CS_G_XB_QW : (dir == 1 ? CS_G_YB_QW : CS_G_ZB_QW);
      const int NF = dir == 0 ? CS_G_XF_N : (dir == 1 ? CS_G_YF_N : CS_G_ZF_N);
      const int nq = dir == 2 ? q : 0, ns = dir == 2 ? 5 : 1;
      const double nx = geo(g, d, NF, nq, p, fx, fy, fz), ny = geo(g, d, NF, ns + nq, p, fx, fy, fz),
                   nz = geo(g, d, NF, 2 * ns + nq, p, fx, fy, fz);
      const double x = (geo(g, d, QP, q, p, fx, fy, fz) - vc0) * obl0;
      const double y = (geo(g, d, QP, 5 + q, p, fx, fy, fz) - vc1) * obl0;
      const double z = (geo(g, d, QP, 10 + q, p, fx, fy, fz) - vc2) * obl0;
      const double bfn[10] = {1.0, x, y, z, x * x - c0[4], y * y - c0[5], z * z - c0[6], x * y - c0[7], y * z - c0[8], x * z - c0[9]};
#pragma unroll
      for (int m = 0; m < 10; ++m) {
        S.Q[lane][m] = m == 0 ? nx : nx * bfn[m];
        S.Q[lane][10 + m] = m == 0 ? ny : ny * bfn[m];
        S.Q[lane][20 + m] = m == 0 ? nz : nz * bfn[m];
      }
      S.wt[lane] = geo(g, d, BW, q, p, fx, fy, fz);
      if (!kFactorOnly) {
        S.bq[lane] = s.Bq[dir][d.at(q, p, fx, fy, fz)];
        S.vB[lane] = Vat(s, d, 5 + lane / 10, lane % 10, p, i, j, k);
      } else {
        S.bq[lane] = 0.0;
        S.vB[lane] = 0.0;
      }
    }
    __syncwarp();
    // 2. constraint rows C, D and the KKT matrix
    for (int e = lane; e < 180; e += 32) {
      const int f = e / 30, m = e % 30;
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < 5; ++q) acc = acc + S.wt[f * 5 + q] * S.Q[f * 5 + q][m];
      S.C[f][m] = acc;
    }
    if (lane < 6) {
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < 5; ++q) acc = acc + S.wt[lane * 5 + q] * S.bq[lane * 5 + q];
      S.D[lane] = acc;
    }
    __syncwarp();
    // divergence-free rows (421:6586-6600) as (column, value) pairs
    const int dcol[4][3] = {{1, 12, 23}, {4, 17, 29}, {7, 15, 28}, {9, 18, 26}};
    const double dval[4][3] = {{1.0, 1.0, 1.0}, {2.0, 1.0, 1.0}, {1.0, 2.0, 1.0}, {1.0, 1.0, 2.0}};
    for (int e = lane; e < 900; e += 32) {
      const int a = e / 30, b = e % 30;
      double acc = 0.0;
      for (int q = 0; q < 30; ++q) acc = acc + S.Q[q][a] * S.Q[q][b];
      if (a == b) acc = acc + 1.0;
      for (int rr = 0; rr < 4; ++rr) {
        double va = 0.0, vb = 0.0;
        for (int c = 0; c < 3; ++c) {
          if (dcol[rr][c] == a) va = dval[rr][c];
          if (dcol[rr][c] == b) vb = dval[rr][c];
        }
        acc = acc + va * vb;
      }
      S.K[a][b] = acc;
    }
    for (int e = lane; e < 180; e += 32) {
      const int f = e / 30, m = e % 30;
      S.K[m][30 + f] = S.C[f][m];
      S.K[30 + f][m] = S.C[f][m];
    }
    for (int e = lane; e < 36; e += 32) {
      S.K[30 + e / 6][30 + e % 6] = 0.0;
    }
    if (lane < 30) {
      double acc = 0.0;
      for (int q = 0; q < 30; ++q) acc = acc + S.Q[q][lane] * S.bq[q];
      S.rhs[lane] = acc + S.vB[lane];
    } else {
      for (int f = lane - 30; f < 6; f += 2) S.rhs[30 + f] = S.D[f];
    }
    __syncwarp();
    // 3. elimination with scaled partial pivoting
    for (int row = lane; row < 36; row += 32) {
      double m = 0.0;
      for (int c = 0; c < 36; ++c) m = fmax(m, fabs(S.K[row][c]));
      S.sc[row] = (m == 0.0) ? 0.0 : 1.0 / m;
      S.piv[row] = row;
    }
    __syncwarp();
    for (int kk = 0; kk < 36; ++kk) {
      double best = -1.0;
      int bi = kk;
      for (int row = kk + lane; row < 36; row += 32) {
        const double v = fabs(S.K[row][kk]) * S.sc[row];
        if (v > best) {
          best = v;
          bi = row;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (bi != kk) {
        for (int c = lane; c < 36; c += 32) {
          const double tmp = S.K[kk][c];
          S.K[kk][c] = S.K[bi][c];
          S.K[bi][c] = tmp;
        }
        if (lane == 0) {
          const double ts = S.sc[kk];
          S.sc[kk] = S.sc[bi];
          S.sc[bi] = ts;
          const int tp = S.piv[kk];
          S.piv[kk] = S.piv[bi];
          S.piv[bi] = tp;
        }
      }
      __syncwarp();
      if (lane == 0 && S.K[kk][kk] == 0.0) S.K[kk][kk] = 1.0e-20;
      __syncwarp();
      const double inv = 1.0 / S.K[kk][kk];
      for (int row = kk + 1 + lane; row < 36; row += 32) {
        const double l = S.K[row][kk] * inv;
        S.K[row][kk] = l;
        for (int c = kk + 1; c < 36; ++c) S.K[row][c] -= l * S.K[kk][c];
      }
      __syncwarp();
    }
    if (kFactorOnly) {
      const long long blk = t / zb, z = t % zb;
      for (int e = lane; e < 36 * 36; e += 32) {
        const int pos = zb == ADP6_ZB ? adp6_stream_pos(e / 36, e % 36) : adp_stream_pos(e / 36, e % 36);
        // panel-shared factors in the state's type, per-panel ones in FP64
        if (zb == ADP6_ZB)
          ((R*)s.adp_lu)[(blk * 1296 + pos) * zb + z] = (R)S.K[e / 36][e % 36];
        else
          ((double*)s.adp_lu)[(blk * 1296 + pos) * zb + z] = S.K[e / 36][e % 36];
      }
      for (int e = lane; e < 36; e += 32) s.adp_piv[(blk * 36 + e) * zb + z] = (int8_t)S.piv[e];
      __syncwarp();
      continue;
    }
    // 4. substitution (one lane, reference order)
    if (lane == 0) {
      double y[36];
      for (int a = 0; a < 36; ++a) {
        double acc = S.rhs[S.piv[a]];
        for (int b = 0; b < a; ++b) acc -= S.K[a][b] * y[b];
        y[a] = acc;
      }
      for (int a = 35; a >= 0; --a) {
        double acc = y[a];
        for (int b = a + 1; b < 36; ++b) acc -= S.K[a][b] * S.sol[b];
        S.sol[a] = acc / S.K[a][a];
      }
    }
    __syncwarp();
    // 5. write back the modes, zone B and the energy adjustment
    if (lane < 30) Vat(s, d, 5 + lane / 10, lane % 10, p, i, j, k) = S.sol[lane];
    if (lane == 0) {
      R* U = s.U;
      const long long o5 = d.at(4, p, i, j, k);
      const double u6 = U[d.at(5, p, i, j, k)], u7 = U[d.at(6, p, i, j, k)], u8 = U[d.at(7, p, i, j, k)];
      const double aa = (u6 * u6 + u7 * u7 + u8 * u8) * ph.ob8pi;
      const double n6 = S.sol[0], n7 = S.sol[10], n8 = S.sol[20];
      U[d.at(5, p, i, j, k)] = n6;
      U[d.at(6, p, i, j, k)] = n7;
      U[d.at(7, p, i, j, k)] = n8;
      const double bb = (n6 * n6 + n7 * n7 + n8 * n8) * ph.ob8pi;
      U[o5] = U[o5] - aa + bb;
    }
    __syncwarp();
  }
}

// STEP 8.d right-hand side with the resident factors: one thread per zone
// forms the 36 entries (the same sums in the same order as k_adp) and
// stores them element-major, [36][zones of the ADP range].
constexpr int ADPR_TPB = 128;
template <typename R>
__global__ void __launch_bounds__(ADPR_TPB) k_adp_rhs(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  const long long n = r.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    double* out = (double*)s.adp_rhs + t;
    if (mask_at(g, d, p, i, j) != 1) {
#pragma unroll
      for (int a = 0; a < 36; ++a) out[(long long)a * n] = 0.0;
      continue;
    }
    const double obl0 = 1.0 / fmax(geo(g, d, CS_G_V_SCALE, 0, p, i, j, k), ph.smallnum);
    const double vc0 = geo(g, d, CS_G_V_CEN, 0, p, i, j, k), vc1 = geo(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 vc2 = geo(g, d, CS_G_V_CEN, 2, p, i, j, k);
    double c0[10];
    coef10(g, d, p, i, j, k, c0);
    double rhs[30];
#pragma unroll
    for (int a = 0; a < 30; ++a) rhs[a] = 0.0;
#pragma unroll 1
    for (int f = 0; f < 6; ++f) {
      const int dir = f / 2;
      const int fx = (f == 1) ? i - 1 : i, fy = (f == 3) ? j - 1 : j, fz = (f == 5) ? k - 1 : k;
      const int QP = dir == 0 ? CS_G_XF_QP : (dir == 1 ? CS_G_YF_QP : CS_G_ZF_QP);
      const int BW = dir == 0 ? CS_G_XB_QW : (dir == 1 ? CS_G_YB_QW : CS_G_ZB_QW);
      const int NF = dir == 0 ? CS_G_XF_N : (dir == 1 ? CS_G_YF_N : CS_G_ZF_N);
      const int ns = dir == 2 ? 5 : 1;
      double dacc = 0.0;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        const int nq = dir == 2 ? q : 0;
        const double nx = geo(g, d, NF, nq, p, fx, fy, fz), ny = geo(g, d, NF, ns + nq, p, fx, fy, fz),
                     nz = geo(g, d, NF, 2 * ns + nq, p, fx, fy, fz);
        const double x = (geo(g, d, QP, q, p, fx, fy, fz) - vc0) * obl0;
        const double y = (geo(g, d, QP, 5 + q, p, fx, fy, fz) - vc1) * obl0;
        const double z = (geo(g, d, QP, 10 + q, p, fx, fy, fz) - vc2) * obl0;
        const double bfn[10] = {1.0, x, y, z, x * x - c0[4], y * y - c0[5], z * z - c0[6], x * y - c0[7],
                                y * z - c0[8], x * z - c0[9]};
        const double bq = s.Bq[dir][d.at(q, p, fx, fy, fz)];
#pragma unroll
        for (int m = 0; m < 10; ++m) {
          rhs[m] = rhs[m] + (m == 0 ? nx : nx * bfn[m]) * bq;
          rhs[10 + m] = rhs[10 + m] + (m == 0 ? ny : ny * bfn[m]) * bq;
          rhs[20 + m] = rhs[20 + m] + (m == 0 ? nz : nz * bfn[m]) * bq;
        }
        dacc = dacc + geo(g, d, BW, q, p, fx, fy, fz) * bq;
      }
      out[(long long)(30 + f) * n] = dacc;
    }
#pragma unroll
    for (int a = 0; a < 30; ++a) out[(long long)a * n] = rhs[a] + Vat(s, d, 5 + a / 10, a % 10, p, i, j, k);
  }
}

// The same right-hand sides for the six panels from panel 1's geometry:
// one thread per zone position forms r1 = sum_q row_1(q) bq_p(q) with
// panel 1's quadrature rows and panel p's face values, then rhs_p =
// T_p r1 + vB_p (the rows of panel p are T_p times panel 1's, see
// k_adp_solve6), so the geometry is read once for six panels.
// Four blocks per SM (128 registers) beat three at 168 (measured).
template <typename R>
__global__ void __launch_bounds__(ADPR_TPB, 4) k_adp_rhs6(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  const long long n = r.count(), n1 = n / 6;
  for (long long t1 = blockIdx.x * (long long)blockDim.x + threadIdx.x; t1 < n1;
       t1 += (long long)gridDim.x * blockDim.x) {
    int p0, i, j, k;
    r.decode(t1, p0, i, j, k);
    const R obl0 = R(1.0) / fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, 0, i, j, k), R(ph.smallnum));
    const R vc0 = geoR<R>(g, d, CS_G_V_CEN, 0, 0, i, j, k), vc1 = geoR<R>(g, d, CS_G_V_CEN, 1, 0, i, j, k),
            vc2 = geoR<R>(g, d, CS_G_V_CEN, 2, 0, i, j, k);
    R c0[10];
    coef10(g, d, 0, i, j, k, c0);
#pragma unroll 1
    for (int p = 0; p < 6; ++p) {
      R* out = (R*)s.adp_rhs + p * n1 + t1;
      if (mask_at(g, d, p, i, j) != 1) {
#pragma unroll
        for (int a = 0; a < 36; ++a) out[(long long)a * n] = R(0.0);
        continue;
      }
      R rhs[30];
#pragma unroll
      for (int a = 0; a < 30; ++a) rhs[a] = R(0.0);
#pragma unroll 1
      for (int f = 0; f < 6; ++f) {
        const int dir = f / 2;
        const int fx = (f == 1) ? i - 1 : i, fy = (f == 3) ? j - 1 : j, fz = (f == 5) ? k - 1 : k;
        const int QP = dir == 0 ? CS_G_XF_QP : (dir == 1 ? CS_G_YF_QP : CS_G_ZF_QP);
        const int BW = dir == 0 ? CS_G_XB_QW : (dir == 1 ? CS_G_YB_QW : CS_G_ZB_QW);
        const int NF = dir == 0 ? CS_G_XF_N : (dir == 1 ? CS_G_YF_N : CS_G_ZF_N);
        const int ns = dir == 2 ? 5 : 1;
        R dacc = R(0.0);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          const int nq = dir == 2 ? q : 0;
          const R nx = geoR<R>(g, d, NF, nq, 0, fx, fy, fz), ny = geoR<R>(g, d, NF, ns + nq, 0, fx, fy, fz),
                  nz = geoR<R>(g, d, NF, 2 * ns + nq, 0, fx, fy, fz);
          const R x = (geoR<R>(g, d, QP, q, 0, fx, fy, fz) - vc0) * obl0;
          const R y = (geoR<R>(g, d, QP, 5 + q, 0, fx, fy, fz) - vc1) * obl0;
          const R z = (geoR<R>(g, d, QP, 10 + q, 0, fx, fy, fz) - vc2) * obl0;
          const R bfn[10] = {R(1.0), x, y, z, x * x - c0[4], y * y - c0[5], z * z - c0[6], x * y - c0[7],
                             y * z - c0[8], x * z - c0[9]};
          const R bq = (R)s.Bq[dir][d.at(q, p, fx, fy, fz)];
#pragma unroll
          for (int m = 0; m < 10; ++m) {
            rhs[m] = rhs[m] + (m == 0 ? nx : nx * bfn[m]) * bq;
            rhs[10 + m] = rhs[10 + m] + (m == 0 ? ny : ny * bfn[m]) * bq;
            rhs[20 + m] = rhs[20 + m] + (m == 0 ? nz : nz * bfn[m]) * bq;
          }
          dacc = dacc + geoR<R>(g, d, BW, q, 0, fx, fy, fz) * bq;
        }
        out[(long long)(30 + f) * n] = dacc;
      }
      const int8_t* umap = s.adp_pmap + p * 72;
#pragma unroll
      for (int v = 0; v < 30; ++v) {
        const int u = __ldg(umap + v);
        out[(long long)u * n] = (R)__ldg(umap + 36 + v) * rhs[v] + Vat(s, d, 5 + u / 10, u % 10, p, i, j, k);
      }
    }
  }
}

// STEP 8.d substitution with the resident factors, one thread per zone.
// The factor stream of the block's 128 zones (1296 x 1 KB, in consumption
// order) flows through a ring of ADPS_NS shared-memory stages of ADPS_CH
// elements (16 KB), filled by bulk asynchronous copies that a producer warp
// issues as soon as the four consumer warps have released a stage
// (full / empty mbarrier pairs).  The solution vector lives in shared
// memory so that the loops stay short; the arithmetic (order included) is
// that of the reference's forward and back substitution.
constexpr int ADPS_TPB = ADP_ZB;             // consumer threads (one per zone)
constexpr int ADPS_THREADS = ADPS_TPB + 32;  // + one producer warp
constexpr int ADPS_CH = 16;
constexpr int ADPS_NS = 4;
constexpr int ADPS_NCH = 1296 / ADPS_CH;
static_assert(1296 % ADPS_CH == 0, "whole chunks");
struct AdpsSmem {
  double stage[ADPS_NS][ADPS_CH][ADPS_TPB];
  double y[36][ADPS_TPB];
  uint64_t full[ADPS_NS];
  uint64_t empty[ADPS_NS];
};

template <typename R>
__global__ void __launch_bounds__(ADPS_THREADS, 2) k_adp_solve(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  extern __shared__ __align__(128) unsigned char adps_raw[];
  AdpsSmem& S = *reinterpret_cast<AdpsSmem*>(adps_raw);
  const int tid = threadIdx.x;
  const long long n = r.count();
  const long long nblk = (n + ADP_ZB - 1) / ADP_ZB;
  if ((long long)blockIdx.x >= nblk) return;
  const long long my_iters = (nblk - 1 - blockIdx.x) / gridDim.x + 1;
  const long long total_chunks = my_iters * ADPS_NCH;
  if (tid == 0) {
    for (int q = 0; q < ADPS_NS; ++q) {
      mbar_init(&S.full[q], 1);
      mbar_init(&S.empty[q], ADPS_TPB / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid >= ADPS_TPB) {
    // producer: chunk gch of this CTA is chunk gch % NCH of zone block
    // blockIdx.x + (gch / NCH) * gridDim.x
    if (tid == ADPS_TPB) {
      for (long long gch = 0; gch < total_chunks; ++gch) {
        const int slot = (int)(gch % ADPS_NS);
        if (gch >= ADPS_NS) mbar_wait(&S.empty[slot], (uint32_t)(((gch / ADPS_NS) - 1) & 1), s.err_flag);
        const long long it = gch / ADPS_NCH, c = gch % ADPS_NCH;
        const long long blk = blockIdx.x + it * gridDim.x;
        const double* src = (const double*)s.adp_lu + (blk * 1296 + c * ADPS_CH) * (long long)ADP_ZB;
        mbar_expect_tx(&S.full[slot], ADPS_CH * ADP_ZB * sizeof(double));
        bulk_g2s(&S.stage[slot][0][0], src, ADPS_CH * ADP_ZB * sizeof(double), &S.full[slot]);
      }
    }
    return;
  }
  const int lane = tid & 31;
  long long gch = 0;  // next chunk to consume
  int within = ADPS_CH;
  const double* cur = nullptr;
  // next factor element of this thread's zone
  auto next = [&]() -> double {
    if (within == ADPS_CH) {
      if (gch > 0) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&S.empty[(int)((gch - 1) % ADPS_NS)]);
      }
      const int slot = (int)(gch % ADPS_NS);
      mbar_wait(&S.full[slot], (uint32_t)((gch / ADPS_NS) & 1), s.err_flag);
      cur = &S.stage[slot][0][tid];
      ++gch;
      within = 0;
    }
    return cur[(within++) * ADPS_TPB];
  };
  for (long long it = 0; it < my_iters; ++it) {
    const long long blk = blockIdx.x + it * gridDim.x;
    const long long t = blk * ADP_ZB + tid;
    const bool inr = t < n;
    const int8_t* pv = s.adp_piv + blk * 36 * ADP_ZB + tid;
    // permuted right-hand side first (36 independent loads), then the
    // substitution in place
#pragma unroll
    for (int a = 0; a < 36; ++a) S.y[a][tid] = inr ? ((const double*)s.adp_rhs)[(long long)pv[a * ADP_ZB] * n + t] : 0.0;
#pragma unroll 1
    for (int a = 1; a < 36; ++a) {
      double acc = S.y[a][tid];
#pragma unroll 4
      for (int b = 0; b < a; ++b) acc -= next() * S.y[b][tid];
      S.y[a][tid] = acc;
    }
#pragma unroll 1
    for (int a = 35; a >= 0; --a) {
      double acc = S.y[a][tid];
#pragma unroll 4
      for (int b = a + 1; b < 36; ++b) acc -= next() * S.y[b][tid];
      S.y[a][tid] = acc / next();
    }
    if (inr) {
      int p, i, j, k;
      r.decode(t, p, i, j, k);
      if (mask_at(g, d, p, i, j) == 1) {
#pragma unroll
        for (int a = 0; a < 30; ++a) Vat(s, d, 5 + a / 10, a % 10, p, i, j, k) = S.y[a][tid];
        R* U = s.U;
        const long long o5 = d.at(4, p, i, j, k);
        const double u6 = U[d.at(5, p, i, j, k)], u7 = U[d.at(6, p, i, j, k)], u8 = U[d.at(7, p, i, j, k)];
        const double aa = (u6 * u6 + u7 * u7 + u8 * u8) * ph.ob8pi;
        const double n6 = S.y[0][tid], n7 = S.y[10][tid], n8 = S.y[20][tid];
        U[d.at(5, p, i, j, k)] = n6;
        U[d.at(6, p, i, j, k)] = n7;
        U[d.at(7, p, i, j, k)] = n8;
        const double bb = (n6 * n6 + n7 * n7 + n8 * n8) * ph.ob8pi;
        U[o5] = U[o5] - aa + bb;
      }
    }
  }
  // release the last chunk (no producer waits for it; keeps the protocol uniform)
  __syncwarp();
  if (lane == 0 && gch > 0) mbar_arrive(&S.empty[(int)((gch - 1) % ADPS_NS)]);
}

// STEP 9.a (421:6700-6790): zone-centred E = -v x B from the point values.
template <typename R>
__global__ void k_efield_a(Dims d, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    R co[10];
    coef10(g, d, p, i, j, k, co);
    R pv[8];
    for (int q = 1; q < 8; ++q) {
      if (q == 4) continue;
      R acc = Vat(s, d, q, 0, p, i, j, k);
      for (int m = 4; m < 10; ++m) acc = acc - Vat(s, d, q, m, p, i, j, k) * co[m];
      pv[q] = acc;
    }
    const R vx = pv[1], vy = pv[2], vz = pv[3], Bx = pv[5], By = pv[6], Bz = pv[7];
    const R ex = -(vy * Bz - vz * By), ey = -(vz * Bx - vx * Bz), ez = -(vx * By - vy * Bx);
    s.E[d.at(0, p, i, j, k)] = ex;
    s.E[d.at(1, p, i, j, k)] = ey;
    s.E[d.at(2, p, i, j, k)] = ez;
    s.Esnap[d.at(0, p, i, j, k)] = ex;
    s.Esnap[d.at(1, p, i, j, k)] = ey;
    s.Esnap[d.at(2, p, i, j, k)] = ez;
  }
}

// STEP 9.b (421:6840-8400): linear WENO slopes of the E point values.
// Three blocks per SM (measured: faster than two at 255 registers, and than
// four).
// Row rr (0: the zone itself, 1..18: the STEP 7.b neighbours) of the
// 19 x 10 interpolation least-squares matrix of STEP 9.c (421:8464-8620).
template <typename R>
__device__ __forceinline__ void e9c_row(const Dims& d, const DGeom& g, int p, int i, int j, int k, const Nbr12& n,
                                        int rr, R cx, R cy, R cz, R obl0, const R* c0, R* A,
                                        long long& off) {
  if (rr == 0) {
    off = d.idx(i, j, k);
    A[0] = R(1.0);
    A[1] = R(0.0);
    A[2] = R(0.0);
    A[3] = R(0.0);
#pragma unroll
    for (int m = 4; m < 10; ++m) A[m] = R(0.0) * R(0.0) - c0[m];
    return;
  }
  const int w = c_n18[rr - 1][0], dz = c_n18[rr - 1][1];
  const int zx = w < 0 ? i : n.x[w], zy = w < 0 ? j : n.y[w], zz = k + dz;
  off = d.idx(zx, zy, zz);
  const R x = (geoR<R>(g, d, CS_G_V_CEN, 0, p, zx, zy, zz) - cx) * obl0;
  const R y = (geoR<R>(g, d, CS_G_V_CEN, 1, p, zx, zy, zz) - cy) * obl0;
  const R z = (geoR<R>(g, d, CS_G_V_CEN, 2, p, zx, zy, zz) - cz) * obl0;
  A[0] = R(1.0);
  A[1] = x;
  A[2] = y;
  A[3] = z;
  A[4] = x * x - c0[4];
  A[5] = y * y - c0[5];
  A[6] = z * z - c0[6];
  A[7] = x * y - c0[7];
  A[8] = y * z - c0[8];
  A[9] = x * z - c0[9];
}

template <typename R>
__device__ __forceinline__ void e9c_minv(const Dims& d, const DGeom& g, int p, int i, int j, int k, const Nbr12& n,
                                         R cx, R cy, R cz, R obl0, const R* c0, R* Minv) {
  R M[100];
#pragma unroll
  for (int t = 0; t < 100; ++t) M[t] = R(0.0);
  for (int rr = 0; rr < 19; ++rr) {
    R A[10];
    long long off;
    e9c_row(d, g, p, i, j, k, n, rr, cx, cy, cz, obl0, c0, A, off);
#pragma unroll
    for (int a = 0; a < 10; ++a)
#pragma unroll
      for (int b = a; b < 10; ++b) M[a * 10 + b] = M[a * 10 + b] + A[a] * A[b];
  }
#pragma unroll
  for (int a = 0; a < 10; ++a)
#pragma unroll
    for (int b = 0; b < a; ++b) M[a * 10 + b] = M[b * 10 + a];
  d_matinv<10>(M, Minv);
}

// STEP 9.c (421:8464-9350): 19-point interpolation least squares
// hybridised with the slopes; the point value is flattened toward E_pt.
// Only the point value (mode 1) is stored: the LLF edge solver consumes
// nothing else.  kCached: the inverse normal matrix comes from the
// operator cache.  Blocks per SM: 4 for FP64, 6 for FP32 (measured).
template <bool kCached, bool kShared, typename R>
__global__ void __launch_bounds__(TPB, sizeof(R) == 4 ? 6 : 4) k_efield_c(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  const R ob12 = R(1.0) / R(12.0), ob180 = R(1.0) / R(180.0), ob144 = R(1.0) / R(144.0);
  const LsqOrder<kShared> ord(r);
  for (long long it = ord.begin(); it < ord.nit; it += ord.stride()) {
    long long t, tw;
    if (!ord.zone(it, t, tw)) continue;
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const Nbr12 n = load_nbr(g, d, p, i, j);
    const R obl0 = R(1.0) / fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, p, i, j, k), R(ph.smallnum));
    R c0[10];
    coef10(g, d, p, i, j, k, c0);
    const R cx = geoR<R>(g, d, CS_G_V_CEN, 0, p, i, j, k), cy = geoR<R>(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 cz = geoR<R>(g, d, CS_G_V_CEN, 2, p, i, j, k);
    // kCached: the solution operator comes from the cache as the row weights
    // W_rr = Minv A_rr^T (geometry only), so X = sum_rr W_rr E_rr directly.
    R Minv[kCached ? 1 : 100];
    if (!kCached) {
      // formed in FP64 in every form, like the cached row weights
      double c0d[10], Md[100];
      coef10(g, d, p, i, j, k, c0d);
      e9c_minv<double>(d, g, p, i, j, k, n, geo(g, d, CS_G_V_CEN, 0, p, i, j, k), geo(g, d, CS_G_V_CEN, 1, p, i, j, k),
                       geo(g, d, CS_G_V_CEN, 2, p, i, j, k), 1.0 / fmax(geo(g, d, CS_G_V_SCALE, 0, p, i, j, k), ph.smallnum),
                       c0d, Md);
#pragma unroll
      for (int e = 0; e < 100; ++e) Minv[e] = (R)Md[e];
    }
    const R* wc = s.op_m10 + tw;
    auto MI = [&](int e) { return Minv[kCached ? 0 : e]; };
    R Y[3][10];
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int a = 0; a < 10; ++a) Y[q][a] = R(0.0);
#pragma unroll 1
    for (int rr = 0; rr < 19; ++rr) {
      R A[10];
      long long off;
      if (kCached) {
        if (rr == 0) {
          off = d.idx(i, j, k);
        } else {
          const int w = c_n18[rr - 1][0];
          off = d.idx(w < 0 ? i : n.x[w], w < 0 ? j : n.y[w], k + c_n18[rr - 1][1]);
        }
#pragma unroll
        for (int a = 0; a < 10; ++a) A[a] = __ldg(wc + (long long)(rr * 10 + a) * ord.nw);
      } else {
        e9c_row(d, g, p, i, j, k, n, rr, cx, cy, cz, obl0, c0, A, off);
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const R Rv = s.Esnap[((long long)q * NPANEL + p) * d.S + off];
#pragma unroll
        for (int a = 0; a < 10; ++a) Y[q][a] = Y[q][a] + A[a] * Rv;
      }
    }
    const R f = s.flatA[d.at(0, p, i, j, k)];
    const R betalo = f + (R(1.0) - f) * R(2.0);
    const R ghi = f * R(0.6) + (R(1.0) - f) * R(0.95), glo = R(1.0) - ghi, obghi = R(1.0) / ghi, grat = glo / ghi;
    const unsigned long long qsrc = kShared ? s.lsq_map10[p].src : LSQ_IDENTITY_SRC;
    const unsigned int qneg = kShared ? s.lsq_map10[p].neg : 0u;
#pragma unroll 1
    for (int q = 0; q < 3; ++q) {
      R X[10];
#pragma unroll
      for (int a = 0; a < 10; ++a) {
        if (kCached) {
          X[a] = kShared ? lsq_rotated<0>(Y[q], a, qsrc, qneg) : Y[q][a];
        } else {
          R acc = R(0.0);
#pragma unroll
          for (int b = 0; b < 10; ++b) acc = acc + MI(a * 10 + b) * Y[q][b];
          X[a] = acc;
        }
      }
      R e[4];
      e[0] = s.Esnap[((long long)q * NPANEL + p) * d.S + d.idx(i, j, k)];
#pragma unroll
      for (int m = 1; m < 4; ++m) e[m] = s.E[d.at(m * 3 + q, p, i, j, k)];
      const R ISlo = betalo * (e[1] * e[1] + e[2] * e[2] + e[3] * e[3]) * ob12;
      R Phi[10];
#pragma unroll
      for (int m = 0; m < 4; ++m) Phi[m] = X[m] * obghi - e[m] * grat;
#pragma unroll
      for (int m = 4; m < 10; ++m) Phi[m] = X[m] * obghi;
      const R IShi = (Phi[1] * Phi[1] + Phi[2] * Phi[2] + Phi[3] * Phi[3]) * ob12 +
                          (Phi[4] * Phi[4]) * (sqr(c0[4] - ob12) + ob180) + (Phi[5] * Phi[5]) * (sqr(c0[5] - ob12) + ob180) +
                          (Phi[6] * Phi[6]) * (sqr(c0[6] - ob12) + ob180) + (Phi[7] * Phi[7]) * (c0[7] * c0[7] + ob144) +
                          (Phi[8] * Phi[8]) * (c0[8] * c0[8] + ob144) + (Phi[9] * Phi[9]) * (c0[9] * c0[9] + ob144);
      const R tau = fabs(IShi - ISlo);
      R Wlo = glo * (R(1.0) + tau / (ISlo + R(ph.smallnum))), Whi = ghi * (R(1.0) + tau / (IShi + R(ph.smallnum)));
      const R aa = R(1.0) / (Wlo + Whi);
      Wlo = Wlo * aa;
      Whi = Whi * aa;
      const R x = R(1.0) - f;
      const R e0 = Whi * Phi[0] + Wlo * e[0];
      s.E[d.at(q, p, i, j, k)] = e[0] * f + e0 * x;
    }
  }
}

template <typename R>
__global__ void k_ops_m10(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  const long long nr_ = s.lsq_map10 ? r.count() / 6 : r.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nr_; t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const Nbr12 n = load_nbr(g, d, p, i, j);
    const double obl0 = 1.0 / fmax(geo(g, d, CS_G_V_SCALE, 0, p, i, j, k), ph.smallnum);
    double c0[10];
    coef10(g, d, p, i, j, k, c0);
    const double cx = geo(g, d, CS_G_V_CEN, 0, p, i, j, k), cy = geo(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 cz = geo(g, d, CS_G_V_CEN, 2, p, i, j, k);
    double Minv[100];
    e9c_minv(d, g, p, i, j, k, n, cx, cy, cz, obl0, c0, Minv);
    // W_rr = Minv A_rr^T for the 19 rows (the zone and its 18 neighbours)
    for (int rr = 0; rr < 19; ++rr) {
      double A[10];
      long long off;
      e9c_row(d, g, p, i, j, k, n, rr, cx, cy, cz, obl0, c0, A, off);
      for (int a = 0; a < 10; ++a) {
        double w = 0.0;
        for (int b = 0; b < 10; ++b) w = w + Minv[a * 10 + b] * A[b];
        s.op_m10[(long long)(rr * 10 + a) * nr_ + t] = (R)w;
      }
    }
  }
}

// ---------------------------------------------------------------------
// LIMIT_ALL_SLOPES_P2 (400riemann_integrate/420limit_all_slopes_p2.f,
// CS_FLAG_P2): STEP 7.a of the primitives (420:2459-5394) and STEP 9.b of E
// (420:8553-12285), the two steps where it differs from P12.
//
// Row rr (0..8) of one-sided stencil st around (i, j, k).  The stencils, in
// the reference's order (420:2596-4329): (R,U,+1), (L,U,+1), (L,D,+1),
// (R,D,+1), then the same with radial offset -1; with a the R / L
// neighbour, b the U / D neighbour and dz the radial direction, the rows are
// a, b, the zone at dz, aa, bb, the zone at 2 dz, the corner between a and
// b, a at dz, b at dz.  With rr a compile-time constant (unrolled loop)
// each neighbour is a select among registers, whatever st is.
__device__ __forceinline__ void p2_zone(const Nbr12& n, int st, int rr, int i, int j, int k, int& zx, int& zy,
                                        int& zz) {
  const int q = st & 3, dz = st < 4 ? 1 : -1;
  const bool R_ = q == 0 || q == 3, U_ = q < 2;
  zx = i;
  zy = j;
  zz = k;
  switch (rr) {
    case 0: case 7:  // a
      zx = R_ ? n.x[0] : n.x[1];
      zy = R_ ? n.y[0] : n.y[1];
      break;
    case 1: case 8:  // b
      zx = U_ ? n.x[2] : n.x[3];
      zy = U_ ? n.y[2] : n.y[3];
      break;
    case 3:  // aa
      zx = R_ ? n.x[4] : n.x[5];
      zy = R_ ? n.y[4] : n.y[5];
      break;
    case 4:  // bb
      zx = U_ ? n.x[6] : n.x[7];
      zy = U_ ? n.y[6] : n.y[7];
      break;
    case 6:  // corner RU, LU, LD, RD
      zx = q == 0 ? n.x[8] : (q == 1 ? n.x[9] : (q == 2 ? n.x[10] : n.x[11]));
      zy = q == 0 ? n.y[8] : (q == 1 ? n.y[9] : (q == 2 ? n.y[10] : n.y[11]));
      break;
    default: break;
  }
  if (rr == 2 || rr == 7 || rr == 8) zz = k + dz;
  if (rr == 5) zz = k + 2 * dz;
}

// The inverses of every zone's eight one-sided stencil matrices (geometry
// only), built once per mesh: STEP 7.a's 9 x 9 RECONSTRUCTION_COEFS systems
// (the modes x .. xz from the zone-average differences) into
// op_p2v[(st * 9 + m) * 9 + rr][zone] and STEP 9.b's 10 x 10
// INTERPOLATION_COEFS systems (the zone itself first, modes 1 .. xz from
// the point values) into op_p2e[(st * 10 + m) * 10 + rr][zone], inverted by
// MATINV's LU (121matinv.f:8).  Shared by the panels: panel 1's zones only.
template <typename R>
__global__ void k_ops_p2(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  const long long nr_ = s.p2_map ? r.count() / 6 : r.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nr_; t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const Nbr12 n = load_nbr(g, d, p, i, j);
    const double l0 = fmax(geo(g, d, CS_G_V_SCALE, 0, p, i, j, k), ph.smallnum), obl0 = 1.0 / l0;
    double c0[10];
    coef10(g, d, p, i, j, k, c0);
    const double cx = geo(g, d, CS_G_V_CEN, 0, p, i, j, k), cy = geo(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 cz = geo(g, d, CS_G_V_CEN, 2, p, i, j, k);
    for (int st = 0; st < 8; ++st) {
      double A[81], Ai[81], B[100], Bi[100];
      for (int m = 0; m < 10; ++m) B[m] = m == 0 ? 1.0 : (m < 4 ? 0.0 : 0.0 * 0.0 - c0[m]);
      for (int rr = 0; rr < 9; ++rr) {
        int zx, zy, zz;
        p2_zone(n, st, rr, i, j, k, zx, zy, zz);
        const double x = (geo(g, d, CS_G_V_CEN, 0, p, zx, zy, zz) - cx) * obl0;
        const double y = (geo(g, d, CS_G_V_CEN, 1, p, zx, zy, zz) - cy) * obl0;
        const double z = (geo(g, d, CS_G_V_CEN, 2, p, zx, zy, zz) - cz) * obl0;
        const double lj = fmax(geo(g, d, CS_G_V_SCALE, 0, p, zx, zy, zz), ph.smallnum);
        const double rt = lj / l0, r2 = rt * rt;
        const double sq[6] = {x * x, y * y, z * z, x * y, y * z, x * z};
        double* a = A + 9 * rr;
        a[0] = x;
        a[1] = y;
        a[2] = z;
        for (int m = 0; m < 6; ++m) a[3 + m] = sq[m] - c0[4 + m] + geo(g, d, CS_G_COEF, 4 + m, p, zx, zy, zz) * r2;
        double* e = B + 10 * (rr + 1);
        e[0] = 1.0;
        e[1] = x;
        e[2] = y;
        e[3] = z;
        for (int m = 0; m < 6; ++m) e[4 + m] = sq[m] - c0[4 + m];
      }
      d_matinv<9>(A, Ai);
      d_matinv<10>(B, Bi);
      for (int e = 0; e < 81; ++e) s.op_p2v[(long long)(st * 81 + e) * nr_ + t] = (R)Ai[e];
      for (int e = 0; e < 100; ++e) s.op_p2e[(long long)(st * 100 + e) * nr_ + t] = (R)Bi[e];
    }
  }
}

// STEP 7.a (kE false) / STEP 9.b (kE true) of LIMIT_ALL_SLOPES_P2.  A block
// takes 32 zones and all the variables (the 8 primitives / the 3 E
// components), a thread one zone and CPT variables: the nine stencils'
// modes (eight one-sided from the resident inverses, the central one from
// P12's resident row weights: STEP 7.b's 18-zone least squares, STEP 9.c's
// 19-zone one), their smoothness indicators over the zone's unit cube
// (420:5245-5257) and WENO weights 1 and 100 over (IS + smallnum)^4 (in
// FP64 in every form), then the weighted modes, summed stencil by stencil
// in the reference's order (the one-sided stencils' modes formed again
// rather than kept: 72 values a variable).  Each operator word is loaded
// once for the CPT variables of the thread (the sums are the same for any
// CPT).  STEP 7.a writes modes 2..10 damped by the flattener; STEP 9.b only
// the point value, flattened toward the unlimited one (the edge solver
// consumes nothing else).  With kShared the inverses are panel 1's, rotated
// per panel like the row weights, and iteration T covers tile T / 6 of
// panel T % 6 so that the six blocks reading one tile's inverses run
// together.
template <bool kE, bool kShared, int CPT, typename R>
__global__ void __launch_bounds__(32 * (kE ? 3 : 8) / CPT) k_p2(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  constexpr int NM = kE ? 10 : 9, NR = kE ? 10 : 9, M0 = kE ? 0 : 1, NO = kE ? 1 : 9;
  constexpr int n18[18][2] = {{0, 0},  {1, 0},  {2, 0},  {3, 0},  {-1, 1}, {-1, -1}, {8, 0}, {9, 0},  {10, 0},
                              {11, 0}, {0, 1},  {1, 1},  {0, -1}, {1, -1}, {2, 1},   {3, 1}, {2, -1}, {3, -1}};
  const int lane = threadIdx.x & 31, q0 = (threadIdx.x >> 5) * CPT;
  const long long nz = r.count(), npp = nz / 6, nw = kShared ? npp : nz;
  const long long ntile = kShared ? 6 * ((npp + 31) / 32) : (nz + 31) / 32;
  const long long cstr = (long long)NPANEL * d.S;  // stride between variables
  for (long long T = blockIdx.x; T < ntile; T += gridDim.x) {
    long long t, tw;
    if (kShared) {
      tw = (T / 6) * 32 + lane;
      t = (T % 6) * npp + tw;
      if (tw >= npp) continue;
    } else {
      t = tw = T * 32 + lane;
      if (t >= nz) continue;
    }
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const Nbr12 n = load_nbr(g, d, p, i, j);
    // smoothness weight of each mode x .. xz over the unit cube
    double wis[9];
    {
      const double ob12 = 1.0 / 12.0, ob180 = 1.0 / 180.0, ob144 = 1.0 / 144.0;
      wis[0] = wis[1] = wis[2] = ob12;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const double cm = geo(g, d, CS_G_COEF, 4 + m, p, i, j, k), cc = geo(g, d, CS_G_COEF, 7 + m, p, i, j, k);
        wis[3 + m] = (cm - ob12) * (cm - ob12) + ob180;
        wis[6 + m] = cc * cc + ob144;
      }
    }
    auto smooth = [&](const R* X) {  // X: modes x .. xz
      return ((double)X[0] * X[0] + (double)X[1] * X[1] + (double)X[2] * X[2]) * wis[0] +
             ((double)X[3] * X[3]) * wis[3] + ((double)X[4] * X[4]) * wis[4] + ((double)X[5] * X[5]) * wis[5] +
             ((double)X[6] * X[6]) * wis[6] + ((double)X[7] * X[7]) * wis[7] + ((double)X[8] * X[8]) * wis[8];
    };
    const R* fb = (kE ? s.Esnap : s.V) + ((long long)q0 * NPANEL + p) * d.S;
    const long long o0 = d.idx(i, j, k);
    R f0[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) f0[c] = fb[c * cstr + o0];
    const unsigned long long qsrc = kShared ? s.p2_map[p].src : LSQ_IDENTITY_SRC;
    const unsigned int qneg = kShared ? s.p2_map[p].neg : 0u;
    const R* op = (kE ? s.op_p2e : s.op_p2v) + tw;
    // The modes of one-sided stencil st for the thread's variables, group
    // by group -- the groups the panel rotations permute within (for E the
    // constant first, then x y z, the squares, the cross terms) -- rotated
    // to this panel and handed to visit(group, X[variable][0..2]); groups
    // g0 .. g1 - 1 only.  Three modes a variable are live at a time.
    constexpr int NG = kE ? 4 : 3;
    auto stencil = [&](int st, int g0, int g1, auto&& visit) {
      R Rv[CPT][NR];
#pragma unroll
      for (int rr = 0; rr < NR; ++rr) {
        int zx = i, zy = j, zz = k;
        if (!kE || rr > 0) p2_zone(n, st, rr - (kE ? 1 : 0), i, j, k, zx, zy, zz);
        const long long off = d.idx(zx, zy, zz);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const R v = fb[c * cstr + off];
          Rv[c][rr] = kE ? v : v - f0[c];
        }
      }
#pragma unroll
      for (int gi = 0; gi < NG; ++gi) {
        if (gi < g0 || gi >= g1) continue;
        const int mb = kE ? (gi == 0 ? 0 : 3 * gi - 2) : 3 * gi + 1;  // first mode of the group
        const int gs = (kE && gi == 0) ? 1 : 3;
        R Y[CPT][3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          if (q < gs) {
            R w[NR];
#pragma unroll
            for (int rr = 0; rr < NR; ++rr) w[rr] = __ldg(op + (long long)((st * NM + mb - M0 + q) * NR + rr) * nw);
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
              R acc = R(0.0);
#pragma unroll
              for (int rr = 0; rr < NR; ++rr) acc = acc + w[rr] * Rv[c][rr];
              Y[c][q] = acc;
            }
          }
        }
        R X[CPT][3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          if (q < gs) {
            const int mm = mb + q;
            const int mu = kShared ? (int)((qsrc >> (4 * mm)) & 15) - mb : q;
            const bool ng = kShared && ((qneg >> mm) & 1u);
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
              const R v = mu == 0 ? Y[c][0] : (mu == 1 ? Y[c][1] : Y[c][2]);
              X[c][q] = ng ? -v : v;
            }
          }
        }
        visit(gi, X);
      }
    };
    double IS[CPT][9];
    R X8[CPT][NM];
    {  // central stencil from the resident row weights
      R Y[CPT][NM];
#pragma unroll
      for (int c = 0; c < CPT; ++c)
#pragma unroll
        for (int m = 0; m < NM; ++m) Y[c][m] = R(0.0);
      const LsqPanelMap* cmap = kE ? s.lsq_map10 : s.lsq_map9;
      const long long tc = cmap ? t - (long long)p * npp : t, ncw = cmap ? npp : nz;
      const R* wc = (kE ? s.op_m10 : s.op_m9) + tc;
      const long long cstride = kE ? ncw : m9_stride(ncw);
#pragma unroll
      for (int rr = 0; rr < NR + 9; ++rr) {
        const int ro = kE ? rr - 1 : rr;  // E: the zone itself first
        const int w = ro < 0 ? -1 : n18[ro][0], dz = ro < 0 ? 0 : n18[ro][1];
        const long long off = d.idx(w < 0 ? i : n.x[w], w < 0 ? j : n.y[w], k + dz);
        R Rv[CPT];
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const R v = fb[c * cstr + off];
          Rv[c] = kE ? v : v - f0[c];
        }
#pragma unroll
        for (int m = 0; m < NM; ++m) {
          const R wv = __ldg(wc + (long long)(rr * NM + m) * cstride);
#pragma unroll
          for (int c = 0; c < CPT; ++c) Y[c][m] = Y[c][m] + wv * Rv[c];
        }
      }
      const unsigned long long csrc = cmap ? cmap[p].src : LSQ_IDENTITY_SRC;
      const unsigned int cneg = cmap ? cmap[p].neg : 0u;
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
#pragma unroll
        for (int m = 0; m < NM; ++m) X8[c][m] = cmap ? lsq_rotated<M0>(Y[c], m + M0, csrc, cneg) : Y[c][m];
        IS[c][8] = smooth(X8[c] + (kE ? 1 : 0));
      }
    }
#pragma unroll 1
    for (int st = 0; st < 8; ++st) {
      double sm[CPT];
      stencil(st, 0, NG, [&](int gi, R (*X)[3]) {
        const int gg = kE ? gi - 1 : gi;  // 0: x y z, 1: the squares, 2: the cross terms
        if (gg < 0) return;               // E's constant has no indicator term
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const double a0 = X[c][0], a1 = X[c][1], a2 = X[c][2];
          if (gg == 0)
            sm[c] = (a0 * a0 + a1 * a1 + a2 * a2) * wis[0];
          else
            sm[c] = sm[c] + (a0 * a0) * wis[3 * gg] + (a1 * a1) * wis[3 * gg + 1] + (a2 * a2) * wis[3 * gg + 2];
        }
      });
#pragma unroll
      for (int c = 0; c < CPT; ++c) IS[c][st] = sm[c];
    }
    double W[CPT][9];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
#pragma unroll
      for (int st = 0; st < 9; ++st) {
        const double tt = IS[c][st] + ph.smallnum, t2 = tt * tt;
        W[c][st] = (st < 8 ? 1.0 : 100.0) / (t2 * t2);
      }
      const double wn =
          1.0 / (W[c][0] + W[c][1] + W[c][2] + W[c][3] + W[c][4] + W[c][5] + W[c][6] + W[c][7] + W[c][8]);
#pragma unroll
      for (int st = 0; st < 9; ++st) W[c][st] = W[c][st] * wn;
    }
    double acc[CPT][NO];
#pragma unroll
    for (int c = 0; c < CPT; ++c)
#pragma unroll
      for (int m = 0; m < NO; ++m) acc[c][m] = 0.0;
#pragma unroll 1
    for (int st = 0; st < 8; ++st) {
      stencil(st, 0, kE ? 1 : NG, [&](int gi, R (*X)[3]) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          const double ws = W[c][st];
#pragma unroll
          for (int q = 0; q < (kE ? 1 : 3); ++q) {
            const int m = kE ? 0 : 3 * gi + q;
            acc[c][m] = st == 0 ? ws * (double)X[c][q] : acc[c][m] + ws * (double)X[c][q];
          }
        }
      });
    }
    const R fl = s.flatA[d.at(0, p, i, j, k)], x = R(1.0) - fl;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
#pragma unroll
      for (int m = 0; m < NO; ++m) acc[c][m] = acc[c][m] + W[c][8] * (double)X8[c][m];
      if (kE) {
        s.E[d.at(q0 + c, p, i, j, k)] = fl * f0[c] + x * (R)acc[c][0];
      } else {
#pragma unroll
        for (int m = 0; m < NO; ++m) Vat(s, d, q0 + c, 1 + m, p, i, j, k) = (R)acc[c][m] * x;
      }
    }
  }
}

inline Range3 zones_all(const Dims& d) { return {1 - d.G, d.N + d.G, 1 - d.G, d.N + d.G, 1 - d.G, d.nr + d.G}; }
inline Range3 shrink(const Dims& d, int s) {
  return {1 - d.G + s, d.N + d.G - s, 1 - d.G + s, d.N + d.G - s, 1 - d.G + s, d.nr + d.G - s};
}

}  // namespace

// STEP 8.d substitution with factors shared by the six panels.  The six
// panels of the cubed sphere are rotations of panel 1 by signed
// permutations R_p (vertex(p, i,j,k) = R_p vertex(1, i,j,k), checked when
// the mesh is uploaded), so the KKT matrix of zone (i,j,k) of panel p is
// T_p K_1 T_p^T, T_p being the signed permutation of the 30 B-mode
// unknowns that R_p induces (identity on the 6 multipliers).  Panel 1's
// factor stream then serves all six panels: r' = T_p^T r, y' = K_1^-1 r',
// y = T_p y'.  A CTA takes ADP6_ZB zone positions and all six panels (one
// consumer warp per panel, one zone per lane, y in registers); a producer
// warp streams the positions' factors (4 KB stages, in consumption order)
// through the ring, so each factor byte read from HBM serves six solves.
// adp_pmap[p][0][v] is the panel-p unknown u fed by panel-1 unknown v,
// adp_pmap[p][1][v] its sign.
constexpr int ADP6_CONS = 6 * 32;
constexpr int ADP6_THREADS = ADP6_CONS + 32;
constexpr int ADP6_CH = 16;
constexpr int ADP6_NS = 12;
constexpr int ADP6_NCH = 1296 / ADP6_CH;
template <typename F>
struct Adp6SmemT {
  F stage[ADP6_NS][ADP6_CH][ADP6_ZB];
  uint64_t full[ADP6_NS];
  uint64_t empty[ADP6_NS];
};

// Element e of the panel-shared factor stream (adp6_stream_pos order):
// row a, column b; b == a is a diagonal entry of the backward pass.
struct AdpElem {
  int a, b;
};
__host__ __device__ constexpr AdpElem adp_elem(int e) {
  if (e < 630) {
    int b = 0;
    while (e >= 35 - b) {
      e -= 35 - b;
      ++b;
    }
    return AdpElem{b + 1 + e, b};
  }
  int r = e - 630, a = 35;
  while (r >= 36 - a) {
    r -= 36 - a;
    --a;
  }
  return r < 35 - a ? AdpElem{a, a + 1 + r} : AdpElem{a, a};
}
static_assert(adp_elem(0).a == 1 && adp_elem(0).b == 0 && adp_elem(34).a == 35 && adp_elem(34).b == 0 &&
                  adp_elem(35).a == 2 && adp_elem(35).b == 1 && adp_elem(629).a == 35 && adp_elem(629).b == 34,
              "forward");
static_assert(adp6_stream_pos(35, 0) == 34 && adp6_stream_pos(2, 1) == 35 && adp6_stream_pos(35, 34) == 629 &&
                  adp6_stream_pos(35, 35) == 630 && adp6_stream_pos(0, 0) == 1295,
              "stream positions");
static_assert(adp_elem(630).a == 35 && adp_elem(630).b == 35 && adp_elem(631).a == 34 && adp_elem(631).b == 35 &&
                  adp_elem(632).b == 34 && adp_elem(1295).a == 0 && adp_elem(1295).b == 0,
              "backward");

// One stream element applied to y in registers (every index a compile-time
// constant): forward and backward eliminations y[a] -= f y[b], the
// diagonal y[a] /= f -- the substitution order of the reference.
template <int E, typename F>
__device__ __forceinline__ void adp6_apply(F (&y)[36], F f) {
  constexpr AdpElem x = adp_elem(E);
  if constexpr (x.a == x.b)
    y[x.a] = y[x.a] / f;
  else
    y[x.a] -= f * y[x.b];
}
template <int C, typename F, int... W>
__device__ __forceinline__ void adp6_chunk(F (&y)[36], const F* cur, std::integer_sequence<int, W...>) {
  (adp6_apply<C * ADP6_CH + W>(y, cur[W * ADP6_ZB]), ...);
}
// The whole stream of one zone block, chunk by chunk through the ring:
// release the previous stage, wait for this one, apply its 16 elements.
template <typename F, int... C>
__device__ __forceinline__ void adp6_substitute(F (&y)[36], Adp6SmemT<F>& S, int lane, long long& gch, int* err,
                                                std::integer_sequence<int, C...>) {
  auto acquire = [&]() -> const F* {
    if (gch > 0) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.empty[(int)((gch - 1) % ADP6_NS)]);
    }
    const int slot = (int)(gch % ADP6_NS);
    mbar_wait(&S.full[slot], (uint32_t)((gch / ADP6_NS) & 1), err);
    ++gch;
    return &S.stage[slot][0][lane];
  };
  (adp6_chunk<C>(y, acquire(), std::make_integer_sequence<int, ADP6_CH>{}), ...);
}

// The factor stream, the right-hand sides and the substitution are in the
// state's type R (FP32 in the precision form: half the stream's bytes).
template <typename R>
__global__ void __launch_bounds__(ADP6_THREADS, sizeof(R) == 4 ? 4 : 2) k_adp_solve6(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  extern __shared__ __align__(128) unsigned char adp6_raw[];
  Adp6SmemT<R>& S = *reinterpret_cast<Adp6SmemT<R>*>(adp6_raw);
  const int tid = threadIdx.x;
  const long long n = r.count(), n1 = n / 6;
  const long long nblk = (n1 + ADP6_ZB - 1) / ADP6_ZB;
  if ((long long)blockIdx.x >= nblk) return;
  const long long my_iters = (nblk - 1 - blockIdx.x) / gridDim.x + 1;
  const long long total_chunks = my_iters * ADP6_NCH;
  if (tid == 0) {
    for (int q = 0; q < ADP6_NS; ++q) {
      mbar_init(&S.full[q], 1);
      mbar_init(&S.empty[q], ADP6_CONS / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid >= ADP6_CONS) {
    if (tid == ADP6_CONS) {
      for (long long gch = 0; gch < total_chunks; ++gch) {
        const int slot = (int)(gch % ADP6_NS);
        if (gch >= ADP6_NS) mbar_wait(&S.empty[slot], (uint32_t)(((gch / ADP6_NS) - 1) & 1), s.err_flag);
        const long long it = gch / ADP6_NCH, c = gch % ADP6_NCH;
        const long long blk = blockIdx.x + it * gridDim.x;
        const R* src = (const R*)s.adp_lu + (blk * 1296 + c * ADP6_CH) * (long long)ADP6_ZB;
        mbar_expect_tx(&S.full[slot], ADP6_CH * ADP6_ZB * sizeof(R));
        bulk_g2s(&S.stage[slot][0][0], src, ADP6_CH * ADP6_ZB * sizeof(R), &S.full[slot]);
      }
    }
    return;
  }
  const int lane = tid & 31, p = tid >> 5;
  const int8_t* umap = s.adp_pmap + p * 72;
  const int8_t* smap = umap + 36;
  long long gch = 0;
  for (long long it = 0; it < my_iters; ++it) {
    const long long blk = blockIdx.x + it * gridDim.x;
    const long long t1 = blk * ADP6_ZB + lane, t = p * n1 + t1;
    const bool inr = t1 < n1;
    const int8_t* pv = s.adp_piv + blk * 36 * ADP6_ZB + lane;
    R y[36];
#pragma unroll
    for (int a = 0; a < 36; ++a) {
      const int v = inr ? pv[a * ADP6_ZB] : 0;
      const int u = __ldg(umap + v);
      y[a] = inr ? (R)__ldg(smap + v) * ((const R*)s.adp_rhs)[(long long)u * n + t] : R(0.0);
    }
    adp6_substitute(y, S, lane, gch, s.err_flag, std::make_integer_sequence<int, ADP6_NCH>{});
    if (inr) {
      int pp, i, j, k;
      r.decode(t, pp, i, j, k);
      if (mask_at(g, d, p, i, j) == 1) {
        double nb[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int v = 0; v < 30; ++v) {
          const int u = __ldg(umap + v);
          const double val = (double)__ldg(smap + v) * (double)y[v];
          Vat(s, d, 5 + u / 10, u % 10, p, i, j, k) = (R)val;
          if (v % 10 == 0) {
            if (u == 0) nb[0] = val;
            if (u == 10) nb[1] = val;
            if (u == 20) nb[2] = val;
          }
        }
        R* U = s.U;
        const long long o5 = d.at(4, p, i, j, k);
        const double u6 = U[d.at(5, p, i, j, k)], u7 = U[d.at(6, p, i, j, k)], u8 = U[d.at(7, p, i, j, k)];
        const double aa = (u6 * u6 + u7 * u7 + u8 * u8) * ph.ob8pi;
        U[d.at(5, p, i, j, k)] = nb[0];
        U[d.at(6, p, i, j, k)] = nb[1];
        U[d.at(7, p, i, j, k)] = nb[2];
        const double bb = (nb[0] * nb[0] + nb[1] * nb[1] + nb[2] * nb[2]) * ph.ob8pi;
        U[o5] = U[o5] - aa + bb;
      }
    }
  }
}

// STEP 10 (421:9354-9976): min and max over the active interior zones of
// the 8 primitives (zone values, B from the ADP solve) and of the zone's
// net face flux of B normalised by the larger of the two sides' |B| and the
// magnetosonic scale msonic sqrt(4 3.14 rho) (the reference's constant).
// Min and max do not depend on order: each warp reduces with shuffles and
// lane 0 folds its 18 values into keys[] by atomicMin / atomicMax on
// order-preserving integer keys of the doubles.
__device__ __forceinline__ unsigned long long minmax_key(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__global__ void k_step10_reset(unsigned long long* keys) {
  if (threadIdx.x < 18) keys[threadIdx.x] = threadIdx.x < 9 ? ~0ULL : 0ULL;
}
template <typename R>
__global__ void k_step10(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r, unsigned long long* keys) {
  double mn[9], mx[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    mn[q] = 1.0e30;
    mx[q] = -1.0e30;
  }
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      v[q] = (double)Vat(s, d, q, 0, p, i, j, k);
      mn[q] = fmin(mn[q], v[q]);
      mx[q] = fmax(mx[q], v[q]);
    }
    const double bxp = s.Bxf[d.at(0, p, i, j, k)], bxm = s.Bxf[d.at(0, p, i - 1, j, k)];
    const double byp = s.Byf[d.at(0, p, i, j, k)], bym = s.Byf[d.at(0, p, i, j - 1, k)];
    const double bzp = s.Bzf[d.at(0, p, i, j, k)], bzm = s.Bzf[d.at(0, p, i, j, k - 1)];
    const double a21 = geo(g, d, CS_G_XF_AREA, 0, p, i, j, k) * bxp + geo(g, d, CS_G_YF_AREA, 0, p, i, j, k) * byp +
                       geo(g, d, CS_G_ZF_AREA, 0, p, i, j, k) * bzp - geo(g, d, CS_G_XF_AREA, 0, p, i - 1, j, k) * bxm -
                       geo(g, d, CS_G_YF_AREA, 0, p, i, j - 1, k) * bym - geo(g, d, CS_G_ZF_AREA, 0, p, i, j, k - 1) * bzm;
    const double a11 = v[5] * v[5] + v[6] * v[6] + v[7] * v[7];
    const double ms = sqrt((ph.gamma * v[4] + ph.ob4pi * a11) / v[0]);
    const double den = fmax(fmax(sqrt(bxp * bxp + byp * byp + bzp * bzp), sqrt(bxm * bxm + bym * bym + bzm * bzm)),
                            ms * sqrt(4.0 * 3.14 * v[0]));
    const double dv = a21 / den;
    mn[8] = fmin(mn[8], dv);
    mx[8] = fmax(mx[8], dv);
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn[q] = fmin(mn[q], __shfl_xor_sync(0xffffffffu, mn[q], o));
      mx[q] = fmax(mx[q], __shfl_xor_sync(0xffffffffu, mx[q], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      atomicMin(keys + q, minmax_key(mn[q]));
      atomicMax(keys + 9 + q, minmax_key(mx[q]));
    }
  }
}

template <typename R>
void launch_step10_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 z = {1, d.N, 1, d.N, 1, d.nr};
  k_step10_reset<<<1, 32, 0, sv.stream>>>(sv.step10_keys);
  mark(sv, "k_step10_reset");
  k_step10<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, z, sv.step10_keys);
  mark(sv, "k_step10");
}

void launch_step10(Solve& sv) {
  if (!sv.step10_keys) return;
  if (sv.fp32)
    launch_step10_t(sv, sv.stF);
  else
    launch_step10_t(sv, sv.st);
}

template <typename R>
void launch_prim_and_masks_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 z = zones_all(d);
  k_prim<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, z);
  mark(sv, "k_prim");
  launch_face_masks(sv);
}

void launch_prim_and_masks(Solve& sv) {
  if (sv.fp32)
    launch_prim_and_masks_t(sv, sv.stF);
  else
    launch_prim_and_masks_t(sv, sv.st);
}

template <typename R>
void launch_face_masks_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 f = {-d.G, d.N + d.G, -d.G, d.N + d.G, -d.G, d.nr + d.G};
  k_zero_masked_faces<R><<<blocks_for(f.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, f);
  mark(sv, "k_zero_masked_faces");
  k_tricorner<R><<<blocks_for(6LL * 4 * d.G * (d.NK - 1), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st);
  mark(sv, "k_tricorner");
}

void launch_face_masks(Solve& sv) {
  if (sv.fp32)
    launch_face_masks_t(sv, sv.stF);
  else
    launch_face_masks_t(sv, sv.st);
}

template <typename R>
void launch_flattener_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 z = zones_all(d);
  const int nb = blocks_for(z.count(), TPB, grid_sms(sv));
  k_flat_a<R><<<nb, TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, z);
  mark(sv, "k_flat_a");
  k_flat_bc<R><<<nb, TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, z, st.flatA, st.flatB, 0);
  mark(sv, "k_flat_bc");
  k_flat_bc<R><<<nb, TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, z, st.flatB, st.flatA, 1);
  mark(sv, "k_flat_bc");
}

void launch_flattener(Solve& sv) {
  if (sv.fp32)
    launch_flattener_t(sv, sv.stF);
  else
    launch_flattener_t(sv, sv.st);
}

// Primitives a thread of STEP 7.a's k_p2 takes (each operator word loaded
// once for all of them; 1 / 2 / 4 measured 233 / 153 / 113 ms per shell128
// step).  STEP 9.b's takes the three E components.
constexpr int P2_CPT = 4;
// Grid of k_p2 over range b: 32-zone tiles (panel-interleaved when shared).
inline int p2_blocks(Solve& sv, const Range3& b, bool shared) {
  const long long npp = b.count() / 6;
  const long long nt = shared ? 6 * ((npp + 31) / 32) : (b.count() + 31) / 32;
  return (int)std::min<long long>(nt, (long long)grid_sms(sv) * 16);
}

template <typename R>
void launch_weno_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 a = shrink(d, 1), b = shrink(d, 2);
  if (sv.p.flags & CS_FLAG_P2) {  // LIMIT_ALL_SLOPES_P2's STEP 7.a
    const long long nt = (b.count() + W7A_ZT - 1) / W7A_ZT;
    const int nb = (int)std::min<long long>(nt, (long long)grid_sms(sv) * 16);
    k_weno_ao_split<false, R, true><<<nb, W7A_ZT * 3, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    mark(sv, "k_p2_entropy");
    if (st.p2_map)
      k_p2<false, true, P2_CPT, R><<<p2_blocks(sv, b, true), 256 / P2_CPT, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    else
      k_p2<false, false, P2_CPT, R><<<p2_blocks(sv, b, false), 256 / P2_CPT, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    mark(sv, "k_p2_prim");
    return;
  }
  {
    const long long nt = (a.count() + W7A_ZT - 1) / W7A_ZT;
    const int nb = (int)std::min<long long>(nt, (long long)grid_sms(sv) * 16);
    k_weno_ao_split<false, R><<<nb, W7A_ZT * 3, 0, sv.stream>>>(d, sv.ph, sv.g, st, a);
    mark(sv, "k_weno7a");
  }
  if (st.op_m9 && st.lsq_map9)
    k_weno7b<true, true, R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
  else if (st.op_m9)
    k_weno7b<true, false, R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
  else
    k_weno7b<false, false, R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
  mark(sv, "k_weno7b");
}

void launch_weno(Solve& sv) {
  if (sv.fp32)
    launch_weno_t(sv, sv.stF);
  else
    launch_weno_t(sv, sv.st);
}

template <typename R>
void launch_positivity_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 z = zones_all(d);
  k_positivity<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, z);
  mark(sv, "k_positivity");
  k_apply_giveup<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, st, z);
  mark(sv, "k_apply_giveup");
}

void launch_positivity(Solve& sv) {
  if (sv.fp32)
    launch_positivity_t(sv, sv.stF);
  else
    launch_positivity_t(sv, sv.st);
}

template <typename R>
void launch_faceB_adp_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  const int G = d.G, N = d.N, nr = d.nr;
  Range3 fx = {1 - G, N + G - 1, 2 - G, N + G - 1, 2 - G, nr + G - 1};
  Range3 fy = {2 - G, N + G - 1, 1 - G, N + G - 1, 2 - G, nr + G - 1};
  Range3 fz = {2 - G, N + G - 1, 2 - G, N + G - 1, 1 - G, nr + G - 1};
  k_faceB<R><<<blocks_for(fx.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, fx, 0);
  mark(sv, "k_faceB");
  k_faceB<R><<<blocks_for(fy.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, fy, 1);
  mark(sv, "k_faceB");
  k_faceB<R><<<blocks_for(fz.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, fz, 2);
  mark(sv, "k_faceB");
  Range3 a = shrink(d, 1);
  if (st.adp_lu && st.adp_pmap) {
    k_adp_rhs6<R><<<blocks_for(a.count() / 6, ADPR_TPB, grid_sms(sv)), ADPR_TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st,
                                                                                                  a);
    mark(sv, "k_adp_rhs6");
    const long long nblk = (a.count() / 6 + ADP6_ZB - 1) / ADP6_ZB;
    const int grid = (int)std::min<long long>(nblk, (long long)grid_sms(sv) * (sizeof(R) == 4 ? 4 : 2));
    k_adp_solve6<R><<<grid, ADP6_THREADS, sizeof(Adp6SmemT<R>), sv.stream>>>(d, sv.ph, sv.g, st, a);
    mark(sv, "k_adp_solve6");
    return;
  }
  if (st.adp_lu) {
    k_adp_rhs<R><<<blocks_for(a.count(), ADPR_TPB, grid_sms(sv)), ADPR_TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, a);
    mark(sv, "k_adp_rhs");
    const long long nblk = (a.count() + ADP_ZB - 1) / ADP_ZB;
    const int grid = (int)std::min<long long>(nblk, (long long)grid_sms(sv) * 2);
    k_adp_solve<R><<<grid, ADPS_THREADS, sizeof(AdpsSmem), sv.stream>>>(d, sv.ph, sv.g, st, a);
    mark(sv, "k_adp_solve");
    return;
  }
  const size_t smem = sizeof(AdpSmem) * ADP_WARPS;
  long long nwarps = a.count();
  long long nblk = (nwarps + ADP_WARPS - 1) / ADP_WARPS;
  long long cap = (long long)grid_sms(sv) * 16;
  if (nblk > cap) nblk = cap;
  k_adp<false, R><<<(int)nblk, 32 * ADP_WARPS, smem, sv.stream>>>(d, sv.ph, sv.g, st, a, a.count(), ADP_ZB);
  mark(sv, "k_adp");
}

void launch_faceB_adp(Solve& sv) {
  if (sv.fp32)
    launch_faceB_adp_t(sv, sv.stF);
  else
    launch_faceB_adp_t(sv, sv.st);
}

long long adp_range_count(const Dims& d) { return shrink(d, 1).count(); }
long long lsq_range_count(const Dims& d) { return shrink(d, 2).count(); }

template <typename R>
void launch_ops_build_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 b = shrink(d, 2);
  if (st.op_m9) {
    k_ops_m9<R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    mark(sv, "k_ops_m9");
  }
  if (st.op_m10) {
    k_ops_m10<R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    mark(sv, "k_ops_m10");
  }
  if (st.op_p2v) {
    k_ops_p2<R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    mark(sv, "k_ops_p2");
  }
}

void launch_ops_build(Solve& sv) {
  if (sv.fp32)
    launch_ops_build_t(sv, sv.stF);
  else
    launch_ops_build_t(sv, sv.st);
}

long long adp_factor_doubles(const Dims& d, bool shared) {
  if (shared) return (shrink(d, 1).count() / 6 + ADP6_ZB - 1) / ADP6_ZB * (long long)ADP6_ZB * 1296;
  return (shrink(d, 1).count() + ADP_ZB - 1) / ADP_ZB * (long long)ADP_ZB * 1296;
}

void set_adp_smem_limits() {
  const int smem = (int)(sizeof(AdpSmem) * ADP_WARPS);
  cudaFuncSetAttribute(k_adp_solve<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(AdpsSmem));
  cudaFuncSetAttribute(k_adp_solve<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(AdpsSmem));
  cudaFuncSetAttribute(k_adp_solve6<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(Adp6SmemT<double>));
  cudaFuncSetAttribute(k_adp_solve6<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Adp6SmemT<float>));
  cudaFuncSetAttribute(k_adp<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(k_adp<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(k_adp<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(k_adp<true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <typename R>
void launch_adp_factor_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 a = shrink(d, 1);
  const size_t smem = sizeof(AdpSmem) * ADP_WARPS;
  // shared factors: panel 1's zones only, in blocks of ADP6_ZB
  const long long tmax = st.adp_pmap ? a.count() / 6 : a.count();
  long long nblk = (tmax + ADP_WARPS - 1) / ADP_WARPS;
  long long cap = (long long)grid_sms(sv) * 16;
  if (nblk > cap) nblk = cap;
  k_adp<true, R><<<(int)nblk, 32 * ADP_WARPS, smem, sv.stream>>>(d, sv.ph, sv.g, st, a, tmax,
                                                                 st.adp_pmap ? ADP6_ZB : ADP_ZB);
  mark(sv, "k_adp_factor");
}

void launch_adp_factor(Solve& sv) {
  if (sv.fp32)
    launch_adp_factor_t(sv, sv.stF);
  else
    launch_adp_factor_t(sv, sv.st);
}

template <typename R>
void launch_efield_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  Range3 z = zones_all(d), a = shrink(d, 1), b = shrink(d, 2);
  k_efield_a<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, z);
  mark(sv, "k_efield_a");
  if (sv.p.flags & CS_FLAG_P2) {  // LIMIT_ALL_SLOPES_P2's STEP 9.b
    if (st.p2_map)
      k_p2<true, true, 3, R><<<p2_blocks(sv, b, true), 32, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    else
      k_p2<true, false, 3, R><<<p2_blocks(sv, b, false), 32, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    mark(sv, "k_p2_efield");
    return;
  }
  {
    const long long nt = (a.count() + W7A_ZT - 1) / W7A_ZT;
    const int nb = (int)std::min<long long>(nt, (long long)grid_sms(sv) * 16);
    k_weno_ao_split<true, R><<<nb, W7A_ZT * 3, 0, sv.stream>>>(d, sv.ph, sv.g, st, a);
    mark(sv, "k_efield_b");
  }
  if (st.op_m10)
    if (st.lsq_map10)
      k_efield_c<true, true, R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
    else
      k_efield_c<true, false, R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
  else
    k_efield_c<false, false, R><<<blocks_for(b.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, b);
  mark(sv, "k_efield_c");
}

void launch_efield(Solve& sv) {
  if (sv.fp32)
    launch_efield_t(sv, sv.stF);
  else
    launch_efield_t(sv, sv.st);
}

}  // namespace cs
