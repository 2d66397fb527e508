// ORACLE -- test infrastructure only (see oracle_core.h for the status
// note).  CPU restatement of the CubeSphere per-stage volume update on the
// six panels of one solve, operating on the same panel-box arrays as the
// library's C ABI.  Exposed to Python through a small extern "C" API.
//
// Each routine below cites the reference routine and the lines it follows.
// Loop extents written in the reference for NGhost = 4 (e.g. "-2, n+3") are
// expressed relative to the ghost depth G ("2-G, n+G-1") so that G = 4
// reproduces them and G = 3 shrinks every stencil range by one layer.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <tuple>
#include <vector>

#include "oracle_core.h"
// The host mesh builder and seeded initial state (a restatement of the
// reference's mesh chain, 201-253, and of 820init_patch_cube_sphere.f, pinned
// by the golden _T/_200mesh/test_quadpoints.out) are compiled into this
// library from their own sources, so a CPU solve needs no other library.
#include "cs_internal.h"

namespace oracle {

enum GF {  // geometry field order of the library's cs_geom_field
  G_VERT = 0, XF_QP, XF_QW, XF_N, XF_AREA, XF_CEN, YF_QP, YF_QW, YF_N, YF_AREA, YF_CEN,
  ZF_QP, ZF_QW, ZF_N, ZF_AREA, ZF_CEN, XB_QW, YB_QW, ZB_QW, V_SCALE, V_VOL, V_CEN, COEF, NGF
};
static const int kNcomp[NGF] = {3, 15, 5, 3, 1, 3, 15, 5, 3, 1, 3, 15, 5, 15, 1, 3, 5, 5, 5, 1, 1, 3, 10};
static const int kNbr[6][4] = {{3, 6, 2, 5}, {1, 4, 3, 6}, {2, 5, 1, 4}, {5, 2, 6, 3}, {6, 3, 4, 1}, {4, 1, 5, 2}};

struct Params {
  int32_t ntp, nr, nghost, radial_mesh;
  double rmin, rmax, radial_ratio, gamma, rhofloor, prsfloor, smallnum, cfl_coef, flatten_coef, prs_flatten_coef, gm;
  int32_t bc_lower, bc_upper, rk_scheme, flags;
};

struct Ctx {
  Params p;
  Phys ph;
  int N, nr, G, NI, NJ, NK;
  size_t S;
  std::vector<double> g[NGF];
  std::vector<int32_t> mask, st;  // mask [6][S]; stencil [6][12][2][NJ][NI]
  // state and work arrays, [comp][6][S]
  std::vector<double> U, ent, Bxf, Byf, Bzf, V, E, msonic, divvel, flat, work, Bqx, Bqy, Bqz, dUdt, SLx, SRx, SDy,
      SUy, SBz, STz, EFx, EFy, EFz, Efx, Efy, Efz, U0, ent0, Bxf0, Byf0, Bzf0;
  // STEP 7.c record per zone: 2 x shrink passes + 1 where the zone gave up
  std::vector<double> pos;
  // STEP 10 per panel: min and max of the 8 primitives and the divergence
  double vmin[6][NV + 1], vmax[6][NV + 1];
  bool step10 = false;
  // IMEX: the first stage's dU/dt, entropy fluxes and EMFs
  std::vector<double> K1, EFx1, EFy1, EFz1, Efx1, Efy1, Efz1;
  double time = 0.0;
  // per-face, per-point flux contributions to the two zones the face
  // updates ([dir]: [point*8 + comp][6][S]) and their target zones
  std::vector<double> cL[3], cR[3];
  std::vector<long long> tL[3], tR[3];
  // panel-edge ownership maps (built on first use)
  struct FaceSync { int dir, pn, i, j, k, odir, opn, oi, oj, ok; };
  struct EdgeSync { int f, pn, i, j, k, of, opn, oi, oj, ok, sign; };
  bool maps_built = false;
  std::vector<FaceSync> fsync;
  std::vector<EdgeSync> esync;
  std::vector<size_t> eclass;  // esync index where each edge's copies start, then esync.size()
  // which value the copies of a shared face or edge take: 0 the
  // lowest-numbered panel's (the library's default), 1 their average (the
  // reference's defect correction; CS_FLAG_PANEL_AVERAGE)
  int panel_rule = 0;

  size_t idx(int i, int j, int k) const { return ((size_t)(k + G) * NJ + (size_t)(j + G)) * NI + (size_t)(i + G); }
  double& a(std::vector<double>& v, int c, int pn, int i, int j, int k) { return v[((size_t)c * 6 + pn) * S + idx(i, j, k)]; }
  double geo(int f, int c, int pn, int i, int j, int k) const { return g[f][((size_t)c * 6 + pn) * S + idx(i, j, k)]; }
  double& geow(int f, int c, int pn, int i, int j, int k) { return g[f][((size_t)c * 6 + pn) * S + idx(i, j, k)]; }
  int m(int pn, int i, int j) const { return mask[(size_t)pn * S + idx(i, j, 0)]; }
  int sti(int pn, int i, int j, int w, int c) const {  // istencil(i, j, c+1, w+1)
    return st[(((size_t)pn * 12 + w) * 2 + c) * ((size_t)NI * NJ) + (size_t)(j + G) * NI + (i + G)];
  }
};

// Zone loops run on all host threads.  Every loop marked OMP_ZONES writes
// only the zone, face or edge of its own iteration and reads values that
// no iteration of the same loop writes, so its results do not depend on
// the thread count or schedule (bit-identical to a serial run).
#define OMP_ZONES _Pragma("omp parallel for collapse(2) schedule(static)")

static inline double sq(double x) { return x * x; }
static inline double pow4(double x) {
  double t = x * x;
  return t * t;
}

// Taylor-basis polynomial value at scaled offset (x,y,z): modes 1..10 of
// the reference's P12 reconstruction with moment coefficients c[0..9].
static inline double poly10(const double* v, const double* c, double x, double y, double z) {
  return v[0] + v[1] * x + v[2] * y + v[3] * z + v[4] * (x * x - c[4]) + v[5] * (y * y - c[5]) +
         v[6] * (z * z - c[6]) + v[7] * (x * y - c[7]) + v[8] * (y * z - c[8]) + v[9] * (x * z - c[9]);
}

void pad_radial(Ctx& c, int pn);

// ------------------------------------------------------------------
// Ghost fill across panel edges plus the radial outflow padding.
// Follows FETCH_BUFFERS_FILL_IN_UX / _UY / _UY_TOP
// (pkg/inc/cubesphere/300riemann_module/330fetch_buffers_fill_in_ux.f:220-714,
//  331fetch_buffers_fill_in_uy.f, 332fetch_buffers_fill_in_uy_top.f) with the
// index transforms of FILL_GHOST2D_GLOBAL (200mesh/203fill_ghost2d_global.f:104-163):
// every value is read from the neighbour's pre-exchange arrays, face-normal
// B changes sign where the two panels' normals are opposite, and the
// coinciding panel-edge faces are averaged.  PAD_BOUNDARY_R
// (800applications_cs/826pad_boundary_r.f:190-420, outflow code 2).
void fill_ghosts(Ctx& c) {
  const int N = c.N, G = c.G, nr = c.nr;
  std::vector<double> U = c.U, ent = c.ent, Bx = c.Bxf, By = c.Byf, Bz = c.Bzf;  // snapshot
  auto src = [&](std::vector<double>& v, int comp, int pn, int i, int j, int k) -> double {
    return v[((size_t)comp * 6 + pn) * c.S + c.idx(i, j, k)];
  };
  auto xmask = [&](int pn, int i, int j) {
    return c.m(pn, std::max(i, 1 - G), j) * c.m(pn, std::min(i + 1, N + G), j);
  };
  auto ymask = [&](int pn, int i, int j) {
    return c.m(pn, i, std::max(j, 1 - G)) * c.m(pn, i, std::min(j + 1, N + G));
  };
  for (int pn = 0; pn < 6; ++pn) {
    const int rt = kNbr[pn][0] - 1, lf = kNbr[pn][1] - 1;
    auto inner = [&](int j, int k) { return j >= 1 && j <= N && k >= 1 && k <= nr; };
    // ---- x direction: right strip
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = N + 1; i <= N + G; ++i) {
          for (int q = 0; q < NV; ++q) c.a(c.U, q, pn, i, j, k) = src(U, q, rt, j, 2 * N + 1 - i, k);
          c.a(c.ent, 0, pn, i, j, k) = src(ent, 0, rt, j, 2 * N + 1 - i, k);
        }
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = N; i <= N + G; ++i) {
          if (xmask(pn, i, j) != 1) continue;
          double v = -src(By, 0, rt, j, 2 * N - i, k);
          double& d = c.a(c.Bxf, 0, pn, i, j, k);
          d = (i == N && inner(j, k)) ? (d + v) * 0.5 : v;
        }
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = -G; j <= N + G; ++j)
        for (int i = N + 1; i <= N + G; ++i) c.a(c.Byf, 0, pn, i, j, k) = src(Bx, 0, rt, j, 2 * N + 1 - i, k);
    OMP_ZONES
    for (int k = -G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = N + 1; i <= N + G; ++i) c.a(c.Bzf, 0, pn, i, j, k) = src(Bz, 0, rt, j, 2 * N + 1 - i, k);
    // ---- x direction: left strip
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= 0; ++i) {
          for (int q = 0; q < NV; ++q) c.a(c.U, q, pn, i, j, k) = src(U, q, lf, 1 - i, N + 1 - j, k);
          c.a(c.ent, 0, pn, i, j, k) = src(ent, 0, lf, 1 - i, N + 1 - j, k);
        }
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = -G; i <= 0; ++i) {
          if (xmask(pn, i, j) != 1) continue;
          double v = -src(Bx, 0, lf, -i, N + 1 - j, k);
          double& d = c.a(c.Bxf, 0, pn, i, j, k);
          d = (i == 0 && inner(j, k)) ? (d + v) * 0.5 : v;
        }
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = -G; j <= N + G; ++j)
        for (int i = 1 - G; i <= 0; ++i) c.a(c.Byf, 0, pn, i, j, k) = -src(By, 0, lf, 1 - i, N - j, k);
    OMP_ZONES
    for (int k = -G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= 0; ++i) c.a(c.Bzf, 0, pn, i, j, k) = src(Bz, 0, lf, 1 - i, N + 1 - j, k);
  }
  for (int pn = 0; pn < 6; ++pn) {
    const int up = kNbr[pn][2] - 1, dn = kNbr[pn][3] - 1;
    auto inner = [&](int i, int k) { return i >= 1 && i <= N && k >= 1 && k <= nr; };
    // ---- y direction: down strip
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= 0; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          for (int q = 0; q < NV; ++q) c.a(c.U, q, pn, i, j, k) = src(U, q, dn, N + 1 - i, 1 - j, k);
          c.a(c.ent, 0, pn, i, j, k) = src(ent, 0, dn, N + 1 - i, 1 - j, k);
        }
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = -G; j <= 0; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          if (ymask(pn, i, j) != 1) continue;
          double v = -src(By, 0, dn, N + 1 - i, -j, k);
          double& d = c.a(c.Byf, 0, pn, i, j, k);
          d = (j == 0 && inner(i, k)) ? (d + v) * 0.5 : v;
        }
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= 0; ++j)
        for (int i = -G; i <= N + G; ++i) c.a(c.Bxf, 0, pn, i, j, k) = -src(Bx, 0, dn, N - i, 1 - j, k);
    OMP_ZONES
    for (int k = -G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= 0; ++j)
        for (int i = 1 - G; i <= N + G; ++i) c.a(c.Bzf, 0, pn, i, j, k) = src(Bz, 0, dn, N + 1 - i, 1 - j, k);
    // ---- y direction: up strip
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = N + 1; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          for (int q = 0; q < NV; ++q) c.a(c.U, q, pn, i, j, k) = src(U, q, up, 2 * N + 1 - j, i, k);
          c.a(c.ent, 0, pn, i, j, k) = src(ent, 0, up, 2 * N + 1 - j, i, k);
        }
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = N; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          if (ymask(pn, i, j) != 1) continue;
          double v = -src(Bx, 0, up, 2 * N - j, i, k);
          double& d = c.a(c.Byf, 0, pn, i, j, k);
          d = (j == N && inner(i, k)) ? (d + v) * 0.5 : v;
        }
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = N + 1; j <= N + G; ++j)
        for (int i = -G; i <= N + G; ++i) c.a(c.Bxf, 0, pn, i, j, k) = src(By, 0, up, 2 * N + 1 - j, i, k);
    OMP_ZONES
    for (int k = -G; k <= nr + G; ++k)
      for (int j = N + 1; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) c.a(c.Bzf, 0, pn, i, j, k) = src(Bz, 0, up, 2 * N + 1 - j, i, k);
  }
  for (int pn = 0; pn < 6; ++pn) pad_radial(c, pn);
}

// PAD_BOUNDARY_R of one panel (826pad_boundary_r.f:190-420, outflow code 2):
// the radial ghost layers of the active columns from the first / last zone.
void pad_radial(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  for (int kk = 1; kk <= G; ++kk)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        if (c.p.bc_lower == 2) {
          int l = 1 - kk, r = 1;
          for (int q = 0; q < NV; ++q) c.a(c.U, q, pn, i, j, l) = c.a(c.U, q, pn, i, j, r);
          c.a(c.Bxf, 0, pn, i, j, l) = c.a(c.Bxf, 0, pn, i, j, r);
          c.a(c.Bxf, 0, pn, i - 1, j, l) = c.a(c.Bxf, 0, pn, i - 1, j, r);
          c.a(c.Byf, 0, pn, i, j, l) = c.a(c.Byf, 0, pn, i, j, r);
          c.a(c.Byf, 0, pn, i, j - 1, l) = c.a(c.Byf, 0, pn, i, j - 1, r);
          c.a(c.Bzf, 0, pn, i, j, l - 1) = c.a(c.Bzf, 0, pn, i, j, r - 1);
        }
      }
  for (int kk = 1; kk <= G; ++kk)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        if (c.p.bc_upper == 2) {
          int l = nr + kk, r = nr;
          for (int q = 0; q < NV; ++q)
            c.a(c.U, q, pn, i, j, l) =
                c.a(c.U, q, pn, i, j, r) * c.geo(V_VOL, 0, pn, i, j, r) / c.geo(V_VOL, 0, pn, i, j, l);
          c.a(c.Bzf, 0, pn, i, j, l) =
              c.a(c.Bzf, 0, pn, i, j, r) * c.geo(ZF_AREA, 0, pn, i, j, r) / c.geo(ZF_AREA, 0, pn, i, j, l);
          c.a(c.Bxf, 0, pn, i, j, l) =
              c.a(c.Bxf, 0, pn, i, j, r) * c.geo(XF_AREA, 0, pn, i, j, r) / c.geo(XF_AREA, 0, pn, i, j, l);
          c.a(c.Byf, 0, pn, i, j, l) =
              c.a(c.Byf, 0, pn, i, j, r) * c.geo(YF_AREA, 0, pn, i, j, r) / c.geo(YF_AREA, 0, pn, i, j, l);
          c.a(c.Bxf, 0, pn, i - 1, j, l) = c.a(c.Bxf, 0, pn, i - 1, j, r) * c.geo(XF_AREA, 0, pn, i - 1, j, r) /
                                            c.geo(XF_AREA, 0, pn, i - 1, j, l);
          c.a(c.Byf, 0, pn, i, j - 1, l) = c.a(c.Byf, 0, pn, i, j - 1, r) * c.geo(YF_AREA, 0, pn, i, j - 1, r) /
                                            c.geo(YF_AREA, 0, pn, i, j - 1, l);
        }
      }
}

// Tri-corner face-B synchronisation at the four panel corners
// (421limit_all_slopes_p12.f:779-962, repeated in 485cleanup_after_update.f:504-687).
static void tricorner_sync(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  for (int i = 1 - G; i <= 0; ++i) {  // LD
    int xd = c.sti(pn, i, 1, 3, 0), yd = c.sti(pn, i, 1, 3, 1);
    for (int k = 1 - G; k <= nr + G; ++k) {
      double a11 = 0.5 * (c.a(c.Byf, 0, pn, i, 0, k) - c.a(c.Bxf, 0, pn, xd - 1, yd, k));
      c.a(c.Byf, 0, pn, i, 0, k) = a11;
      c.a(c.Bxf, 0, pn, xd - 1, yd, k) = -a11;
    }
  }
  for (int i = N + 1; i <= N + G; ++i) {  // RD
    int xd = c.sti(pn, i, 1, 3, 0), yd = c.sti(pn, i, 1, 3, 1);
    for (int k = 1 - G; k <= nr + G; ++k) {
      double a11 = 0.5 * (c.a(c.Byf, 0, pn, i, 0, k) + c.a(c.Bxf, 0, pn, xd, yd, k));
      c.a(c.Byf, 0, pn, i, 0, k) = a11;
      c.a(c.Bxf, 0, pn, xd, yd, k) = a11;
    }
  }
  for (int i = N + 1; i <= N + G; ++i) {  // RU
    int xu = c.sti(pn, i, N, 2, 0), yu = c.sti(pn, i, N, 2, 1);
    for (int k = 1 - G; k <= nr + G; ++k) {
      double a11 = 0.5 * (c.a(c.Byf, 0, pn, i, N, k) - c.a(c.Bxf, 0, pn, xu, yu, k));
      c.a(c.Byf, 0, pn, i, N, k) = a11;
      c.a(c.Bxf, 0, pn, xu, yu, k) = -a11;
    }
  }
  for (int i = 1 - G; i <= 0; ++i) {  // LU
    int xu = c.sti(pn, i, N, 2, 0), yu = c.sti(pn, i, N, 2, 1);
    for (int k = 1 - G; k <= nr + G; ++k) {
      double a11 = 0.5 * (c.a(c.Byf, 0, pn, i, N, k) + c.a(c.Bxf, 0, pn, xu - 1, yu, k));
      c.a(c.Byf, 0, pn, i, N, k) = a11;
      c.a(c.Bxf, 0, pn, xu - 1, yu, k) = a11;
    }
  }
}

static void zero_masked_faces(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = -G; i <= N + G; ++i)
        if (c.m(pn, std::max(i, 1 - G), j) == 0 && c.m(pn, std::min(i + 1, N + G), j) == 0)
          c.a(c.Bxf, 0, pn, i, j, k) = 0.0;
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = -G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i)
        if (c.m(pn, i, std::max(j, 1 - G)) == 0 && c.m(pn, i, std::min(j + 1, N + G)) == 0)
          c.a(c.Byf, 0, pn, i, j, k) = 0.0;
  OMP_ZONES
  for (int k = -G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i)
        if (c.m(pn, i, j) == 0) c.a(c.Bzf, 0, pn, i, j, k) = 0.0;
}

// Neighbour zone w (0..11 = R,L,U,D,RR,LL,UU,DD,RU,LU,LD,RD) of (i,j).
struct Nb {
  int x[12], y[12];
};
static inline Nb nbrs(const Ctx& c, int pn, int i, int j) {
  Nb n;
  for (int w = 0; w < 12; ++w) {
    n.x[w] = c.sti(pn, i, j, w, 0);
    n.y[w] = c.sti(pn, i, j, w, 1);
  }
  return n;
}

// The eight one-sided 3-zone stencils of STEP 7.a, as (neighbour in plane
// 1, neighbour in plane 2, radial offset): (R,U,+1),(R,U,-1),(L,U,+1),
// (L,U,-1),(R,D,+1),(R,D,-1),(L,D,+1),(L,D,-1).
static const int kSt8[8][3] = {{0, 2, 1}, {0, 2, -1}, {1, 2, 1}, {1, 2, -1}, {0, 3, 1}, {0, 3, -1}, {1, 3, 1}, {1, 3, -1}};

// 3x3 inverses of the eight stencils (421limit_all_slopes_p12.f:2561-3110).
static void stencil_inverses(Ctx& c, int pn, int i, int j, int k, const Nb& n, double Ai[8][3][3]) {
  double obl0 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, i, j, k), c.p.smallnum);
  double cx = c.geo(V_CEN, 0, pn, i, j, k), cy = c.geo(V_CEN, 1, pn, i, j, k), cz = c.geo(V_CEN, 2, pn, i, j, k);
  for (int s = 0; s < 8; ++s) {
    int w1 = kSt8[s][0], w2 = kSt8[s][1], dz = kSt8[s][2];
    double a11 = (c.geo(V_CEN, 0, pn, n.x[w1], n.y[w1], k) - cx) * obl0;
    double a12 = (c.geo(V_CEN, 1, pn, n.x[w1], n.y[w1], k) - cy) * obl0;
    double a13 = (c.geo(V_CEN, 2, pn, n.x[w1], n.y[w1], k) - cz) * obl0;
    double a21 = (c.geo(V_CEN, 0, pn, n.x[w2], n.y[w2], k) - cx) * obl0;
    double a22 = (c.geo(V_CEN, 1, pn, n.x[w2], n.y[w2], k) - cy) * obl0;
    double a23 = (c.geo(V_CEN, 2, pn, n.x[w2], n.y[w2], k) - cz) * obl0;
    double a31 = (c.geo(V_CEN, 0, pn, i, j, k + dz) - cx) * obl0;
    double a32 = (c.geo(V_CEN, 1, pn, i, j, k + dz) - cy) * obl0;
    double a33 = (c.geo(V_CEN, 2, pn, i, j, k + dz) - cz) * obl0;
    double ob = (-a13 * a22 * a31 + a12 * a23 * a31 + a13 * a21 * a32 - a11 * a23 * a32 - a12 * a21 * a33 +
                 a11 * a22 * a33);
    ob = std::copysign(1.0, ob) / std::max(1.0e-32, std::fabs(ob));
    Ai[s][0][0] = (-a23 * a32 + a22 * a33) * ob;
    Ai[s][0][1] = (a13 * a32 - a12 * a33) * ob;
    Ai[s][0][2] = (-a13 * a22 + a12 * a23) * ob;
    Ai[s][1][0] = (a23 * a31 - a21 * a33) * ob;
    Ai[s][1][1] = (-a13 * a31 + a11 * a33) * ob;
    Ai[s][1][2] = (a13 * a21 - a11 * a23) * ob;
    Ai[s][2][0] = (-a22 * a31 + a21 * a32) * ob;
    Ai[s][2][1] = (a12 * a31 - a11 * a32) * ob;
    Ai[s][2][2] = (-a12 * a21 + a11 * a22) * ob;
  }
}

// WENO combination of the eight stencil gradients plus their mean with
// central weight 100 (421limit_all_slopes_p12.f:3116-3432): f(pn,ii,jj,kk)
// returns the zone value being limited; grad gets modes 2..4.
template <class F>
static void weno8(const Ctx& c, const Nb& n, int i, int j, int k, double Ai[8][3][3], F f, double grad[3]) {
  double X[3][9];
  double f0 = f(i, j, k);
  for (int s = 0; s < 8; ++s) {
    int w1 = kSt8[s][0], w2 = kSt8[s][1], dz = kSt8[s][2];
    double R[3] = {f(n.x[w1], n.y[w1], k) - f0, f(n.x[w2], n.y[w2], k) - f0, f(i, j, k + dz) - f0};
    for (int r = 0; r < 3; ++r) X[r][s] = Ai[s][r][0] * R[0] + Ai[s][r][1] * R[1] + Ai[s][r][2] * R[2];
  }
  for (int r = 0; r < 3; ++r)
    X[r][8] = 0.125 * (X[r][0] + X[r][1] + X[r][2] + X[r][3] + X[r][4] + X[r][5] + X[r][6] + X[r][7]);
  double W[9];
  for (int s = 0; s < 9; ++s) {
    double IS = X[0][s] * X[0][s] + X[1][s] * X[1][s] + X[2][s] * X[2][s];
    W[s] = (s < 8 ? 1.0 : 100.0) / pow4(IS + c.p.smallnum);
  }
  double a11 = 1.0 / (W[0] + W[1] + W[2] + W[3] + W[4] + W[5] + W[6] + W[7] + W[8]);
  for (int s = 0; s < 9; ++s) W[s] = W[s] * a11;
  for (int r = 0; r < 3; ++r) {
    double t = W[0] * X[r][0];
    for (int s = 1; s < 9; ++s) t = t + W[s] * X[r][s];
    grad[r] = t;
  }
}

// The 18 neighbours of the central quadratic stencil: (w, radial offset)
// with w = -1 for the zone itself (421limit_all_slopes_p12.f:3960-4351).
static const int kN18[18][2] = {{0, 0},  {1, 0},  {2, 0},  {3, 0},  {-1, 1}, {-1, -1}, {8, 0}, {9, 0},  {10, 0},
                                {11, 0}, {0, 1},  {1, 1},  {0, -1}, {1, -1}, {2, 1},   {3, 1}, {2, -1}, {3, -1}};

// RECONSTRUCTION_COEFS at third order (200mesh/251reconstruction_coefs.f:55-81).
static void recon_row(double x, double y, double z, double l0, double lj, const double* c0, const double* cj,
                      double* row) {
  double r = lj / l0;
  double r2 = r * r;
  row[0] = x;
  row[1] = y;
  row[2] = z;
  row[3] = x * x - c0[4] + cj[4] * r2;
  row[4] = y * y - c0[5] + cj[5] * r2;
  row[5] = z * z - c0[6] + cj[6] * r2;
  row[6] = x * y - c0[7] + cj[7] * r2;
  row[7] = y * z - c0[8] + cj[8] * r2;
  row[8] = x * z - c0[9] + cj[9] * r2;
}

// INTERPOLATION_COEFS at third order (200mesh/252interpolation_coefs.f:53-75).
static void interp_row(double x, double y, double z, const double* c0, double* row) {
  row[0] = 1.0;
  row[1] = x;
  row[2] = y;
  row[3] = z;
  row[4] = x * x - c0[4];
  row[5] = y * y - c0[5];
  row[6] = z * z - c0[6];
  row[7] = x * y - c0[7];
  row[8] = y * z - c0[8];
  row[9] = x * z - c0[9];
}

// CMat_Row_Coefs_P2 (200mesh/253cmat_row_coefs_p2.f:7-96).
static void cmat_row(double x, double y, double z, double nx, double ny, double nz, const double* c0, double* row) {
  double b[10] = {1.0, x, y, z, x * x - c0[4], y * y - c0[5], z * z - c0[6], x * y - c0[7], y * z - c0[8], x * z - c0[9]};
  for (int t = 0; t < 10; ++t) {
    row[t] = (t == 0) ? nx : nx * b[t];
    row[10 + t] = (t == 0) ? ny : ny * b[t];
    row[20 + t] = (t == 0) ? nz : nz * b[t];
  }
}

static void coef_at(const Ctx& c, int pn, int i, int j, int k, double* co) {
  for (int t = 0; t < 10; ++t) co[t] = c.geo(COEF, t, pn, i, j, k);
}

// ------------------------------------------------------------------
// LIMIT_ALL_SLOPES_P2 (pkg/inc/cubesphere/400riemann_integrate/420limit_all_slopes_p2.f)
// differs from P12 in STEP 7.a and STEP 9.b only.  Its eight one-sided
// quadratic stencils, in the reference's order (R,U,+1), (L,U,+1), (L,D,+1),
// (R,D,+1), then the same with radial offset -1 (420:2596-4329, 8687-10120):
// in-plane neighbour a (R = 0 / L = 1), in-plane neighbour b (U = 2 / D = 3),
// radial direction dz and the corner zone between a and b.
static const int kP2St[8][4] = {{0, 2, 1, 8},  {1, 2, 1, 9},  {1, 3, 1, 10},  {0, 3, 1, 11},
                                {0, 2, -1, 8}, {1, 2, -1, 9}, {1, 3, -1, 10}, {0, 3, -1, 11}};

// The nine zones of stencil s around (i, j, k): a, b, the zone at dz, aa,
// bb, the zone at 2 dz, the corner, a at dz, b at dz.
static void p2_zones(const Nb& n, int s, int i, int j, int k, int* zx, int* zy, int* zz) {
  const int a = kP2St[s][0], b = kP2St[s][1], dz = kP2St[s][2], cn = kP2St[s][3];
  const int w[9] = {a, b, -1, a + 4, b + 4, -1, cn, a, b};
  const int o[9] = {0, 0, dz, 0, 0, 2 * dz, 0, dz, dz};
  for (int r = 0; r < 9; ++r) {
    zx[r] = w[r] < 0 ? i : n.x[w[r]];
    zy[r] = w[r] < 0 ? j : n.y[w[r]];
    zz[r] = k + o[r];
  }
}

// Smoothness indicator of the nine non-constant modes X (x, y, z, xx, yy,
// zz, xy, yz, xz) over the zone's unit cube (420:5245-5257, 10990-11002).
static double p2_smoothness(const double* X, const double* c0) {
  const double ob12 = 1.0 / 12.0, ob180 = 1.0 / 180.0, ob144 = 1.0 / 144.0;
  return (X[0] * X[0] + X[1] * X[1] + X[2] * X[2]) * ob12 + (X[3] * X[3]) * (sq(c0[4] - ob12) + ob180) +
         (X[4] * X[4]) * (sq(c0[5] - ob12) + ob180) + (X[5] * X[5]) * (sq(c0[6] - ob12) + ob180) +
         (X[6] * X[6]) * (c0[7] * c0[7] + ob144) + (X[7] * X[7]) * (c0[8] * c0[8] + ob144) +
         (X[8] * X[8]) * (c0[9] * c0[9] + ob144);
}

// Normalised WENO weights of the nine stencils: linear weights 1 (one-sided)
// and 100 (central), divided by (IS + smallnum)^4 (420:5264-5277).
static void p2_weights(const double* IS, double sm, double* W) {
  for (int s = 0; s < 9; ++s) W[s] = (s < 8 ? 1.0 : 100.0) / pow4(IS[s] + sm);
  double x = 1.0 / (W[0] + W[1] + W[2] + W[3] + W[4] + W[5] + W[6] + W[7] + W[8]);
  for (int s = 0; s < 9; ++s) W[s] = W[s] * x;
}

// Scaled centroid offset of zone (x, y, z) from zone (i, j, k).
static void p2_offset(const Ctx& c, int pn, int i, int j, int k, int zx, int zy, int zz, double obl0, double* o) {
  for (int a = 0; a < 3; ++a) o[a] = (c.geo(V_CEN, a, pn, zx, zy, zz) - c.geo(V_CEN, a, pn, i, j, k)) * obl0;
}

// STEP 7.a of LIMIT_ALL_SLOPES_P2 (420:2459-5394) for the primitives: per
// zone, the eight one-sided stencils' 9 x 9 reconstruction matrices
// (RECONSTRUCTION_COEFS rows) inverted by MATINV and the central 18-zone
// least squares (the STEP 7.b matrix of P12); per primitive, the nine
// stencils' modes, their smoothness indicators and WENO weights, the
// weighted modes 2..10 and the flattener.
static void p2_limit_primitives(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  const double sm = c.p.smallnum;
  auto V = [&](int comp, int mode, int i, int j, int k) -> double& { return c.a(c.V, mode * NV + comp, pn, i, j, k); };
  OMP_ZONES
  for (int k = 3 - G; k <= nr + G - 2; ++k)
    for (int j = 3 - G; j <= N + G - 2; ++j)
      for (int i = 3 - G; i <= N + G - 2; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        Nb n = nbrs(c, pn, i, j);
        const double l0 = std::max(c.geo(V_SCALE, 0, pn, i, j, k), sm), obl0 = 1.0 / l0;
        double c0[10];
        coef_at(c, pn, i, j, k, c0);
        double Ai[8][81];
        int zx[8][9], zy[8][9], zz[8][9];
        for (int s = 0; s < 8; ++s) {
          p2_zones(n, s, i, j, k, zx[s], zy[s], zz[s]);
          double A[81];
          for (int r = 0; r < 9; ++r) {
            double o[3], cj[10];
            p2_offset(c, pn, i, j, k, zx[s][r], zy[s][r], zz[s][r], obl0, o);
            const double lj = std::max(c.geo(V_SCALE, 0, pn, zx[s][r], zy[s][r], zz[s][r]), sm);
            coef_at(c, pn, zx[s][r], zy[s][r], zz[s][r], cj);
            recon_row(o[0], o[1], o[2], l0, lj, c0, cj, A + 9 * r);
          }
          matinv(9, A, Ai[s]);
        }
        double A18[18][9];
        int cx[18], cy[18], cz[18];
        for (int r = 0; r < 18; ++r) {
          const int w = kN18[r][0];
          cx[r] = (w < 0) ? i : n.x[w];
          cy[r] = (w < 0) ? j : n.y[w];
          cz[r] = k + kN18[r][1];
          double o[3], cj[10];
          p2_offset(c, pn, i, j, k, cx[r], cy[r], cz[r], obl0, o);
          const double lj = std::max(c.geo(V_SCALE, 0, pn, cx[r], cy[r], cz[r]), sm);
          coef_at(c, pn, cx[r], cy[r], cz[r], cj);
          recon_row(o[0], o[1], o[2], l0, lj, c0, cj, A18[r]);
        }
        double M[81], Minv[81];
        for (int a2 = 0; a2 < 9; ++a2)
          for (int b2 = 0; b2 < 9; ++b2) {
            double s = 0.0;
            for (int r = 0; r < 18; ++r) s = s + A18[r][a2] * A18[r][b2];
            M[a2 * 9 + b2] = s;
          }
        matinv(9, M, Minv);
        const double x = 1.0 - c.a(c.flat, 0, pn, i, j, k);
        for (int q = 0; q < NV; ++q) {
          const double v0 = V(q, 0, i, j, k);
          double X[9][9], IS[9], W[9];  // X[stencil][mode]
          for (int s = 0; s < 8; ++s) {
            double R[9];
            for (int r = 0; r < 9; ++r) R[r] = V(q, 0, zx[s][r], zy[s][r], zz[s][r]) - v0;
            for (int a2 = 0; a2 < 9; ++a2) {
              double t = 0.0;
              for (int r = 0; r < 9; ++r) t = t + Ai[s][a2 * 9 + r] * R[r];
              X[s][a2] = t;
            }
          }
          double Y[9];
          for (int a2 = 0; a2 < 9; ++a2) {
            double t = 0.0;
            for (int r = 0; r < 18; ++r) t = t + A18[r][a2] * (V(q, 0, cx[r], cy[r], cz[r]) - v0);
            Y[a2] = t;
          }
          for (int a2 = 0; a2 < 9; ++a2) {
            double t = 0.0;
            for (int b2 = 0; b2 < 9; ++b2) t = t + Minv[a2 * 9 + b2] * Y[b2];
            X[8][a2] = t;
          }
          for (int s = 0; s < 9; ++s) IS[s] = p2_smoothness(X[s], c0);
          p2_weights(IS, sm, W);
          for (int a2 = 0; a2 < 9; ++a2) {
            double t = W[0] * X[0][a2];
            for (int s = 1; s < 9; ++s) t = t + W[s] * X[s][a2];
            V(q, 1 + a2, i, j, k) = t * x;
          }
        }
        // entropy: P12's eight linear stencils and their mean (420:5396-6306)
        double Al[8][3][3], gr[3];
        stencil_inverses(c, pn, i, j, k, n, Al);
        weno8(c, n, i, j, k, Al, [&](int x2, int y2, int z2) { return c.a(c.ent, 0, pn, x2, y2, z2); }, gr);
        for (int r = 0; r < 3; ++r) c.a(c.ent, 1 + r, pn, i, j, k) = gr[r] * x;
      }
}

// STEP 9.b of LIMIT_ALL_SLOPES_P2 (420:8553-12285): third-order
// interpolation WENO of the zone-centred E components: the eight one-sided
// 10-zone stencils (the zone and the nine zones of the primitive stencil,
// INTERPOLATION_COEFS rows, 10 x 10 MATINV) and the central 19-zone least
// squares (the STEP 9.c matrix of P12), WENO-weighted; the point value is
// flattened toward the unlimited one and modes 2..10 damped.  Each zone
// rewrites its own point value, so neighbours are read from the values
// before the loop (parallel-loop semantics, order-free).
static void p2_limit_efield(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  const double sm = c.p.smallnum;
  auto E = [&](int comp, int mode, int i, int j, int k) -> double& { return c.a(c.E, mode * 3 + comp, pn, i, j, k); };
  std::vector<double> esnap(3 * c.S);
  for (int q = 0; q < 3; ++q)
    std::memcpy(&esnap[(size_t)q * c.S], &c.E[((size_t)q * 6 + pn) * c.S], c.S * sizeof(double));
  auto Es = [&](int q, int x, int y, int z) { return esnap[(size_t)q * c.S + c.idx(x, y, z)]; };
  OMP_ZONES
  for (int k = 3 - G; k <= nr + G - 2; ++k)
    for (int j = 3 - G; j <= N + G - 2; ++j)
      for (int i = 3 - G; i <= N + G - 2; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        Nb n = nbrs(c, pn, i, j);
        const double obl0 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, i, j, k), sm);
        double c0[10];
        coef_at(c, pn, i, j, k, c0);
        double Ai[8][100];
        int zx[8][10], zy[8][10], zz[8][10];
        for (int s = 0; s < 8; ++s) {
          zx[s][0] = i;
          zy[s][0] = j;
          zz[s][0] = k;
          p2_zones(n, s, i, j, k, zx[s] + 1, zy[s] + 1, zz[s] + 1);
          double A[100];
          for (int r = 0; r < 10; ++r) {
            double o[3];
            p2_offset(c, pn, i, j, k, zx[s][r], zy[s][r], zz[s][r], obl0, o);
            if (r == 0) o[0] = o[1] = o[2] = 0.0;
            interp_row(o[0], o[1], o[2], c0, A + 10 * r);
          }
          matinv(10, A, Ai[s]);
        }
        double A19[19][10];
        int cx[19], cy[19], cz[19];
        cx[0] = i;
        cy[0] = j;
        cz[0] = k;
        interp_row(0.0, 0.0, 0.0, c0, A19[0]);
        for (int r = 0; r < 18; ++r) {
          const int w = kN18[r][0];
          cx[r + 1] = (w < 0) ? i : n.x[w];
          cy[r + 1] = (w < 0) ? j : n.y[w];
          cz[r + 1] = k + kN18[r][1];
          double o[3];
          p2_offset(c, pn, i, j, k, cx[r + 1], cy[r + 1], cz[r + 1], obl0, o);
          interp_row(o[0], o[1], o[2], c0, A19[r + 1]);
        }
        double M[100], Minv[100];
        for (int a2 = 0; a2 < 10; ++a2)
          for (int b2 = 0; b2 < 10; ++b2) {
            double s = 0.0;
            for (int r = 0; r < 19; ++r) s = s + A19[r][a2] * A19[r][b2];
            M[a2 * 10 + b2] = s;
          }
        matinv(10, M, Minv);
        const double f = c.a(c.flat, 0, pn, i, j, k), x = 1.0 - f;
        for (int q = 0; q < 3; ++q) {
          double X[9][10], IS[9], W[9];
          for (int s = 0; s < 8; ++s) {
            double R[10];
            for (int r = 0; r < 10; ++r) R[r] = Es(q, zx[s][r], zy[s][r], zz[s][r]);
            for (int a2 = 0; a2 < 10; ++a2) {
              double t = 0.0;
              for (int r = 0; r < 10; ++r) t = t + Ai[s][a2 * 10 + r] * R[r];
              X[s][a2] = t;
            }
          }
          double Y[10];
          for (int a2 = 0; a2 < 10; ++a2) {
            double t = 0.0;
            for (int r = 0; r < 19; ++r) t = t + A19[r][a2] * Es(q, cx[r], cy[r], cz[r]);
            Y[a2] = t;
          }
          for (int a2 = 0; a2 < 10; ++a2) {
            double t = 0.0;
            for (int b2 = 0; b2 < 10; ++b2) t = t + Minv[a2 * 10 + b2] * Y[b2];
            X[8][a2] = t;
          }
          for (int s = 0; s < 9; ++s) IS[s] = p2_smoothness(X[s] + 1, c0);
          p2_weights(IS, sm, W);
          const double Ept = Es(q, i, j, k);
          double e[10];
          for (int a2 = 0; a2 < 10; ++a2) {
            double t = W[0] * X[0][a2];
            for (int s = 1; s < 9; ++s) t = t + W[s] * X[s][a2];
            e[a2] = t;
          }
          E(q, 0, i, j, k) = f * Ept + x * e[0];
          for (int a2 = 1; a2 < 10; ++a2) E(q, a2, i, j, k) = e[a2] * x;
        }
      }
}

// ------------------------------------------------------------------
// LIMIT_ALL_SLOPES_P12 (pkg/inc/cubesphere/400riemann_integrate/421limit_all_slopes_p12.f:9-9985)
// without its STEP 10 diagnostics, for one panel.
void limit_all_slopes_p12(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  const double g = c.p.gamma, sm = c.p.smallnum;
  const double ob12 = 1.0 / 12.0, ob180 = 1.0 / 180.0, ob144 = 1.0 / 144.0;
  auto V = [&](int comp, int mode, int i, int j, int k) -> double& { return c.a(c.V, mode * NV + comp, pn, i, j, k); };
  auto E = [&](int comp, int mode, int i, int j, int k) -> double& { return c.a(c.E, mode * 3 + comp, pn, i, j, k); };
  // STEP 2 (:597-759)
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        c.a(c.msonic, 0, pn, i, j, k) = sm;
        for (int q = 1; q < 4; ++q) c.a(c.ent, q, pn, i, j, k) = 0.0;
        for (int t = 0; t < NV * 10; ++t) c.a(c.V, t, pn, i, j, k) = 0.0;
        if (c.m(pn, i, j) == 0) {
          for (int q = 0; q < NV; ++q) c.a(c.U, q, pn, i, j, k) = 0.0;
          c.a(c.U, 0, pn, i, j, k) = c.p.rhofloor;
          c.a(c.U, 4, pn, i, j, k) = c.p.prsfloor / (g - 1.0);
          c.geow(V_SCALE, 0, pn, i, j, k) = sm;
        }
      }
  zero_masked_faces(c, pn);
  // STEP 3 (:779-962)
  tricorner_sync(c, pn);
  // STEP 5 (:1497-1628)
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        double Up[NV], Vp[NV];
        for (int q = 0; q < NV; ++q) Up[q] = c.a(c.U, q, pn, i, j, k);
        double en = c.a(c.ent, 0, pn, i, j, k);
        cons_to_prim(c.ph, en, Up, Vp);
        for (int q = 0; q < NV; ++q) {
          V(q, 0, i, j, k) = Vp[q];
          c.a(c.U, q, pn, i, j, k) = Up[q];
        }
        c.a(c.ent, 0, pn, i, j, k) = en;
        for (int q = 1; q < 4; ++q) c.a(c.ent, q, pn, i, j, k) = 0.0;
        double a12 = (sq(V(5, 0, i, j, k)) + sq(V(6, 0, i, j, k)) + sq(V(7, 0, i, j, k))) * c.ph.ob4pi;
        double ms = g * V(4, 0, i, j, k) + a12;
        c.a(c.msonic, 0, pn, i, j, k) = std::sqrt(ms / V(0, 0, i, j, k));
      }
  // STEP 6 flattener (:1797-2458)
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) c.a(c.flat, 0, pn, i, j, k) = 0.0;
  OMP_ZONES
  for (int k = 2 - G; k <= nr + G - 1; ++k)
    for (int j = 2 - G; j <= N + G - 1; ++j)
      for (int i = 2 - G; i <= N + G - 1; ++i) {
        Nb n = nbrs(c, pn, i, j);
        double obl0 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, i, j, k), sm);
        auto ms = [&](int x, int y, int z) { return c.a(c.msonic, 0, pn, x, y, z); };
        double w = std::min({ms(i, j, k), ms(n.x[0], n.y[0], k), ms(n.x[1], n.y[1], k), ms(n.x[2], n.y[2], k),
                             ms(n.x[3], n.y[3], k), ms(i, j, k + 1), ms(i, j, k - 1)});
        c.a(c.work, 0, pn, i, j, k) = w;
        double dv = 0.0;
        auto cen = [&](int q, int x, int y, int z) { return c.geo(V_CEN, q, pn, x, y, z); };
        // (zone a, zone b) with b - a along the face normal (nx,ny,nz)
        auto term = [&](int ax, int ay, int az, int bx, int by, int bz, double nx, double ny, double nz) {
          double x = (cen(0, bx, by, bz) - cen(0, ax, ay, az)) * obl0;
          double y = (cen(1, bx, by, bz) - cen(1, ax, ay, az)) * obl0;
          double z = (cen(2, bx, by, bz) - cen(2, ax, ay, az)) * obl0;
          double a11 = 0.5 / std::max(std::sqrt(x * x + y * y + z * z), sm);
          dv = dv + nx * a11 * (V(1, 0, bx, by, bz) - V(1, 0, ax, ay, az)) +
               ny * a11 * (V(2, 0, bx, by, bz) - V(2, 0, ax, ay, az)) +
               nz * a11 * (V(3, 0, bx, by, bz) - V(3, 0, ax, ay, az));
        };
        term(i, j, k, n.x[0], n.y[0], k, c.geo(XF_N, 0, pn, i, j, k), c.geo(XF_N, 1, pn, i, j, k), c.geo(XF_N, 2, pn, i, j, k));
        term(n.x[1], n.y[1], k, i, j, k, c.geo(XF_N, 0, pn, i - 1, j, k), c.geo(XF_N, 1, pn, i - 1, j, k),
             c.geo(XF_N, 2, pn, i - 1, j, k));
        term(i, j, k, n.x[2], n.y[2], k, c.geo(YF_N, 0, pn, i, j, k), c.geo(YF_N, 1, pn, i, j, k), c.geo(YF_N, 2, pn, i, j, k));
        term(n.x[3], n.y[3], k, i, j, k, c.geo(YF_N, 0, pn, i, j - 1, k), c.geo(YF_N, 1, pn, i, j - 1, k),
             c.geo(YF_N, 2, pn, i, j - 1, k));
        double nx = c.geo(ZF_CEN, 0, pn, i, j, k), ny = c.geo(ZF_CEN, 1, pn, i, j, k), nz = c.geo(ZF_CEN, 2, pn, i, j, k);
        double a12 = 1.0 / std::max(std::sqrt(nx * nx + ny * ny + nz * nz), sm);
        nx = nx * a12;
        ny = ny * a12;
        nz = nz * a12;
        term(i, j, k, i, j, k + 1, nx, ny, nz);
        term(i, j, k - 1, i, j, k, nx, ny, nz);
        c.a(c.divvel, 0, pn, i, j, k) = dv;
        double a13 = std::fabs(dv) / (c.p.flatten_coef * w);
        a13 = a13 - 1.0;
        double fl = (a13 <= 0.0) ? 0.0 : std::min(1.0, a13);
        if (c.m(pn, i, j) != 1) fl = 0.0;
        c.a(c.flat, 0, pn, i, j, k) = fl;
      }
  for (int pass = 0; pass < 2; ++pass) {
    // pass 0: STEP 6.b (pressure-ratio raise), pass 1: STEP 6.c (upwinding)
    OMP_ZONES
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) c.a(c.work, 0, pn, i, j, k) = c.a(c.flat, 0, pn, i, j, k);
    OMP_ZONES
    for (int k = 2 - G; k <= nr + G - 1; ++k)
      for (int j = 2 - G; j <= N + G - 1; ++j)
        for (int i = 2 - G; i <= N + G - 1; ++i) {
          Nb n = nbrs(c, pn, i, j);
          int xs[6] = {n.x[0], n.x[1], n.x[2], n.x[3], i, i}, ys[6] = {n.y[0], n.y[1], n.y[2], n.y[3], j, j};
          int zs[6] = {k, k, k, k, k + 1, k - 1};
          double& fl = c.a(c.flat, 0, pn, i, j, k);
          for (int t = 0; t < 6; ++t) {
            bool take = (pass == 1) || (V(4, 0, xs[t], ys[t], zs[t]) > c.p.prs_flatten_coef * V(4, 0, i, j, k));
            if (take) fl = std::max(fl, c.a(c.work, 0, pn, xs[t], ys[t], zs[t]));
          }
        }
  }
  // CS_FLAG_P2: STEP 7.a of LIMIT_ALL_SLOPES_P2 in place of STEPS 7.a and 7.b
  const bool p2 = (c.p.flags & CS_FLAG_P2) != 0;
  if (p2) p2_limit_primitives(c, pn);
  if (!p2) {  // P12 STEPS 7.a, 7.b
  // STEP 7.a (:2515-3804)
  OMP_ZONES
  for (int k = 2 - G; k <= nr + G - 1; ++k)
    for (int j = 2 - G; j <= N + G - 1; ++j)
      for (int i = 2 - G; i <= N + G - 1; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        Nb n = nbrs(c, pn, i, j);
        double Ai[8][3][3];
        stencil_inverses(c, pn, i, j, k, n, Ai);
        for (int q = 0; q < NV; ++q) {
          double gr[3];
          weno8(c, n, i, j, k, Ai, [&](int x, int y, int z) { return V(q, 0, x, y, z); }, gr);
          V(q, 1, i, j, k) = gr[0];
          V(q, 2, i, j, k) = gr[1];
          V(q, 3, i, j, k) = gr[2];
        }
        double gr[3];
        weno8(c, n, i, j, k, Ai, [&](int x, int y, int z) { return c.a(c.ent, 0, pn, x, y, z); }, gr);
        double om = 1.0 - c.a(c.flat, 0, pn, i, j, k);
        for (int r = 0; r < 3; ++r) c.a(c.ent, 1 + r, pn, i, j, k) = gr[r] * om;
      }
  // STEP 7.b (:3869-4551)
  OMP_ZONES
  for (int k = 3 - G; k <= nr + G - 2; ++k)
    for (int j = 3 - G; j <= N + G - 2; ++j)
      for (int i = 3 - G; i <= N + G - 2; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        Nb n = nbrs(c, pn, i, j);
        double l0 = std::max(c.geo(V_SCALE, 0, pn, i, j, k), sm), obl0 = 1.0 / l0;
        double c0[10];
        coef_at(c, pn, i, j, k, c0);
        double A[18][9];
        int zx[18], zy[18], zz[18];
        for (int r = 0; r < 18; ++r) {
          int w = kN18[r][0], dz = kN18[r][1];
          zx[r] = (w < 0) ? i : n.x[w];
          zy[r] = (w < 0) ? j : n.y[w];
          zz[r] = k + dz;
          double x = (c.geo(V_CEN, 0, pn, zx[r], zy[r], zz[r]) - c.geo(V_CEN, 0, pn, i, j, k)) * obl0;
          double y = (c.geo(V_CEN, 1, pn, zx[r], zy[r], zz[r]) - c.geo(V_CEN, 1, pn, i, j, k)) * obl0;
          double z = (c.geo(V_CEN, 2, pn, zx[r], zy[r], zz[r]) - c.geo(V_CEN, 2, pn, i, j, k)) * obl0;
          double lj = std::max(c.geo(V_SCALE, 0, pn, zx[r], zy[r], zz[r]), sm);
          double cj[10];
          coef_at(c, pn, zx[r], zy[r], zz[r], cj);
          recon_row(x, y, z, l0, lj, c0, cj, A[r]);
        }
        double M[81], Minv[81];
        for (int a2 = 0; a2 < 9; ++a2)
          for (int b2 = 0; b2 < 9; ++b2) {
            double s = 0.0;
            for (int r = 0; r < 18; ++r) s = s + A[r][a2] * A[r][b2];
            M[a2 * 9 + b2] = s;
          }
        matinv(9, M, Minv);
        double f = c.a(c.flat, 0, pn, i, j, k);
        for (int q = 0; q < NV; ++q) {
          double R[18], Y[9], X[9];
          double v0 = V(q, 0, i, j, k);
          for (int r = 0; r < 18; ++r) R[r] = V(q, 0, zx[r], zy[r], zz[r]) - v0;
          for (int a2 = 0; a2 < 9; ++a2) {
            double s = 0.0;
            for (int r = 0; r < 18; ++r) s = s + A[r][a2] * R[r];
            Y[a2] = s;
          }
          for (int a2 = 0; a2 < 9; ++a2) {
            double s = 0.0;
            for (int b2 = 0; b2 < 9; ++b2) s = s + Minv[a2 * 9 + b2] * Y[b2];
            X[a2] = s;
          }
          double betalo = f + (1.0 - f) * 2.0;
          double ghi = f * 0.6 + (1.0 - f) * 0.95, glo = 1.0 - ghi, obghi = 1.0 / ghi, grat = glo / ghi;
          double v2 = V(q, 1, i, j, k), v3 = V(q, 2, i, j, k), v4 = V(q, 3, i, j, k);
          double ISlo = betalo * (v2 * v2 + v3 * v3 + v4 * v4) * ob12;
          double Phi[9];
          Phi[0] = X[0] * obghi - v2 * grat;
          Phi[1] = X[1] * obghi - v3 * grat;
          Phi[2] = X[2] * obghi - v4 * grat;
          for (int t = 3; t < 9; ++t) Phi[t] = X[t] * obghi;
          double IShi = (Phi[0] * Phi[0] + Phi[1] * Phi[1] + Phi[2] * Phi[2]) * ob12 +
                        (Phi[3] * Phi[3]) * (sq(c0[4] - ob12) + ob180) + (Phi[4] * Phi[4]) * (sq(c0[5] - ob12) + ob180) +
                        (Phi[5] * Phi[5]) * (sq(c0[6] - ob12) + ob180) + (Phi[6] * Phi[6]) * (c0[7] * c0[7] + ob144) +
                        (Phi[7] * Phi[7]) * (c0[8] * c0[8] + ob144) + (Phi[8] * Phi[8]) * (c0[9] * c0[9] + ob144);
          double tau = std::fabs(IShi - ISlo);
          double Wlo = glo * (1.0 + tau / (ISlo + sm)), Whi = ghi * (1.0 + tau / (IShi + sm));
          double aa = 1.0 / (Wlo + Whi);
          Wlo = Wlo * aa;
          Whi = Whi * aa;
          V(q, 1, i, j, k) = Whi * Phi[0] + Wlo * v2;
          V(q, 2, i, j, k) = Whi * Phi[1] + Wlo * v3;
          V(q, 3, i, j, k) = Whi * Phi[2] + Wlo * v4;
          for (int t = 4; t < 10; ++t) V(q, t, i, j, k) = Whi * Phi[t - 1];
          double x = 1.0 - f;
          for (int t = 1; t < 10; ++t) V(q, t, i, j, k) = V(q, t, i, j, k) * x;
        }
      }
  }  // P12 STEPS 7.a, 7.b
  // STEP 7.c ENFORCE_PRESSURE_POSITIVITY_PRIM (440enforce_pressure_positivity_prim.f:204-829).
  // The zone loop is a parallel loop in the reference's GPU path; neighbour
  // entropy is read from the values before the loop (a zone that gives up
  // zeroes its own entropy, 440:569-575), so the result is order-free.
  {
    const std::vector<double> ent_snap(c.ent.begin() + (size_t)pn * c.S, c.ent.begin() + (size_t)(pn + 1) * c.S);
    std::fill(c.pos.begin() + (size_t)pn * c.S, c.pos.begin() + (size_t)(pn + 1) * c.S, 0.0);
    const int niter = 15;
    const double ratio = std::pow(0.10, 1.0 / (double)niter), ef = 0.2;
    OMP_ZONES
    for (int k = 2 - G; k <= nr + G - 1; ++k)
      for (int j = 2 - G; j <= N + G - 1; ++j)
        for (int i = 2 - G; i <= N + G - 1; ++i) {
          Nb n = nbrs(c, pn, i, j);
          double obl0 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, i, j, k), sm);
          double vc[3] = {c.geo(V_CEN, 0, pn, i, j, k), c.geo(V_CEN, 1, pn, i, j, k), c.geo(V_CEN, 2, pn, i, j, k)};
          double c0[10];
          coef_at(c, pn, i, j, k, c0);
          int px[9] = {i, n.x[0], n.x[1], n.x[2], n.x[3], n.x[8], n.x[9], n.x[10], n.x[11]};
          int py[9] = {j, n.y[0], n.y[1], n.y[2], n.y[3], n.y[8], n.y[9], n.y[10], n.y[11]};
          double Vmin[NV], Vmax[NV], emin = 1e300, emax = -1e300;
          for (int q = 0; q < NV; ++q) {
            Vmin[q] = 1e300;
            Vmax[q] = -1e300;
          }
          for (int s = 0; s < 9; ++s)
            for (int dz = -1; dz <= 1; ++dz) {
              for (int q = 0; q < NV; ++q) {
                double v = V(q, 0, px[s], py[s], k + dz);
                Vmin[q] = std::min(Vmin[q], v);
                Vmax[q] = std::max(Vmax[q], v);
              }
              double e = ent_snap[c.idx(px[s], py[s], k + dz)];
              emin = std::min(emin, e);
              emax = std::max(emax, e);
            }
          double Vd[NV];
          for (int q = 0; q < NV; ++q) Vd[q] = Vmax[q] - Vmin[q];
          double ff = std::max(std::min((c.a(c.flat, 0, pn, i, j, k) - 0.1) / 0.4, 1.0), 0.0);
          double omff = 1.0 - ff;
          Vmin[0] = std::max(Vmin[0] * (1.0 - ef * omff), c.p.rhofloor);
          Vmax[0] = std::max(Vmax[0] * (1.0 + ef * omff), c.p.rhofloor);
          Vmin[4] = std::max(Vmin[4] * (1.0 - ef * omff), c.p.prsfloor);
          Vmax[4] = std::max(Vmax[4] * (1.0 + ef * omff), c.p.prsfloor);
          for (int q : {1, 2, 3, 5, 6, 7}) {
            Vmin[q] = Vmin[q] - 0.5 * ef * omff * Vd[q];
            Vmax[q] = Vmax[q] + 0.5 * ef * omff * Vd[q];
          }
          emin = emin * (1.0 - ef * omff);
          emax = emax * (1.0 + ef * omff);
          double Vp[NV][10], ep[4];
          for (int q = 0; q < NV; ++q)
            for (int t = 0; t < 10; ++t) Vp[q][t] = V(q, t, i, j, k);
          for (int t = 0; t < 4; ++t) ep[t] = c.a(c.ent, t, pn, i, j, k);
          double vert[27][3];
          auto vx = [&](int node, int x, int y, int z) {
            for (int q = 0; q < 3; ++q) vert[node][q] = c.geo(G_VERT, q, pn, x, y, z);
          };
          vx(0, i - 1, j - 1, k - 1);
          vx(1, i, j - 1, k - 1);
          vx(2, i - 1, j, k - 1);
          vx(3, i, j, k - 1);
          vx(4, i - 1, j - 1, k);
          vx(5, i, j - 1, k);
          vx(6, i - 1, j, k);
          vx(7, i, j, k);
          for (int q = 0; q < 3; ++q) {
            vert[8][q] = c.geo(XF_CEN, q, pn, i, j, k);
            vert[9][q] = c.geo(XF_CEN, q, pn, i - 1, j, k);
            vert[10][q] = c.geo(YF_CEN, q, pn, i, j, k);
            vert[11][q] = c.geo(YF_CEN, q, pn, i, j - 1, k);
            vert[12][q] = c.geo(ZF_CEN, q, pn, i, j, k);
            vert[13][q] = c.geo(ZF_CEN, q, pn, i, j, k - 1);
          }
          static const int pr[12][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3},
                                        {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
          for (int e = 0; e < 12; ++e)
            for (int q = 0; q < 3; ++q) vert[14 + e][q] = (vert[pr[e][0]][q] + vert[pr[e][1]][q]) * 0.5;
          for (int q = 0; q < 3; ++q) vert[26][q] = vc[q];
          double xyz[27][3];
          for (int nd = 0; nd < 27; ++nd)
            for (int q = 0; q < 3; ++q) xyz[nd][q] = (vert[nd][q] - vc[q]) * obl0;
          int shrinks = 0, gave_up = 0;
          for (int iter = 1; iter <= niter + 1; ++iter) {
            if (iter == niter + 1) {
              for (int q = 0; q < NV; ++q)
                for (int t = 1; t < 10; ++t) Vp[q][t] = 0.0;
              for (int t = 0; t < 4; ++t) ep[t] = 0.0;
              gave_up = 1;
              break;
            }
            bool pass = true;
            for (int nd = 0; nd < 27; ++nd) {
              double x = xyz[nd][0], y = xyz[nd][1], z = xyz[nd][2];
              double v1 = poly10(Vp[0], c0, x, y, z), v5 = poly10(Vp[4], c0, x, y, z);
              double en = ep[0] + ep[1] * x + ep[2] * y + ep[3] * z;
              if (v1 < Vmin[0] || v1 > Vmax[0]) pass = false;
              if (v5 < Vmin[4] || v5 > Vmax[4]) pass = false;
              if (en < emin || en > emax) pass = false;
            }
            if (pass) break;
            for (int q = 0; q < NV; ++q)
              for (int t = 1; t < 10; ++t) Vp[q][t] = ratio * Vp[q][t];
            for (int t = 1; t < 4; ++t) ep[t] = ratio * ep[t];
            ++shrinks;
          }
          c.a(c.pos, 0, pn, i, j, k) = gave_up + 2 * shrinks;
          for (int q = 0; q < NV; ++q)
            for (int t = 0; t < 10; ++t) V(q, t, i, j, k) = Vp[q][t];
          for (int t = 0; t < 4; ++t) c.a(c.ent, t, pn, i, j, k) = ep[t];
        }
  }
  // STEP 8.a-c: B at the five quadrature points of every face from both sides,
  // shifted to the facial mean (421limit_all_slopes_p12.f:4686-5567).
  for (int dir = 0; dir < 3; ++dir) {
    std::vector<double>& Bq = dir == 0 ? c.Bqx : (dir == 1 ? c.Bqy : c.Bqz);
    std::vector<double>& Bf = dir == 0 ? c.Bxf : (dir == 1 ? c.Byf : c.Bzf);
    const int QP = dir == 0 ? XF_QP : (dir == 1 ? YF_QP : ZF_QP);
    const int BW = dir == 0 ? XB_QW : (dir == 1 ? YB_QW : ZB_QW);
    int lo[3] = {2 - G, 2 - G, 2 - G}, hi[3] = {N + G - 1, N + G - 1, nr + G - 1};
    lo[dir] = 1 - G;
    OMP_ZONES
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          int lx, ly, rx, ry, lz = k, rz = k;
          bool skip = false;
          if (dir == 0) {
            int mL = c.m(pn, i, j), mR = c.m(pn, i + 1, j);
            if (mL == 1 && mR == 1) { lx = i; ly = j; rx = i + 1; ry = j; }
            else if (mL == 0 && mR == 1) { rx = i + 1; ry = j; lx = c.sti(pn, rx, ry, 1, 0); ly = c.sti(pn, rx, ry, 1, 1); }
            else if (mL == 1 && mR == 0) { lx = i; ly = j; rx = c.sti(pn, lx, ly, 0, 0); ry = c.sti(pn, lx, ly, 0, 1); }
            else skip = true;
          } else if (dir == 1) {
            int mL = c.m(pn, i, j), mR = c.m(pn, i, j + 1);
            if (mL == 1 && mR == 1) { lx = i; ly = j; rx = i; ry = j + 1; }
            else if (mL == 0 && mR == 1) { rx = i; ry = j + 1; lx = c.sti(pn, rx, ry, 3, 0); ly = c.sti(pn, rx, ry, 3, 1); }
            else if (mL == 1 && mR == 0) { lx = i; ly = j; rx = c.sti(pn, lx, ly, 2, 0); ry = c.sti(pn, lx, ly, 2, 1); }
            else skip = true;
          } else {
            if (c.m(pn, i, j) == 0) skip = true;
            lx = rx = i;
            ly = ry = j;
            rz = k + 1;
          }
          if (skip) {
            for (int q = 0; q < 5; ++q) c.a(Bq, q, pn, i, j, k) = 0.0;
            continue;
          }
          double obl0 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, lx, ly, lz), sm);
          double obl02 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, rx, ry, rz), sm);
          double c0[10], cj[10];
          coef_at(c, pn, lx, ly, lz, c0);
          coef_at(c, pn, rx, ry, rz, cj);
          for (int q = 0; q < 5; ++q) {
            double nx, ny, nz;
            if (dir == 0) { nx = c.geo(XF_N, 0, pn, i, j, k); ny = c.geo(XF_N, 1, pn, i, j, k); nz = c.geo(XF_N, 2, pn, i, j, k); }
            else if (dir == 1) { nx = c.geo(YF_N, 0, pn, i, j, k); ny = c.geo(YF_N, 1, pn, i, j, k); nz = c.geo(YF_N, 2, pn, i, j, k); }
            else { nx = c.geo(ZF_N, 0 * 5 + q, pn, i, j, k); ny = c.geo(ZF_N, 1 * 5 + q, pn, i, j, k); nz = c.geo(ZF_N, 2 * 5 + q, pn, i, j, k); }
            double px = c.geo(QP, 0 * 5 + q, pn, i, j, k), py = c.geo(QP, 1 * 5 + q, pn, i, j, k),
                   pz = c.geo(QP, 2 * 5 + q, pn, i, j, k);
            double x = (px - c.geo(V_CEN, 0, pn, lx, ly, lz)) * obl0, y = (py - c.geo(V_CEN, 1, pn, lx, ly, lz)) * obl0,
                   z = (pz - c.geo(V_CEN, 2, pn, lx, ly, lz)) * obl0;
            double x2 = (px - c.geo(V_CEN, 0, pn, rx, ry, rz)) * obl02, y2 = (py - c.geo(V_CEN, 1, pn, rx, ry, rz)) * obl02,
                   z2 = (pz - c.geo(V_CEN, 2, pn, rx, ry, rz)) * obl02;
            double vl[3][10], vr[3][10];
            for (int t = 0; t < 10; ++t)
              for (int b = 0; b < 3; ++b) {
                vl[b][t] = V(5 + b, t, lx, ly, lz);
                vr[b][t] = V(5 + b, t, rx, ry, rz);
              }
            double bx = poly10(vl[0], c0, x, y, z), by = poly10(vl[1], c0, x, y, z), bz = poly10(vl[2], c0, x, y, z);
            double bx2 = poly10(vr[0], cj, x2, y2, z2), by2 = poly10(vr[1], cj, x2, y2, z2), bz2 = poly10(vr[2], cj, x2, y2, z2);
            c.a(Bq, q, pn, i, j, k) = 0.5 * (nx * (bx + bx2) + ny * (by + by2) + nz * (bz + bz2));
          }
        }
    OMP_ZONES
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          double bd = c.a(Bf, 0, pn, i, j, k);
          for (int q = 0; q < 5; ++q) bd = bd - c.geo(BW, q, pn, i, j, k) * c.a(Bq, q, pn, i, j, k);
          for (int q = 0; q < 5; ++q) c.a(Bq, q, pn, i, j, k) = c.a(Bq, q, pn, i, j, k) + bd;
        }
  }
  // STEP 8.d ADP constrained least squares (:5617-6677)
  OMP_ZONES
  for (int k = 2 - G; k <= nr + G - 1; ++k)
    for (int j = 2 - G; j <= N + G - 1; ++j)
      for (int i = 2 - G; i <= N + G - 1; ++i) {
        if (c.m(pn, i, j) == 0) continue;
        double C[6][30] = {}, D[6] = {}, A[64][30] = {}, Bv[64] = {};
        double c0[10];
        coef_at(c, pn, i, j, k, c0);
        double obl0 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, i, j, k), sm);
        double vc[3] = {c.geo(V_CEN, 0, pn, i, j, k), c.geo(V_CEN, 1, pn, i, j, k), c.geo(V_CEN, 2, pn, i, j, k)};
        // faces: x+ (i), x- (i-1), y+ (j), y- (j-1), z+ (k), z- (k-1)
        for (int f = 0; f < 6; ++f) {
          int dir = f / 2, fx = i, fy = j, fz = k;
          if (f == 1) fx = i - 1;
          if (f == 3) fy = j - 1;
          if (f == 5) fz = k - 1;
          const int QP = dir == 0 ? XF_QP : (dir == 1 ? YF_QP : ZF_QP);
          const int BW = dir == 0 ? XB_QW : (dir == 1 ? YB_QW : ZB_QW);
          std::vector<double>& Bq = dir == 0 ? c.Bqx : (dir == 1 ? c.Bqy : c.Bqz);
          for (int q = 0; q < 5; ++q) {
            double nx, ny, nz;
            if (dir == 0) { nx = c.geo(XF_N, 0, pn, fx, fy, fz); ny = c.geo(XF_N, 1, pn, fx, fy, fz); nz = c.geo(XF_N, 2, pn, fx, fy, fz); }
            else if (dir == 1) { nx = c.geo(YF_N, 0, pn, fx, fy, fz); ny = c.geo(YF_N, 1, pn, fx, fy, fz); nz = c.geo(YF_N, 2, pn, fx, fy, fz); }
            else { nx = c.geo(ZF_N, q, pn, fx, fy, fz); ny = c.geo(ZF_N, 5 + q, pn, fx, fy, fz); nz = c.geo(ZF_N, 10 + q, pn, fx, fy, fz); }
            double wt = c.geo(BW, q, pn, fx, fy, fz);
            double x = (c.geo(QP, q, pn, fx, fy, fz) - vc[0]) * obl0;
            double y = (c.geo(QP, 5 + q, pn, fx, fy, fz) - vc[1]) * obl0;
            double z = (c.geo(QP, 10 + q, pn, fx, fy, fz) - vc[2]) * obl0;
            double row[30];
            cmat_row(x, y, z, nx, ny, nz, c0, row);
            for (int t = 0; t < 30; ++t) C[f][t] = C[f][t] + wt * row[t];
            double bq = c.a(Bq, q, pn, fx, fy, fz);
            D[f] = D[f] + wt * bq;
            for (int t = 0; t < 30; ++t) A[f * 5 + q][t] = row[t];
            Bv[f * 5 + q] = bq;
          }
        }
        for (int b = 0; b < 3; ++b)
          for (int t = 0; t < 10; ++t) {
            A[30 + b * 10 + t][b * 10 + t] = 1.0;
            Bv[30 + b * 10 + t] = V(5 + b, t, i, j, k);
          }
        A[60][1] = 1.0; A[60][12] = 1.0; A[60][23] = 1.0;
        A[61][4] = 2.0; A[61][17] = 1.0; A[61][29] = 1.0;
        A[62][7] = 1.0; A[62][15] = 2.0; A[62][28] = 1.0;
        A[63][9] = 1.0; A[63][18] = 1.0; A[63][26] = 2.0;
        double K[36 * 36], rhs[36], sol[36];
        int piv[36];
        for (int a2 = 0; a2 < 30; ++a2) {
          for (int b2 = 0; b2 < 30; ++b2) {
            double s = 0.0;
            for (int r = 0; r < 64; ++r) s = s + A[r][a2] * A[r][b2];
            K[a2 * 36 + b2] = s;
          }
          for (int f = 0; f < 6; ++f) K[a2 * 36 + 30 + f] = C[f][a2];
          double s = 0.0;
          for (int r = 0; r < 64; ++r) s = s + A[r][a2] * Bv[r];
          rhs[a2] = s;
        }
        for (int f = 0; f < 6; ++f) {
          for (int b2 = 0; b2 < 30; ++b2) K[(30 + f) * 36 + b2] = C[f][b2];
          for (int b2 = 0; b2 < 6; ++b2) K[(30 + f) * 36 + 30 + b2] = 0.0;
          rhs[30 + f] = D[f];
        }
        lu_factor(36, K, piv);
        lu_solve(36, K, piv, rhs, sol);
        double aa = (sq(c.a(c.U, 5, pn, i, j, k)) + sq(c.a(c.U, 6, pn, i, j, k)) + sq(c.a(c.U, 7, pn, i, j, k))) * c.ph.ob8pi;
        for (int b = 0; b < 3; ++b) {
          for (int t = 0; t < 10; ++t) V(5 + b, t, i, j, k) = sol[b * 10 + t];
          c.a(c.U, 5 + b, pn, i, j, k) = V(5 + b, 0, i, j, k);
        }
        double bb = (sq(c.a(c.U, 5, pn, i, j, k)) + sq(c.a(c.U, 6, pn, i, j, k)) + sq(c.a(c.U, 7, pn, i, j, k))) * c.ph.ob8pi;
        c.a(c.U, 4, pn, i, j, k) = c.a(c.U, 4, pn, i, j, k) - aa + bb;
      }
  // STEP 9.a zone-centred E = -v x B at the centroid (:6700-6790)
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        double co[10];
        coef_at(c, pn, i, j, k, co);
        auto pt = [&](int q) {
          double s = V(q, 0, i, j, k);
          for (int t = 4; t < 10; ++t) s = s - V(q, t, i, j, k) * co[t];
          return s;
        };
        double Bx = pt(5), By = pt(6), Bz = pt(7), vx = pt(1), vy = pt(2), vz = pt(3);
        for (int t = 0; t < 30; ++t) c.a(c.E, t, pn, i, j, k) = 0.0;
        E(0, 0, i, j, k) = -(vy * Bz - vz * By);
        E(1, 0, i, j, k) = -(vz * Bx - vx * Bz);
        E(2, 0, i, j, k) = -(vx * By - vy * Bx);
      }
  // CS_FLAG_P2: STEP 9.b of LIMIT_ALL_SLOPES_P2 in place of STEPS 9.b and 9.c
  if (p2) p2_limit_efield(c, pn);
  if (!p2) {  // P12 STEPS 9.b, 9.c
  // STEP 9.b WENO gradients of E (:6840-8400)
  OMP_ZONES
  for (int k = 2 - G; k <= nr + G - 1; ++k)
    for (int j = 2 - G; j <= N + G - 1; ++j)
      for (int i = 2 - G; i <= N + G - 1; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        Nb n = nbrs(c, pn, i, j);
        double Ai[8][3][3];
        stencil_inverses(c, pn, i, j, k, n, Ai);
        for (int q = 0; q < 3; ++q) {
          double gr[3];
          weno8(c, n, i, j, k, Ai, [&](int x, int y, int z) { return E(q, 0, x, y, z); }, gr);
          E(q, 1, i, j, k) = gr[0];
          E(q, 2, i, j, k) = gr[1];
          E(q, 3, i, j, k) = gr[2];
        }
      }
  // STEP 9.c point-value (FD) WENO hybridisation of E (:8464-9350).  Each
  // zone rewrites its own point value; neighbours are read from the values
  // before the loop (parallel-loop semantics, order-free).
  std::vector<double> esnap(3 * c.S);
  for (int q = 0; q < 3; ++q)
    std::memcpy(&esnap[(size_t)q * c.S], &c.E[((size_t)q * 6 + pn) * c.S], c.S * sizeof(double));
  auto E1s = [&](int q, int x, int y, int z) { return esnap[(size_t)q * c.S + c.idx(x, y, z)]; };
  OMP_ZONES
  for (int k = 3 - G; k <= nr + G - 2; ++k)
    for (int j = 3 - G; j <= N + G - 2; ++j)
      for (int i = 3 - G; i <= N + G - 2; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        Nb n = nbrs(c, pn, i, j);
        double obl0 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, i, j, k), sm);
        double c0[10];
        coef_at(c, pn, i, j, k, c0);
        double A[19][10];
        int zx[19], zy[19], zz[19];
        zx[0] = i; zy[0] = j; zz[0] = k;
        interp_row(0.0, 0.0, 0.0, c0, A[0]);
        for (int r = 0; r < 18; ++r) {
          int w = kN18[r][0], dz = kN18[r][1];
          zx[r + 1] = (w < 0) ? i : n.x[w];
          zy[r + 1] = (w < 0) ? j : n.y[w];
          zz[r + 1] = k + dz;
          double x = (c.geo(V_CEN, 0, pn, zx[r + 1], zy[r + 1], zz[r + 1]) - c.geo(V_CEN, 0, pn, i, j, k)) * obl0;
          double y = (c.geo(V_CEN, 1, pn, zx[r + 1], zy[r + 1], zz[r + 1]) - c.geo(V_CEN, 1, pn, i, j, k)) * obl0;
          double z = (c.geo(V_CEN, 2, pn, zx[r + 1], zy[r + 1], zz[r + 1]) - c.geo(V_CEN, 2, pn, i, j, k)) * obl0;
          interp_row(x, y, z, c0, A[r + 1]);
        }
        double M[100], Minv[100];
        for (int a2 = 0; a2 < 10; ++a2)
          for (int b2 = 0; b2 < 10; ++b2) {
            double s = 0.0;
            for (int r = 0; r < 19; ++r) s = s + A[r][a2] * A[r][b2];
            M[a2 * 10 + b2] = s;
          }
        matinv(10, M, Minv);
        double f = c.a(c.flat, 0, pn, i, j, k);
        for (int q = 0; q < 3; ++q) {
          double Ept = E1s(q, i, j, k);
          double R[19], Y[10], X[10];
          for (int r = 0; r < 19; ++r) R[r] = E1s(q, zx[r], zy[r], zz[r]);
          for (int a2 = 0; a2 < 10; ++a2) {
            double s = 0.0;
            for (int r = 0; r < 19; ++r) s = s + A[r][a2] * R[r];
            Y[a2] = s;
          }
          for (int a2 = 0; a2 < 10; ++a2) {
            double s = 0.0;
            for (int b2 = 0; b2 < 10; ++b2) s = s + Minv[a2 * 10 + b2] * Y[b2];
            X[a2] = s;
          }
          double betalo = f + (1.0 - f) * 2.0;
          double ghi = f * 0.6 + (1.0 - f) * 0.95, glo = 1.0 - ghi, obghi = 1.0 / ghi, grat = glo / ghi;
          double e[10];
          for (int t = 0; t < 10; ++t) e[t] = E(q, t, i, j, k);
          e[0] = Ept;
          double ISlo = betalo * (e[1] * e[1] + e[2] * e[2] + e[3] * e[3]) * ob12;
          double Phi[10];
          for (int t = 0; t < 4; ++t) Phi[t] = X[t] * obghi - e[t] * grat;
          for (int t = 4; t < 10; ++t) Phi[t] = X[t] * obghi;
          double IShi = (Phi[1] * Phi[1] + Phi[2] * Phi[2] + Phi[3] * Phi[3]) * ob12 +
                        (Phi[4] * Phi[4]) * (sq(c0[4] - ob12) + ob180) + (Phi[5] * Phi[5]) * (sq(c0[5] - ob12) + ob180) +
                        (Phi[6] * Phi[6]) * (sq(c0[6] - ob12) + ob180) + (Phi[7] * Phi[7]) * (c0[7] * c0[7] + ob144) +
                        (Phi[8] * Phi[8]) * (c0[8] * c0[8] + ob144) + (Phi[9] * Phi[9]) * (c0[9] * c0[9] + ob144);
          double tau = std::fabs(IShi - ISlo);
          double Wlo = glo * (1.0 + tau / (ISlo + sm)), Whi = ghi * (1.0 + tau / (IShi + sm));
          double aa = 1.0 / (Wlo + Whi);
          Wlo = Wlo * aa;
          Whi = Whi * aa;
          for (int t = 0; t < 4; ++t) e[t] = Whi * Phi[t] + Wlo * e[t];
          for (int t = 4; t < 10; ++t) e[t] = Whi * Phi[t];
          double x = 1.0 - f;
          e[0] = Ept * f + e[0] * x;
          for (int t = 1; t < 10; ++t) e[t] = e[t] * x;
          for (int t = 0; t < 10; ++t) E(q, t, i, j, k) = e[t];
        }
      }
  }  // P12 STEPS 9.b, 9.c
  // STEP 10 (:9354-9976): min and max over the active interior zones of the
  // zone primitives (B from STEP 8.d) and of the zone's net face flux of B
  // over max(|B| of the upper faces, |B| of the lower faces,
  // msonic sqrt(4 x 3.14 x rho)), with msonic from these primitives.
  for (int q = 0; q <= NV; ++q) {
    c.vmin[pn][q] = 1.0e30;
    c.vmax[pn][q] = -1.0e30;
  }
  for (int k = 1; k <= nr; ++k)
    for (int j = 1; j <= N; ++j)
      for (int i = 1; i <= N; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        for (int q = 0; q < NV; ++q) {
          c.vmin[pn][q] = std::min(c.vmin[pn][q], V(q, 0, i, j, k));
          c.vmax[pn][q] = std::max(c.vmax[pn][q], V(q, 0, i, j, k));
        }
        auto B = [&](std::vector<double>& f, int x, int y, int z) { return c.a(f, 0, pn, x, y, z); };
        double a21 = c.geo(XF_AREA, 0, pn, i, j, k) * B(c.Bxf, i, j, k) + c.geo(YF_AREA, 0, pn, i, j, k) * B(c.Byf, i, j, k) +
                     c.geo(ZF_AREA, 0, pn, i, j, k) * B(c.Bzf, i, j, k) -
                     c.geo(XF_AREA, 0, pn, i - 1, j, k) * B(c.Bxf, i - 1, j, k) -
                     c.geo(YF_AREA, 0, pn, i, j - 1, k) * B(c.Byf, i, j - 1, k) -
                     c.geo(ZF_AREA, 0, pn, i, j, k - 1) * B(c.Bzf, i, j, k - 1);
        double a11 = sq(V(5, 0, i, j, k)) + sq(V(6, 0, i, j, k)) + sq(V(7, 0, i, j, k));
        double ms = std::sqrt((g * V(4, 0, i, j, k) + c.ph.ob4pi * a11) / V(0, 0, i, j, k));
        a21 = a21 / std::max({std::sqrt(sq(B(c.Bxf, i, j, k)) + sq(B(c.Byf, i, j, k)) + sq(B(c.Bzf, i, j, k))),
                              std::sqrt(sq(B(c.Bxf, i - 1, j, k)) + sq(B(c.Byf, i, j - 1, k)) + sq(B(c.Bzf, i, j, k - 1))),
                              ms * std::sqrt(4.0 * 3.14 * V(0, 0, i, j, k))});
        c.vmin[pn][NV] = std::min(c.vmin[pn][NV], a21);
        c.vmax[pn][NV] = std::max(c.vmax[pn][NV], a21);
      }
  c.step10 = true;
}

// ------------------------------------------------------------------
// MAKE_FACIAL_FLUXES (400riemann_integrate/450make_facial_fluxes.f:405-2933), one panel.
void make_facial_fluxes(Ctx& c, int pn) {
  const int N = c.N, nr = c.nr;
  const double sm = c.p.smallnum;
  auto V = [&](int comp, int mode, int i, int j, int k) -> double& { return c.a(c.V, mode * NV + comp, pn, i, j, k); };
  for (int dir = 0; dir < 3; ++dir) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int t = 0; t < 5 * NV; ++t)
      for (long long o = 0; o < (long long)c.S; ++o) {
        c.cL[dir][((size_t)t * 6 + pn) * c.S + o] = 0.0;
        c.cR[dir][((size_t)t * 6 + pn) * c.S + o] = 0.0;
      }
#pragma omp parallel for schedule(static)
    for (long long o = 0; o < (long long)c.S; ++o) {
      c.tL[dir][(size_t)pn * c.S + o] = -1;
      c.tR[dir][(size_t)pn * c.S + o] = -1;
    }
  }
  for (int dir = 0; dir < 3; ++dir) {
    const int QP = dir == 0 ? XF_QP : (dir == 1 ? YF_QP : ZF_QP);
    const int QW = dir == 0 ? XF_QW : (dir == 1 ? YF_QW : ZF_QW);
    const int AR = dir == 0 ? XF_AREA : (dir == 1 ? YF_AREA : ZF_AREA);
    std::vector<double>& SLo = dir == 0 ? c.SLx : (dir == 1 ? c.SDy : c.SBz);
    std::vector<double>& SHi = dir == 0 ? c.SRx : (dir == 1 ? c.SUy : c.STz);
    std::vector<double>& EF = dir == 0 ? c.EFx : (dir == 1 ? c.EFy : c.EFz);
    int lo[3] = {0, 0, 0}, hi[3] = {N + 1, N + 1, nr + 1};
    lo[dir] = -1;
    for (int jq = 0; jq < 5; ++jq) {
      OMP_ZONES
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            int lx, ly, rx, ry, lz = k, rz = k;
            if (dir == 0) {
              int mL = c.m(pn, i, j), mR = c.m(pn, i + 1, j);
              if (mL == 1 && mR == 1) { lx = i; ly = j; rx = i + 1; ry = j; }
              else if (mL == 0 && mR == 1) { rx = i + 1; ry = j; lx = c.sti(pn, rx, ry, 1, 0); ly = c.sti(pn, rx, ry, 1, 1); }
              else if (mL == 1 && mR == 0) { lx = i; ly = j; rx = c.sti(pn, lx, ly, 0, 0); ry = c.sti(pn, lx, ly, 0, 1); }
              else continue;
            } else if (dir == 1) {
              int mL = c.m(pn, i, j), mR = c.m(pn, i, j + 1);
              if (mL == 1 && mR == 1) { lx = i; ly = j; rx = i; ry = j + 1; }
              else if (mL == 0 && mR == 1) { rx = i; ry = j + 1; lx = c.sti(pn, rx, ry, 3, 0); ly = c.sti(pn, rx, ry, 3, 1); }
              else if (mL == 1 && mR == 0) { lx = i; ly = j; rx = c.sti(pn, lx, ly, 2, 0); ry = c.sti(pn, lx, ly, 2, 1); }
              else continue;
            } else {
              if (c.m(pn, i, j) == 0) continue;
              lx = rx = i;
              ly = ry = j;
              rz = k + 1;
            }
            double obl0 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, lx, ly, lz), sm);
            double obl02 = 1.0 / std::max(c.geo(V_SCALE, 0, pn, rx, ry, rz), sm);
            double Ax, Ay, Az, Bx, By, Bz, Cx, Cy, Cz;
            if (dir == 0) {
              Ax = c.geo(XF_N, 0, pn, i, j, k); Ay = c.geo(XF_N, 1, pn, i, j, k); Az = c.geo(XF_N, 2, pn, i, j, k);
              Cx = c.geo(XF_CEN, 0, pn, i, j, k); Cy = c.geo(XF_CEN, 1, pn, i, j, k); Cz = c.geo(XF_CEN, 2, pn, i, j, k);
              double t = 1.0 / std::max(std::sqrt(Cx * Cx + Cy * Cy + Cz * Cz), sm);
              Cx = Cx * t; Cy = Cy * t; Cz = Cz * t;
              Bx = Cy * Az - Cz * Ay; By = Cz * Ax - Cx * Az; Bz = Cx * Ay - Cy * Ax;
            } else if (dir == 1) {
              Ax = c.geo(YF_N, 0, pn, i, j, k); Ay = c.geo(YF_N, 1, pn, i, j, k); Az = c.geo(YF_N, 2, pn, i, j, k);
              Bx = c.geo(YF_CEN, 0, pn, i, j, k); By = c.geo(YF_CEN, 1, pn, i, j, k); Bz = c.geo(YF_CEN, 2, pn, i, j, k);
              double t = 1.0 / std::max(std::sqrt(Bx * Bx + By * By + Bz * Bz), sm);
              Bx = Bx * t; By = By * t; Bz = Bz * t;
              Cx = Ay * Bz - Az * By; Cy = Az * Bx - Ax * Bz; Cz = Ax * By - Ay * Bx;
            } else {
              Ax = c.geo(ZF_N, jq, pn, i, j, k); Ay = c.geo(ZF_N, 5 + jq, pn, i, j, k); Az = c.geo(ZF_N, 10 + jq, pn, i, j, k);
              double t = 1.0 / std::max(std::sqrt(Ax * Ax + Ay * Ay + Az * Az), sm);
              Ax = Ax * t; Ay = Ay * t; Az = Az * t;
              auto vt = [&](int q, int x, int y) { return c.geo(G_VERT, q, pn, x, y, k); };
              Bx = vt(0, i, j) + vt(0, i, j - 1) - vt(0, i - 1, j) - vt(0, i - 1, j - 1);
              By = vt(1, i, j) + vt(1, i, j - 1) - vt(1, i - 1, j) - vt(1, i - 1, j - 1);
              Bz = vt(2, i, j) + vt(2, i, j - 1) - vt(2, i - 1, j) - vt(2, i - 1, j - 1);
              t = Bx * Ax + By * Ay + Bz * Az;
              Bx = Bx - t * Ax; By = By - t * Ay; Bz = Bz - t * Az;
              t = 1.0 / std::max(std::sqrt(Bx * Bx + By * By + Bz * Bz), sm);
              Bx = Bx * t; By = By * t; Bz = Bz * t;
              Cx = Ay * Bz - Az * By; Cy = Az * Bx - Ax * Bz; Cz = Ax * By - Ay * Bx;
              t = 1.0 / std::max(std::sqrt(Cx * Cx + Cy * Cy + Cz * Cz), sm);
              Cx = Cx * t; Cy = Cy * t; Cz = Cz * t;
            }
            double px = c.geo(QP, jq, pn, i, j, k), py = c.geo(QP, 5 + jq, pn, i, j, k), pz = c.geo(QP, 10 + jq, pn, i, j, k);
            double x = (px - c.geo(V_CEN, 0, pn, lx, ly, lz)) * obl0, y = (py - c.geo(V_CEN, 1, pn, lx, ly, lz)) * obl0,
                   z = (pz - c.geo(V_CEN, 2, pn, lx, ly, lz)) * obl0;
            double x2 = (px - c.geo(V_CEN, 0, pn, rx, ry, rz)) * obl02, y2 = (py - c.geo(V_CEN, 1, pn, rx, ry, rz)) * obl02,
                   z2 = (pz - c.geo(V_CEN, 2, pn, rx, ry, rz)) * obl02;
            double wt = c.geo(QW, jq, pn, i, j, k);
            double cL[10], cR[10], VL[NV], VR[NV];
            coef_at(c, pn, lx, ly, lz, cL);
            coef_at(c, pn, rx, ry, rz, cR);
            for (int q = 0; q < NV; ++q) {
              double vl[10], vr[10];
              for (int t = 0; t < 10; ++t) {
                vl[t] = V(q, t, lx, ly, lz);
                vr[t] = V(q, t, rx, ry, rz);
              }
              VL[q] = poly10(vl, cL, x, y, z);
              VR[q] = poly10(vr, cR, x2, y2, z2);
            }
            double entL = c.a(c.ent, 0, pn, lx, ly, lz) + c.a(c.ent, 1, pn, lx, ly, lz) * x +
                          c.a(c.ent, 2, pn, lx, ly, lz) * y + c.a(c.ent, 3, pn, lx, ly, lz) * z;
            double entR = c.a(c.ent, 0, pn, rx, ry, rz) + c.a(c.ent, 1, pn, rx, ry, rz) * x2 +
                          c.a(c.ent, 2, pn, rx, ry, rz) * y2 + c.a(c.ent, 3, pn, rx, ry, rz) * z2;
            auto rot = [&](double* W, int o) {
              double a1 = Ax * W[o] + Ay * W[o + 1] + Az * W[o + 2];
              double b1 = Bx * W[o] + By * W[o + 1] + Bz * W[o + 2];
              double c1 = Cx * W[o] + Cy * W[o + 1] + Cz * W[o + 2];
              W[o] = a1; W[o + 1] = b1; W[o + 2] = c1;
            };
            rot(VL, 1); rot(VL, 5); rot(VR, 1); rot(VR, 5);
            RSOut o;
            oned_rs_hll(c.ph, VL, VR, entL, entR, o);
            if (jq == 0) {
              c.a(SLo, 0, pn, i, j, k) = o.SL;
              c.a(SHi, 0, pn, i, j, k) = o.SR;
            }
            auto back = [&](const double* W, double* Out) {
              Out[0] = W[0];
              Out[1] = Ax * W[1] + Bx * W[2] + Cx * W[3];
              Out[2] = Ay * W[1] + By * W[2] + Cy * W[3];
              Out[3] = Az * W[1] + Bz * W[2] + Cz * W[3];
              Out[4] = W[4];
              Out[5] = Ax * W[5] + Bx * W[6] + Cx * W[7];
              Out[6] = Ay * W[5] + By * W[6] + Cy * W[7];
              Out[7] = Az * W[5] + Bz * W[6] + Cz * W[7];
            };
            double Fp[NV], Fm[NV], FLL[NV], FRR[NV];
            back(o.FlR, Fp);
            back(o.FlL, Fm);
            back(o.FL, FLL);
            back(o.FR, FRR);
            double area = c.geo(AR, 0, pn, i, j, k);
            double volL = c.geo(V_VOL, 0, pn, lx, ly, lz), volR = c.geo(V_VOL, 0, pn, rx, ry, rz);
            const size_t fo = c.idx(i, j, k);
            for (int q = 0; q < NV; ++q) {
              c.cL[dir][((size_t)(jq * NV + q) * 6 + pn) * c.S + fo] = wt * (Fm[q] + FLL[q]) * area / volL;
              c.cR[dir][((size_t)(jq * NV + q) * 6 + pn) * c.S + fo] = wt * (Fp[q] - FRR[q]) * area / volR;
            }
            c.tL[dir][(size_t)pn * c.S + fo] = (long long)c.idx(lx, ly, lz);
            c.tR[dir][(size_t)pn * c.S + fo] = (long long)c.idx(rx, ry, rz);
            if (jq == 0) c.a(EF, 0, pn, i, j, k) = o.entF;
          }
    }
  }
}

// Second half of MAKE_FACIAL_FLUXES: every face's per-point contributions
// are subtracted from the time derivatives of the zones it updates, in the
// reference's order (direction, quadrature point, face).  The x and y faces
// of plane k update zones of plane k only, so whole planes go to one thread
// each and every zone still receives its terms in that order; a z face k
// updates zones k (its lower side) and k + 1 (its upper side), so each zone
// collects the upper-side term of face k - 1 and then the lower-side term of
// face k, point by point, as the face loop would apply them.
void scatter_facial_fluxes(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i)
        for (int q = 0; q < NV; ++q) c.a(c.dUdt, q, pn, i, j, k) = 0.0;
  auto sub = [&](int jq, size_t fo, long long z, const std::vector<double>& cc) {
    for (int q = 0; q < NV; ++q) {
      double& d = c.dUdt[((size_t)q * 6 + pn) * c.S + (size_t)z];
      d = d - cc[((size_t)(jq * NV + q) * 6 + pn) * c.S + fo];
    }
  };
  for (int dir = 0; dir < 2; ++dir) {
    int lo[3] = {0, 0, 0}, hi[3] = {N + 1, N + 1, nr + 1};
    lo[dir] = -1;
#pragma omp parallel for schedule(static)
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int jq = 0; jq < 5; ++jq)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            const size_t fo = c.idx(i, j, k);
            const long long l = c.tL[dir][(size_t)pn * c.S + fo], r = c.tR[dir][(size_t)pn * c.S + fo];
            if (l < 0) continue;
            sub(jq, fo, l, c.cL[dir]);
            sub(jq, fo, r, c.cR[dir]);
          }
  }
  // z faces k in [-1, nr + 1] over (i, j) in [0, N + 1]^2: lower side zone
  // (i, j, k), upper side (i, j, k + 1)
  OMP_ZONES
  for (int kz = -1; kz <= nr + 2; ++kz)
    for (int j = 0; j <= N + 1; ++j)
      for (int i = 0; i <= N + 1; ++i) {
        const long long z = (long long)c.idx(i, j, kz);
        const bool below = kz - 1 >= -1, above = kz <= nr + 1;
        const size_t fb = below ? c.idx(i, j, kz - 1) : 0, fa = above ? c.idx(i, j, kz) : 0;
        const bool ub = below && c.tL[2][(size_t)pn * c.S + fb] >= 0;
        const bool ua = above && c.tL[2][(size_t)pn * c.S + fa] >= 0;
        if (ub && c.tR[2][(size_t)pn * c.S + fb] != z) std::abort();
        if (ua && c.tL[2][(size_t)pn * c.S + fa] != z) std::abort();
        for (int jq = 0; jq < 5; ++jq) {
          if (ub) sub(jq, fb, z, c.cR[2]);
          if (ua) sub(jq, fa, z, c.cL[2]);
        }
      }
}

// ------------------------------------------------------------------
// Panel-edge ownership (the single-device counterpart of the reference's
// defect correction, DRV:3200-3461 with 485update_defect_imex_rk.f): the
// face fluxes of the faces on a panel edge and the EMFs of the edges on a
// panel boundary are computed by both panels (three at a cube corner);
// every copy takes the value of the copy owned by the lowest-numbered
// panel, so each face and edge has one value, the update is conservative
// and CT keeps div B at round-off across panel edges.
//
// Vertex identity across panels follows the ghost-fill index maps of
// FILL_GHOST2D_GLOBAL (203:104-163): right edge (N, j) ~ right neighbour
// (j, N); left (0, j) ~ (0, N - j); down (i, 0) ~ (N - i, 0); up (i, N) ~ (N, i).
static void build_sync_maps(Ctx& c) {
  const int N = c.N, nr = c.nr;
  const int NV1 = N + 1;
  std::vector<int> par((size_t)6 * NV1 * NV1);
  for (size_t t = 0; t < par.size(); ++t) par[t] = (int)t;
  auto vid = [&](int p, int i, int j) { return (p * NV1 + j) * NV1 + i; };
  std::function<int(int)> root = [&](int x) {
    while (par[x] != x) x = par[x] = par[par[x]];
    return x;
  };
  auto unite = [&](int a, int b) {
    a = root(a);
    b = root(b);
    if (a != b) par[std::max(a, b)] = std::min(a, b);
  };
  for (int p = 0; p < 6; ++p) {
    const int rt = kNbr[p][0] - 1, lf = kNbr[p][1] - 1, up = kNbr[p][2] - 1, dn = kNbr[p][3] - 1;
    for (int t = 0; t <= N; ++t) {
      unite(vid(p, N, t), vid(rt, t, N));
      unite(vid(p, 0, t), vid(lf, 0, N - t));
      unite(vid(p, t, 0), vid(dn, N - t, 0));
      unite(vid(p, t, N), vid(up, N, t));
    }
  }
  // check the identities against the vertex coordinates
  for (int p = 0; p < 6; ++p)
    for (int j = 0; j <= N; ++j)
      for (int i = 0; i <= N; ++i) {
        const int r = root(vid(p, i, j));
        const int rp = r / (NV1 * NV1), ri = r % NV1, rj = (r / NV1) % NV1;
        for (int q = 0; q < 3; ++q) {
          const double a = c.geo(G_VERT, q, p, i, j, 0), b = c.geo(G_VERT, q, rp, ri, rj, 0);
          if (std::fabs(a - b) > 1e-9 * (std::fabs(c.geo(G_VERT, 0, p, i, j, 0)) + std::fabs(c.geo(G_VERT, 1, p, i, j, 0)) +
                                          std::fabs(c.geo(G_VERT, 2, p, i, j, 0)))) {
            std::fprintf(stderr, "oracle: panel-edge vertex map mismatch at panel %d (%d,%d)\n", p, i, j);
            std::abort();
          }
        }
      }
  // faces on panel edges: (p, dir, i, j) ~ partner, k = 1..nr; the copy of
  // the higher-numbered panel takes the owner's values
  c.fsync.clear();
  for (int p = 0; p < 6; ++p) {
    const int rt = kNbr[p][0] - 1, lf = kNbr[p][1] - 1, up = kNbr[p][2] - 1, dn = kNbr[p][3] - 1;
    for (int t = 1; t <= N; ++t)
      for (int k = 1; k <= nr; ++k) {
        const Ctx::FaceSync cand[4] = {{0, p, N, t, k, 1, rt, t, N, k},
                                       {0, p, 0, t, k, 0, lf, 0, N + 1 - t, k},
                                       {1, p, t, 0, k, 1, dn, N + 1 - t, 0, k},
                                       {1, p, t, N, k, 0, up, N, t, k}};
        for (const auto& f : cand)
          if (f.opn < f.pn) c.fsync.push_back(f);
      }
  }
  // edges on panel boundaries, grouped by their end vertices
  struct Copy { int f, p, i, j, k, a, b; };  // a -> b: vertex roots in the edge's direction
  std::map<std::tuple<int, int, int>, std::vector<Copy>> cls;
  for (int p = 0; p < 6; ++p) {
    for (int j = 0; j <= N; ++j)
      for (int i = 0; i <= N; ++i) {
        const bool bnd = i == 0 || i == N || j == 0 || j == N;
        if (!bnd) continue;
        for (int k = 1; k <= nr; ++k) {
          const int r = root(vid(p, i, j));
          cls[std::make_tuple(r, -1, k)].push_back({2, p, i, j, k, r, r});
        }
      }
    for (int k = 0; k <= nr; ++k) {
      for (int i : {0, N})
        for (int j = 1; j <= N; ++j) {
          const int a = root(vid(p, i, j - 1)), b = root(vid(p, i, j));
          cls[std::make_tuple(std::min(a, b), std::max(a, b), k)].push_back({1, p, i, j, k, a, b});
        }
      for (int j : {0, N})
        for (int i = 1; i <= N; ++i) {
          const int a = root(vid(p, i - 1, j)), b = root(vid(p, i, j));
          cls[std::make_tuple(std::min(a, b), std::max(a, b), k)].push_back({0, p, i, j, k, a, b});
        }
    }
  }
  c.esync.clear();
  c.eclass.clear();
  for (auto& kv : cls) {
    auto& v = kv.second;
    if (v.size() < 2) {
      std::fprintf(stderr, "oracle: unshared panel-boundary edge\n");
      std::abort();
    }
    std::sort(v.begin(), v.end(), [](const Copy& x, const Copy& y) { return x.p < y.p; });
    const Copy& o = v[0];
    c.eclass.push_back(c.esync.size());
    for (size_t m = 1; m < v.size(); ++m) {
      const Copy& x = v[m];
      const int sign = (x.a == o.a && x.b == o.b) ? 1 : -1;
      c.esync.push_back({x.f, x.p, x.i, x.j, x.k, o.f, o.p, o.i, o.j, o.k, sign});
    }
  }
  c.eclass.push_back(c.esync.size());
  c.maps_built = true;
}

static bool sync_on(const Ctx& c) { return !(c.p.flags & CS_FLAG_NO_PANEL_SYNC); }

// Non-owner copies of panel-edge faces take the owner's contributions with
// the two sides exchanged (the normals are opposite) and the negated
// entropy flux.
//
// With panel_rule 1 the copies take their average instead, as in the
// reference's defect correction: FETCH_BUFFERS_FILL_IN_FLUX_X / _Y set each
// coinciding face's fluctuations and entropy flux and each coinciding edge's
// EMF to (own + neighbour's) * 0.5 (334fetch_buffers_fill_in_flux_x.f:295-309,
// :341-350, :384-395, 335 likewise), the three copies of a cube-corner radial
// edge to their sum / 3 (335:761-795), and UPDATE_DEFECT_IMEX_RK applies the
// differences from the per-panel values with the stage's dtmove
// (1000riemann_geomesh_cs_mhd.f:2777, :3200-3470), which is the update with
// the averages up to round-off.
void sync_facial_fluxes(Ctx& c) {
  if (!sync_on(c)) return;
  if (!c.maps_built) build_sync_maps(c);
  if (c.panel_rule == 1) {
    for (const auto& f : c.fsync) {
      const size_t d = c.idx(f.i, f.j, f.k), o = c.idx(f.oi, f.oj, f.ok);
      for (int t = 0; t < 5 * NV; ++t) {
        double& Ld = c.cL[f.dir][((size_t)t * 6 + f.pn) * c.S + d];
        double& Rd = c.cR[f.dir][((size_t)t * 6 + f.pn) * c.S + d];
        double& Lo = c.cL[f.odir][((size_t)t * 6 + f.opn) * c.S + o];
        double& Ro = c.cR[f.odir][((size_t)t * 6 + f.opn) * c.S + o];
        const double a = (Ld + Ro) * 0.5, b = (Rd + Lo) * 0.5;
        Ld = Ro = a;
        Rd = Lo = b;
      }
      std::vector<double>& EFd = f.dir == 0 ? c.EFx : (f.dir == 1 ? c.EFy : c.EFz);
      std::vector<double>& EFo = f.odir == 0 ? c.EFx : (f.odir == 1 ? c.EFy : c.EFz);
      const double a = (EFd[(size_t)f.pn * c.S + d] - EFo[(size_t)f.opn * c.S + o]) * 0.5;
      EFd[(size_t)f.pn * c.S + d] = a;
      EFo[(size_t)f.opn * c.S + o] = -a;
    }
    return;
  }
  for (const auto& f : c.fsync) {
    const size_t d = c.idx(f.i, f.j, f.k), o = c.idx(f.oi, f.oj, f.ok);
    for (int t = 0; t < 5 * NV; ++t) {
      c.cL[f.dir][((size_t)t * 6 + f.pn) * c.S + d] = c.cR[f.odir][((size_t)t * 6 + f.opn) * c.S + o];
      c.cR[f.dir][((size_t)t * 6 + f.pn) * c.S + d] = c.cL[f.odir][((size_t)t * 6 + f.opn) * c.S + o];
    }
    std::vector<double>& EFd = f.dir == 0 ? c.EFx : (f.dir == 1 ? c.EFy : c.EFz);
    const std::vector<double>& EFo = f.odir == 0 ? c.EFx : (f.odir == 1 ? c.EFy : c.EFz);
    EFd[(size_t)f.pn * c.S + d] = -EFo[(size_t)f.opn * c.S + o];
  }
}

void sync_edge_efields(Ctx& c) {
  if (!sync_on(c)) return;
  if (!c.maps_built) build_sync_maps(c);
  auto E = [&](int f) -> std::vector<double>& { return f == 0 ? c.Efx : (f == 1 ? c.Efy : c.Efz); };
  if (c.panel_rule == 1) {
    for (size_t q = 0; q + 1 < c.eclass.size(); ++q) {
      const Ctx::EdgeSync& h = c.esync[c.eclass[q]];
      double& Eo = E(h.of)[(size_t)h.opn * c.S + c.idx(h.oi, h.oj, h.ok)];
      double sum = Eo;
      for (size_t m = c.eclass[q]; m < c.eclass[q + 1]; ++m) {
        const Ctx::EdgeSync& e = c.esync[m];
        sum += e.sign * E(e.f)[(size_t)e.pn * c.S + c.idx(e.i, e.j, e.k)];
      }
      const double avg = c.eclass[q + 1] - c.eclass[q] == 1 ? sum * 0.5 : sum / 3.0;
      Eo = avg;
      for (size_t m = c.eclass[q]; m < c.eclass[q + 1]; ++m) {
        const Ctx::EdgeSync& e = c.esync[m];
        E(e.f)[(size_t)e.pn * c.S + c.idx(e.i, e.j, e.k)] = e.sign * avg;
      }
    }
    return;
  }
  for (const auto& e : c.esync) {
    std::vector<double>& Ed = e.f == 0 ? c.Efx : (e.f == 1 ? c.Efy : c.Efz);
    const std::vector<double>& Eo = e.of == 0 ? c.Efx : (e.of == 1 ? c.Efy : c.Efz);
    Ed[(size_t)e.pn * c.S + c.idx(e.i, e.j, e.k)] = e.sign * Eo[(size_t)e.opn * c.S + c.idx(e.oi, e.oj, e.ok)];
  }
}

// ------------------------------------------------------------------
// MAKE_EDGE_EFIELDS_P1 with USE_2D_LLF_RS_FOR_EZ = 1
// (400riemann_integrate/460make_edge_fields_p1.f:335-7037), one panel.
void make_edge_efields(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  auto E1 = [&](int q, int x, int y, int z) { return c.a(c.E, q, pn, x, y, z); };  // mode 1
  auto vt = [&](int q, int x, int y, int z) { return c.geo(G_VERT, q, pn, x, y, z); };
  auto Bq = [&](std::vector<double>& B, int q, int x, int y, int z) { return c.a(B, q, pn, x, y, z); };
  auto S = [&](std::vector<double>& s, int x, int y, int z) { return c.a(s, 0, pn, x, y, z); };
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        c.a(c.Efx, 0, pn, i, j, k) = 0.0;
        c.a(c.Efy, 0, pn, i, j, k) = 0.0;
        c.a(c.Efz, 0, pn, i, j, k) = 0.0;
      }
  // Simpson point on the edge a-b: centre rescaled to |a| for angular edges.
  auto edge_pt = [&](int jq, int ax, int ay, int az, int bx, int by, int bz, bool rescale, double* e) {
    if (jq == 0) {
      for (int q = 0; q < 3; ++q) e[q] = 0.5 * (vt(q, ax, ay, az) + vt(q, bx, by, bz));
      if (rescale) {
        double t = std::sqrt(sq(vt(0, ax, ay, az)) + sq(vt(1, ax, ay, az)) + sq(vt(2, ax, ay, az))) /
                   std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        for (int q = 0; q < 3; ++q) e[q] = e[q] * t;
      }
    } else if (jq == 1) {
      for (int q = 0; q < 3; ++q) e[q] = vt(q, ax, ay, az);
    } else {
      for (int q = 0; q < 3; ++q) e[q] = vt(q, bx, by, bz);
    }
  };
  auto unit = [](double* v) {
    double t = 1.0 / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int q = 0; q < 3; ++q) v[q] = v[q] * t;
  };
  auto orth = [&](double* v, const double* n) {
    double t = v[0] * n[0] + v[1] * n[1] + v[2] * n[2];
    for (int q = 0; q < 3; ++q) v[q] = v[q] - t * n[q];
    unit(v);
  };
  auto avg4 = [&](int q, const int z[4][3]) {
    return (E1(q, z[0][0], z[0][1], z[0][2]) + E1(q, z[1][0], z[1][1], z[1][2]) + E1(q, z[2][0], z[2][1], z[2][2]) +
            E1(q, z[3][0], z[3][1], z[3][2])) * 0.25;
  };
  auto llf = [](double& SR, double& SL, double& SU, double& SD) {
    double t = std::max({std::fabs(SR), std::fabs(SL), std::fabs(SU), std::fabs(SD)});
    SR = t; SL = -t; SU = t; SD = -t;
  };
  for (int jq = 0; jq < 3; ++jq) {
    double wt = (jq == 0) ? 4.0 / 6.0 : 1.0 / 6.0;
    // x-edges (:393-1493): zones LD (i,j,k), RD (i,j+1,k), RU (i,j+1,k+1), LU (i,j,k+1)
    OMP_ZONES
    for (int k = 0; k <= nr; ++k)
      for (int j = 0; j <= N; ++j)
        for (int i = 1; i <= N; ++i) {
          double e[3], n2[3], n3[3];
          edge_pt(jq, i, j, k, i - 1, j, k, true, e);
          for (int q = 0; q < 3; ++q) n2[q] = e[q];
          unit(n2);
          for (int q = 0; q < 3; ++q) n3[q] = vt(q, i, j, k) - vt(q, i - 1, j, k);
          orth(n3, n2);
          const int z[4][3] = {{i, j, k}, {i, j + 1, k}, {i, j + 1, k + 1}, {i, j, k + 1}};
          double Ex = avg4(0, z), Ey = avg4(1, z), Ez = avg4(2, z);
          double Ezl = Ex * n3[0] + Ey * n3[1] + Ez * n3[2];
          double ByR = Bq(c.Bqz, 4, i, j + 1, k), ByL = Bq(c.Bqz, 3, i, j, k);
          double BnU = Bq(c.Bqy, 2, i, j, k + 1), BnD = Bq(c.Bqy, 1, i, j, k);
          double SR = std::max(S(c.SUy, i, j, k + 1), S(c.SUy, i, j, k));
          double SL = std::min(S(c.SDy, i, j, k + 1), S(c.SDy, i, j, k));
          double SU = std::max(S(c.STz, i, j + 1, k), S(c.STz, i, j, k));
          double SD = std::min(S(c.SBz, i, j + 1, k), S(c.SBz, i, j, k));
          llf(SR, SL, SU, SD);
          double ess = twod_rs_ez_4state(SR, SL, SU, SD, 0.0, 1.0, Ezl, Ezl, Ezl, Ezl, BnU, BnD, ByR, ByL);
          c.a(c.Efx, 0, pn, i, j, k) = c.a(c.Efx, 0, pn, i, j, k) + wt * ess;
        }
    // y-edges (:1497-2587): LD (i,j,k), RD (i,j,k+1), LU (i+1,j,k), RU (i+1,j,k+1)
    OMP_ZONES
    for (int k = 0; k <= nr; ++k)
      for (int i = 0; i <= N; ++i)
        for (int j = 1; j <= N; ++j) {
          double e[3], n1[3], n3[3];
          edge_pt(jq, i, j, k, i, j - 1, k, true, e);
          for (int q = 0; q < 3; ++q) n1[q] = e[q];
          unit(n1);
          for (int q = 0; q < 3; ++q) n3[q] = vt(q, i, j, k) - vt(q, i, j - 1, k);
          orth(n3, n1);
          const int z[4][3] = {{i, j, k}, {i, j, k + 1}, {i + 1, j, k + 1}, {i + 1, j, k}};
          double Ex = avg4(0, z), Ey = avg4(1, z), Ez = avg4(2, z);
          double Ezl = Ex * n3[0] + Ey * n3[1] + Ez * n3[2];
          double ByR = Bq(c.Bqx, 4, i, j, k + 1), ByL = Bq(c.Bqx, 3, i, j, k);
          double BnU = Bq(c.Bqz, 2, i + 1, j, k), BnD = Bq(c.Bqz, 1, i, j, k);
          double SR = std::max(S(c.STz, i + 1, j, k), S(c.STz, i, j, k));
          double SL = std::min(S(c.SBz, i + 1, j, k), S(c.SBz, i, j, k));
          double SU = std::max(S(c.SRx, i, j, k), S(c.SRx, i, j, k + 1));
          double SD = std::min(S(c.SLx, i, j, k), S(c.SLx, i, j, k + 1));
          llf(SR, SL, SU, SD);
          double ess = twod_rs_ez_4state(SR, SL, SU, SD, 0.0, 1.0, Ezl, Ezl, Ezl, Ezl, BnU, BnD, ByR, ByL);
          c.a(c.Efy, 0, pn, i, j, k) = c.a(c.Efy, 0, pn, i, j, k) + wt * ess;
        }
    // z-edges (:2591-3721): LD (i,j,k), RD (i+1,j,k), RU (i+1,j+1,k), LU (i,j+1,k)
    OMP_ZONES
    for (int i = 0; i <= N; ++i)
      for (int j = 0; j <= N; ++j)
        for (int k = 1; k <= nr; ++k) {
          if (c.m(pn, i, j) == 0 || c.m(pn, i + 1, j) == 0 || c.m(pn, i + 1, j + 1) == 0 || c.m(pn, i, j + 1) == 0) continue;
          double e[3], n1[3], n3[3], tau[3];
          edge_pt(jq, i, j, k, i, j, k - 1, false, e);
          for (int q = 0; q < 3; ++q) n3[q] = e[q];
          unit(n3);
          for (int q = 0; q < 3; ++q) n1[q] = vt(q, i + 1, j, k) - vt(q, i - 1, j, k);
          orth(n1, n3);
          for (int q = 0; q < 3; ++q) tau[q] = vt(q, i, j + 1, k) - vt(q, i, j - 1, k);
          orth(tau, n3);
          double cos_t = tau[0] * n1[0] + tau[1] * n1[1] + tau[2] * n1[2];
          double sin_t = std::sqrt(1.0 - cos_t * cos_t);
          const int z[4][3] = {{i, j, k}, {i + 1, j, k}, {i + 1, j + 1, k}, {i, j + 1, k}};
          double Ex = avg4(0, z), Ey = avg4(1, z), Ez = avg4(2, z);
          double Ezl = Ex * n3[0] + Ey * n3[1] + Ez * n3[2];
          double ByR = Bq(c.Bqy, 4, i + 1, j, k), ByL = Bq(c.Bqy, 3, i, j, k);
          double BnU = Bq(c.Bqx, 2, i, j + 1, k), BnD = Bq(c.Bqx, 1, i, j, k);
          double SR = std::max(S(c.SRx, i, j + 1, k), S(c.SRx, i, j, k));
          double SL = std::min(S(c.SLx, i, j + 1, k), S(c.SLx, i, j, k));
          double SU = std::max(S(c.SUy, i + 1, j, k), S(c.SUy, i, j, k));
          double SD = std::min(S(c.SDy, i + 1, j, k), S(c.SDy, i, j, k));
          llf(SR, SL, SU, SD);
          double ess = twod_rs_ez_4state(SR, SL, SU, SD, cos_t, sin_t, Ezl, Ezl, Ezl, Ezl, BnU, BnD, ByR, ByL);
          c.a(c.Efz, 0, pn, i, j, k) = c.a(c.Efz, 0, pn, i, j, k) + wt * ess;
        }
    // tri-corner z-edges (:3725-7037) with the 3-state solver.
    for (int corner = 0; corner < 4; ++corner) {
      int i = (corner == 1 || corner == 2) ? N : 0, j = (corner >= 2) ? N : 0;
      int z1[2], z2[2], z3[2];
      if (corner == 0) { z1[0] = i + 1; z1[1] = j + 1; z2[0] = i; z2[1] = j + 1; z3[0] = i + 1; z3[1] = j; }
      else if (corner == 1) { z1[0] = i + 1; z1[1] = j + 1; z2[0] = i; z2[1] = j + 1; z3[0] = i; z3[1] = j; }
      else if (corner == 2) { z1[0] = i; z1[1] = j + 1; z2[0] = i; z2[1] = j; z3[0] = i + 1; z3[1] = j; }
      else { z1[0] = i + 1; z1[1] = j + 1; z2[0] = i; z2[1] = j; z3[0] = i + 1; z3[1] = j; }
      for (int k = 1; k <= nr; ++k) {
        double e[3], n3[3];
        edge_pt(jq, i, j, k, i, j, k - 1, false, e);
        for (int q = 0; q < 3; ++q) n3[q] = e[q];
        unit(n3);
        double Ex = (E1(0, z1[0], z1[1], k) + E1(0, z2[0], z2[1], k) + E1(0, z3[0], z3[1], k)) * (1.0 / 3.0);
        double Ey = (E1(1, z1[0], z1[1], k) + E1(1, z2[0], z2[1], k) + E1(1, z3[0], z3[1], k)) * (1.0 / 3.0);
        double Ez = (E1(2, z1[0], z1[1], k) + E1(2, z2[0], z2[1], k) + E1(2, z3[0], z3[1], k)) * (1.0 / 3.0);
        double Ezl = Ex * n3[0] + Ey * n3[1] + Ez * n3[2];
        double Bn1, Bn2, Bn3, SR1, SL1, SR2, SL2, SR3, SL3;
        if (corner == 0) {
          Bn1 = -Bq(c.Bqy, 4, z3[0], z3[1], k); Bn2 = Bq(c.Bqx, 2, z2[0], z2[1], k); Bn3 = Bq(c.Bqy, 3, z2[0], z2[1] - 1, k);
          SR1 = -S(c.SDy, z3[0], z3[1], k); SL1 = -S(c.SUy, z3[0], z3[1], k);
          SR2 = S(c.SRx, z2[0], z2[1], k); SL2 = S(c.SLx, z2[0], z2[1], k);
          SR3 = S(c.SUy, z2[0], z2[1] - 1, k); SL3 = S(c.SDy, z2[0], z2[1] - 1, k);
        } else if (corner == 1) {
          Bn1 = -Bq(c.Bqy, 4, z1[0], z1[1] - 1, k); Bn2 = Bq(c.Bqx, 2, z2[0], z2[1], k); Bn3 = Bq(c.Bqy, 3, z3[0], z3[1], k);
          SR1 = -S(c.SLx, z3[0], z3[1], k); SL1 = -S(c.SRx, z3[0], z3[1], k);
          SR2 = S(c.SRx, z2[0], z2[1], k); SL2 = S(c.SLx, z2[0], z2[1], k);
          SR3 = S(c.SUy, z3[0], z3[1], k); SL3 = S(c.SDy, z3[0], z3[1], k);
        } else if (corner == 2) {
          Bn1 = Bq(c.Bqx, 2, z1[0], z1[1], k); Bn2 = Bq(c.Bqy, 3, z2[0], z2[1], k); Bn3 = -Bq(c.Bqx, 1, z2[0], z2[1], k);
          SR1 = S(c.SRx, z1[0], z1[1], k); SL1 = S(c.SLx, z1[0], z1[1], k);
          SR2 = S(c.SUy, z2[0], z2[1], k); SL2 = S(c.SDy, z2[0], z2[1], k);
          SR3 = -S(c.SLx, z2[0], z2[1], k); SL3 = -S(c.SRx, z2[0], z2[1], k);
        } else {
          Bn1 = -Bq(c.Bqy, 4, z3[0], z3[1], k); Bn2 = Bq(c.Bqy, 3, z2[0], z2[1], k); Bn3 = -Bq(c.Bqx, 1, z2[0], z2[1], k);
          SR1 = -S(c.SDy, z3[0], z3[1], k); SL1 = -S(c.SUy, z3[0], z3[1], k);
          SR2 = S(c.SUy, z2[0], z2[1], k); SL2 = S(c.SDy, z2[0], z2[1], k);
          SR3 = -S(c.SLx, z2[0], z2[1], k); SL3 = -S(c.SRx, z2[0], z2[1], k);
        }
        double t = std::max({std::fabs(SR1), std::fabs(SL1), std::fabs(SR2), std::fabs(SL2), std::fabs(SR3), std::fabs(SL3)});
        SR1 = t; SL1 = -t; SR2 = t; SL2 = -t; SR3 = t; SL3 = -t;
        double ess = twod_rs_ez_3state(SR1, SL1, SR2, SL2, SR3, SL3, Ezl, Ezl, Ezl, Bn1, Bn2, Bn3);
        c.a(c.Efz, 0, pn, i, j, k) = c.a(c.Efz, 0, pn, i, j, k) + wt * ess;
      }
    }
  }
}

// BUILD_NON_STIFF_SOURCES, point-mass gravity only (400riemann_integrate/470build_non_stiff_sources.f:95-247).
void build_non_stiff_sources(Ctx& c, int pn) {
  if (!(c.p.gm > c.p.smallnum)) return;
  const int N = c.N, nr = c.nr;
  auto V = [&](int comp, int i, int j, int k) -> double& { return c.a(c.V, comp, pn, i, j, k); };
  OMP_ZONES
  for (int k = 0; k <= nr + 1; ++k)
    for (int j = 0; j <= N + 1; ++j)
      for (int i = 0; i <= N + 1; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        double x = c.geo(V_CEN, 0, pn, i, j, k), y = c.geo(V_CEN, 1, pn, i, j, k), z = c.geo(V_CEN, 2, pn, i, j, k);
        double rho = V(0, i, j, k), vx = V(1, i, j, k), vy = V(2, i, j, k), vz = V(3, i, j, k);
        double rad = std::sqrt(x * x + y * y + z * z);
        double obr3 = 1.0 / (rad * rad * rad);
        double gmb = c.p.gm * obr3;
        double S2 = -(gmb * x * rho), S3 = -(gmb * y * rho), S4 = -(gmb * z * rho);
        double S5 = vx * S2 + vy * S3 + vz * S4;
        c.a(c.dUdt, 1, pn, i, j, k) = c.a(c.dUdt, 1, pn, i, j, k) + S2;
        c.a(c.dUdt, 2, pn, i, j, k) = c.a(c.dUdt, 2, pn, i, j, k) + S3;
        c.a(c.dUdt, 3, pn, i, j, k) = c.a(c.dUdt, 3, pn, i, j, k) + S4;
        c.a(c.dUdt, 4, pn, i, j, k) = c.a(c.dUdt, 4, pn, i, j, k) + S5;
      }
}

// UPDATE_IMEX_RK_STEP_P1 for ideal MHD (400riemann_integrate/484update_imex_rk_step_p1.f:212-906).
void update(Ctx& c, int pn, double dt) {
  const int N = c.N, G = c.G, nr = c.nr;
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i)
        for (int q = 0; q < NV; ++q)
          c.a(c.U, q, pn, i, j, k) = c.a(c.U, q, pn, i, j, k) + dt * c.a(c.dUdt, q, pn, i, j, k);
  OMP_ZONES
  for (int k = 1; k <= nr; ++k)
    for (int j = 1; j <= N; ++j)
      for (int i = 1; i <= N; ++i) {
        auto A = [&](int f, int x, int y, int z) { return c.geo(f, 0, pn, x, y, z); };
        double div = A(XF_AREA, i, j, k) * c.a(c.EFx, 0, pn, i, j, k) - A(XF_AREA, i - 1, j, k) * c.a(c.EFx, 0, pn, i - 1, j, k) +
                     A(YF_AREA, i, j, k) * c.a(c.EFy, 0, pn, i, j, k) - A(YF_AREA, i, j - 1, k) * c.a(c.EFy, 0, pn, i, j - 1, k) +
                     A(ZF_AREA, i, j, k) * c.a(c.EFz, 0, pn, i, j, k) - A(ZF_AREA, i, j, k - 1) * c.a(c.EFz, 0, pn, i, j, k - 1);
        c.a(c.ent, 0, pn, i, j, k) = c.a(c.ent, 0, pn, i, j, k) - dt * div / A(V_VOL, i, j, k);
        double Up[NV], Vp[NV];
        for (int q = 0; q < NV; ++q) Up[q] = c.a(c.U, q, pn, i, j, k);
        double en = c.a(c.ent, 0, pn, i, j, k);
        cons_to_prim(c.ph, en, Up, Vp);
        for (int q = 0; q < NV; ++q) c.a(c.U, q, pn, i, j, k) = Up[q];
        c.a(c.ent, 0, pn, i, j, k) = en;
      }
  auto vt = [&](int q, int x, int y, int z) { return c.geo(G_VERT, q, pn, x, y, z); };
  auto rad = [&](int x, int y, int z) { return std::sqrt(sq(vt(0, x, y, z)) + sq(vt(1, x, y, z)) + sq(vt(2, x, y, z))); };
  auto ang = [&](int ax, int ay, int bx, int by, int z, double inv) {
    double d = (vt(0, ax, ay, z) * inv) * (vt(0, bx, by, z) * inv) + (vt(1, ax, ay, z) * inv) * (vt(1, bx, by, z) * inv) +
               (vt(2, ax, ay, z) * inv) * (vt(2, bx, by, z) * inv);
    return std::acos(d);
  };
  OMP_ZONES
  for (int k = 1; k <= nr; ++k)
    for (int j = 1; j <= N; ++j)
      for (int i = 0; i <= N; ++i) {
        double rout = rad(i, j, k), rin = rad(i, j, k - 1), dr = rout - rin;
        double th = ang(i, j, i, j - 1, k, 1.0 / rout);
        double lin = rin * th, lout = rout * th;
        double s = dr * c.a(c.Efz, 0, pn, i, j, k) - dr * c.a(c.Efz, 0, pn, i, j - 1, k) - lout * c.a(c.Efy, 0, pn, i, j, k) +
                   lin * c.a(c.Efy, 0, pn, i, j, k - 1);
        c.a(c.Bxf, 0, pn, i, j, k) = c.a(c.Bxf, 0, pn, i, j, k) - dt * s / c.geo(XF_AREA, 0, pn, i, j, k);
      }
  OMP_ZONES
  for (int k = 1; k <= nr; ++k)
    for (int j = 0; j <= N; ++j)
      for (int i = 1; i <= N; ++i) {
        double rout = rad(i, j, k), rin = rad(i, j, k - 1), dr = rout - rin;
        double th = ang(i, j, i - 1, j, k, 1.0 / rout);
        double lin = rin * th, lout = rout * th;
        double s = -dr * c.a(c.Efz, 0, pn, i, j, k) + dr * c.a(c.Efz, 0, pn, i - 1, j, k) + lout * c.a(c.Efx, 0, pn, i, j, k) -
                   lin * c.a(c.Efx, 0, pn, i, j, k - 1);
        c.a(c.Byf, 0, pn, i, j, k) = c.a(c.Byf, 0, pn, i, j, k) - dt * s / c.geo(YF_AREA, 0, pn, i, j, k);
      }
  OMP_ZONES
  for (int k = 0; k <= nr; ++k)
    for (int j = 1; j <= N; ++j)
      for (int i = 1; i <= N; ++i) {
        double rout = rad(i, j, k), inv = 1.0 / rout;
        double lxp = rout * ang(i, j, i - 1, j, k, inv);
        double lxm = rout * ang(i, j - 1, i - 1, j - 1, k, inv);
        double lyp = rout * ang(i, j, i, j - 1, k, inv);
        double lym = rout * ang(i - 1, j, i - 1, j - 1, k, inv);
        double s = lyp * c.a(c.Efy, 0, pn, i, j, k) - lym * c.a(c.Efy, 0, pn, i - 1, j, k) - lxp * c.a(c.Efx, 0, pn, i, j, k) +
                   lxm * c.a(c.Efx, 0, pn, i, j - 1, k);
        c.a(c.Bzf, 0, pn, i, j, k) = c.a(c.Bzf, 0, pn, i, j, k) - dt * s / c.geo(ZF_AREA, 0, pn, i, j, k);
      }
}

// CLEANUP_AFTER_UPDATE (400riemann_integrate/485cleanup_after_update.f:383-1273).
void cleanup(Ctx& c, int pn) {
  const int N = c.N, G = c.G, nr = c.nr;
  const double sm = c.p.smallnum;
  zero_masked_faces(c, pn);
  tricorner_sync(c, pn);
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        double nv[3] = {c.geo(ZF_CEN, 0, pn, i, j, k), c.geo(ZF_CEN, 1, pn, i, j, k), c.geo(ZF_CEN, 2, pn, i, j, k)};
        double a = 1.0 / std::max(sm, std::sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]));
        for (int q = 0; q < 3; ++q) nv[q] = nv[q] * a;
        double Am[6][3];
        for (int q = 0; q < 3; ++q) {
          Am[0][q] = c.geo(XF_N, q, pn, i, j, k);
          Am[1][q] = c.geo(XF_N, q, pn, i - 1, j, k);
          Am[2][q] = c.geo(YF_N, q, pn, i, j, k);
          Am[3][q] = c.geo(YF_N, q, pn, i, j - 1, k);
          Am[4][q] = nv[q];
          Am[5][q] = nv[q];
        }
        double Rm[6] = {c.a(c.Bxf, 0, pn, i, j, k), c.a(c.Bxf, 0, pn, i - 1, j, k), c.a(c.Byf, 0, pn, i, j, k),
                        c.a(c.Byf, 0, pn, i, j - 1, k), c.a(c.Bzf, 0, pn, i, j, k), c.a(c.Bzf, 0, pn, i, j, k - 1)};
        double M[3][3], R[3];
        for (int r = 0; r < 3; ++r) {
          for (int s2 = 0; s2 < 3; ++s2) {
            double s = 0.0;
            for (int t = 0; t < 6; ++t) s = s + Am[t][r] * Am[t][s2];
            M[r][s2] = s;
          }
          double s = 0.0;
          for (int t = 0; t < 6; ++t) s = s + Am[t][r] * Rm[t];
          R[r] = s;
        }
        double a11 = M[0][0], a12 = M[0][1], a13 = M[0][2], a21 = M[1][0], a22 = M[1][1], a23 = M[1][2], a31 = M[2][0],
               a32 = M[2][1], a33 = M[2][2];
        double det = a11 * (a22 * a33 - a32 * a23) - a12 * (a21 * a33 - a31 * a23) + a13 * (a21 * a32 - a31 * a22);
        double ob = std::copysign(1.0, det) / std::max(1.0e-32, std::fabs(det));
        double b11 = (a22 * a33 - a23 * a32) * ob, b12 = (a13 * a32 - a12 * a33) * ob, b13 = (a12 * a23 - a22 * a13) * ob;
        double b21 = (a23 * a31 - a21 * a33) * ob, b22 = (a11 * a33 - a13 * a31) * ob, b23 = (a13 * a21 - a11 * a23) * ob;
        double b31 = (a21 * a32 - a22 * a31) * ob, b32 = (a12 * a31 - a11 * a32) * ob, b33 = (a11 * a22 - a12 * a21) * ob;
        double Bx = c.a(c.U, 5, pn, i, j, k), By = c.a(c.U, 6, pn, i, j, k), Bz = c.a(c.U, 7, pn, i, j, k);
        double nb[3] = {b11 * R[0] + b12 * R[1] + b13 * R[2], b21 * R[0] + b22 * R[1] + b23 * R[2],
                        b31 * R[0] + b32 * R[1] + b33 * R[2]};
        for (int q = 0; q < 3; ++q) c.a(c.U, 5 + q, pn, i, j, k) = nb[q];
        c.a(c.U, 4, pn, i, j, k) = c.a(c.U, 4, pn, i, j, k) - (Bx * Bx + By * By + Bz * Bz) * c.ph.ob8pi +
                                   (nb[0] * nb[0] + nb[1] * nb[1] + nb[2] * nb[2]) * c.ph.ob8pi;
      }
  OMP_ZONES
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        double Up[NV], Vp[NV];
        for (int q = 0; q < NV; ++q) Up[q] = c.a(c.U, q, pn, i, j, k);
        double en = c.a(c.ent, 0, pn, i, j, k);
        cons_to_prim(c.ph, en, Up, Vp);
        for (int q = 0; q < NV; ++q) {
          c.a(c.U, q, pn, i, j, k) = Up[q];
          c.a(c.V, q, pn, i, j, k) = Vp[q];
        }
        c.a(c.ent, 0, pn, i, j, k) = en;
      }
}

// EVALUATE_TIMESTEP (400riemann_integrate/490evaluate_timestep.f:121-286), all panels.
double evaluate_timestep(Ctx& c, double dtcur, unsigned panels = 63u) {
  double dt = 1.1 * dtcur;
  const int N = c.N, nr = c.nr;
#pragma omp parallel for collapse(3) schedule(static) reduction(min : dt)
  for (int pn = 0; pn < 6; ++pn)
    for (int k = 1; k <= nr; ++k)
      for (int j = 1; j <= N; ++j)
        for (int i = 1; i <= N; ++i) {
          if (((panels >> pn) & 1u) == 0 || c.m(pn, i, j) == 0) continue;
          double Up[NV], Vp[NV];
          for (int q = 0; q < NV; ++q) Up[q] = c.a(c.U, q, pn, i, j, k);
          double en = c.a(c.ent, 0, pn, i, j, k);
          cons_to_prim(c.ph, en, Up, Vp);
          for (int q = 0; q < NV; ++q) {
            c.a(c.U, q, pn, i, j, k) = Up[q];
            c.a(c.V, q, pn, i, j, k) = Vp[q];
          }
          double b2 = Vp[5] * Vp[5] + Vp[6] * Vp[6] + Vp[7] * Vp[7];
          double ms = std::sqrt((c.p.gamma * Vp[4] + c.ph.ob4pi * b2) / Vp[0]);
          c.a(c.msonic, 0, pn, i, j, k) = ms;
          double a21 = std::sqrt(Vp[1] * Vp[1] + Vp[2] * Vp[2] + Vp[3] * Vp[3]) + ms;
          dt = std::min(dt, c.p.cfl_coef * c.geo(V_SCALE, 0, pn, i, j, k) / a21);
        }
  return dt;
}

// IMEX-RK2 pieces (ARS(2,2,2), gravity implicit).  Gravity S(U) = (0,
// -rho g, -m . g) with g = GM x / r^3 on the active zones 0..N+1; the
// implicit stage U = U* + a S(U) is closed-form because rho is unchanged.
static void gravity_implicit(Ctx& c, int pn, double a) {
  if (!(c.p.gm > c.p.smallnum)) return;
  const int N = c.N, nr = c.nr;
  OMP_ZONES
  for (int k = 0; k <= nr + 1; ++k)
    for (int j = 0; j <= N + 1; ++j)
      for (int i = 0; i <= N + 1; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        double x = c.geo(V_CEN, 0, pn, i, j, k), y = c.geo(V_CEN, 1, pn, i, j, k), z = c.geo(V_CEN, 2, pn, i, j, k);
        double rad = std::sqrt(x * x + y * y + z * z);
        double gmb = c.p.gm * (1.0 / (rad * rad * rad));
        double gx = gmb * x, gy = gmb * y, gz = gmb * z;
        double rho = c.a(c.U, 0, pn, i, j, k);
        double& m1 = c.a(c.U, 1, pn, i, j, k);
        double& m2 = c.a(c.U, 2, pn, i, j, k);
        double& m3 = c.a(c.U, 3, pn, i, j, k);
        m1 = m1 - a * (gx * rho);
        m2 = m2 - a * (gy * rho);
        m3 = m3 - a * (gz * rho);
        double& e = c.a(c.U, 4, pn, i, j, k);
        e = e - a * (gx * m1 + gy * m2 + gz * m3);
      }
}

static void add_gravity(Ctx& c, int pn, double cc) {
  if (!(c.p.gm > c.p.smallnum)) return;
  const int N = c.N, nr = c.nr;
  OMP_ZONES
  for (int k = 0; k <= nr + 1; ++k)
    for (int j = 0; j <= N + 1; ++j)
      for (int i = 0; i <= N + 1; ++i) {
        if (c.m(pn, i, j) != 1) continue;
        double x = c.geo(V_CEN, 0, pn, i, j, k), y = c.geo(V_CEN, 1, pn, i, j, k), z = c.geo(V_CEN, 2, pn, i, j, k);
        double rad = std::sqrt(x * x + y * y + z * z);
        double gmb = c.p.gm * (1.0 / (rad * rad * rad));
        double gx = gmb * x, gy = gmb * y, gz = gmb * z;
        double rho = c.a(c.U, 0, pn, i, j, k);
        double m1 = c.a(c.U, 1, pn, i, j, k), m2 = c.a(c.U, 2, pn, i, j, k), m3 = c.a(c.U, 3, pn, i, j, k);
        c.a(c.dUdt, 1, pn, i, j, k) += cc * (-(gx * rho));
        c.a(c.dUdt, 2, pn, i, j, k) += cc * (-(gy * rho));
        c.a(c.dUdt, 3, pn, i, j, k) += cc * (-(gz * rho));
        c.a(c.dUdt, 4, pn, i, j, k) += cc * (-(gx * m1 + gy * m2 + gz * m3));
      }
}

static bool owns(unsigned panels, int pn) { return (panels >> pn) & 1u; }

// A stage in phases over a set of panels (bit p of `panels` = panel p), so
// that ranks holding some of the panels can run them with the exchanges
// between: the ghost fill before stage_fluxes, the face-flux ownership
// before stage_emfs, the EMF ownership before stage_finish.  Reconstruction
// and face fluxes:
void stage_fluxes(Ctx& c, unsigned panels) {
  for (int pn = 0; pn < 6; ++pn)
    if (owns(panels, pn)) {
      limit_all_slopes_p12(c, pn);
      make_facial_fluxes(c, pn);
    }
}

// The face-flux scatter into the zones and the edge EMFs.
void stage_emfs(Ctx& c, unsigned panels) {
  for (int pn = 0; pn < 6; ++pn)
    if (owns(panels, pn)) {
      scatter_facial_fluxes(c, pn);
      make_edge_efields(c, pn);
    }
}

// The rest of one ARS(2,2,2) stage: fluxes, entropy transport and CT
// explicit, gravity implicit; gamma = 1 - 1/sqrt(2), delta = 1 - 1/(2 gamma).
//   stage 1: U* = U^n + gamma dt F(U^n);  U2 = U* + gamma dt S(U2)
//   stage 2: U* = U^n + delta dt F(U^n) + (1-delta) dt F(U2) + (1-gamma) dt S(U2)
//            U^{n+1} = U* + gamma dt S(U^{n+1})
static void stage_imex_finish(Ctx& c, int irk, double dtcur, unsigned panels) {
  const double gam = 1.0 - 1.0 / std::sqrt(2.0), del = 1.0 - 1.0 / (2.0 * gam);
  if (irk == 1) {
    c.U0 = c.U;
    std::memcpy(c.ent0.data(), c.ent.data(), 6 * c.S * sizeof(double));
    c.Bxf0 = c.Bxf;
    c.Byf0 = c.Byf;
    c.Bzf0 = c.Bzf;
    c.K1 = c.dUdt;
    c.EFx1 = c.EFx; c.EFy1 = c.EFy; c.EFz1 = c.EFz;
    c.Efx1 = c.Efx; c.Efy1 = c.Efy; c.Efz1 = c.Efz;
    for (int pn = 0; pn < 6; ++pn)
      if (owns(panels, pn)) update(c, pn, gam * dtcur);
  } else {
    for (int pn = 0; pn < 6; ++pn)
      if (owns(panels, pn)) add_gravity(c, pn, (1.0 - gam) / (1.0 - del));
    c.U = c.U0;
    std::memcpy(c.ent.data(), c.ent0.data(), 6 * c.S * sizeof(double));
    c.Bxf = c.Bxf0;
    c.Byf = c.Byf0;
    c.Bzf = c.Bzf0;
    auto swap1 = [&]() {
      std::swap(c.dUdt, c.K1);
      std::swap(c.EFx, c.EFx1); std::swap(c.EFy, c.EFy1); std::swap(c.EFz, c.EFz1);
      std::swap(c.Efx, c.Efx1); std::swap(c.Efy, c.Efy1); std::swap(c.Efz, c.Efz1);
    };
    swap1();
    for (int pn = 0; pn < 6; ++pn)
      if (owns(panels, pn)) update(c, pn, del * dtcur);
    swap1();
    for (int pn = 0; pn < 6; ++pn)
      if (owns(panels, pn)) update(c, pn, (1.0 - del) * dtcur);
  }
  for (int pn = 0; pn < 6; ++pn)
    if (owns(panels, pn)) {
      gravity_implicit(c, pn, gam * dtcur);
      cleanup(c, pn);
    }
}

// The rest of an RK2 / SSP-RK3 stage: sources, the stage combine, the
// update and the clean-up.
static void stage_rk_finish(Ctx& c, int irk, double dtcur, unsigned panels) {
  double dtmove = dtcur;
  double a0 = 0.0;  // weight of the saved state in the combine
  int scheme = c.p.rk_scheme;
  if (scheme == 2) {
    if (irk == 2) dtmove = 0.5 * dtcur;
  } else if (scheme == 3) {
    if (irk == 2) { a0 = 0.75; dtmove = 0.25 * dtcur; }
    if (irk == 3) { a0 = 1.0 / 3.0; dtmove = (2.0 / 3.0) * dtcur; }
  }
  for (int pn = 0; pn < 6; ++pn) {
    if (!owns(panels, pn)) continue;
    build_non_stiff_sources(c, pn);
    const size_t S = c.S;
    if (irk == 1) {
      for (int q = 0; q < NV; ++q)
        std::memcpy(&c.U0[((size_t)q * 6 + pn) * S], &c.U[((size_t)q * 6 + pn) * S], S * sizeof(double));
      std::memcpy(&c.ent0[(size_t)pn * S], &c.ent[(size_t)pn * S], S * sizeof(double));
      std::memcpy(&c.Bxf0[(size_t)pn * S], &c.Bxf[(size_t)pn * S], S * sizeof(double));
      std::memcpy(&c.Byf0[(size_t)pn * S], &c.Byf[(size_t)pn * S], S * sizeof(double));
      std::memcpy(&c.Bzf0[(size_t)pn * S], &c.Bzf[(size_t)pn * S], S * sizeof(double));
    } else {
      auto comb = [&](double* x, const double* x0, size_t n) {
        if (scheme == 3) {
          double a1 = 1.0 - a0;
          for (size_t t = 0; t < n; ++t) x[t] = a0 * x0[t] + a1 * x[t];
        } else {
          for (size_t t = 0; t < n; ++t) x[t] = (x[t] + x0[t]) * 0.5;
        }
      };
      for (int q = 0; q < NV; ++q) comb(&c.U[((size_t)q * 6 + pn) * S], &c.U0[((size_t)q * 6 + pn) * S], S);
      comb(&c.ent[(size_t)pn * S], &c.ent0[(size_t)pn * S], S);
      comb(&c.Bxf[(size_t)pn * S], &c.Bxf0[(size_t)pn * S], S);
      comb(&c.Byf[(size_t)pn * S], &c.Byf0[(size_t)pn * S], S);
      comb(&c.Bzf[(size_t)pn * S], &c.Bzf0[(size_t)pn * S], S);
    }
    update(c, pn, dtmove);
    cleanup(c, pn);
  }
}

void stage_finish(Ctx& c, int irk, double dtcur, unsigned panels) {
  if (c.p.rk_scheme == 4)
    stage_imex_finish(c, irk, dtcur, panels);
  else
    stage_rk_finish(c, irk, dtcur, panels);
}

// One RK stage in the driver's order (1000riemann_geomesh_cs_mhd.f:1746-2887):
// ghost fill, then per panel reconstruction, fluxes, EMFs, sources, the
// stage combine, the update and the clean-up, with the panel-edge
// ownership applied to the fluxes and EMFs before they are used.  Panels
// are independent between the exchanges (each reads only its own,
// ghost-filled arrays); the zone loops inside every routine run on all host
// threads.
void stage(Ctx& c, int irk, double dtcur) {
  fill_ghosts(c);
  stage_fluxes(c, 63u);
  sync_facial_fluxes(c);
  stage_emfs(c, 63u);
  sync_edge_efields(c);
  stage_finish(c, irk, dtcur, 63u);
}

}  // namespace oracle

using namespace oracle;

extern "C" {

void* oracle_create(const void* params) {
  Ctx* c = new Ctx();
  std::memcpy(&c->p, params, sizeof(Params));
  c->panel_rule = (c->p.flags & CS_FLAG_PANEL_AVERAGE) ? 1 : 0;
  c->N = c->p.ntp;
  c->nr = c->p.nr;
  c->G = c->p.nghost;
  c->NI = c->NJ = c->N + 2 * c->G + 1;
  c->NK = c->nr + 2 * c->G + 1;
  c->S = (size_t)c->NI * c->NJ * c->NK;
  c->ph.gamma = c->p.gamma;
  c->ph.rhofloor = c->p.rhofloor;
  c->ph.prsfloor = c->p.prsfloor;
  c->ph.smallnum = c->p.smallnum;
  c->ph.pi = 4.0 * std::atan(1.0);
  c->ph.ob4pi = 1.0 / (4.0 * c->ph.pi);
  c->ph.ob8pi = 1.0 / (8.0 * c->ph.pi);
  const size_t S6 = 6 * c->S;
  auto al = [&](std::vector<double>& v, int n) { v.assign((size_t)n * S6, 0.0); };
  al(c->U, 8); al(c->ent, 4); al(c->Bxf, 1); al(c->Byf, 1); al(c->Bzf, 1); al(c->V, 80); al(c->E, 30);
  al(c->msonic, 1); al(c->divvel, 1); al(c->flat, 1); al(c->work, 1); al(c->Bqx, 5); al(c->Bqy, 5); al(c->Bqz, 5);
  al(c->dUdt, 8); al(c->SLx, 1); al(c->SRx, 1); al(c->SDy, 1); al(c->SUy, 1); al(c->SBz, 1); al(c->STz, 1);
  al(c->EFx, 1); al(c->EFy, 1); al(c->EFz, 1); al(c->Efx, 1); al(c->Efy, 1); al(c->Efz, 1);
  al(c->U0, 8); al(c->ent0, 1); al(c->Bxf0, 1); al(c->Byf0, 1); al(c->Bzf0, 1); al(c->pos, 1);
  if (c->p.rk_scheme == 4) {
    al(c->K1, 8); al(c->EFx1, 1); al(c->EFy1, 1); al(c->EFz1, 1); al(c->Efx1, 1); al(c->Efy1, 1); al(c->Efz1, 1);
  }
  for (int d = 0; d < 3; ++d) {
    al(c->cL[d], 5 * 8);
    al(c->cR[d], 5 * 8);
    c->tL[d].assign(S6, -1);
    c->tR[d].assign(S6, -1);
  }
  return c;
}

void oracle_destroy(void* h) { delete (Ctx*)h; }

// The solve's own mesh: geometry, mask and stencil from the host mesh
// builder for the parameters given at creation.  Returns 0, or 1 with the
// reason in why (a buffer of nwhy bytes).
int oracle_build_mesh(void* h, char* why, int nwhy) {
  Ctx* c = (Ctx*)h;
  static_assert(sizeof(Params) == sizeof(cs_params), "oracle Params mirrors cs_params");
  cs_params cp;
  std::memcpy(&cp, &c->p, sizeof(cp));
  cs::GeomHost gh;
  const std::string e = cs::build_geometry(cp, gh);
  if (!e.empty()) {
    if (why && nwhy > 0) std::snprintf(why, (size_t)nwhy, "%s", e.c_str());
    return 1;
  }
  for (int f = 0; f < NGF; ++f) c->g[f] = std::move(gh.f[f]);
  c->mask = std::move(gh.mask);
  c->st = std::move(gh.stencil);
  c->maps_built = false;
  return 0;
}

// The seeded initial state (cs_init_desc) written into the solve's state on
// its own mesh (oracle_build_mesh first).  Returns 0, or 1 with the reason.
int oracle_init_problem(void* h, const void* desc, char* why, int nwhy) {
  Ctx* c = (Ctx*)h;
  cs_params cp;
  std::memcpy(&cp, &c->p, sizeof(cp));
  cs_init_desc d;
  std::memcpy(&d, desc, sizeof(d));
  cs::GeomHost gh;  // borrows the solve's geometry for the call
  gh.box = cs::Box(c->N, c->nr, c->G);
  for (int f = 0; f < NGF; ++f) gh.f[f] = std::move(c->g[f]);
  gh.mask = std::move(c->mask);
  gh.stencil = std::move(c->st);
  const std::string e = cs::init_problem_host(cp, d, gh, c->U.data(), c->ent.data(), c->Bxf.data(), c->Byf.data(),
                                              c->Bzf.data());
  for (int f = 0; f < NGF; ++f) c->g[f] = std::move(gh.f[f]);
  c->mask = std::move(gh.mask);
  c->st = std::move(gh.stencil);
  if (!e.empty()) {
    if (why && nwhy > 0) std::snprintf(why, (size_t)nwhy, "%s", e.c_str());
    return 1;
  }
  for (size_t t = 6 * c->S; t < c->ent.size(); ++t) c->ent[t] = 0.0;
  return 0;
}

// Geometry field f, mask and stencil of the solve (for comparisons).
void oracle_get_geometry(void* h, int f, double* out) {
  Ctx* c = (Ctx*)h;
  std::memcpy(out, c->g[f].data(), c->g[f].size() * sizeof(double));
}
void oracle_get_mask_stencil(void* h, int32_t* mask, int32_t* st) {
  Ctx* c = (Ctx*)h;
  std::memcpy(mask, c->mask.data(), c->mask.size() * sizeof(int32_t));
  std::memcpy(st, c->st.data(), c->st.size() * sizeof(int32_t));
}

// Geometry field f (cs_geom_field order), [comp][6][box] doubles.
void oracle_set_geometry(void* h, int f, const double* data) {
  Ctx* c = (Ctx*)h;
  c->g[f].assign(data, data + (size_t)kNcomp[f] * 6 * c->S);
}
void oracle_set_mask_stencil(void* h, const int32_t* mask, const int32_t* st) {
  Ctx* c = (Ctx*)h;
  c->mask.assign(mask, mask + 6 * c->S);
  c->st.assign(st, st + (size_t)6 * 24 * c->NI * c->NJ);
}
void oracle_set_state(void* h, const double* U, const double* ent, const double* bx, const double* by, const double* bz) {
  Ctx* c = (Ctx*)h;
  const size_t S6 = 6 * c->S;
  std::memcpy(c->U.data(), U, 8 * S6 * sizeof(double));
  std::memcpy(c->ent.data(), ent, S6 * sizeof(double));
  std::memcpy(c->Bxf.data(), bx, S6 * sizeof(double));
  std::memcpy(c->Byf.data(), by, S6 * sizeof(double));
  std::memcpy(c->Bzf.data(), bz, S6 * sizeof(double));
}
void oracle_get_state(void* h, double* U, double* ent, double* bx, double* by, double* bz) {
  Ctx* c = (Ctx*)h;
  const size_t S6 = 6 * c->S;
  std::memcpy(U, c->U.data(), 8 * S6 * sizeof(double));
  std::memcpy(ent, c->ent.data(), S6 * sizeof(double));
  std::memcpy(bx, c->Bxf.data(), S6 * sizeof(double));
  std::memcpy(by, c->Byf.data(), S6 * sizeof(double));
  std::memcpy(bz, c->Bzf.data(), S6 * sizeof(double));
}
// which: same numbering as cs_debug_get.
int oracle_debug_get(void* h, int which, double* out) {
  Ctx* c = (Ctx*)h;
  const size_t S6 = 6 * c->S;
  auto cp = [&](const std::vector<double>& v) { std::memcpy(out, v.data(), v.size() * sizeof(double)); };
  switch (which) {
    case 0: cp(c->V); break;
    case 1: cp(c->ent); break;
    case 2: cp(c->flat); break;
    case 3: cp(c->dUdt); break;
    case 4: cp(c->Efx); break;
    case 5: cp(c->Efy); break;
    case 6: cp(c->Efz); break;
    case 7: cp(c->Bqx); break;
    case 8: cp(c->Bqy); break;
    case 9: cp(c->Bqz); break;
    case 10:
      for (int q = 0; q < 3; ++q) std::memcpy(out + q * S6, c->E.data() + q * S6, S6 * sizeof(double));
      break;
    case 11: {
      const std::vector<double>* s[6] = {&c->SLx, &c->SRx, &c->SDy, &c->SUy, &c->SBz, &c->STz};
      for (int q = 0; q < 6; ++q) std::memcpy(out + q * S6, s[q]->data(), S6 * sizeof(double));
      break;
    }
    case 12: {
      const std::vector<double>* s[3] = {&c->EFx, &c->EFy, &c->EFz};
      for (int q = 0; q < 3; ++q) std::memcpy(out + q * S6, s[q]->data(), S6 * sizeof(double));
      break;
    }
    case 13: cp(c->pos); break;
    default: return 1;
  }
  return 0;
}
void oracle_fill_ghosts(void* h) { fill_ghosts(*(Ctx*)h); }
void oracle_limit_all_slopes_p12(void* h) {
  for (int p = 0; p < 6; ++p) limit_all_slopes_p12(*(Ctx*)h, p);
}
void oracle_make_facial_fluxes(void* h) {
  Ctx& c = *(Ctx*)h;
  for (int p = 0; p < 6; ++p) make_facial_fluxes(c, p);
  sync_facial_fluxes(c);
  for (int p = 0; p < 6; ++p) scatter_facial_fluxes(c, p);
}
void oracle_make_edge_efields(void* h) {
  Ctx& c = *(Ctx*)h;
  for (int p = 0; p < 6; ++p) make_edge_efields(c, p);
  sync_edge_efields(c);
}
void oracle_build_non_stiff_sources(void* h) {
  for (int p = 0; p < 6; ++p) build_non_stiff_sources(*(Ctx*)h, p);
}
void oracle_update(void* h, double dt) {
  for (int p = 0; p < 6; ++p) update(*(Ctx*)h, p, dt);
}
void oracle_cleanup(void* h) {
  for (int p = 0; p < 6; ++p) cleanup(*(Ctx*)h, p);
}
double oracle_evaluate_timestep(void* h, double dtcur) { return evaluate_timestep(*(Ctx*)h, dtcur); }
void oracle_stage(void* h, int irk, double dtcur) { stage(*(Ctx*)h, irk, dtcur); }
// One phase of a stage over the panels in the bit set `panels`: 0 the radial
// padding (after the ghost fill), 1 reconstruction and face fluxes, 2 the
// flux scatter and the edge EMFs, 3 the rest of the stage; the exchanges go
// between them (pad_radial / stage_fluxes / stage_emfs / stage_finish).
int oracle_stage_phase(void* h, int phase, int irk, double dtcur, unsigned panels) {
  Ctx& c = *(Ctx*)h;
  switch (phase) {
    case 0:
      for (int pn = 0; pn < 6; ++pn)
        if ((panels >> pn) & 1u) pad_radial(c, pn);
      return 0;
    case 1: stage_fluxes(c, panels); return 0;
    case 2: stage_emfs(c, panels); return 0;
    case 3: stage_finish(c, irk, dtcur, panels); return 0;
    default: return 1;
  }
}
// Rule for the copies of shared faces and edges: 0 the lowest-numbered
// panel's (the library's), 1 their average (the reference's).
void oracle_set_panel_rule(void* h, int rule) { ((Ctx*)h)->panel_rule = rule; }
double oracle_evaluate_timestep_panels(void* h, double dtcur, unsigned panels) {
  return evaluate_timestep(*(Ctx*)h, dtcur, panels);
}
// The stage arrays the panel-edge ownership acts on, in place: which 0 / 1
// the two one-sided face contributions cL / cR of direction `dir` (5
// quadrature points x NV per face, [point * NV + var][panel][box]), 2 the
// entropy flux of direction `dir`, 3 EMF component `dir`.  Null for any
// other request; *n is the array's length.
double* oracle_stage_array(void* h, int which, int dir, size_t* n) {
  Ctx& c = *(Ctx*)h;
  if (dir < 0 || dir > 2) return nullptr;
  std::vector<double>* EF[3] = {&c.EFx, &c.EFy, &c.EFz};
  std::vector<double>* Ef[3] = {&c.Efx, &c.Efy, &c.Efz};
  std::vector<double>* v = which == 0 ? &c.cL[dir] : which == 1 ? &c.cR[dir] : which == 2 ? EF[dir]
                         : which == 3 ? Ef[dir] : nullptr;
  if (!v) return nullptr;
  *n = v->size();
  return v->data();
}
// One full time step; returns the next dt (min over panels, grown at most 10%).
double oracle_step(void* h, double dtcur) {
  Ctx* c = (Ctx*)h;
  int ns = (c->p.rk_scheme == 3) ? 3 : 2;
  for (int irk = 1; irk <= ns; ++irk) stage(*c, irk, dtcur);
  c->time += dtcur;
  return evaluate_timestep(*c, dtcur);
}

// STEP 10 of the last LIMIT_ALL_SLOPES_P12 over the six panels (the
// driver's reduction over patches, 1000riemann_geomesh_cs_mhd.f:2447-2448).
int oracle_limit_minmax(void* h, double* vmin, double* vmax) {
  const Ctx* c = (const Ctx*)h;
  if (!c->step10) return 1;
  for (int q = 0; q <= NV; ++q) {
    vmin[q] = 1.0e32;
    vmax[q] = -1.0e32;
    for (int pn = 0; pn < 6; ++pn) {
      vmin[q] = std::min(vmin[q], c->vmin[pn][q]);
      vmax[q] = std::max(vmax[q], c->vmax[pn][q]);
    }
  }
  return 0;
}

// The pointwise physics on n cases, with the solve's constants; the same
// cases and layouts as the library's cs_pointwise: kind 0 PRIM_TO_CONS,
// kind 1 CONS_TO_PRIM, kind 2 the HLL solve of OneD_RS_MHD_Ptwise.
int oracle_pointwise(void* h, int kind, int n, const double* in, double* out) {
  const Ctx* c = (const Ctx*)h;
  for (int t = 0; t < n; ++t) {
    if (kind == 0) {
      const double* a = in + (size_t)t * 9;
      double V[NV], U[NV];
      for (int q = 0; q < NV; ++q) V[q] = a[q];
      prim_to_cons(c->ph, a[8], U, V);
      for (int q = 0; q < NV; ++q) out[(size_t)t * 8 + q] = U[q];
    } else if (kind == 1) {
      const double* a = in + (size_t)t * 9;
      double V[NV], U[NV];
      for (int q = 0; q < NV; ++q) U[q] = a[q];
      double ent = a[8];
      const int flag = cons_to_prim(c->ph, ent, U, V);
      double* o = out + (size_t)t * 18;
      for (int q = 0; q < NV; ++q) o[q] = V[q];
      o[8] = ent;
      o[9] = flag;
      for (int q = 0; q < NV; ++q) o[10 + q] = U[q];
    } else if (kind == 2) {
      const double* a = in + (size_t)t * 18;
      double VL[NV], VR[NV];
      for (int q = 0; q < NV; ++q) {
        VL[q] = a[q];
        VR[q] = a[8 + q];
      }
      RSOut r;
      oned_rs_hll(c->ph, VL, VR, a[16], a[17], r);
      double* o = out + (size_t)t * 35;
      for (int q = 0; q < NV; ++q) {
        o[q] = r.FlL[q];
        o[8 + q] = r.FlR[q];
        o[16 + q] = r.FL[q];
        o[24 + q] = r.FR[q];
      }
      o[32] = r.SL;
      o[33] = r.SR;
      o[34] = r.entF;
    } else {
      return 1;
    }
  }
  return 0;
}

// The two multidimensional Riemann solvers with four / three separate Ez
// (the reference's argument lists), for known-answer tests.
double oracle_twod_rs_ez_4state(const double* a) {
  return twod_rs_ez_4state(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11], a[12], a[13]);
}
double oracle_twod_rs_ez_3state(const double* a) {
  return twod_rs_ez_3state(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11]);
}

}  // extern "C"
