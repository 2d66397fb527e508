// Device-side layout, accessors and pointwise physics of the B200 stage
// update.  All state lives in HBM as FP64 panel boxes (component-major SoA,
// i fastest) so that a warp along i reads 32 consecutive doubles per field.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cs_internal.h"

namespace cs {

// Sizes of one solve.
struct Dims {
  int N, nr, G, NI, NJ, NK;
  long long S;  // points per panel box
  __host__ __device__ long long idx(int i, int j, int k) const {
    return ((long long)(k + G) * NJ + (long long)(j + G)) * NI + (long long)(i + G);
  }
  __host__ __device__ long long at(int c, int p, int i, int j, int k) const {
    return ((long long)c * NPANEL + p) * S + idx(i, j, k);
  }
};

// Physical constants of one solve.
struct PhysC {
  double gamma, rhofloor, prsfloor, smallnum, ob4pi, ob8pi, fourpi, cfl, flatten_coef, prs_flatten_coef, gm;
};

// Geometry resident on the device (read only during stages).
struct DGeom {
  const double* f[CS_G_NFIELDS];
  const int32_t* mask;  // [6][S]
  const int32_t* st;    // [6][12][2][NJ][NI]
};

// How panel p reads panel 1's least-squares row weights: mode m (0 the
// constant, 1-3 x y z, 4-6 xx yy zz, 7-9 xy yz xz) takes panel 1's mode
// (src >> 4m) & 15, negated where bit m of neg is set.
struct LsqPanelMap {
  unsigned long long src;
  unsigned int neg;
  unsigned int pad;
};
constexpr unsigned long long LSQ_IDENTITY_SRC = 0x9876543210ULL;

// Mutable per-solve arrays.  R is the storage and arithmetic type of the
// state, the reconstruction, the face states and fluxes and the stage update
// (double in the plain form, float in the precision form); face B, its
// quadrature values, the EMFs and the ADP factors are FP64 always.
template <typename R>
struct DStateT {
  using real = R;
  R *U, *ent;                            // state (U: 8 comps, ent: 4 modes)
  double *Bxf, *Byf, *Bzf;               // face-normal B
  R *V, *E, *Esnap;                      // V: 80 (mode*8+comp), E: 30 (mode*3+comp), Esnap: 3
  R *msonic, *flatA, *flatB;             // flattener work
  double *Bq[3];                         // B at face quadrature points (5 each)
  R *fcon[3];                            // per-face flux contributions: [16][..] (L 8, R 8)
  R *S[6];                               // S_L,S_R (x), S_D,S_U (y), S_B,S_T (z) at j=1
  R *EF[3];                              // entropy fluxes
  double *Ef[3];                         // edge EMFs
  R *dUdt;                               // 8
  R *U0, *ent0;                          // saved stage-1 state
  double *B0[3];
  R *K1, *EF1[3];                        // IMEX: first stage's dU/dt and entropy fluxes
  double *Ef1[3];                        // IMEX: first stage's EMFs
  R* op_m9;                              // STEP 7.b row weights Minv A_rr^T, [18 x 9][zones of shrink(2)], or null
  R* op_m10;                             // STEP 9.c row weights Minv A_rr^T, [19 x 10][zones of shrink(2)], or null
  const LsqPanelMap* lsq_map9;           // op_m9 shared by the panels (panel 1's zones only), or null
  const LsqPanelMap* lsq_map10;          // op_m10 likewise
  R* op_p2v;                             // CS_FLAG_P2 STEP 7.a stencil inverses, [8 x 9 x 9][zones of shrink(2)], or null
  R* op_p2e;                             // CS_FLAG_P2 STEP 9.b stencil inverses, [8 x 10 x 10][zones of shrink(2)], or null
  const LsqPanelMap* p2_map;             // op_p2v / op_p2e shared by the panels, or null
  void* adp_lu;                          // ADP KKT factors, per block of zones [1296 in use order][block], or null:
                                         // FP64 per panel; panel 1's (adp_pmap set) in the state's type R
  int8_t* adp_piv;                       // their row permutation, per block [36][block]
  void* adp_rhs;                         // ADP right-hand sides, [36][zones of the ADP range], typed as adp_lu
  const int8_t* adp_pmap;                // factors shared by the panels: per panel [unknown map 36][sign 36], or null
  int* err_flag;                         // device-side error bits (bounded waits that gave up)
  int32_t* giveup;                       // positivity give-up flags per zone
  unsigned long long* dtmin;             // CFL reduction target (bit pattern of a positive double)
  double* dt;                            // the solve's current time step (device scalar)
};
using DState = DStateT<double>;

__device__ __forceinline__ int mask_at(const DGeom& g, const Dims& d, int p, int i, int j) {
  return g.mask[(long long)p * d.S + d.idx(i, j, 0)];
}
__device__ __forceinline__ int sten(const DGeom& g, const Dims& d, int p, int i, int j, int w, int c) {
  return g.st[(((long long)p * 12 + w) * 2 + c) * ((long long)d.NI * d.NJ) + (long long)(j + d.G) * d.NI + (i + d.G)];
}
__device__ __forceinline__ double geo(const DGeom& g, const Dims& d, int f, int c, int p, int i, int j, int k) {
  return __ldg(g.f[f] + d.at(c, p, i, j, k));
}

template <typename R>
__device__ __forceinline__ R geoR(const DGeom& g, const Dims& d, int f, int c, int p, int i, int j, int k) {
  return (R)__ldg(g.f[f] + d.at(c, p, i, j, k));
}

// Decode a flat thread index over panels x a 3-D index range.
struct Range3 {
  int i0, i1, j0, j1, k0, k1;
  __host__ __device__ long long count() const {
    return 6LL * (long long)(i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1);
  }
  __device__ void decode(long long t, int& p, int& i, int& j, int& k) const {
    const long long ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
    i = (int)(t % ni) + i0;
    t /= ni;
    j = (int)(t % nj) + j0;
    t /= nj;
    k = (int)(t % nk) + k0;
    p = (int)(t / nk);
  }
};

// ---------------- pointwise physics (ideal MHD, adiabatic) ----------------
template <typename R>
__device__ __forceinline__ R sqr(R x) { return x * x; }

// Conserved -> primitive with density/pressure floors and the entropy
// fallback; updates ent and re-derives the total energy.  Returns the
// floor flag.
template <typename R>
__device__ __forceinline__ int d_cons_to_prim(const PhysC& ph, R& ent, R* U, R* V) {
  int flag = 0;
  U[0] = fmax(U[0], R(ph.rhofloor));
  V[0] = U[0];
  const R a = V[0] / (V[0] * V[0] + R(ph.rhofloor) * R(ph.rhofloor));
  V[1] = U[1] * a;
  V[2] = U[2] * a;
  V[3] = U[3] * a;
  V[5] = U[5];
  V[6] = U[6];
  V[7] = U[7];
  const R v2 = V[1] * V[1] + V[2] * V[2] + V[3] * V[3];
  const R b2 = V[5] * V[5] + V[6] * V[6] + V[7] * V[7];
  V[4] = (R(ph.gamma) - R(1.0)) * (U[4] - R(0.5) * V[0] * v2 - R(ph.ob8pi) * b2);
  if (V[4] <= R(ph.prsfloor)) {
    V[4] = fmax(R(ph.prsfloor), ent * pow(V[0], R(ph.gamma) - R(1.0)));
    flag = 1;
  }
  ent = V[4] / pow(V[0], R(ph.gamma) - R(1.0));
  U[4] = V[4] / (R(ph.gamma) - R(1.0)) + R(0.5) * V[0] * v2 + R(ph.ob8pi) * b2;
  return flag;
}

template <typename R>
__device__ __forceinline__ void d_prim_to_cons(const PhysC& ph, R ent, R* U, R* V) {
  V[0] = fmax(V[0], R(ph.rhofloor));
  if (V[4] <= R(ph.prsfloor)) V[4] = fmax(R(ph.prsfloor), ent * pow(V[0], R(ph.gamma) - R(1.0)));
  U[0] = V[0];
  U[1] = V[0] * V[1];
  U[2] = V[0] * V[2];
  U[3] = V[0] * V[3];
  U[5] = V[5];
  U[6] = V[6];
  U[7] = V[7];
  U[4] = V[4] / (R(ph.gamma) - R(1.0)) + R(0.5) * V[0] * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]) +
         R(ph.ob8pi) * (V[5] * V[5] + V[6] * V[6] + V[7] * V[7]);
}

// Fast magnetosonic extremal speeds along the local x axis.
template <typename R>
__device__ __forceinline__ void d_wavespeeds(const PhysC& ph, const R* V, R& smin, R& smax) {
  const R cs2 = R(ph.gamma) * V[4] / V[0];
  const R b2r = (V[5] * V[5] + V[6] * V[6] + V[7] * V[7]) / (R(ph.fourpi) * V[0]);
  const R bb = -(cs2 + b2r);
  const R cc = cs2 * V[5] * V[5] / (R(ph.fourpi) * V[0]);
  const R mf = sqrt((-bb + sqrt(bb * bb - R(4.0) * cc)) / R(2.0));
  smin = V[1] - mf;
  smax = V[1] + mf;
}

template <typename R>
__device__ __forceinline__ void d_flux_x(const PhysC& ph, const R* V, R* F) {
  const R u4 = V[4] / (R(ph.gamma) - R(1.0)) + R(0.5) * V[0] * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]) +
                    R(ph.ob8pi) * (V[5] * V[5] + V[6] * V[6] + V[7] * V[7]);
  const R b2 = V[5] * V[5] + V[6] * V[6] + V[7] * V[7];
  const R vdb = V[1] * V[5] + V[2] * V[6] + V[3] * V[7];
  const R pt = V[4] + R(ph.ob8pi) * b2;
  F[0] = V[1] * V[0];
  F[1] = V[1] * (V[0] * V[1]) + pt - R(ph.ob4pi) * V[5] * V[5];
  F[2] = V[1] * (V[0] * V[2]) - R(ph.ob4pi) * V[5] * V[6];
  F[3] = V[1] * (V[0] * V[3]) - R(ph.ob4pi) * V[5] * V[7];
  F[4] = V[1] * u4 + pt * V[1] - R(ph.ob4pi) * V[5] * vdb;
  F[5] = R(0.0);
  F[6] = V[1] * V[6] - V[5] * V[2];
  F[7] = V[1] * V[7] - V[5] * V[3];
}

// HLL solve at one quadrature point in the face frame.  Outputs the left
// and right fluctuations, the two physical fluxes (all in the face frame),
// the extremal speeds and the entropy flux.
template <typename R>
__device__ __forceinline__ void d_hll(const PhysC& ph, R* VL, R* VR, R entL, R entR, R* FlL,
                                      R* FlR, R* FL, R* FR, R& SL, R& SR, R& entF) {
  const R bx = R(0.5) * (VL[5] + VR[5]);
  VL[5] = bx;
  VR[5] = bx;
  R UL[8], UR[8];
  d_prim_to_cons(ph, entL, UL, VL);
  d_prim_to_cons(ph, entR, UR, VR);
  d_flux_x(ph, VL, FL);
  d_flux_x(ph, VR, FR);
  R smin, smax;
  SR = -R(1.0e30);
  SL = R(1.0e30);
  d_wavespeeds(ph, VL, smin, smax);
  SL = fmin(SL, smin);
  SR = fmax(SR, smax);
  d_wavespeeds(ph, VR, smin, smax);
  SL = fmin(SL, smin);
  SR = fmax(SR, smax);
  R Vm[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) Vm[c] = R(0.5) * (VL[c] + VR[c]);
  d_wavespeeds(ph, Vm, smin, smax);
  SL = fmin(SL, smin);
  SR = fmax(SR, smax);
  const R t3 = R(1.0) / (SR - SL), t1 = SR * t3, t2 = SL * t3;
  R Us[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) Us[c] = t1 * UR[c] - t2 * UL[c] - t3 * (FR[c] - FL[c]);
  const R entU = t1 * entR - t2 * entL - t3 * (entR * VR[1] - entL * VL[1]);
  const R peng = (R(ph.gamma) - R(1.0)) * (Us[4] - R(0.5) * (Us[1] * Us[1] + Us[2] * Us[2] + Us[3] * Us[3]) / Us[0] -
                                          R(ph.ob8pi) * (Us[5] * Us[5] + Us[6] * Us[6] + Us[7] * Us[7]));
  // The entropy pressure (a pow) is formed only where the floor needs it.
  if (peng <= R(ph.prsfloor)) {
    const R pent = entU * pow(Us[0], R(ph.gamma) - R(1.0));
    Us[4] = Us[4] + (pent - peng) / (R(ph.gamma) - R(1.0));
  }
  if (SL >= R(0.0)) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      FlR[c] = SL * (UL[c] - UL[c]) + SR * (UR[c] - UL[c]);
      FlL[c] = R(0.0);
    }
    entF = entL * VL[1];
  } else if (SR <= R(0.0)) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      FlL[c] = SL * (UR[c] - UL[c]) + SR * (UR[c] - UR[c]);
      FlR[c] = R(0.0);
    }
    entF = entR * VR[1];
  } else {
    const R s1 = t3, s2 = SR * SL * s1;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      FlL[c] = SL * (Us[c] - UL[c]);
      FlR[c] = SR * (UR[c] - Us[c]);
    }
    entF = (SR * entL * VL[1] - SL * entR * VR[1]) * s1 + (entR - entL) * s2;
  }
}

// Multidimensional HLL solver for the induction equation with four states
// (general branch reached when all four speeds straddle zero, which the
// symmetrised LLF speeds always do).
__device__ __forceinline__ double d_rs4(double SR, double SL, double SU, double SD, double cos_t, double sin_t,
                                        double Ez, double BnU, double BnD, double ByR, double ByL) {
  const double EzRU = Ez, EzLU = Ez, EzLD = Ez, EzRD = Ez;
  const double obSx = 1.0 / (SR - SL), obSy = 1.0 / (SU - SD);
  const double csc = 1.0 / sin_t, cot = cos_t / sin_t;
  const double BxRU = (BnU + ByR * cos_t) / sin_t, BxLU = (BnU + ByL * cos_t) / sin_t;
  const double BxRD = (BnD + ByR * cos_t) / sin_t, BxLD = (BnD + ByL * cos_t) / sin_t;
  const double BtRU = BxRU * cos_t + ByR * sin_t, BtLU = BxLU * cos_t + ByL * sin_t;
  const double BtRD = BxRD * cos_t + ByR * sin_t, BtLD = BxLD * cos_t + ByL * sin_t;
  if (SL >= 0.0 && SD >= 0.0) return EzLD;
  if (SR <= 0.0 && SD >= 0.0) return EzRD;
  if (SR <= 0.0 && SU <= 0.0) return EzRU;
  if (SL >= 0.0 && SU <= 0.0) return EzLU;
  if (SL >= 0.0) return (SU * EzLD - SD * EzLU) * obSy + SU * SD * (BxLU - BxLD) * obSy;
  if (SR <= 0.0) return (SU * EzRD - SD * EzRU) * obSy + SU * SD * (BxRU - BxRD) * obSy;
  if (SD >= 0.0) return (SR * EzLD - SL * EzRD) * obSx - SR * SL * (BtRD - BtLD) * obSx;
  if (SU <= 0.0) return (SR * EzLU - SL * EzRU) * obSx - SR * SL * (BtRU - BtLU) * obSx;
  const double BSxL = (SU * BxLU - SD * BxLD) * obSy - (EzLU - EzLD) * obSy, BSyL = ByL;
  const double ESzL = (SU * EzLD - SD * EzLU) * obSy + SU * SD * (BxLU - BxLD) * obSy;
  const double BSxR = (SU * BxRU - SD * BxRD) * obSy - (EzRU - EzRD) * obSy, BSyR = ByR;
  const double ESzR = (SU * EzRD - SD * EzRU) * obSy + SU * SD * (BxRU - BxRD) * obSy;
  double BSt = (SR * BtRD - SL * BtLD) * obSx + (EzRD - EzLD) * obSx;
  const double BSxD = BnD * sin_t + BSt * cos_t, BSyD = -BnD * cos_t + BSt * sin_t;
  const double ESzD = (SR * EzLD - SL * EzRD) * obSx - SR * SL * (BtRD - BtLD) * obSx;
  BSt = (SR * BtRU - SL * BtLU) * obSx + (EzRU - EzLU) * obSx;
  const double BSxU = BnU * sin_t + BSt * cos_t, BSyU = -BnU * cos_t + BSt * sin_t;
  const double ESzU = (SR * EzLU - SL * EzRU) * obSx - SR * SL * (BtRU - BtLU) * obSx;
  const double xc = 0.5 * ((SU + SD) * cos_t + (SR + SL)) / sin_t, yc = 0.5 * (SU + SD);
  const double BSSx = -0.5 * ((-cos_t * ESzR - SR * BSxR) * obSx + (ESzU - SU * BSxU) * obSy +
                              (cos_t * ESzL + SL * BSxL) * obSx + (-ESzD + SD * BSxD) * obSy);
  const double BSSy = -0.5 * ((-sin_t * ESzR - SR * BSyR) * obSx + (-SU * BSyU) * obSy +
                              (sin_t * ESzL + SL * BSyL) * obSx + (SD * BSyD) * obSy);
  const double E1 = -xc * BSSy - 0.5 * (csc * (-sin_t * ESzR - SR * BSyR) + cot * (-SU * BSyU) -
                                        csc * (sin_t * ESzL + SL * BSyL) - cot * (SD * BSyD));
  const double E2 = yc * BSSx + 0.5 * ((ESzU - SU * BSxU) - (-ESzD + SD * BSxD));
  return 0.5 * (E1 + E2);
}

// Three-state multidimensional HLL solver at a cube corner (tri-corner).
__device__ __forceinline__ double d_rs3(double SR1, double SL1, double SR2, double SL2, double SR3, double SL3,
                                        double Ez, double Bn1, double Bn2, double Bn3) {
  const double Ez1 = Ez, Ez2 = Ez, Ez3 = Ez;
  const double sq3_2 = sqrt(3.0) / 2.0, obsq3 = 1.0 / sqrt(3.0);
  const double obS1 = 1.0 / (SR1 - SL1), obS2 = 1.0 / (SR2 - SL2), obS3 = 1.0 / (SR3 - SL3);
  const double Ax = (SL1 + 2.0 * SR2) * obsq3, Ay = -SL1, Bx = (SL2 - SR3) * obsq3, By = SL2 + SR3;
  const double Cx = -(SR1 + 2.0 * SL3) * obsq3, Cy = -SR1;
  const double xc = (Ax + Bx + Cx) / 3.0, yc = (Ay + By + Cy) / 3.0;
  const double l1x = Ax - Cx, l2x = Bx - Ax, l3x = Cx - Bx, l1y = Ay - Cy, l2y = By - Ay, l3y = Cy - By;
  const double l1 = sqrt(l1x * l1x + l1y * l1y), l2 = sqrt(l2x * l2x + l2y * l2y), l3 = sqrt(l3x * l3x + l3y * l3y);
  const double X13x = l1y / l1, X13y = -l1x / l1, X21x = l2y / l2, X21y = -l2x / l2, X32x = l3y / l3, X32y = -l3x / l3;
  const double S13 = X13x * Ax + X13y * Ay, S21 = X21x * Bx + X21y * By, S32 = X32x * Cx + X32y * Cy;
  const double xb13 = 0.5 * (Ax + Cx), yb13 = 0.5 * (Ay + Cy), xb21 = 0.5 * (Bx + Ax), yb21 = 0.5 * (By + Ay);
  const double xb32 = 0.5 * (Cx + Bx), yb32 = 0.5 * (Cy + By);
  const double s = (l1 + l2 + l3) / 2.0;
  const double Area = sqrt(s * (s - l1) * (s - l2) * (s - l3));
  const double Bx1 = (2.0 * Bn2 + Bn1) * obsq3, Bx2 = (Bn2 - Bn3) * obsq3, Bx3 = -(2.0 * Bn3 + Bn1) * obsq3;
  const double By2 = Bn2 + Bn3;
  const double Bt1U1 = Bx1, Bt1U3 = Bx3;
  const double Bt2U1 = -0.5 * Bx1 + sq3_2 * (-Bn1), Bt2U2 = -0.5 * Bx2 + sq3_2 * By2;
  const double Bt3U2 = -0.5 * Bx2 - sq3_2 * By2, Bt3U3 = -0.5 * Bx3 - sq3_2 * (-Bn1);
  const double BSt13 = (SR1 * Bt1U3 - SL1 * Bt1U1 + Ez3 - Ez1) * obS1;
  const double ESz13 = (SR1 * Ez1 - SL1 * Ez3 - SR1 * SL1 * (Bt1U3 - Bt1U1)) * obS1;
  const double BSx13 = BSt13, BSy13 = -Bn1;
  const double BSt21 = (SR2 * Bt2U1 - SL2 * Bt2U2 + Ez1 - Ez2) * obS2;
  const double ESz21 = (SR2 * Ez2 - SL2 * Ez1 - SR2 * SL2 * (Bt2U1 - Bt2U2)) * obS2;
  const double BSx21 = -0.5 * BSt21 + sq3_2 * Bn2, BSy21 = sq3_2 * BSt21 + 0.5 * Bn2;
  const double BSt32 = (SR3 * Bt3U2 - SL3 * Bt3U3 + Ez2 - Ez3) * obS3;
  const double ESz32 = (SR3 * Ez3 - SL3 * Ez2 - SR3 * SL3 * (Bt3U2 - Bt3U3)) * obS3;
  const double BSx32 = -0.5 * BSt32 - sq3_2 * Bn3, BSy32 = -sq3_2 * BSt32 + 0.5 * Bn3;
  if (SL1 >= 0.0 && SR2 <= 0.0) return Ez1;
  if (SL2 >= 0.0 && SR3 <= 0.0) return Ez2;
  if (SL3 >= 0.0 && SR1 <= 0.0) return Ez3;
  if ((SL1 * (SR1 + 2.0 * SL3) + SR1 * (SL1 + 2.0 * SR2)) <= 0) return ESz13;
  if (((SL2 + SR3) * (SL1 + 2.0 * SR2) + (SL2 - SR3) * SL1) <= 0) return ESz21;
  if (((SL2 + SR3) * (SR1 + 2.0 * SL3) - (SL2 - SR3) * SR1) <= 0) return ESz32;
  const double BSSx = ((X13y * ESz13 - S13 * BSx13) * l1 + (X21y * ESz21 - S21 * BSx21) * l2 +
                       (X32y * ESz32 - S32 * BSx32) * l3) / (-2.0 * Area);
  const double BSSy = ((-X13x * ESz13 - S13 * BSy13) * l1 + (-X21x * ESz21 - S21 * BSy21) * l2 +
                       (-X32x * ESz32 - S32 * BSy32) * l3) / (-2.0 * Area);
  const double E1 = -xc * BSSy - ((xb13 - xc) * (-X13x * ESz13 - S13 * BSy13) * l1 +
                                  (xb21 - xc) * (-X21x * ESz21 - S21 * BSy21) * l2 +
                                  (xb32 - xc) * (-X32x * ESz32 - S32 * BSy32) * l3) / Area;
  const double E2 = yc * BSSx + ((yb13 - yc) * (X13y * ESz13 - S13 * BSx13) * l1 +
                                 (yb21 - yc) * (X21y * ESz21 - S21 * BSx21) * l2 +
                                 (yb32 - yc) * (X32y * ESz32 - S32 * BSx32) * l3) / Area;
  return 0.5 * (E1 + E2);
}

// Taylor polynomial (10 modes) at scaled offset (x,y,z).
template <typename R>
__device__ __forceinline__ R d_poly10(const R* v, const R* c, R x, R y, R z) {
  return v[0] + v[1] * x + v[2] * y + v[3] * z + v[4] * (x * x - c[4]) + v[5] * (y * y - c[5]) +
         v[6] * (z * z - c[6]) + v[7] * (x * y - c[7]) + v[8] * (y * z - c[8]) + v[9] * (x * z - c[9]);
}

// In-register Gaussian elimination with scaled partial pivoting for the
// small (9x9, 10x10) normal matrices; returns the inverse, row-major.
template <int n, typename R>
__device__ __forceinline__ void d_matinv(const R* A, R* Ainv) {
  R M[n * n];
  R sc[n];
  int pv[n];
#pragma unroll
  for (int t = 0; t < n * n; ++t) M[t] = A[t];
#pragma unroll
  for (int i = 0; i < n; ++i) {
    R m = R(0.0);
#pragma unroll
    for (int j = 0; j < n; ++j) m = fmax(m, fabs(M[i * n + j]));
    sc[i] = (m == R(0.0)) ? R(0.0) : R(1.0) / m;
    pv[i] = i;
  }
#pragma unroll
  for (int k = 0; k < n; ++k) {
    int p = k;
    R best = -R(1.0);
#pragma unroll
    for (int i = k; i < n; ++i) {
      const R v = fabs(M[i * n + k]) * sc[i];
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (p != k) {
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const R t = M[k * n + j];
        M[k * n + j] = M[p * n + j];
        M[p * n + j] = t;
      }
      const R t = sc[k];
      sc[k] = sc[p];
      sc[p] = t;
      const int ti = pv[k];
      pv[k] = pv[p];
      pv[p] = ti;
    }
    if (M[k * n + k] == R(0.0)) M[k * n + k] = R(1.0e-20);
    const R inv = R(1.0) / M[k * n + k];
#pragma unroll
    for (int i = k + 1; i < n; ++i) {
      const R l = M[i * n + k] * inv;
      M[i * n + k] = l;
#pragma unroll
      for (int j = k + 1; j < n; ++j) M[i * n + j] -= l * M[k * n + j];
    }
  }
#pragma unroll
  for (int c = 0; c < n; ++c) {
    R y[n];
#pragma unroll
    for (int i = 0; i < n; ++i) {
      R s = (pv[i] == c) ? R(1.0) : R(0.0);
#pragma unroll
      for (int j = 0; j < i; ++j) s -= M[i * n + j] * y[j];
      y[i] = s;
    }
#pragma unroll
    for (int i = n - 1; i >= 0; --i) {
      R s = y[i];
#pragma unroll
      for (int j = i + 1; j < n; ++j) s -= M[i * n + j] * Ainv[j * n + c];
      Ainv[i * n + c] = s / M[i * n + i];
    }
  }
}

// Row stride of STEP 7.b's resident row weights [162][stride]: the zone
// count rounded up to 4 elements, so each row starts on a 16-byte (FP32) or
// 32-byte (FP64) boundary.
__host__ __device__ constexpr long long m9_stride(long long n) { return (n + 3) / 4 * 4; }

// Host-side launch helpers implemented in the .cu files.
struct Solve;  // defined in cs_capi.cu
void launch_prim_and_masks(Solve& s);
void launch_face_masks(Solve& s);
void launch_flattener(Solve& s);
void launch_weno(Solve& s);
void launch_positivity(Solve& s);
void launch_faceB_adp(Solve& s);
void launch_adp_factor(Solve& s);
void set_adp_smem_limits();
long long adp_range_count(const Dims& d);
long long adp_factor_doubles(const Dims& d, bool shared);
long long lsq_range_count(const Dims& d);
void launch_ops_build(Solve& s);
void launch_efield(Solve& s);
// STEP 10 min / max into Solve::step10_keys (no-op without CS_FLAG_STEP10).
void launch_step10(Solve& s);
void launch_fluxes(Solve& s);
void launch_edges(Solve& s);
void launch_sources(Solve& s);
void launch_save_stage0(Solve& s);
void launch_combine(Solve& s, double a0, int kind);
// Update, CT and implicit gravity advance by scale times the device-resident
// time step (DStateT::dt), which launch_set_dt sets and launch_timestep
// replaces with the next step.
void launch_update(Solve& s, double scale);
template <typename R>
void launch_update_with(Solve& s, const DStateT<R>& st, double scale);
void launch_gravity_implicit(Solve& s, double scale);
void launch_add_gravity(Solve& s, double c);
void launch_save_stage1_rates(Solve& s);
void launch_restore_stage0(Solve& s);
void launch_cleanup(Solve& s);
void launch_timestep(Solve& s);
void launch_set_dt(Solve& s, double dt);
// Mass, energy and max |div B| of the interior into out[0..2] (part: the
// diag_scratch_doubles() partial sums).
void launch_diag(Solve& s, double* part, double* out);
size_t diag_scratch_doubles();
void launch_fill_ghosts(Solve& s);

}  // namespace cs
