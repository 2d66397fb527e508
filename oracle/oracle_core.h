// ORACLE -- test infrastructure only.  A plain C++ restatement, on the CPU,
// of the SPGEOMESH/CubeSphere per-stage volume update, used as the checker
// for the CUDA implementation.  Nothing here is linked into or called by the
// product library; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline use it.
//
// Parity status: the stage dynamics are unpinned by the reference (the
// Fortran cannot be built here and its tests assert nothing); this file is
// a line-by-line restatement of the cited routines, checked against the
// reference's fixed-input programs and invariants (see tests/).  The mesh
// geometry it consumes is produced by the library's host mesh builder and
// pinned by the golden _T/_200mesh/test_quadpoints.out.
//
// Pointwise physics and linear algebra used by the stage routines.
#pragma once

#include <algorithm>
#include <cmath>

namespace oracle {

constexpr int NV = 8;

struct Phys {
  double gamma, rhofloor, prsfloor, smallnum, pi, ob4pi, ob8pi;
};

// PRIM_TO_CONS, ideal MHD, adiabatic, PRESSURE_POSITIVITY 1
// (pkg/inc/cubesphere/660pde_3d/661pde_3d_prim_to_cons.f:14-125).
inline void prim_to_cons(const Phys& ph, double ent, double* U, double* V) {
  V[0] = std::max(V[0], ph.rhofloor);
  double rho = V[0];
  if (V[4] <= ph.prsfloor) V[4] = std::max(ph.prsfloor, ent * std::pow(rho, ph.gamma - 1.0));
  U[0] = V[0];
  U[1] = V[0] * V[1];
  U[2] = V[0] * V[2];
  U[3] = V[0] * V[3];
  U[5] = V[5];
  U[6] = V[6];
  U[7] = V[7];
  U[4] = V[4] / (ph.gamma - 1.0) + 0.5 * V[0] * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]) +
         ph.ob8pi * (V[5] * V[5] + V[6] * V[6] + V[7] * V[7]);
}

// CONS_TO_PRIM (662pde_3d_cons_to_prim.f:14-151); ent is in/out, returns iprs_flag.
inline int cons_to_prim(const Phys& ph, double& ent, double* U, double* V) {
  int flag = 0;
  U[0] = std::max(U[0], ph.rhofloor);
  V[0] = U[0];
  double a = V[0] / (V[0] * V[0] + ph.rhofloor * ph.rhofloor);
  V[1] = U[1] * a;
  V[2] = U[2] * a;
  V[3] = U[3] * a;
  V[5] = U[5];
  V[6] = U[6];
  V[7] = U[7];
  double V2 = V[1] * V[1] + V[2] * V[2] + V[3] * V[3];
  double B2 = V[5] * V[5] + V[6] * V[6] + V[7] * V[7];
  V[4] = (ph.gamma - 1.0) * (U[4] - 0.5 * V[0] * V2 - ph.ob8pi * B2);
  double rho = V[0];
  if (V[4] <= ph.prsfloor) {
    V[4] = std::max(ph.prsfloor, ent * std::pow(rho, ph.gamma - 1.0));
    flag = 1;
  }
  ent = V[4] / std::pow(V[0], ph.gamma - 1.0);
  U[4] = V[4] / (ph.gamma - 1.0) + 0.5 * V[0] * V2 + ph.ob8pi * B2;
  return flag;
}

// PRIM_TO_WAVSPD, x-direction (660pde_3d_prim_to_wavspd.f:54-87).
inline void prim_to_wavspd_x(const Phys& ph, const double* V, double& smin, double& smax) {
  double rho = V[0], prs = V[4];
  double bfx = V[5], bfy = V[6], bfz = V[7];
  double cs = std::sqrt(ph.gamma * prs / rho);
  double b2 = (bfx * bfx + bfy * bfy + bfz * bfz) / (4.0 * ph.pi * rho);
  double bb = -(cs * cs + b2);
  double cc = cs * cs * bfx * bfx / (4.0 * ph.pi * rho);
  double mf = std::sqrt((-bb + std::sqrt(bb * bb - 4.0 * 1.0 * cc)) / (2.0 * 1.0));
  smin = V[1] - mf;
  smax = V[1] + mf;
}

// Ideal-MHD x-flux F(V) with B0 = 0, the in-tree statement of MHD_V_TO_UFG
// (620riemann_2d/620_2d_rs_mhd_v_to_ufg.f:23-105), standing in for the
// CONS_PRIM_TO_FLUX_3D that the 1D solver calls but the tree does not define.
inline void flux_x(const Phys& ph, const double* V, double* F) {
  double U[NV];
  U[0] = V[0];
  U[1] = V[0] * V[1];
  U[2] = V[0] * V[2];
  U[3] = V[0] * V[3];
  U[4] = V[4] / (ph.gamma - 1.0) + 0.5 * V[0] * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]) +
         ph.ob8pi * (V[5] * V[5] + V[6] * V[6] + V[7] * V[7]);
  U[5] = V[5];
  U[6] = V[6];
  U[7] = V[7];
  double B2 = V[5] * V[5] + V[6] * V[6] + V[7] * V[7];
  double vdb = V[1] * V[5] + V[2] * V[6] + V[3] * V[7];
  double ptot = V[4] + ph.ob8pi * B2;
  for (int c = 0; c < NV; ++c) F[c] = V[1] * U[c];
  F[1] = F[1] + ptot - ph.ob4pi * V[5] * V[5];
  F[2] = F[2] - ph.ob4pi * V[5] * V[6];
  F[3] = F[3] - ph.ob4pi * V[5] * V[7];
  F[4] = F[4] + ptot * V[1] - ph.ob4pi * V[5] * vdb;
  F[5] = 0.0;
  F[6] = F[6] - V[5] * V[2];
  F[7] = F[7] - V[5] * V[3];
}

// OneD_RS_MHD_Ptwise, HLL branch for ideal MHD with PRESSURE_POSITIVITY 1
// (600riemann_1d/610_1d_rs_oned_rs_mhd_ptwise.f:100-237, :644-705).
// V_L / V_R are modified (the normal B is averaged), as in the reference.
struct RSOut {
  double SL, SR, Ustar[NV], Fstar[NV], entF, FlL[NV], FlR[NV], UL[NV], UR[NV], FL[NV], FR[NV];
};
inline void oned_rs_hll(const Phys& ph, double* VL, double* VR, double entL, double entR, RSOut& o) {
  double bx = 0.5 * (VL[5] + VR[5]);
  VL[5] = bx;
  VR[5] = bx;
  prim_to_cons(ph, entL, o.UL, VL);
  prim_to_cons(ph, entR, o.UR, VR);
  flux_x(ph, VL, o.FL);
  flux_x(ph, VR, o.FR);
  double SR = -1.0e30, SL = 1.0e30, smin, smax;
  prim_to_wavspd_x(ph, VL, smin, smax);
  SL = std::min(SL, smin);
  SR = std::max(SR, smax);
  prim_to_wavspd_x(ph, VR, smin, smax);
  SL = std::min(SL, smin);
  SR = std::max(SR, smax);
  double Vm[NV];
  for (int c = 0; c < NV; ++c) Vm[c] = 0.5 * (VL[c] + VR[c]);
  prim_to_wavspd_x(ph, Vm, smin, smax);
  SL = std::min(SL, smin);
  SR = std::max(SR, smax);
  double t3 = 1.0 / (SR - SL), t1 = SR * t3, t2 = SL * t3;
  for (int c = 0; c < NV; ++c) o.Ustar[c] = t1 * o.UR[c] - t2 * o.UL[c] - t3 * (o.FR[c] - o.FL[c]);
  double entU = t1 * entR - t2 * entL - t3 * (entR * VR[1] - entL * VL[1]);
  double *Us = o.Ustar;
  double p_ent = entU * std::pow(Us[0], ph.gamma - 1.0);
  double p_eng = (ph.gamma - 1.0) * (Us[4] - 0.5 * (Us[1] * Us[1] + Us[2] * Us[2] + Us[3] * Us[3]) / Us[0] -
                                     ph.ob8pi * (Us[5] * Us[5] + Us[6] * Us[6] + Us[7] * Us[7]));
  if (p_eng <= ph.prsfloor) Us[4] = Us[4] + (p_ent - p_eng) / (ph.gamma - 1.0);
  if (SL >= 0.0) {
    for (int c = 0; c < NV; ++c) {
      o.Ustar[c] = o.UL[c];
      o.Fstar[c] = o.FL[c];
    }
    o.entF = entL * VL[1];
    for (int c = 0; c < NV; ++c) {
      o.FlR[c] = SL * (o.Ustar[c] - o.UL[c]) + SR * (o.UR[c] - o.Ustar[c]);
      o.FlL[c] = 0.0;
    }
  } else if (SR <= 0.0) {
    for (int c = 0; c < NV; ++c) {
      o.Ustar[c] = o.UR[c];
      o.Fstar[c] = o.FR[c];
    }
    o.entF = entR * VR[1];
    for (int c = 0; c < NV; ++c) {
      o.FlL[c] = SL * (o.Ustar[c] - o.UL[c]) + SR * (o.UR[c] - o.Ustar[c]);
      o.FlR[c] = 0.0;
    }
  } else {
    double s1 = 1.0 / (SR - SL), s2 = SR * SL * s1;
    for (int c = 0; c < NV; ++c) {
      o.Fstar[c] = 0.5 * (o.FL[c] + o.FR[c]) + 0.5 * SL * (o.Ustar[c] - o.UL[c]) - 0.5 * SR * (o.UR[c] - o.Ustar[c]);
      o.FlL[c] = SL * (o.Ustar[c] - o.UL[c]);
      o.FlR[c] = SR * (o.UR[c] - o.Ustar[c]);
    }
    o.entF = (SR * entL * VL[1] - SL * entR * VR[1]) * s1 + (entR - entL) * s2;
  }
  o.SL = SL;
  o.SR = SR;
}

// Two_D_RS_Ez_4State_HLL (620riemann_2d/630_2d_rs_ez_two_d_rs_ez_4state_hll.f:10-372); returns ESSz.
inline double twod_rs_ez_4state(double SR, double SL, double SU, double SD, double cos_t, double sin_t,
                                double EzRU, double EzLU, double EzLD, double EzRD, double BnU, double BnD,
                                double ByR, double ByL) {
  double obSx = 1.0 / (SR - SL), obSy = 1.0 / (SU - SD);
  double csc = 1.0 / sin_t, cot = cos_t / sin_t;
  double BxRU = (BnU + ByR * cos_t) / sin_t, ByRU = ByR;
  double BxLU = (BnU + ByL * cos_t) / sin_t, ByLU = ByL;
  double BxRD = (BnD + ByR * cos_t) / sin_t, ByRD = ByR;
  double BxLD = (BnD + ByL * cos_t) / sin_t, ByLD = ByL;
  double BtRU = BxRU * cos_t + ByRU * sin_t;
  double BtLU = BxLU * cos_t + ByLU * sin_t;
  double BtRD = BxRD * cos_t + ByRD * sin_t;
  double BtLD = BxLD * cos_t + ByLD * sin_t;
  if (SL >= 0.0 && SD >= 0.0) return EzLD;
  if (SR <= 0.0 && SD >= 0.0) return EzRD;
  if (SR <= 0.0 && SU <= 0.0) return EzRU;
  if (SL >= 0.0 && SU <= 0.0) return EzLU;
  if (SL >= 0.0) return (SU * EzLD - SD * EzLU) * obSy + SU * SD * (BxLU - BxLD) * obSy;
  if (SR <= 0.0) return (SU * EzRD - SD * EzRU) * obSy + SU * SD * (BxRU - BxRD) * obSy;
  if (SD >= 0.0) return (SR * EzLD - SL * EzRD) * obSx - SR * SL * (BtRD - BtLD) * obSx;
  if (SU <= 0.0) return (SR * EzLU - SL * EzRU) * obSx - SR * SL * (BtRU - BtLU) * obSx;
  double BSxL = (SU * BxLU - SD * BxLD) * obSy - (EzLU - EzLD) * obSy;
  double BSyL = ByL;
  double ESzL = (SU * EzLD - SD * EzLU) * obSy + SU * SD * (BxLU - BxLD) * obSy;
  double BSxR = (SU * BxRU - SD * BxRD) * obSy - (EzRU - EzRD) * obSy;
  double BSyR = ByR;
  double ESzR = (SU * EzRD - SD * EzRU) * obSy + SU * SD * (BxRU - BxRD) * obSy;
  double BSn = BnD;
  double BSt = (SR * BtRD - SL * BtLD) * obSx + (EzRD - EzLD) * obSx;
  double BSxD = BSn * sin_t + BSt * cos_t;
  double BSyD = -BSn * cos_t + BSt * sin_t;
  double ESzD = (SR * EzLD - SL * EzRD) * obSx - SR * SL * (BtRD - BtLD) * obSx;
  BSn = BnU;
  BSt = (SR * BtRU - SL * BtLU) * obSx + (EzRU - EzLU) * obSx;
  double BSxU = BSn * sin_t + BSt * cos_t;
  double BSyU = -BSn * cos_t + BSt * sin_t;
  double ESzU = (SR * EzLU - SL * EzRU) * obSx - SR * SL * (BtRU - BtLU) * obSx;
  double xc = 0.5 * ((SU + SD) * cos_t + (SR + SL)) / sin_t;
  double yc = 0.5 * (SU + SD);
  double BSSx = -0.5 * ((-cos_t * ESzR - SR * BSxR) * obSx + (ESzU - SU * BSxU) * obSy +
                        (cos_t * ESzL + SL * BSxL) * obSx + (-ESzD + SD * BSxD) * obSy);
  double BSSy = -0.5 * ((-sin_t * ESzR - SR * BSyR) * obSx + (-SU * BSyU) * obSy +
                        (sin_t * ESzL + SL * BSyL) * obSx + (SD * BSyD) * obSy);
  double E1 = -xc * BSSy - 0.5 * (csc * (-sin_t * ESzR - SR * BSyR) + cot * (-SU * BSyU) -
                                  csc * (sin_t * ESzL + SL * BSyL) - cot * (SD * BSyD));
  double E2 = yc * BSSx + 0.5 * ((ESzU - SU * BSxU) - (-ESzD + SD * BSxD));
  return 0.5 * (E1 + E2);
}

// Two_D_RS_Ez_3State_HLL (620riemann_2d/631_2d_rs_ez_two_d_rs_ez_3state_hll.f:9-338); returns ESSz.
inline double twod_rs_ez_3state(double SR1, double SL1, double SR2, double SL2, double SR3, double SL3,
                                double Ez1, double Ez2, double Ez3, double Bn1, double Bn2, double Bn3) {
  double sq3_2 = std::sqrt(3.0) / 2.0, obsq3 = 1.0 / std::sqrt(3.0);
  double obS1 = 1.0 / (SR1 - SL1), obS2 = 1.0 / (SR2 - SL2), obS3 = 1.0 / (SR3 - SL3);
  double Ax = (SL1 + 2.0 * SR2) * obsq3, Ay = -SL1;
  double Bx = (SL2 - SR3) * obsq3, By = SL2 + SR3;
  double Cx = -(SR1 + 2.0 * SL3) * obsq3, Cy = -SR1;
  double xc = (Ax + Bx + Cx) / 3.0, yc = (Ay + By + Cy) / 3.0;
  double l1x = Ax - Cx, l2x = Bx - Ax, l3x = Cx - Bx;
  double l1y = Ay - Cy, l2y = By - Ay, l3y = Cy - By;
  double l1 = std::sqrt(l1x * l1x + l1y * l1y), l2 = std::sqrt(l2x * l2x + l2y * l2y),
         l3 = std::sqrt(l3x * l3x + l3y * l3y);
  double X13x = l1y / l1, X13y = -l1x / l1, X21x = l2y / l2, X21y = -l2x / l2, X32x = l3y / l3, X32y = -l3x / l3;
  double S13 = X13x * Ax + X13y * Ay, S21 = X21x * Bx + X21y * By, S32 = X32x * Cx + X32y * Cy;
  double xb13 = 0.5 * (Ax + Cx), yb13 = 0.5 * (Ay + Cy), xb21 = 0.5 * (Bx + Ax), yb21 = 0.5 * (By + Ay);
  double xb32 = 0.5 * (Cx + Bx), yb32 = 0.5 * (Cy + By);
  double s = (l1 + l2 + l3) / 2.0;
  double Area = std::sqrt(s * (s - l1) * (s - l2) * (s - l3));
  double Bx1 = (2.0 * Bn2 + Bn1) * obsq3, Bx2 = (Bn2 - Bn3) * obsq3, Bx3 = -(2.0 * Bn3 + Bn1) * obsq3;
  double By1 = -Bn1, By2 = Bn2 + Bn3, By3 = -Bn1;
  (void)By1; (void)By3;
  double Bt1U1 = Bx1, Bt1U3 = Bx3;
  double Bt2U1 = -0.5 * Bx1 + sq3_2 * (-Bn1), Bt2U2 = -0.5 * Bx2 + sq3_2 * By2;
  double Bt3U2 = -0.5 * Bx2 - sq3_2 * By2, Bt3U3 = -0.5 * Bx3 - sq3_2 * (-Bn1);
  double BSn13 = Bn1;
  double BSt13 = (SR1 * Bt1U3 - SL1 * Bt1U1 + Ez3 - Ez1) * obS1;
  double ESz13 = (SR1 * Ez1 - SL1 * Ez3 - SR1 * SL1 * (Bt1U3 - Bt1U1)) * obS1;
  double BSx13 = BSt13, BSy13 = -BSn13;
  double BSn21 = Bn2;
  double BSt21 = (SR2 * Bt2U1 - SL2 * Bt2U2 + Ez1 - Ez2) * obS2;
  double ESz21 = (SR2 * Ez2 - SL2 * Ez1 - SR2 * SL2 * (Bt2U1 - Bt2U2)) * obS2;
  double BSx21 = -0.5 * BSt21 + sq3_2 * BSn21, BSy21 = sq3_2 * BSt21 + 0.5 * BSn21;
  double BSn32 = Bn3;
  double BSt32 = (SR3 * Bt3U2 - SL3 * Bt3U3 + Ez2 - Ez3) * obS3;
  double ESz32 = (SR3 * Ez3 - SL3 * Ez2 - SR3 * SL3 * (Bt3U2 - Bt3U3)) * obS3;
  double BSx32 = -0.5 * BSt32 - sq3_2 * BSn32, BSy32 = -sq3_2 * BSt32 + 0.5 * BSn32;
  if (SL1 >= 0.0 && SR2 <= 0.0) return Ez1;
  if (SL2 >= 0.0 && SR3 <= 0.0) return Ez2;
  if (SL3 >= 0.0 && SR1 <= 0.0) return Ez3;
  if ((SL1 * (SR1 + 2.0 * SL3) + SR1 * (SL1 + 2.0 * SR2)) <= 0) return ESz13;
  if (((SL2 + SR3) * (SL1 + 2.0 * SR2) + (SL2 - SR3) * SL1) <= 0) return ESz21;
  if (((SL2 + SR3) * (SR1 + 2.0 * SL3) - (SL2 - SR3) * SR1) <= 0) return ESz32;
  double BSSx = ((X13y * ESz13 - S13 * BSx13) * l1 + (X21y * ESz21 - S21 * BSx21) * l2 +
                 (X32y * ESz32 - S32 * BSx32) * l3) / (-2.0 * Area);
  double BSSy = ((-X13x * ESz13 - S13 * BSy13) * l1 + (-X21x * ESz21 - S21 * BSy21) * l2 +
                 (-X32x * ESz32 - S32 * BSy32) * l3) / (-2.0 * Area);
  double E1 = -xc * BSSy - ((xb13 - xc) * (-X13x * ESz13 - S13 * BSy13) * l1 +
                            (xb21 - xc) * (-X21x * ESz21 - S21 * BSy21) * l2 +
                            (xb32 - xc) * (-X32x * ESz32 - S32 * BSy32) * l3) / Area;
  double E2 = yc * BSSx + ((yb13 - yc) * (X13y * ESz13 - S13 * BSx13) * l1 +
                           (yb21 - yc) * (X21y * ESz21 - S21 * BSx21) * l2 +
                           (yb32 - yc) * (X32y * ESz32 - S32 * BSx32) * l3) / Area;
  return 0.5 * (E1 + E2);
}

// LU with scaled partial pivoting, written from the textbook algorithm
// (Golub & Van Loan, Matrix Computations, sec. 3.4), standing in for the
// MATSOLVE / MATINV the reference builds on its vendored LU
// (pkg/inc/cubesphere/100math/120matsolve.f:7, 121matinv.f:8).
// A is n x n row-major, overwritten by its factors; piv gets the row order.
inline void lu_factor(int n, double* A, int* piv) {
  double scale[64];
  for (int i = 0; i < n; ++i) {
    double m = 0.0;
    for (int j = 0; j < n; ++j) m = std::max(m, std::fabs(A[i * n + j]));
    scale[i] = (m == 0.0) ? 0.0 : 1.0 / m;
    piv[i] = i;
  }
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = -1.0;
    for (int i = k; i < n; ++i) {
      double v = std::fabs(A[i * n + k]) * scale[i];
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
      std::swap(scale[k], scale[p]);
      std::swap(piv[k], piv[p]);
    }
    if (A[k * n + k] == 0.0) A[k * n + k] = 1.0e-20;
    double inv = 1.0 / A[k * n + k];
    for (int i = k + 1; i < n; ++i) {
      double l = A[i * n + k] * inv;
      A[i * n + k] = l;
      for (int j = k + 1; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
    }
  }
}
inline void lu_solve(int n, const double* LU, const int* piv, const double* b, double* x) {
  double y[64];
  for (int i = 0; i < n; ++i) {
    double s = b[piv[i]];
    for (int j = 0; j < i; ++j) s -= LU[i * n + j] * y[j];
    y[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = y[i];
    for (int j = i + 1; j < n; ++j) s -= LU[i * n + j] * x[j];
    x[i] = s / LU[i * n + i];
  }
}
// Inverse of A (row-major) into Ainv (row-major).
inline void matinv(int n, const double* A, double* Ainv) {
  double LU[64 * 64];
  int piv[64];
  for (int t = 0; t < n * n; ++t) LU[t] = A[t];
  lu_factor(n, LU, piv);
  double e[64], x[64];
  for (int c = 0; c < n; ++c) {
    for (int i = 0; i < n; ++i) e[i] = (i == c) ? 1.0 : 0.0;
    lu_solve(n, LU, piv, e, x);
    for (int i = 0; i < n; ++i) Ainv[i * n + c] = x[i];
  }
}

}  // namespace oracle
