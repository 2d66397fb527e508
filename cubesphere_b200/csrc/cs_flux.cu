// Face fluxes of the stage: five-point quadrature per face, rotation to
// the face frame, HLL solve, rotation back, and the race-free gather of
// the per-face contributions into the zone time derivative; plus the
// explicit point-mass gravity source.
//
// Follows MAKE_FACIAL_FLUXES (pkg/inc/cubesphere/400riemann_integrate/
// 450make_facial_fluxes.f:405-2933), OneD_RS_MHD_Ptwise
// (600riemann_1d/610_1d_rs_oned_rs_mhd_ptwise.f) and
// BUILD_NON_STIFF_SOURCES (470build_non_stiff_sources.f:147-244).
// The reference scatters each face into both neighbours inside one
// parallel loop; here each face writes its two one-sided contributions and
// each zone sums its own six faces in a fixed order.
#include <algorithm>

#include "cs_solve.h"

namespace cs {

namespace {

constexpr int TPB = 128;

template <typename R>
__device__ __forceinline__ R Vm(const DStateT<R>& s, const Dims& d, int comp, int mode, int p, long long o) {
  return s.V[((long long)(mode * NVAR + comp) * NPANEL + p) * d.S + o];
}

// A block takes 32 faces, in two phases.  Face states (450:545-2931): the
// first two warps put each side's five quadrature points, in the side
// zone's scaled coordinates, and its basis moments in shared memory; then
// the five warps evaluate the 18 (side, primitive or entropy) polynomials
// of each face at the five points, each reading that variable's modes once,
// into shared memory, so no face state goes through HBM.  Fluxes: one face
// quadrature point per thread (warp = point) rotates
// the two states to the face frame, solves the HLL problem and rotates the
// contributions back; they meet in shared memory and are summed in point
// order (the order of the reference's quadrature loop).  One launch covers
// the three face directions: tile T is tile T / 3 of direction T % 3, so the
// x, y and z faces of about the same zone rows run side by side and L2
// serves a zone's modes to all three.
constexpr int FLUX_FACES = 32;
// Registers / occupancy: 4 blocks per SM suit the FP64 instantiation, 7 the
// FP32 one (measured on the 6 x 128^2 x 64 shell).
template <typename R>
__global__ void __launch_bounds__(FLUX_FACES * 5, sizeof(R) == 4 ? 7 : 4) k_flux(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r0, Range3 r1, Range3 r2) {
  // the point coordinates and moments are dead once the face states are
  // formed, so they share their space with the flux contributions
  union Scratch {
    R red[5][16][FLUX_FACES];
    struct {
      R pc[2][5][3][FLUX_FACES];  // [side][point][x y z][face]
      R cf[2][6][FLUX_FACES];     // [side][moments 4-9][face]
    } g;
  };
  __shared__ Scratch sc;
  R(&red)[5][16][FLUX_FACES] = sc.red;
  __shared__ R fs[2][9][5][FLUX_FACES];  // [side][primitive 0-7, entropy][point][face]
  __shared__ long long zo[2][FLUX_FACES];  // box offset of each side's zone
  const int lane = threadIdx.x % FLUX_FACES, jq = threadIdx.x / FLUX_FACES;
  const long long nt0 = (r0.count() + FLUX_FACES - 1) / FLUX_FACES, nt1 = (r1.count() + FLUX_FACES - 1) / FLUX_FACES,
                  nt2 = (r2.count() + FLUX_FACES - 1) / FLUX_FACES;
  const long long ntile = 3 * max(nt0, max(nt1, nt2));
  for (long long T = blockIdx.x; T < ntile; T += gridDim.x) {
    const int dir = (int)(T % 3);
    const long long tile = T / 3;
    const Range3 r = dir == 0 ? r0 : (dir == 1 ? r1 : r2);
    if (tile >= (dir == 0 ? nt0 : (dir == 1 ? nt1 : nt2))) continue;  // uniform over the block
    const long long nf = r.count();
    const int QP = dir == 0 ? CS_G_XF_QP : (dir == 1 ? CS_G_YF_QP : CS_G_ZF_QP);
    const int QW = dir == 0 ? CS_G_XF_QW : (dir == 1 ? CS_G_YF_QW : CS_G_ZF_QW);
    const int AR = dir == 0 ? CS_G_XF_AREA : (dir == 1 ? CS_G_YF_AREA : CS_G_ZF_AREA);
    R* F = s.fcon[dir];
    R* SLo = s.S[2 * dir];
    R* SHi = s.S[2 * dir + 1];
    R* EF = s.EF[dir];
    const long long t = tile * FLUX_FACES + lane;
    const bool valid = t < nf;
    int p = 0, i = 0, j = 0, k = 0;
    if (valid) r.decode(t, p, i, j, k);
    int lx = i, ly = j, lz = k, rx = i, ry = j, rz = k;
    bool skip = !valid;
    if (valid) {
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
    }
    // phase 1a: each side's points and moments (a side remapped through
    // istencil at a panel corner is the remapped zone)
    if (jq < 2 && !skip) {
      const int side = jq;
      const int zx = side ? rx : lx, zy = side ? ry : ly, zz = side ? rz : lz;
      zo[side][lane] = d.idx(zx, zy, zz);
      const R obl = R(1.0) / fmax(geoR<R>(g, d, CS_G_V_SCALE, 0, p, zx, zy, zz), R(ph.smallnum));
      const R cx = geoR<R>(g, d, CS_G_V_CEN, 0, p, zx, zy, zz), cy = geoR<R>(g, d, CS_G_V_CEN, 1, p, zx, zy, zz),
              cz = geoR<R>(g, d, CS_G_V_CEN, 2, p, zx, zy, zz);
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        sc.g.pc[side][q][0][lane] = (geoR<R>(g, d, QP, q, p, i, j, k) - cx) * obl;
        sc.g.pc[side][q][1][lane] = (geoR<R>(g, d, QP, 5 + q, p, i, j, k) - cy) * obl;
        sc.g.pc[side][q][2][lane] = (geoR<R>(g, d, QP, 10 + q, p, i, j, k) - cz) * obl;
      }
#pragma unroll
      for (int m = 4; m < 10; ++m) sc.g.cf[side][m - 4][lane] = geoR<R>(g, d, CS_G_COEF, m, p, zx, zy, zz);
    }
    __syncthreads();
    // phase 1b: task v = 0..17 (side v / 9, variable v % 9) of this face;
    // warp jq takes tasks jq, jq + 5, jq + 10, jq + 15
    if (!skip) {
#pragma unroll 1
      for (int v = jq; v < 18; v += 5) {
        const int side = v / 9, var = v % 9;
        const long long oz = zo[side][lane];
        R cc[10];
        cc[0] = cc[1] = cc[2] = cc[3] = R(0.0);
#pragma unroll
        for (int m = 4; m < 10; ++m) cc[m] = sc.g.cf[side][m - 4][lane];
        if (var < 8) {
          R w[10];
#pragma unroll
          for (int m = 0; m < 10; ++m) w[m] = Vm(s, d, var, m, p, oz);
#pragma unroll
          for (int q = 0; q < 5; ++q)
            fs[side][var][q][lane] =
                d_poly10(w, cc, sc.g.pc[side][q][0][lane], sc.g.pc[side][q][1][lane], sc.g.pc[side][q][2][lane]);
        } else {
          const R* E = s.ent;
          const R e0 = E[((long long)0 * NPANEL + p) * d.S + oz], e1 = E[((long long)1 * NPANEL + p) * d.S + oz],
                  e2 = E[((long long)2 * NPANEL + p) * d.S + oz], e3 = E[((long long)3 * NPANEL + p) * d.S + oz];
#pragma unroll
          for (int q = 0; q < 5; ++q)
            fs[side][8][q][lane] = e0 + e1 * sc.g.pc[side][q][0][lane] + e2 * sc.g.pc[side][q][1][lane] +
                                   e3 * sc.g.pc[side][q][2][lane];
        }
      }
    }
    __syncthreads();
    // phase 2: the flux at point jq of face lane
    if (skip) {
#pragma unroll
      for (int c = 0; c < 16; ++c) red[jq][c][lane] = R(0.0);
    } else {
      R Ax, Ay, Az, Bx, By, Bz, Cx, Cy, Cz;
      if (dir == 0) {
        Ax = geoR<R>(g, d, CS_G_XF_N, 0, p, i, j, k);
        Ay = geoR<R>(g, d, CS_G_XF_N, 1, p, i, j, k);
        Az = geoR<R>(g, d, CS_G_XF_N, 2, p, i, j, k);
        Cx = geoR<R>(g, d, CS_G_XF_CEN, 0, p, i, j, k);
        Cy = geoR<R>(g, d, CS_G_XF_CEN, 1, p, i, j, k);
        Cz = geoR<R>(g, d, CS_G_XF_CEN, 2, p, i, j, k);
        const R tt = R(1.0) / fmax(sqrt(Cx * Cx + Cy * Cy + Cz * Cz), R(ph.smallnum));
        Cx = Cx * tt;
        Cy = Cy * tt;
        Cz = Cz * tt;
        Bx = Cy * Az - Cz * Ay;
        By = Cz * Ax - Cx * Az;
        Bz = Cx * Ay - Cy * Ax;
      } else if (dir == 1) {
        Ax = geoR<R>(g, d, CS_G_YF_N, 0, p, i, j, k);
        Ay = geoR<R>(g, d, CS_G_YF_N, 1, p, i, j, k);
        Az = geoR<R>(g, d, CS_G_YF_N, 2, p, i, j, k);
        Bx = geoR<R>(g, d, CS_G_YF_CEN, 0, p, i, j, k);
        By = geoR<R>(g, d, CS_G_YF_CEN, 1, p, i, j, k);
        Bz = geoR<R>(g, d, CS_G_YF_CEN, 2, p, i, j, k);
        const R tt = R(1.0) / fmax(sqrt(Bx * Bx + By * By + Bz * Bz), R(ph.smallnum));
        Bx = Bx * tt;
        By = By * tt;
        Bz = Bz * tt;
        Cx = Ay * Bz - Az * By;
        Cy = Az * Bx - Ax * Bz;
        Cz = Ax * By - Ay * Bx;
      } else {
        auto vt = [&](int q, int x, int y) { return geoR<R>(g, d, CS_G_VERT, q, p, x, y, k); };
        Ax = geoR<R>(g, d, CS_G_ZF_N, jq, p, i, j, k);
        Ay = geoR<R>(g, d, CS_G_ZF_N, 5 + jq, p, i, j, k);
        Az = geoR<R>(g, d, CS_G_ZF_N, 10 + jq, p, i, j, k);
        R tt = R(1.0) / fmax(sqrt(Ax * Ax + Ay * Ay + Az * Az), R(ph.smallnum));
        Ax = Ax * tt;
        Ay = Ay * tt;
        Az = Az * tt;
        Bx = vt(0, i, j) + vt(0, i, j - 1) - vt(0, i - 1, j) - vt(0, i - 1, j - 1);
        By = vt(1, i, j) + vt(1, i, j - 1) - vt(1, i - 1, j) - vt(1, i - 1, j - 1);
        Bz = vt(2, i, j) + vt(2, i, j - 1) - vt(2, i - 1, j) - vt(2, i - 1, j - 1);
        tt = Bx * Ax + By * Ay + Bz * Az;
        Bx = Bx - tt * Ax;
        By = By - tt * Ay;
        Bz = Bz - tt * Az;
        tt = R(1.0) / fmax(sqrt(Bx * Bx + By * By + Bz * Bz), R(ph.smallnum));
        Bx = Bx * tt;
        By = By * tt;
        Bz = Bz * tt;
        Cx = Ay * Bz - Az * By;
        Cy = Az * Bx - Ax * Bz;
        Cz = Ax * By - Ay * Bx;
        tt = R(1.0) / fmax(sqrt(Cx * Cx + Cy * Cy + Cz * Cz), R(ph.smallnum));
        Cx = Cx * tt;
        Cy = Cy * tt;
        Cz = Cz * tt;
      }
      R VL[8], VR[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        VL[c] = fs[0][c][jq][lane];
        VR[c] = fs[1][c][jq][lane];
      }
      const R entL = fs[0][8][jq][lane], entR = fs[1][8][jq][lane];
#pragma unroll
      for (int o = 1; o <= 5; o += 4) {
        R a1 = Ax * VL[o] + Ay * VL[o + 1] + Az * VL[o + 2];
        R b1 = Bx * VL[o] + By * VL[o + 1] + Bz * VL[o + 2];
        R c1 = Cx * VL[o] + Cy * VL[o + 1] + Cz * VL[o + 2];
        VL[o] = a1;
        VL[o + 1] = b1;
        VL[o + 2] = c1;
        a1 = Ax * VR[o] + Ay * VR[o + 1] + Az * VR[o + 2];
        b1 = Bx * VR[o] + By * VR[o + 1] + Bz * VR[o + 2];
        c1 = Cx * VR[o] + Cy * VR[o + 1] + Cz * VR[o + 2];
        VR[o] = a1;
        VR[o + 1] = b1;
        VR[o + 2] = c1;
      }
      R FlL[8], FlR[8], FL[8], FR[8], SL, SR, entF;
      d_hll(ph, VL, VR, entL, entR, FlL, FlR, FL, FR, SL, SR, entF);
      const long long fo = d.idx(i, j, k);
      if (jq == 0) {
        SLo[((long long)p) * d.S + fo] = SL;
        SHi[((long long)p) * d.S + fo] = SR;
        EF[((long long)p) * d.S + fo] = entF;
      }
      const R wt = geoR<R>(g, d, QW, jq, p, i, j, k);
      const R area = geoR<R>(g, d, AR, 0, p, i, j, k);
      const R volL = geoR<R>(g, d, CS_G_V_VOL, 0, p, lx, ly, lz), volR = geoR<R>(g, d, CS_G_V_VOL, 0, p, rx, ry, rz);
      // rotate back to global components: fluctuation + flux on each side
      auto back = [&](const R* W, int c) {
        if (c == 0 || c == 4) return W[c];
        const int o = c < 4 ? 1 : 5, a = c - o;
        const R ea = a == 0 ? Ax : (a == 1 ? Ay : Az), eb = a == 0 ? Bx : (a == 1 ? By : Bz),
                     ec = a == 0 ? Cx : (a == 1 ? Cy : Cz);
        return ea * W[o] + eb * W[o + 1] + ec * W[o + 2];
      };
      // the two sides' net contributions (fluctuation + flux) summed in the
      // face frame and rotated back once, and area / volume once per side
      // (the reference rotates each term and divides every term; the
      // results differ from it in the last bits only)
      R GL[8], GR[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        GL[c] = FlL[c] + FL[c];
        GR[c] = FlR[c] - FR[c];
      }
      const R aL = area / volL, aR = area / volR;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        red[jq][c][lane] = wt * back(GL, c) * aL;
        red[jq][8 + c][lane] = wt * back(GR, c) * aR;
      }
    }
    __syncthreads();
    if (valid) {
      const long long fo = d.idx(i, j, k);
      for (int c = jq; c < 16; c += 5) {
        R acc = R(0.0);
#pragma unroll
        for (int q = 0; q < 5; ++q) acc = acc + red[q][c][lane];
        F[((long long)c * NPANEL + p) * d.S + fo] = acc;
      }
    }
    __syncthreads();
  }
}

// Panel-edge ownership for the face fluxes: a non-owner copy of a shared
// face takes the owner's two one-sided contributions with the sides
// exchanged (their normals are opposite) and the negated entropy flux.
template <typename R>
__global__ void k_sync_flux(Dims d, DStateT<R> s, PanelSync ps) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ps.nf; t += (long long)gridDim.x * blockDim.x) {
    const long long dst = ps.f_dst[t], src = ps.f_src[t];
    const int dd = ps.f_ddir[t], sd = ps.f_sdir[t];
    const int dp = (int)(dst / d.S), sp = (int)(src / d.S);
    const long long dof = dst % d.S, sof = src % d.S;
    R* Fd = s.fcon[dd];
    const R* Fs = s.fcon[sd];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      Fd[((long long)c * NPANEL + dp) * d.S + dof] = Fs[((long long)(8 + c) * NPANEL + sp) * d.S + sof];
      Fd[((long long)(8 + c) * NPANEL + dp) * d.S + dof] = Fs[((long long)c * NPANEL + sp) * d.S + sof];
    }
    s.EF[dd][dst] = -s.EF[sd][src];
  }
}

// The reference's rule for a shared face (CS_FLAG_PANEL_AVERAGE): both
// copies take the average of the two panels' one-sided contributions (the
// sides exchanged between them) and of their entropy fluxes (negated), as
// its defect correction does (FETCH_BUFFERS_FILL_IN_FLUX_X / _Y,
// 334fetch_buffers_fill_in_flux_x.f:295-309).  Each face is in one entry.
template <typename R>
__global__ void k_avg_flux(Dims d, DStateT<R> s, PanelSync ps) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ps.nf; t += (long long)gridDim.x * blockDim.x) {
    const long long dst = ps.f_dst[t], src = ps.f_src[t];
    const int dd = ps.f_ddir[t], sd = ps.f_sdir[t];
    const int dp = (int)(dst / d.S), sp = (int)(src / d.S);
    const long long dof = dst % d.S, sof = src % d.S;
    R* Fd = s.fcon[dd];
    R* Fs = s.fcon[sd];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      R& dl = Fd[((long long)c * NPANEL + dp) * d.S + dof];
      R& dr = Fd[((long long)(8 + c) * NPANEL + dp) * d.S + dof];
      R& sl = Fs[((long long)c * NPANEL + sp) * d.S + sof];
      R& sr = Fs[((long long)(8 + c) * NPANEL + sp) * d.S + sof];
      const R a = (dl + sr) * R(0.5), b = (dr + sl) * R(0.5);
      dl = a;
      sr = a;
      dr = b;
      sl = b;
    }
    const R e = (s.EF[dd][dst] - s.EF[sd][src]) * R(0.5);
    s.EF[dd][dst] = e;
    s.EF[sd][src] = -e;
  }
}

// dU/dt of each zone from its six faces (x, then y, then z; lower face,
// upper face) for the zones whose faces were all computed.
template <typename R>
__global__ void k_gather(Dims d, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    R acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = R(0.0);
    if (mask_at(g, d, p, i, j) == 1) {
      const long long ox[2] = {d.idx(i - 1, j, k), d.idx(i, j, k)};
      const long long oy[2] = {d.idx(i, j - 1, k), d.idx(i, j, k)};
      const long long oz[2] = {d.idx(i, j, k - 1), d.idx(i, j, k)};
      const long long* os[3] = {ox, oy, oz};
      for (int dir = 0; dir < 3; ++dir) {
        const R* F = s.fcon[dir];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          acc[c] = acc[c] - F[((long long)(8 + c) * NPANEL + p) * d.S + os[dir][0]];
          acc[c] = acc[c] - F[((long long)c * NPANEL + p) * d.S + os[dir][1]];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) s.dUdt[d.at(c, p, i, j, k)] = acc[c];
  }
}

// Point-mass gravity on zones 0..N+1 (470:147-244).
template <typename R>
__global__ void k_sources(Dims d, PhysC ph, DGeom g, DStateT<R> s, Range3 r) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < r.count(); t += (long long)gridDim.x * blockDim.x) {
    int p, i, j, k;
    r.decode(t, p, i, j, k);
    if (mask_at(g, d, p, i, j) != 1) continue;
    const R x = geoR<R>(g, d, CS_G_V_CEN, 0, p, i, j, k), y = geoR<R>(g, d, CS_G_V_CEN, 1, p, i, j, k),
                 z = geoR<R>(g, d, CS_G_V_CEN, 2, p, i, j, k);
    const R rho = s.V[d.at(0, p, i, j, k)], vx = s.V[d.at(1, p, i, j, k)], vy = s.V[d.at(2, p, i, j, k)],
                 vz = s.V[d.at(3, p, i, j, k)];
    const R rad = sqrt(x * x + y * y + z * z);
    const R gmb = R(ph.gm) * (R(1.0) / (rad * rad * rad));
    const R S2 = -(gmb * x * rho), S3 = -(gmb * y * rho), S4 = -(gmb * z * rho);
    const R S5 = vx * S2 + vy * S3 + vz * S4;
    s.dUdt[d.at(1, p, i, j, k)] += S2;
    s.dUdt[d.at(2, p, i, j, k)] += S3;
    s.dUdt[d.at(3, p, i, j, k)] += S4;
    s.dUdt[d.at(4, p, i, j, k)] += S5;
  }
}

}  // namespace

template <typename R>
void launch_fluxes_t(Solve& sv, DStateT<R>& st) {
  const Dims& d = sv.d;
  const int N = d.N, nr = d.nr;
  Range3 fx = {-1, N + 1, 0, N + 1, 0, nr + 1};
  Range3 fy = {0, N + 1, -1, N + 1, 0, nr + 1};
  Range3 fz = {0, N + 1, 0, N + 1, -1, nr + 1};
  {
    const long long nt = 3 * ((std::max(fx.count(), std::max(fy.count(), fz.count())) + FLUX_FACES - 1) / FLUX_FACES);
    const int nb = (int)std::min<long long>(nt, (long long)grid_sms(sv) * 32);
    k_flux<R><<<nb, FLUX_FACES * 5, 0, sv.stream>>>(d, sv.ph, sv.g, st, fx, fy, fz);
    mark(sv, "k_flux");
  }
  if (sv.psync.nf > 0 && (sv.p.flags & CS_FLAG_PANEL_AVERAGE)) {
    k_avg_flux<R><<<blocks_for(sv.psync.nf, 128, grid_sms(sv)), 128, 0, sv.stream>>>(d, st, sv.psync);
    mark(sv, "k_avg_flux");
  } else if (sv.psync.nf > 0) {
    k_sync_flux<R><<<blocks_for(sv.psync.nf, 128, grid_sms(sv)), 128, 0, sv.stream>>>(d, st, sv.psync);
    mark(sv, "k_sync_flux");
  }
  Range3 z = {0, N + 1, 0, N + 1, 0, nr + 1};
  k_gather<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.g, st, z);
  mark(sv, "k_gather");
}

void launch_fluxes(Solve& sv) {
  if (sv.fp32)
    launch_fluxes_t(sv, sv.stF);
  else
    launch_fluxes_t(sv, sv.st);
}

template <typename R>
void launch_sources_t(Solve& sv, DStateT<R>& st) {
  if (!(sv.ph.gm > sv.p.smallnum)) return;
  const Dims& d = sv.d;
  Range3 z = {0, d.N + 1, 0, d.N + 1, 0, d.nr + 1};
  k_sources<R><<<blocks_for(z.count(), TPB, grid_sms(sv)), TPB, 0, sv.stream>>>(d, sv.ph, sv.g, st, z);
  mark(sv, "k_sources");
}

void launch_sources(Solve& sv) {
  if (sv.fp32)
    launch_sources_t(sv, sv.stF);
  else
    launch_sources_t(sv, sv.st);
}

}  // namespace cs
