// Host-side mesh build of the 6-panel cubed sphere: equiangular gnomonic
// sector meshes with ghost rows, radial meshes, per-panel vertex extraction
// with the tri-corner mask, the 12-neighbour stencil table and the degree-2
// isoparametric face / B-field / volume geometry plus the Taylor-basis
// moments.  Runs once per solve; the result is copied to the device.
//
// Restates, from SPGEOMESH/CubeSphere:
//   SWIVEL_N, Mesh_Sector_General     pkg/inc/cubesphere/200mesh/201mesh_sector_general.f:12-827
//   GENERATE_GLOBAL_RADIAL_{UNIFORM,LOG,STRETCHED}_MESH  200mesh/202generate_global_radial_mesh.f:10-235
//   FILL_GHOST2D_GLOBAL               200mesh/203fill_ghost2d_global.f:7-167
//   EXTRACT_VERT_COORDS_PATCH         200mesh/210extract_vert_coords_patch.f:7-355
//   STENCIL_INDEXING_TRICORNERS       200mesh/211stencil_indexing_tricorners.f:6-653
//   COORDS_TO_WT_QUADPTS_FACES_ISO2   200mesh/220coords_to_wt_quadpts_faces_iso2.f:7-2299
//   COORDS_TO_WT_QUADPTS_BFLD_ISO2    200mesh/230coords_to_wt_quadpts_bfld_iso2.f:8 (weights only:
//                                      its points and normals equal the face ones)
//   COORDS_TO_WT_QUADPTS_VOLUME_ISO2  200mesh/240coords_to_wt_quadpts_volume_iso2.f:7-1166
//   BUILD_MODE_INDICES / INIT_BASIS_FUNCTION_COEFS  200mesh/204build_mode_indices.f:7,
//                                      200mesh/250init_basis_function_coefs.f:5-267
#include <cmath>
#include <cstring>

#include "cs_internal.h"

namespace cs {

namespace {

struct V3 {
  double x = 0, y = 0, z = 0;
};
inline V3 vsub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 vscale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double vnorm(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
// Integer power by repeated multiplication (x**n with integer n).
inline double ipow(double x, int n) {
  double r = 1.0;
  for (int t = 0; t < n; ++t) r *= x;
  return r;
}
inline V3 vcross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// Great-circle subdivision of the arc a1 -> a2 into n equal angles.
void swivel(V3 a1, V3 a2, int n, std::vector<V3>& out) {
  out.assign(n + 1, V3{});
  double dot = a1.x * a2.x + a1.y * a2.y + a1.z * a2.z;
  double theta = std::acos(dot);
  double dth = theta / (double)n;
  out[0] = a1;
  out[n] = a2;
  V3 x = a1;
  V3 y = vsub(a2, vscale(x, dot));
  double t = vnorm(y);
  y = vscale(y, 1.0 / t);
  for (int i = 1; i < n; ++i) {
    double ang = dth * (double)i;
    out[i] = vadd(vscale(x, std::cos(ang)), vscale(y, std::sin(ang)));
  }
}

// Corners of the six cube faces projected to the unit sphere, in the order
// (lower-left, lower-right, upper-left, upper-right) of each sector.
void sector_corners(int isector, V3 v[4]) {
  const double s = 1.0 / std::sqrt(3.0);
  static const int tab[6][4][3] = {
      {{-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}},
      {{-1, 1, -1}, {-1, 1, 1}, {1, 1, -1}, {1, 1, 1}},
      {{1, -1, -1}, {1, 1, -1}, {1, -1, 1}, {1, 1, 1}},
      {{1, 1, -1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, -1}},
      {{1, -1, 1}, {-1, -1, 1}, {1, -1, -1}, {-1, -1, -1}},
      {{-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}}};
  for (int c = 0; c < 4; ++c)
    v[c] = {tab[isector - 1][c][0] * s, tab[isector - 1][c][1] * s, tab[isector - 1][c][2] * s};
}

// Unit-sphere vertices of one sector, (n+2g+1)^2 points, interior only;
// ghost rows are filled afterwards from the neighbours.
void sector_mesh(int isector, int n, int g, std::vector<V3>& coords) {
  const int w = n + 2 * g + 1;
  coords.assign((size_t)w * w, V3{});
  V3 c[4];
  sector_corners(isector, c);
  std::vector<V3> a1, a2, a3, a4;
  swivel(c[0], c[1], n, a1);
  swivel(c[2], c[3], n, a2);
  swivel(c[0], c[2], n, a3);
  swivel(c[1], c[3], n, a4);
  for (int j = 0; j <= n; ++j)
    for (int i = 0; i <= n; ++i) {
      V3 A = vcross(a1[i], a2[i]);
      V3 B = vcross(a3[j], a4[j]);
      V3 C = vcross(B, A);
      bool flip = (isector == 1 && C.z < 0) || (isector == 4 && C.z > 0) || (isector == 2 && C.y < 0) ||
                  (isector == 5 && C.y > 0) || (isector == 3 && C.x < 0) || (isector == 6 && C.x > 0);
      if (flip) C = vscale(C, -1.0);
      double t = 1.0 / vnorm(C);
      coords[(size_t)(j + g) * w + (i + g)] = vscale(C, t);
    }
}

// Panel adjacency: right, left, up, down neighbour of each sector (1-based).
const int kNbr[6][4] = {{3, 6, 2, 5}, {1, 4, 3, 6}, {2, 5, 1, 4}, {5, 2, 6, 3}, {6, 3, 4, 1}, {4, 1, 5, 2}};

void fill_ghost2d(int n, int g, std::vector<V3> sec[6]) {
  const int w = n + 2 * g + 1;
  auto at = [&](int s, int i, int j) -> V3& { return sec[s][(size_t)(j + g) * w + (i + g)]; };
  for (int s = 0; s < 6; ++s) {
    int rt = kNbr[s][0] - 1, lf = kNbr[s][1] - 1, up = kNbr[s][2] - 1, dn = kNbr[s][3] - 1;
    for (int i = n + 1; i <= n + g; ++i) {
      int jy = n - 1 - (i - n - 1);
      for (int j = 0; j <= n; ++j) at(s, i, j) = at(rt, j, jy);
    }
    for (int i = -1; i >= -g; --i) {
      int ix = 1 - (i + 1);
      for (int j = 0; j <= n; ++j) at(s, i, j) = at(lf, ix, n - j);
    }
    for (int j = n + 1; j <= n + g; ++j) {
      int ix = n - 1 - (j - n - 1);
      for (int i = 0; i <= n; ++i) at(s, i, j) = at(up, ix, i);
    }
    for (int j = -1; j >= -g; --j) {
      int jy = 1 - (j + 1);
      for (int i = 0; i <= n; ++i) at(s, i, j) = at(dn, n - i, jy);
    }
  }
}

std::string radial_mesh(int kind, int nr, int g, double rmin, double rmax, double ratio, double smallnum,
                        std::vector<double>& rb) {
  rb.assign(nr + 2 * g + 1, 0.0);
  auto R = [&](int i) -> double& { return rb[i + g]; };
  if (kind == CS_RADIAL_UNIFORM) {
    for (int i = -g; i <= nr + g; ++i) R(i) = rmin + (rmax - rmin) * ((double)i / (double)nr);
  } else if (kind == CS_RADIAL_LOG) {
    for (int i = -g; i <= nr + g; ++i) R(i) = rmin * std::pow(rmax / rmin, (double)i / (double)nr);
  } else if (kind == CS_RADIAL_STRETCHED) {
    int N = nr + 1;
    double dx1;
    if (ratio > 1.0 + smallnum) {
      dx1 = (rmax - rmin) / ((std::pow(ratio, N) - 1.0) / (ratio - 1.0));
    } else {
      dx1 = (rmax - rmin) / nr;
      ratio = 1.0;
    }
    R(0) = rmin;
    for (int i = 1; i <= nr; ++i) R(i) = dx1 * std::pow(ratio, i - 1) + R(i - 1);
    double dx0 = R(1) - R(0);
    for (int i = -g; i <= -1; ++i) R(i) = R(0) + i * dx0;
    double dxN = R(nr) - R(nr - 1);
    for (int i = nr + 1; i <= nr + g; ++i) R(i) = R(nr) + (i - nr) * dxN;
  } else {
    return "unknown radial mesh kind";
  }
  return "";
}

// ---------------- isoparametric elements ----------------
// 8-node serendipity quadrilateral on [-1/2,1/2]^2 and its derivatives.
void quad8(double x, double y, double N[8], double dx[8], double dy[8]) {
  N[0] = (0.5 - x) * (0.5 - y) * (-2.0 * x - 2.0 * y - 1.0);
  N[1] = (0.5 + x) * (0.5 - y) * (2.0 * x - 2.0 * y - 1.0);
  N[2] = (0.5 + x) * (0.5 + y) * (2.0 * x + 2.0 * y - 1.0);
  N[3] = (0.5 - x) * (0.5 + y) * (-2.0 * x + 2.0 * y - 1.0);
  N[4] = (1.0 - 4.0 * x * x) * (0.5 - y);
  N[5] = (0.5 + x) * (1.0 - 4.0 * y * y);
  N[6] = (1.0 - 4.0 * x * x) * (0.5 + y);
  N[7] = (0.5 - x) * (1.0 - 4.0 * y * y);
  dx[0] = (0.5 - y) * (4.0 * x + 2.0 * y);
  dy[0] = (0.5 - x) * (2.0 * x + 4.0 * y);
  dx[1] = (0.5 - y) * (4.0 * x - 2.0 * y);
  dy[1] = (0.5 + x) * (-2.0 * x + 4.0 * y);
  dx[2] = (0.5 + y) * (4.0 * x + 2.0 * y);
  dy[2] = (0.5 + x) * (2.0 * x + 4.0 * y);
  dx[3] = (0.5 + y) * (4.0 * x - 2.0 * y);
  dy[3] = (0.5 - x) * (-2.0 * x + 4.0 * y);
  dx[4] = -8.0 * x * (0.5 - y);
  dy[4] = -(1.0 - 4.0 * x * x);
  dx[5] = 1.0 - 4.0 * y * y;
  dy[5] = -8.0 * y * (0.5 + x);
  dx[6] = -8.0 * x * (0.5 + y);
  dy[6] = 1.0 - 4.0 * x * x;
  dx[7] = -(1.0 - 4.0 * y * y);
  dy[7] = -8.0 * y * (0.5 - x);
}

// 20-node serendipity hexahedron: corners 1..8 in the reference order
// (-,-,-),(+,-,-),(+,+,-),(-,+,-),(-,-,+),(+,-,+),(+,+,+),(-,+,+); then the
// x-edge, y-edge and radial-edge midpoints.
void hex20(double x, double y, double z, double N[20], double dx[20], double dy[20], double dz[20]) {
  static const int sg[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                               {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  for (int n = 0; n < 8; ++n) {
    double sx = sg[n][0], sy = sg[n][1], sz = sg[n][2];
    double fx = 0.5 + sx * x, fy = 0.5 + sy * y, fz = 0.5 + sz * z;
    double l = 2.0 * sx * x + 2.0 * sy * y + 2.0 * sz * z - 2.0;
    N[n] = fx * fy * fz * l;
    dx[n] = sx * fy * fz * (4.0 * sx * x + 2.0 * sy * y + 2.0 * sz * z - 1.0);
    dy[n] = sy * fx * fz * (2.0 * sx * x + 4.0 * sy * y + 2.0 * sz * z - 1.0);
    dz[n] = sz * fx * fy * (2.0 * sx * x + 2.0 * sy * y + 4.0 * sz * z - 1.0);
  }
  // x-edges: (y,z) signs (-,-),(+,-),(+,+),(-,+)
  static const int ex[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
  for (int e = 0; e < 4; ++e) {
    double sy = ex[e][0], sz = ex[e][1];
    double gx = 1.0 - 4.0 * x * x, fy = 0.5 + sy * y, fz = 0.5 + sz * z;
    N[8 + e] = gx * fy * fz;
    dx[8 + e] = -8.0 * x * fy * fz;
    dy[8 + e] = sy * gx * fz;
    dz[8 + e] = sz * gx * fy;
  }
  // y-edges: (x,z) signs (-,-),(-,+),(+,+),(+,-)
  static const int ey[4][2] = {{-1, -1}, {-1, 1}, {1, 1}, {1, -1}};
  for (int e = 0; e < 4; ++e) {
    double sx = ey[e][0], sz = ey[e][1];
    double gy = 1.0 - 4.0 * y * y, fx = 0.5 + sx * x, fz = 0.5 + sz * z;
    N[12 + e] = fx * gy * fz;
    dx[12 + e] = sx * gy * fz;
    dy[12 + e] = -8.0 * y * fx * fz;
    dz[12 + e] = sz * fx * gy;
  }
  // radial edges: (x,y) signs (-,-),(+,-),(+,+),(-,+)
  static const int ez[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
  for (int e = 0; e < 4; ++e) {
    double sx = ez[e][0], sy = ez[e][1];
    double gz = 1.0 - 4.0 * z * z, fx = 0.5 + sx * x, fy = 0.5 + sy * y;
    N[16 + e] = fx * fy * gz;
    dx[16 + e] = sx * fy * gz;
    dy[16 + e] = sy * fx * gz;
    dz[16 + e] = -8.0 * z * fx * fy;
  }
}

// Five-point face rule on the 8-node element: centre and the four edge
// midpoints (reference coordinates +-1/2).
const double kFaceX[NQ] = {0.0, 0.5, -0.5, 0.0, 0.0};
const double kFaceY[NQ] = {0.0, 0.0, 0.0, 0.5, -0.5};
const double kFaceW[NQ] = {1.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};

struct FaceRule {
  double N[NQ][8], dx[NQ][8], dy[NQ][8];
  FaceRule() {
    for (int q = 0; q < NQ; ++q) quad8(kFaceX[q], kFaceY[q], N[q], dx[q], dy[q]);
  }
};

struct VolRule {
  double N[27][20], dx[27][20], dy[27][20], dz[27][20], w[27];
  VolRule() {
    const double g = 0.5 * std::sqrt(3.0 / 5.0);
    const double xg[3] = {-g, 0.0, g};
    const double lw[3] = {5.0 / 18.0, 8.0 / 18.0, 5.0 / 18.0};
    int q = 0;
    for (int iz = 0; iz < 3; ++iz)
      for (int iy = 0; iy < 3; ++iy)
        for (int ix = 0; ix < 3; ++ix, ++q) {
          hex20(xg[ix], xg[iy], xg[iz], N[q], dx[q], dy[q], dz[q]);
          w[q] = lw[ix] * lw[iy] * lw[iz];
        }
  }
};

}  // namespace

void vol_rule_pack(double* out) {
  static const VolRule VR;
  for (int q = 0; q < 27; ++q)
    for (int n = 0; n < 20; ++n) {
      out[q * 20 + n] = VR.N[q][n];
      out[540 + q * 20 + n] = VR.dx[q][n];
      out[1080 + q * 20 + n] = VR.dy[q][n];
      out[1620 + q * 20 + n] = VR.dz[q][n];
    }
  for (int q = 0; q < 27; ++q) out[2160 + q] = VR.w[q];
}

namespace {

inline V3 onto_radius(V3 mid, double r, double smallnum) {
  double t = std::fmax(smallnum, vnorm(mid));
  return vscale(mid, r / t);
}

// One face of the mesh: the 8 element nodes, then points, weights, normals.
struct FaceOut {
  V3 qp[NQ];
  double qw_raw[NQ];
  V3 nq[NQ];  // normal at each point
  double area;
  double qw[NQ];   // area-normalised weights (220)
  double bqw[NQ];  // B-field weights (230)
  V3 cen;
};

void face_geometry(const FaceRule& R, const V3 v[8], double smallnum, FaceOut& o) {
  for (int q = 0; q < NQ; ++q) {
    V3 p{}, A{}, B{};
    for (int n = 0; n < 8; ++n) {
      p = vadd(p, vscale(v[n], R.N[q][n]));
      A = vadd(A, vscale(v[n], R.dx[q][n]));
      B = vadd(B, vscale(v[n], R.dy[q][n]));
    }
    V3 C = vcross(A, B);
    double cm = vnorm(C);
    o.qp[q] = p;
    o.qw_raw[q] = kFaceW[q] * cm;
    double inv = 1.0 / std::fmax(cm, smallnum);
    o.nq[q] = vscale(C, inv);
  }
  double area = 0.0;
  for (int q = 0; q < NQ; ++q) area += o.qw_raw[q];
  area = std::fmax(smallnum, area);
  o.area = area;
  for (int q = 0; q < NQ; ++q) o.qw[q] = o.qw_raw[q] / area;
  double a = o.qw_raw[0] + o.qw_raw[1] + o.qw_raw[2] + o.qw_raw[3] + o.qw_raw[4];
  a = 1.0 / std::fmax(a, smallnum);
  for (int q = 0; q < NQ; ++q) o.bqw[q] = a * o.qw_raw[q];
  V3 c{};
  for (int q = 0; q < NQ; ++q) c = vadd(c, vscale(o.qp[q], o.qw[q]));
  o.cen = c;
}

}  // namespace

int geom_ncomp(int field) {
  switch (field) {
    case CS_G_VERT: return 3;
    case CS_G_XF_QP: case CS_G_YF_QP: case CS_G_ZF_QP: return 3 * NQ;
    case CS_G_XF_QW: case CS_G_YF_QW: case CS_G_ZF_QW: return NQ;
    case CS_G_XF_N: case CS_G_YF_N: return 3;
    case CS_G_ZF_N: return 3 * NQ;
    case CS_G_XF_AREA: case CS_G_YF_AREA: case CS_G_ZF_AREA: return 1;
    case CS_G_XF_CEN: case CS_G_YF_CEN: case CS_G_ZF_CEN: return 3;
    case CS_G_XB_QW: case CS_G_YB_QW: case CS_G_ZB_QW: return NQ;
    case CS_G_V_SCALE: case CS_G_V_VOL: return 1;
    case CS_G_V_CEN: return 3;
    case CS_G_COEF: return NMODE;
    default: return 0;
  }
}

namespace {

// 27-point isoparametric volume rule of one zone from its 8 corners (in the
// reference order): points and un-normalised weights w_q * |det J|.
void zone_rule_raw(const V3 c8[8], double smallnum, double qp[27][3], double qw[27]) {
  static const VolRule VR;
  V3 v[20];
  for (int n = 0; n < 8; ++n) v[n] = c8[n];
  double r1 = vnorm(v[0]), r2 = vnorm(v[4]);
  v[8] = onto_radius(vscale(vadd(v[0], v[1]), 0.5), r1, smallnum);
  v[9] = onto_radius(vscale(vadd(v[2], v[3]), 0.5), r1, smallnum);
  v[10] = onto_radius(vscale(vadd(v[6], v[7]), 0.5), r2, smallnum);
  v[11] = onto_radius(vscale(vadd(v[4], v[5]), 0.5), r2, smallnum);
  v[12] = onto_radius(vscale(vadd(v[0], v[3]), 0.5), r1, smallnum);
  v[15] = onto_radius(vscale(vadd(v[1], v[2]), 0.5), r1, smallnum);
  v[13] = onto_radius(vscale(vadd(v[4], v[7]), 0.5), r2, smallnum);
  v[14] = onto_radius(vscale(vadd(v[5], v[6]), 0.5), r2, smallnum);
  v[16] = vscale(vadd(v[0], v[4]), 0.5);
  v[17] = vscale(vadd(v[1], v[5]), 0.5);
  v[18] = vscale(vadd(v[2], v[6]), 0.5);
  v[19] = vscale(vadd(v[3], v[7]), 0.5);
  for (int q = 0; q < 27; ++q) {
    V3 p{}, A{}, B{}, C{};
    for (int n = 0; n < 20; ++n) {
      p = vadd(p, vscale(v[n], VR.N[q][n]));
      A = vadd(A, vscale(v[n], VR.dx[q][n]));
      B = vadd(B, vscale(v[n], VR.dy[q][n]));
      C = vadd(C, vscale(v[n], VR.dz[q][n]));
    }
    V3 D = vcross(A, B);
    double det = std::fabs(C.x * D.x + C.y * D.y + C.z * D.z);
    qp[q][0] = p.x;
    qp[q][1] = p.y;
    qp[q][2] = p.z;
    qw[q] = VR.w[q] * det;
  }
}

// Computes every per-panel geometry field from the vertex array and mask.
void panel_geometry(const Box& b, int p, double smallnum, GeomHost& g) {
  static const FaceRule FR;
  const size_t S = b.size();
  auto F = [&](int field, int c, size_t o) -> double& { return g.f[field][((size_t)c * NPANEL + p) * S + o]; };
  auto vert = [&](int i, int j, int k) -> V3 {
    size_t o = b.idx(i, j, k);
    return {F(CS_G_VERT, 0, o), F(CS_G_VERT, 1, o), F(CS_G_VERT, 2, o)};
  };
  auto mask = [&](int i, int j) -> int { return g.mask[(size_t)p * S + b.idx(i, j, 0)]; };
  const int N = b.N, G = b.G, nr = b.nr;

  // x-faces: i in [-G, N+G], j,k in [1-G, ...]
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = -G; i <= N + G; ++i) {
        V3 v[8];
        v[0] = vert(i, j - 1, k - 1);
        v[1] = vert(i, j, k - 1);
        v[2] = vert(i, j, k);
        v[3] = vert(i, j - 1, k);
        double r1 = vnorm(v[0]), r2 = vnorm(v[2]);
        v[4] = onto_radius(vscale(vadd(v[0], v[1]), 0.5), r1, smallnum);
        v[5] = vscale(vadd(v[1], v[2]), 0.5);
        v[6] = onto_radius(vscale(vadd(v[2], v[3]), 0.5), r2, smallnum);
        v[7] = vscale(vadd(v[3], v[0]), 0.5);
        FaceOut o;
        face_geometry(FR, v, smallnum, o);
        size_t ix = b.idx(i, j, k);
        for (int q = 0; q < NQ; ++q) {
          F(CS_G_XF_QP, 0 * NQ + q, ix) = o.qp[q].x;
          F(CS_G_XF_QP, 1 * NQ + q, ix) = o.qp[q].y;
          F(CS_G_XF_QP, 2 * NQ + q, ix) = o.qp[q].z;
          F(CS_G_XF_QW, q, ix) = o.qw[q];
          F(CS_G_XB_QW, q, ix) = o.bqw[q];
        }
        F(CS_G_XF_N, 0, ix) = o.nq[0].x;
        F(CS_G_XF_N, 1, ix) = o.nq[0].y;
        F(CS_G_XF_N, 2, ix) = o.nq[0].z;
        F(CS_G_XF_AREA, 0, ix) = o.area;
        F(CS_G_XF_CEN, 0, ix) = o.cen.x;
        F(CS_G_XF_CEN, 1, ix) = o.cen.y;
        F(CS_G_XF_CEN, 2, ix) = o.cen.z;
      }

  // y-faces: j in [-G, N+G]
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = -G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        V3 v[8];
        v[0] = vert(i - 1, j, k - 1);
        v[1] = vert(i - 1, j, k);
        v[2] = vert(i, j, k);
        v[3] = vert(i, j, k - 1);
        double r1 = vnorm(v[0]), r2 = vnorm(v[2]);
        v[4] = vscale(vadd(v[0], v[1]), 0.5);
        v[5] = onto_radius(vscale(vadd(v[1], v[2]), 0.5), r2, smallnum);
        v[6] = vscale(vadd(v[2], v[3]), 0.5);
        v[7] = onto_radius(vscale(vadd(v[3], v[0]), 0.5), r1, smallnum);
        FaceOut o;
        face_geometry(FR, v, smallnum, o);
        size_t ix = b.idx(i, j, k);
        for (int q = 0; q < NQ; ++q) {
          F(CS_G_YF_QP, 0 * NQ + q, ix) = o.qp[q].x;
          F(CS_G_YF_QP, 1 * NQ + q, ix) = o.qp[q].y;
          F(CS_G_YF_QP, 2 * NQ + q, ix) = o.qp[q].z;
          F(CS_G_YF_QW, q, ix) = o.qw[q];
          F(CS_G_YB_QW, q, ix) = o.bqw[q];
        }
        F(CS_G_YF_N, 0, ix) = o.nq[0].x;
        F(CS_G_YF_N, 1, ix) = o.nq[0].y;
        F(CS_G_YF_N, 2, ix) = o.nq[0].z;
        F(CS_G_YF_AREA, 0, ix) = o.area;
        F(CS_G_YF_CEN, 0, ix) = o.cen.x;
        F(CS_G_YF_CEN, 1, ix) = o.cen.y;
        F(CS_G_YF_CEN, 2, ix) = o.cen.z;
      }

  // z-faces: k in [-G, nr+G]; spherical, normal per quadrature point.
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = -G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        V3 v[8];
        v[0] = vert(i - 1, j - 1, k);
        v[1] = vert(i, j - 1, k);
        v[2] = vert(i, j, k);
        v[3] = vert(i - 1, j, k);
        double r1 = vnorm(v[0]);
        v[4] = onto_radius(vscale(vadd(v[0], v[1]), 0.5), r1, smallnum);
        v[5] = onto_radius(vscale(vadd(v[1], v[2]), 0.5), r1, smallnum);
        v[6] = onto_radius(vscale(vadd(v[2], v[3]), 0.5), r1, smallnum);
        v[7] = onto_radius(vscale(vadd(v[3], v[0]), 0.5), r1, smallnum);
        FaceOut o;
        face_geometry(FR, v, smallnum, o);
        size_t ix = b.idx(i, j, k);
        for (int q = 0; q < NQ; ++q) {
          F(CS_G_ZF_QP, 0 * NQ + q, ix) = o.qp[q].x;
          F(CS_G_ZF_QP, 1 * NQ + q, ix) = o.qp[q].y;
          F(CS_G_ZF_QP, 2 * NQ + q, ix) = o.qp[q].z;
          F(CS_G_ZF_QW, q, ix) = o.qw[q];
          F(CS_G_ZB_QW, q, ix) = o.bqw[q];
          F(CS_G_ZF_N, 0 * NQ + q, ix) = o.nq[q].x;
          F(CS_G_ZF_N, 1 * NQ + q, ix) = o.nq[q].y;
          F(CS_G_ZF_N, 2 * NQ + q, ix) = o.nq[q].z;
        }
        F(CS_G_ZF_AREA, 0, ix) = o.area;
        F(CS_G_ZF_CEN, 0, ix) = o.cen.x;
        F(CS_G_ZF_CEN, 1, ix) = o.cen.y;
        F(CS_G_ZF_CEN, 2, ix) = o.cen.z;
      }

  // Zones: volume rule, centroid, scale length and basis moments.
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1 - G; k <= nr + G; ++k)
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        V3 v[8];
        v[0] = vert(i - 1, j - 1, k - 1);
        v[1] = vert(i, j - 1, k - 1);
        v[2] = vert(i, j, k - 1);
        v[3] = vert(i - 1, j, k - 1);
        v[4] = vert(i - 1, j - 1, k);
        v[5] = vert(i, j - 1, k);
        v[6] = vert(i, j, k);
        v[7] = vert(i - 1, j, k);
        double qpa[27][3], qw[27];
        zone_rule_raw(v, smallnum, qpa, qw);
        V3 qp[27];
        for (int q = 0; q < 27; ++q) qp[q] = {qpa[q][0], qpa[q][1], qpa[q][2]};
        double vol = 0.0;
        for (int q = 0; q < 27; ++q) vol += qw[q];
        vol = std::fmax(smallnum, vol);
        for (int q = 0; q < 27; ++q) qw[q] /= vol;
        V3 c0{};
        for (int n = 0; n < 8; ++n) c0 = vadd(c0, v[n]);
        c0 = vscale(c0, 0.125);
        V3 sh{};
        for (int q = 0; q < 27; ++q) sh = vadd(sh, vscale(vsub(qp[q], c0), qw[q]));
        V3 cen = vadd(c0, sh);
        // Scale length: radial edge length and the four angular chords of the
        // inner face.
        double sl = vnorm(vsub(vert(i, j, k), vert(i, j, k - 1)));
        sl = std::fmin(sl, std::fmin(vnorm(vsub(vert(i - 1, j, k - 1), vert(i, j, k - 1))),
                                     vnorm(vsub(vert(i - 1, j - 1, k - 1), vert(i, j - 1, k - 1)))));
        sl = std::fmin(sl, std::fmin(vnorm(vsub(vert(i, j - 1, k - 1), vert(i, j, k - 1))),
                                     vnorm(vsub(vert(i - 1, j - 1, k - 1), vert(i - 1, j, k - 1)))));
        size_t ix = b.idx(i, j, k);
        F(CS_G_V_VOL, 0, ix) = vol;
        F(CS_G_V_CEN, 0, ix) = cen.x;
        F(CS_G_V_CEN, 1, ix) = cen.y;
        F(CS_G_V_CEN, 2, ix) = cen.z;
        F(CS_G_V_SCALE, 0, ix) = sl;
        static const int pw[NMODE][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                         {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}};
        for (int m = 0; m < NMODE; ++m) F(CS_G_COEF, m, ix) = 0.0;
        if (mask(i, j) == 1) {
          double aa = 1.0 / std::fmax(smallnum, std::fabs(sl));
          for (int m = 1; m < NMODE; ++m) {
            double s = 0.0;
            for (int q = 0; q < 27; ++q) {
              double x = (qp[q].x - cen.x) * aa, y = (qp[q].y - cen.y) * aa, z = (qp[q].z - cen.z) * aa;
              double t = ipow(x, pw[m][0]) * ipow(y, pw[m][1]) * ipow(z, pw[m][2]);
              s += qw[q] * t;
            }
            F(CS_G_COEF, m, ix) = s;
          }
        }
      }
}

void build_stencil(const Box& b, int32_t* st /* [12][2][NJ][NI] */) {
  const int N = b.N, G = b.G;
  const size_t P = b.plane();
  auto S = [&](int i, int j, int which, int c) -> int32_t& {
    return st[((size_t)which * 2 + c) * P + (size_t)(j + G) * b.NI + (i + G)];
  };
  for (size_t t = 0; t < 24 * P; ++t) st[t] = 0;
  const int lo = 1 - G, hi = N + G;
  for (int i = lo; i <= hi; ++i)
    for (int j = lo; j <= hi; ++j) {
      int ip1 = std::min(i + 1, hi), jp1 = std::min(j + 1, hi), ip2 = std::min(i + 2, hi), jp2 = std::min(j + 2, hi);
      int im1 = std::max(i - 1, lo), jm1 = std::max(j - 1, lo), im2 = std::max(i - 2, lo), jm2 = std::max(j - 2, lo);
      const int tab[12][2] = {{ip1, j}, {im1, j}, {i, jp1}, {i, jm1}, {ip2, j},   {im2, j},
                              {i, jp2}, {i, jm2}, {ip1, jp1}, {im1, jp1}, {im1, jm1}, {ip1, jm1}};
      for (int w = 0; w < 12; ++w) {
        S(i, j, w, 0) = tab[w][0];
        S(i, j, w, 1) = tab[w][1];
      }
    }
  auto set = [&](int i, int j, int w1, int a, int bb) {
    S(i, j, w1 - 1, 0) = a;
    S(i, j, w1 - 1, 1) = bb;
  };
  // Left-down tri-corner.
  for (int i = lo; i <= 0; ++i) {
    int j = 1;
    set(i, j, 4, 1, i);
    set(i, j, 8, 2, i);
    set(i, j, 11, 1, std::max(i - 1, lo));
    set(i, j, 12, 1, i + 1);
    if (i == 0) set(i, j, 12, 2, i - 1);
    set(i, j + 1, 8, 1, i);
  }
  for (int j = lo; j <= 0; ++j) {
    int i = 1;
    set(i, j, 2, j, 1);
    set(i, j, 6, j, 2);
    set(i, j, 10, j + 1, 1);
    if (j == 0) set(i, j, 10, j - 1, 2);
    set(i, j, 11, std::max(j - 1, lo), 1);
    set(i + 1, j, 6, j, 1);
  }
  set(1, 1, 11, 2, -1);
  // Right-down tri-corner.
  for (int i = N + 1; i <= hi; ++i) {
    int j = 1;
    set(i, j, 4, N, N - i + 1);
    set(i, j, 8, N - 1, N - i + 1);
    set(i, j, 11, N, N - i + 2);
    if (i == N + 1) set(i, j, 11, N - 1, N - i);
    set(i, j, 12, N, std::max(N - i, lo));
    set(i, j + 1, 8, N, N - i + 1);
  }
  for (int j = lo; j <= 0; ++j) {
    int i = N;
    set(i, j, 1, N + 1 - j, 1);
    set(i, j, 5, N + 1 - j, 2);
    set(i, j, 9, N - j, 1);
    if (j == 0) set(i, j, 9, N + 2 - j, 2);
    set(i, j, 12, std::min(N + 2 - j, hi), 1);
    set(i - 1, j, 5, N + 1 - j, 1);
  }
  set(N, 1, 12, N - 1, -1);
  // Right-up tri-corner.
  for (int i = N + 1; i <= hi; ++i) {
    int j = N;
    set(i, j, 3, N, i);
    set(i, j, 7, N - 1, i);
    set(i, j, 10, N, i - 1);
    if (i == N + 1) set(i, j, 10, N - 1, i + 1);
    set(i, j, 9, N, std::min(i + 1, hi));
    set(i, j - 1, 7, N, i);
  }
  for (int j = N + 1; j <= hi; ++j) {
    int i = N;
    set(i, j, 1, j, N);
    set(i, j, 5, j, N - 1);
    set(i, j, 12, j - 1, N);
    if (j == N + 1) set(i, j, 12, j + 1, N - 1);
    set(i, j, 9, std::min(j + 1, hi), N);
    set(i - 1, j, 5, j, N);
  }
  set(N, N, 9, N - 1, N + 2);
  // Left-up tri-corner.
  for (int j = N + 1; j <= hi; ++j) {
    int i = 1;
    set(i, j, 2, N - j + 1, N);
    set(i, j, 6, N - j + 1, N - 1);
    set(i, j, 11, N - j + 2, N);
    if (j == N + 1) set(i, j, 11, N - j, N - 1);
    set(i, j, 10, std::max(N - j, lo), N);
    set(i + 1, j, 6, N - j + 1, N);
  }
  for (int i = lo; i <= 0; ++i) {
    int j = N;
    set(i, j, 3, 1, N - i + 1);
    set(i, j, 7, 2, N - i + 1);
    set(i, j, 9, 1, N - i);
    if (i == 0) set(i, j, 9, 2, N - i + 2);
    set(i, j, 10, 1, std::min(N - i + 2, hi));
    set(i, j - 1, 7, 1, N - i + 1);
  }
  set(1, N, 10, 2, N + 2);
}

std::string build_from_unit_vertices(const cs_params& p, const std::vector<V3> sec[6], int iscale, int nglobal,
                                     int ghost_global, const std::vector<double>& rb_global, GeomHost& g) {
  const Box b(p.ntp, p.nr, p.nghost);
  g.box = b;
  const size_t S = b.size();
  // The fields hold ≈126 words a point (6 GB at 6 x 128^2 x 64): their first
  // touch (page faults and zeroing) runs one field a thread.
#pragma omp parallel for schedule(dynamic, 1)
  for (int f = 0; f < CS_G_NFIELDS; ++f) g.f[f].assign((size_t)geom_ncomp(f) * NPANEL * S, 0.0);
  g.mask.assign((size_t)NPANEL * S, 0);
  g.stencil.assign((size_t)NPANEL * 24 * b.plane(), 0);
  const int N = b.N, G = b.G, nr = b.nr;
  const int wg = nglobal + 2 * ghost_global + 1;
  g.rb.assign(nr + 2 * G + 1, 0.0);
  for (int k = -G; k <= nr + G; ++k) g.rb[k + G] = rb_global[(size_t)(k * iscale + ghost_global)];
  for (int s = 0; s < NPANEL; ++s) {
    // One radial layer of unit vectors, then scaled by the vertex radii.
    std::vector<V3> layer((size_t)b.plane());
    for (int j = -G; j <= N + G; ++j)
      for (int i = -G; i <= N + G; ++i) {
        int iu = i * iscale, ju = j * iscale;
        layer[(size_t)(j + G) * b.NI + (i + G)] = sec[s][(size_t)(ju + ghost_global) * wg + (iu + ghost_global)];
      }
    for (int j = 1 - G; j <= N + G; ++j)
      for (int i = 1 - G; i <= N + G; ++i) {
        auto L = [&](int a, int c) { return layer[(size_t)(c + G) * b.NI + (a + G)]; };
        bool bad = vnorm(L(i, j)) < p.smallnum || vnorm(L(i - 1, j)) < p.smallnum ||
                   vnorm(L(i, j - 1)) < p.smallnum || vnorm(L(i - 1, j - 1)) < p.smallnum;
        for (int k = -G; k <= nr + G; ++k) g.mask[(size_t)s * S + b.idx(i, j, k)] = bad ? 0 : 1;
      }
    for (int k = -G; k <= nr + G; ++k)
      for (int j = -G; j <= N + G; ++j)
        for (int i = -G; i <= N + G; ++i) {
          V3 u = layer[(size_t)(j + G) * b.NI + (i + G)];
          double r = g.rb[k + G];
          size_t o = b.idx(i, j, k);
          g.f[CS_G_VERT][((size_t)0 * NPANEL + s) * S + o] = r * u.x;
          g.f[CS_G_VERT][((size_t)1 * NPANEL + s) * S + o] = r * u.y;
          g.f[CS_G_VERT][((size_t)2 * NPANEL + s) * S + o] = r * u.z;
        }
    build_stencil(b, &g.stencil[(size_t)s * 24 * b.plane()]);
    panel_geometry(b, s, p.smallnum, g);
  }
  return "";
}

}  // namespace

void zone_volume_rule(const GeomHost& g, int pn, int i, int j, int k, double smallnum, double qp[27][3],
                      double qw[27]) {
  const Box& b = g.box;
  const size_t S = b.size();
  auto vert = [&](int a, int c, int d) -> V3 {
    size_t o = b.idx(a, c, d);
    return {g.f[CS_G_VERT][((size_t)0 * NPANEL + pn) * S + o], g.f[CS_G_VERT][((size_t)1 * NPANEL + pn) * S + o],
            g.f[CS_G_VERT][((size_t)2 * NPANEL + pn) * S + o]};
  };
  V3 v[8] = {vert(i - 1, j - 1, k - 1), vert(i, j - 1, k - 1), vert(i, j, k - 1), vert(i - 1, j, k - 1),
             vert(i - 1, j - 1, k),     vert(i, j - 1, k),     vert(i, j, k),     vert(i - 1, j, k)};
  zone_rule_raw(v, smallnum, qp, qw);
  double vol = 0.0;
  for (int q = 0; q < 27; ++q) vol += qw[q];
  vol = std::fmax(smallnum, vol);
  for (int q = 0; q < 27; ++q) qw[q] /= vol;
}

std::string build_geometry(const cs_params& p, GeomHost& g) {
  if (p.ntp < 2 || p.nr < 1 || p.nghost < 1 || p.nghost >= p.ntp) return "bad mesh sizes (need ntp>=2, nr>=1, 1<=nghost<ntp)";
  std::vector<V3> sec[6];
  for (int s = 0; s < 6; ++s) sector_mesh(s + 1, p.ntp, p.nghost, sec[s]);
  fill_ghost2d(p.ntp, p.nghost, sec);
  std::vector<double> rb;
  std::string e = radial_mesh(p.radial_mesh, p.nr, p.nghost, p.rmin, p.rmax, p.radial_ratio, p.smallnum, rb);
  if (!e.empty()) return e;
  return build_from_unit_vertices(p, sec, 1, p.ntp, p.nghost, rb, g);
}

std::string build_geometry_single_zone(int isector, int ntp_global, int nr_global, int iscale, double rmin,
                                       double rmax, int radial_mesh_kind, GeomHost& g) {
  std::vector<V3> sec[6];
  for (int s = 0; s < 6; ++s) sector_mesh(s + 1, ntp_global, 0, sec[s]);
  std::vector<double> rb;
  std::string e = radial_mesh(radial_mesh_kind, nr_global, 0, rmin, rmax, 1.0, 1e-12, rb);
  if (!e.empty()) return e;
  // Only the requested sector matters; the others are built for uniformity.
  std::vector<V3> one[6];
  for (int s = 0; s < 6; ++s) one[s] = sec[isector - 1];
  cs_params p{};
  p.ntp = ntp_global / iscale;
  p.nr = nr_global / iscale;
  p.nghost = 0;
  p.smallnum = 1e-12;
  return build_from_unit_vertices(p, one, iscale, ntp_global, 0, rb, g);
}

}  // namespace cs
