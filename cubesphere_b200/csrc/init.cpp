// Seeded initial states of the benchmark configurations, built with the
// reference's initialisation mechanism (INIT_PATCH_CUBE_SPHERE,
// pkg/inc/cubesphere/800applications_cs/820init_patch_cube_sphere.f:319-689):
//   * zone averages of the conserved variables are volume-quadrature sums
//     of point values over the 27 points of the isoparametric zone;
//   * face B is the circulation of a vector potential A around the face
//     divided by the face area (midpoint rule per edge, arcs measured as
//     r * angle), so div B is zero to round-off from the first step;
//   * the entropy variable is p / rho^(gamma-1) of the zone average.
// The problems themselves are new generator cases (seeded harmonic sums):
//   kind 0 (surface): rho = 1 + rho_amp*Y, p = p0, v = v_amp * (z-hat x r),
//          A = a_amp * Psi * r-hat;
//   kind 1 (shell):   rho = r^-2 (1 + rho_amp*Y), p = gm/(3 r^3) + p0,
//          v = 0, A = a_amp * Psi * r-hat.
// Y and Psi are seeded random polynomials of degree <= lmax in the unit
// vector r-hat (i.e. spherical-harmonic sums up to degree lmax), normalised
// to max |.| = 1 on a fixed 96 x 192 latitude-longitude sampling grid.
#include <cmath>
#include <random>

#include "cs_internal.h"

namespace cs {

namespace {

struct Harm {
  std::vector<int> a, b, c;
  std::vector<double> w;
  int deg = 0;
  double scale = 1.0;
  // powers x^0 .. x^deg by repeated multiplication
  static void powers(double x, int deg, double* p) {
    p[0] = 1.0;
    for (int e = 1; e <= deg; ++e) p[e] = p[e - 1] * x;
  }
  double value(double u, double v, double t) const {
    double pu[16], pv[16], pt[16];
    powers(u, deg, pu);
    powers(v, deg, pv);
    powers(t, deg, pt);
    double s = 0.0;
    for (size_t n = 0; n < w.size(); ++n) s += w[n] * pu[a[n]] * pv[b[n]] * pt[c[n]];
    return s * scale;
  }
  void grad(double u, double v, double t, double g[3]) const {
    double pu[16], pv[16], pt[16];
    powers(u, deg, pu);
    powers(v, deg, pv);
    powers(t, deg, pt);
    g[0] = g[1] = g[2] = 0.0;
    for (size_t n = 0; n < w.size(); ++n) {
      if (a[n] > 0) g[0] += w[n] * a[n] * pu[a[n] - 1] * pv[b[n]] * pt[c[n]];
      if (b[n] > 0) g[1] += w[n] * b[n] * pu[a[n]] * pv[b[n] - 1] * pt[c[n]];
      if (c[n] > 0) g[2] += w[n] * c[n] * pu[a[n]] * pv[b[n]] * pt[c[n] - 1];
    }
    for (int q = 0; q < 3; ++q) g[q] *= scale;
  }
};

// Box-Muller normal deviates from a 64-bit Mersenne twister (same stream on
// every platform: only integer draws and IEEE arithmetic are used).
struct Normal {
  std::mt19937_64 eng;
  explicit Normal(uint64_t s) : eng(s) {}
  double uni() { return ((eng() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
  double operator()() {
    double u1 = uni(), u2 = uni();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
  }
};

Harm make_harm(Normal& rnd, int lmax) {
  Harm h;
  h.deg = lmax;
  for (int d = 1; d <= lmax; ++d)
    for (int a = d; a >= 0; --a)
      for (int b = d - a; b >= 0; --b) {
        h.a.push_back(a);
        h.b.push_back(b);
        h.c.push_back(d - a - b);
        h.w.push_back(rnd());
      }
  double mx = 0.0;
  const int nt = 96, np = 192;
  for (int it = 0; it < nt; ++it) {
    double th = M_PI * (it + 0.5) / nt;
    for (int ip = 0; ip < np; ++ip) {
      double ph = 2.0 * M_PI * ip / np;
      double v = h.value(std::sin(th) * std::cos(ph), std::sin(th) * std::sin(ph), std::cos(th));
      mx = std::max(mx, std::fabs(v));
    }
  }
  h.scale = (mx > 0.0) ? 1.0 / mx : 1.0;
  return h;
}

struct Problem {
  int kind;
  double gamma, rho_amp, a_amp, v_amp, p0, gm, ob8pi;
  Harm Y, Psi;
  // Point conserved state at (x,y,z).
  void point(double x, double y, double z, double U[8]) const {
    double r = std::sqrt(x * x + y * y + z * z);
    double u = x / r, v = y / r, t = z / r;
    double rho, p, vx, vy, vz;
    if (kind == 0) {
      rho = 1.0 + rho_amp * Y.value(u, v, t);
      p = p0;
      vx = -v_amp * y;
      vy = v_amp * x;
      vz = 0.0;
    } else {
      rho = (1.0 / (r * r)) * (1.0 + rho_amp * Y.value(u, v, t));
      p = gm / (3.0 * r * r * r) + p0;
      vx = vy = vz = 0.0;
    }
    double g[3];
    Psi.grad(u, v, t, g);
    // B = curl(a Psi(r-hat) r-hat) = (a / r) grad_u Psi x r-hat
    double bx = (a_amp / r) * (g[1] * t - g[2] * v);
    double by = (a_amp / r) * (g[2] * u - g[0] * t);
    double bz = (a_amp / r) * (g[0] * v - g[1] * u);
    U[0] = rho;
    U[1] = rho * vx;
    U[2] = rho * vy;
    U[3] = rho * vz;
    U[4] = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + ob8pi * (bx * bx + by * by + bz * bz);
    U[5] = bx;
    U[6] = by;
    U[7] = bz;
  }
  // A . dl along the edge a -> b (midpoint rule; for an arc the midpoint is
  // rescaled to the radius of a and dl is r*angle along the chord direction).
  double a_dot_dl(const double* pa, const double* pb, bool arc) const {
    double m[3], dl[3];
    for (int q = 0; q < 3; ++q) {
      m[q] = 0.5 * (pa[q] + pb[q]);
      dl[q] = pb[q] - pa[q];
    }
    if (arc) {
      double ra = std::sqrt(pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]);
      double rb = std::sqrt(pb[0] * pb[0] + pb[1] * pb[1] + pb[2] * pb[2]);
      double rm = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
      for (int q = 0; q < 3; ++q) m[q] *= ra / rm;
      double cosang = (pa[0] * pb[0] + pa[1] * pb[1] + pa[2] * pb[2]) / (ra * rb);
      cosang = std::max(-1.0, std::min(1.0, cosang));
      double ang = std::acos(cosang);
      double dn = std::sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
      for (int q = 0; q < 3; ++q) dl[q] = ra * ang * dl[q] / dn;
    }
    double r = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    double psi = Psi.value(m[0] / r, m[1] / r, m[2] / r);
    double ar = a_amp * psi / r;  // A = a Psi r-hat -> components a Psi m / r
    return ar * (m[0] * dl[0] + m[1] * dl[1] + m[2] * dl[2]);
  }
};

}  // namespace

std::string init_harmonics(const cs_init_desc& d, InitHarmonics& Y, InitHarmonics& Psi) {
  const int lmax = d.lmax > 0 ? d.lmax : 4;
  if (lmax > 15) return "init lmax must be <= 15";
  Normal rnd(d.seed);
  const Harm hy = make_harm(rnd, lmax);
  const Harm hp = make_harm(rnd, lmax);
  for (int q = 0; q < 2; ++q) {
    const Harm& h = q ? hp : hy;
    InitHarmonics& o = q ? Psi : Y;
    o.deg = h.deg;
    o.a = h.a;
    o.b = h.b;
    o.c = h.c;
    o.w = h.w;
    o.scale = h.scale;
  }
  return "";
}

std::string init_problem_host(const cs_params& p, const cs_init_desc& d, const GeomHost& g, double* U, double* ent,
                              double* bx, double* by, double* bz) {
  const Box& b = g.box;
  const size_t S = b.size();
  const int N = b.N, G = b.G, nr = b.nr;
  Normal rnd(d.seed);
  Problem pr;
  pr.kind = d.kind;
  pr.gamma = p.gamma;
  pr.rho_amp = d.rho_amp;
  pr.a_amp = d.a_amp;
  pr.v_amp = d.v_amp;
  pr.p0 = d.p0;
  pr.gm = p.gm;
  pr.ob8pi = 1.0 / (8.0 * (4.0 * std::atan(1.0)));
  int lmax = d.lmax > 0 ? d.lmax : 4;
  if (lmax > 15) return "init lmax must be <= 15";
  pr.Y = make_harm(rnd, lmax);
  pr.Psi = make_harm(rnd, lmax);
  for (size_t t = 0; t < 8 * NPANEL * S; ++t) U[t] = 0.0;
  for (size_t t = 0; t < NPANEL * S; ++t) ent[t] = bx[t] = by[t] = bz[t] = 0.0;
  auto F = [&](int f, int c, int pn, size_t o) { return g.f[f][((size_t)c * NPANEL + pn) * S + o]; };
  for (int pn = 0; pn < NPANEL; ++pn) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          size_t o = b.idx(i, j, k);
          if (g.mask[(size_t)pn * S + o] != 1) continue;
          // Volume-quadrature average over the 27 isoparametric points
          // (weights normalised by the zone volume), 820:333-395.
          double qp[27][3], qw[27];
          zone_volume_rule(g, pn, i, j, k, p.smallnum, qp, qw);
          double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
          for (int q27 = 0; q27 < 27; ++q27) {
            double Up[8];
            pr.point(qp[q27][0], qp[q27][1], qp[q27][2], Up);
            for (int q = 0; q < 8; ++q) acc[q] = acc[q] + Up[q] * qw[q27];
          }
          for (int q = 0; q < 8; ++q) U[((size_t)q * NPANEL + pn) * S + o] = acc[q];
          double rho = std::max(U[((size_t)0 * NPANEL + pn) * S + o], p.rhofloor);
          double v0 = rho / (rho * rho + p.rhofloor * p.rhofloor);
          double vx = U[((size_t)1 * NPANEL + pn) * S + o] * v0, vy = U[((size_t)2 * NPANEL + pn) * S + o] * v0,
                 vz = U[((size_t)3 * NPANEL + pn) * S + o] * v0;
          double bfx = U[((size_t)5 * NPANEL + pn) * S + o], bfy = U[((size_t)6 * NPANEL + pn) * S + o],
                 bfz = U[((size_t)7 * NPANEL + pn) * S + o];
          double prs = (p.gamma - 1.0) * (U[((size_t)4 * NPANEL + pn) * S + o] - 0.5 * rho * (vx * vx + vy * vy + vz * vz) -
                                           (bfx * bfx + bfy * bfy + bfz * bfz) * pr.ob8pi);
          prs = std::max(prs, p.prsfloor);
          ent[(size_t)pn * S + o] = prs / std::pow(rho, p.gamma - 1.0);
        }
    // Face B from edge circulations.  Each edge integral is computed once per
    // face from the same endpoint pair, so neighbouring faces share it.
    auto V = [&](int i, int j, int k, double* out) {
      for (int q = 0; q < 3; ++q) out[q] = F(CS_G_VERT, q, pn, b.idx(i, j, k));
    };
    auto edge = [&](int ai, int aj, int ak, int bi, int bj, int bk, bool arc) {
      double pa[3], pb[3];
      V(ai, aj, ak, pa);
      V(bi, bj, bk, pb);
      // canonical direction (lexicographic) so both faces see the same number
      bool swap = (ak > bk) || (ak == bk && (aj > bj || (aj == bj && ai > bi)));
      double s = swap ? -1.0 : 1.0;
      return swap ? s * pr.a_dot_dl(pb, pa, arc) : pr.a_dot_dl(pa, pb, arc);
    };
    auto nonzero = [&](int i, int j, int k) {
      double pa[3];
      V(i, j, k, pa);
      return (pa[0] * pa[0] + pa[1] * pa[1] + pa[2] * pa[2]) > 0.0;
    };
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = -G; i <= N + G; ++i) {
          if (!(nonzero(i, j - 1, k - 1) && nonzero(i, j, k - 1) && nonzero(i, j, k) && nonzero(i, j - 1, k))) continue;
          // loop (i,j-1,k-1) -> (i,j,k-1) -> (i,j,k) -> (i,j-1,k), positive about +x
          double c = edge(i, j - 1, k - 1, i, j, k - 1, true) + edge(i, j, k - 1, i, j, k, false) +
                     edge(i, j, k, i, j - 1, k, true) + edge(i, j - 1, k, i, j - 1, k - 1, false);
          bx[(size_t)pn * S + b.idx(i, j, k)] = c / F(CS_G_XF_AREA, 0, pn, b.idx(i, j, k));
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = -G; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          if (!(nonzero(i - 1, j, k - 1) && nonzero(i - 1, j, k) && nonzero(i, j, k) && nonzero(i, j, k - 1))) continue;
          // loop (i-1,j,k-1) -> (i-1,j,k) -> (i,j,k) -> (i,j,k-1), positive about +y
          double c = edge(i - 1, j, k - 1, i - 1, j, k, false) + edge(i - 1, j, k, i, j, k, true) +
                     edge(i, j, k, i, j, k - 1, false) + edge(i, j, k - 1, i - 1, j, k - 1, true);
          by[(size_t)pn * S + b.idx(i, j, k)] = c / F(CS_G_YF_AREA, 0, pn, b.idx(i, j, k));
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = -G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) {
          if (!(nonzero(i - 1, j - 1, k) && nonzero(i, j - 1, k) && nonzero(i, j, k) && nonzero(i - 1, j, k))) continue;
          // loop (i-1,j-1,k) -> (i,j-1,k) -> (i,j,k) -> (i-1,j,k), positive about +z (radial)
          double c = edge(i - 1, j - 1, k, i, j - 1, k, true) + edge(i, j - 1, k, i, j, k, true) +
                     edge(i, j, k, i - 1, j, k, true) + edge(i - 1, j, k, i - 1, j - 1, k, true);
          bz[(size_t)pn * S + b.idx(i, j, k)] = c / F(CS_G_ZF_AREA, 0, pn, b.idx(i, j, k));
        }
  }
  return "";
}

}  // namespace cs
