// Internal declarations shared by the host mesh builder, the CUDA stage
// kernels and the C ABI.  Not part of the public interface.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "cubesphere_b200.h"

namespace cs {

constexpr int NPANEL = 6;
constexpr int NQ = 5;     // NAREA_QUAD_PTS == NBFLD_QUAD_PTS in the reference directives
constexpr int NMODE = 10; // n_cc_modes at NUMORDER 3
constexpr int NVAR = 8;   // ideal MHD (IPDE_SYSTEM 1)

// Panel box: all per-panel arrays (zones, faces, vertices) share one padded
// index space [-G, N+G]^2 x [-G, nr+G] with i fastest.
struct Box {
  int N = 0, nr = 0, G = 0;
  int NI = 0, NJ = 0, NK = 0;
  Box() = default;
  Box(int n, int r, int g) : N(n), nr(r), G(g), NI(n + 2 * g + 1), NJ(n + 2 * g + 1), NK(r + 2 * g + 1) {}
  size_t size() const { return (size_t)NI * NJ * NK; }
  size_t plane() const { return (size_t)NI * NJ; }
  size_t idx(int i, int j, int k) const {
    return ((size_t)(k + G) * NJ + (size_t)(j + G)) * NI + (size_t)(i + G);
  }
};

// Components per geometry field (enum cs_geom_field order).
int geom_ncomp(int field);

// Host geometry: every field is [comp][panel][box] doubles; mask is
// [panel][box] ints (imask_active, identical for every k like the
// reference), stencil is [panel][12][2][NJ][NI] ints holding
// istencil_patch(i, j, 1:2, 1:12) for the zone (i, j).
struct GeomHost {
  Box box;
  std::vector<double> f[CS_G_NFIELDS];
  std::vector<int32_t> mask;
  std::vector<int32_t> stencil;
  std::vector<double> rb;  // radial vertex radii rb_save_global(k), k in [-G, nr+G]
};

// Builds the complete 6-panel geometry of one solve (host, OpenMP).
// Returns an empty string on success, otherwise the reason.
std::string build_geometry(const cs_params& p, GeomHost& g);

// Normalised 27-point volume rule of zone (i,j,k) of panel pn.
void zone_volume_rule(const GeomHost& g, int pn, int i, int j, int k, double smallnum, double qp[27][3],
                      double qw[27]);

// Seeded initial state (host), written into panel-box arrays.
std::string init_problem_host(const cs_params& p, const cs_init_desc& d, const GeomHost& g, double* U, double* ent,
                              double* bx, double* by, double* bz);

// The two seeded harmonic sums of an initial-state description (Y for the
// density, Psi for the vector potential), as init_problem_host draws them:
// terms w_n u^a_n v^b_n t^c_n of degree 1..deg, times scale.
struct InitHarmonics {
  int deg = 0;
  std::vector<int> a, b, c;
  std::vector<double> w;
  double scale = 1.0;
};
std::string init_harmonics(const cs_init_desc& d, InitHarmonics& Y, InitHarmonics& Psi);

// The 27-point isoparametric volume rule of the 20-node zone element:
// shape functions N[27][20], derivatives dx, dy, dz [27][20], weights w[27],
// packed in that order (2187 doubles).
void vol_rule_pack(double* out);

// Golden-vector helper: geometry of a single coarse zone extracted with a
// refinement stride (the reference's iscale) from a sector mesh of
// ntp_global zones, with no ghost layers.  Used by the quadrature-point test
// that mirrors _T/_200mesh/004test_quadpoints.f.
std::string build_geometry_single_zone(int isector, int ntp_global, int nr_global, int iscale,
                                       double rmin, double rmax, int radial_mesh, GeomHost& g);

}  // namespace cs
