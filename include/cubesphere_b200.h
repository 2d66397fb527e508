/*
 * cubesphere_b200.h -- C ABI of the B200 per-stage volume update of the
 * CubeSphere cubed-sphere MHD code.
 *
 * Every entry point returns 0 on success and a nonzero cs_status otherwise;
 * nothing aborts.  cs_last_error() returns a one-line reason for the last
 * failure on a context.  One host thread and one CUDA stream per context;
 * contexts are independent.
 *
 * Array layout shared by every host<->device entry point ("panel box"):
 *   each of the 6 panels (sectors) is a box of NI x NJ x NK points with
 *   NI = NJ = ntp + 2*nghost + 1, NK = nr + 2*nghost + 1; the point (i,j,k),
 *   i,j in [-nghost, ntp+nghost], k in [-nghost, nr+nghost], sits at offset
 *     ((k+nghost)*NJ + (j+nghost))*NI + (i+nghost)
 *   (i fastest, like the reference's column-major patch arrays).  Zone (cell)
 *   arrays use i,j,k >= 1-nghost; x-face arrays use i >= -nghost (the
 *   reference's 0-NGhost lower bound), y- and z-faces likewise in j and k.
 *   A field with C components is stored component-major:
 *     field[(c*6 + panel)*box + offset].
 *
 * Reference interfaces replaced (paths inside SPGEOMESH/CubeSphere):
 *   cs_mesh_build        _I/_1000riemann_geomesh_cs_mhd/1000riemann_geomesh_cs_mhd.f:860-1341
 *                        (BUILD_BASE_PATCHES, GENERATE_GLOBAL_RADIAL_*, Mesh_Sector_General,
 *                         FILL_GHOST2D_GLOBAL, EXTRACT_VERT_COORDS_PATCH,
 *                         STENCIL_INDEXING_TRICORNERS, COORDS_TO_WT_QUADPTS_{FACES,BFLD,VOLUME}_ISO2,
 *                         INIT_BASIS_FUNCTION_COEFS)
 *   cs_init_problem      pkg/inc/cubesphere/800applications_cs/820init_patch_cube_sphere.f:8
 *   cs_state_put/get     the !$acc update device/host copies of the driver
 *                        (1000riemann_geomesh_cs_mhd.f:2160-2198, :3051-3073)
 *   cs_fill_ghosts       pkg/inc/cubesphere/300riemann_module/320-333 (LOAD_LOCAL_BUFFERS_UXY/UZ,
 *                        FETCH_BUFFERS_FILL_IN_{UX,UY,UY_TOP,UZ}) and
 *                        pkg/inc/cubesphere/800applications_cs/826pad_boundary_r.f:11
 *   cs_limit_all_slopes_p12  pkg/inc/cubesphere/400riemann_integrate/421limit_all_slopes_p12.f:9
 *   cs_make_facial_fluxes    pkg/inc/cubesphere/400riemann_integrate/450make_facial_fluxes.f:5
 *   cs_make_edge_efields_p1  pkg/inc/cubesphere/400riemann_integrate/460make_edge_fields_p1.f:1
 *   cs_build_non_stiff_sources pkg/inc/cubesphere/400riemann_integrate/470build_non_stiff_sources.f:6
 *   cs_update_imex_rk_step_p1 pkg/inc/cubesphere/400riemann_integrate/484update_imex_rk_step_p1.f:7
 *   cs_cleanup_after_update   pkg/inc/cubesphere/400riemann_integrate/485cleanup_after_update.f:4
 *   cs_evaluate_timestep      pkg/inc/cubesphere/400riemann_integrate/490evaluate_timestep.f:7
 *   cs_stage / cs_step        the per-stage call sequence and RK combine of
 *                             1000riemann_geomesh_cs_mhd.f:1738-2908
 */
#ifndef CUBESPHERE_B200_H
#define CUBESPHERE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum cs_status {
  CS_OK = 0,
  CS_ERR_ARG = 1,      /* bad argument / size */
  CS_ERR_CUDA = 2,     /* a CUDA call failed */
  CS_ERR_STATE = 3,    /* called out of order (e.g. stage before mesh build) */
  CS_ERR_NOMEM = 4,    /* device allocation failed */
  CS_ERR_NUMERIC = 5   /* non-finite value detected by a checking entry point */
};

/* Radial mesh choices (reference CHOOSE_RADIAL_MESH values). */
enum cs_radial_mesh { CS_RADIAL_UNIFORM = 0, CS_RADIAL_LOG = 1, CS_RADIAL_STRETCHED = 2 };

/* Time integrators.  CS_RK2 is the reference's two-stage combine
 * (1000riemann_geomesh_cs_mhd.f:2661-2773); CS_SSPRK3 the three-stage
 * Shu-Osher scheme in the same combine form; CS_IMEX_RK2 the two-stage
 * ARS(2,2,2) scheme with fluxes, entropy transport and CT explicit and the
 * point-mass gravity implicit (closed form: gravity leaves rho unchanged). */
enum cs_rk_scheme { CS_RK2 = 2, CS_SSPRK3 = 3, CS_IMEX_RK2 = 4 };

/* Runtime parameters: the reference's compile-time directives, module
 * sizes and COMMON /RIEMANN_COM/ constants (pkg/inc/cubesphere/000com/riemann.com:42-74). */
typedef struct cs_params {
  int32_t ntp;          /* zones along each panel edge (ntp_zones) */
  int32_t nr;           /* radial zones (nr_zones) */
  int32_t nghost;       /* ghost layers (NGhost); 4 in the reference */
  int32_t radial_mesh;  /* enum cs_radial_mesh */
  double rmin, rmax;    /* radial extent */
  double radial_ratio;  /* geometric stretch ratio (CS_RADIAL_STRETCHED) */
  double gamma;         /* ratio of specific heats */
  double rhofloor, prsfloor, smallnum;
  double cfl_coef, flatten_coef, prs_flatten_coef;
  double gm;            /* newtonsc * Mstar for the point-mass gravity source */
  int32_t bc_lower, bc_upper; /* radial boundary codes: 2 = outflow */
  int32_t rk_scheme;    /* enum cs_rk_scheme */
  int32_t flags;        /* CS_FLAG_* bits */
} cs_params;

/* cs_params.flags: do not keep the per-zone factors of the (geometry-only)
 * ADP constrained least-squares system resident (10.4 KB per zone); factor
 * it in every stage instead.  The cache is also skipped automatically when
 * the device lacks the memory.  Results are identical either way. */
#define CS_FLAG_NO_ADP_CACHE 1
/* cs_params.flags: likewise for the least-squares solution operators of
 * the reconstructions of the primitives and of E (STEPS 7.b / 9.c): per
 * zone, each stencil row's weights W = Minv A_row^T (1.55 KB per zone in
 * FP64 and 0.23 KB in the precision form, shared by the panels by default:
 * see CS_FLAG_LSQ_PER_PANEL); without them every stage rebuilds
 * the rows and the normal matrices and inverts them (same results to
 * round-off). */
#define CS_FLAG_NO_OP_CACHE 2
/* cs_params.flags: keep each panel's own fluxes and EMFs on the faces and
 * edges it shares with other panels instead of giving every shared face and
 * edge the value of its owner (the lowest-numbered panel holding it).  The
 * default ownership is this library's single-device form of the reference's
 * defect correction (DRV:3200-3461), whose values are the copies' average
 * instead (CS_FLAG_PANEL_AVERAGE): conservative, and div B stays at round-off
 * across panel edges; without it div B grows at the cube corners. */
#define CS_FLAG_NO_PANEL_SYNC 4
/* cs_params.flags: the reference's rule for the shared copies instead of
 * ownership: every copy of a face or edge that two panels compute takes
 * their average, the three copies of a cube-corner radial edge their sum / 3
 * (the values its defect correction applies: FETCH_BUFFERS_FILL_IN_FLUX_X /
 * _Y, 334fetch_buffers_fill_in_flux_x.f:295-395, 335:761-795, through
 * UPDATE_DEFECT_IMEX_RK with the stage's dtmove, DRV:2777, 3200-3470).
 * Conservative, div B at round-off, and unlike ownership it keeps the cube's
 * rotation symmetry.  Not with CS_FLAG_NO_PANEL_SYNC (CS_ERR_ARG). */
#define CS_FLAG_PANEL_AVERAGE 256
/* cs_params.flags: the precision form.  The bulk of the stage (conserved
 * state, entropy, primitives and their modes, the flattener, face states and
 * fluxes, dU/dt, the stage copies, the resident least-squares inverses, the
 * face-B quadrature evaluations and the ADP constrained least squares:
 * right-hand sides, panel-shared factors, substitution) is stored and
 * computed in FP32; the geometry, face B, the shift of the quadrature
 * values to the FP64 face mean, the ADP factorisation itself (stored
 * rounded), the edge EMFs, the CT update, the positivity fix and the
 * global reductions stay FP64, so div B stays at FP64 round-off.
 * The WENO nonlinear weights are formed in FP64.  The reference has no
 * such form (it computes everything in REAL*8); the state read and written
 * through cs_state_get / cs_state_put stays FP64 at the boundary. */
#define CS_FLAG_FP32 8
/* cs_params.flags: keep one set of ADP factors per panel.  By default the
 * resident ADP factors are panel 1's only and serve all six panels: the
 * panels are rotations of panel 1 by signed permutations (checked on the
 * vertices when the mesh is uploaded), under which the KKT matrix of a zone
 * transforms by the induced signed permutation of the unknowns, so one
 * factor read from HBM serves six solves and the cache takes 1/6 of the
 * memory (1.7 KB per zone).  The reference factors every zone's system
 * (420/421 STEP 8.d); its solutions agree with the per-panel factors to
 * round-off.  This flag restores per-panel factors; meshes without the
 * symmetry use them anyway. */
#define CS_FLAG_ADP_PER_PANEL 16
/* cs_params.flags: keep one set of least-squares row weights per panel.  By
 * default the resident row weights W_r = Minv A_r^T of STEP 9.c (and of
 * STEP 7.b in the precision form) are panel 1's only: where every panel is
 * a signed-permutation rotation of panel 1 with the same stencil table and
 * mask, a zone's rows transform by the induced signed permutation Q of the
 * modes, so W_r(panel p) = Q^T W_r(panel 1); the stage sums over panel 1's
 * weights and rotates the sums (a select and a sign per mode), and the six
 * blocks that read one tile's weights run side by side so five of them hit
 * L2.  The row weights then take 1.55 KB per zone in FP64 (STEP 7.b's stay
 * per panel there: its kernel, at its register limit, measured slower
 * shared) and 0.23 KB in the precision form, against 2.8 and 1.4 KB.  The
 * results agree with per-panel weights to round-off.  This flag restores
 * per-panel weights; meshes without the symmetry use them anyway. */
#define CS_FLAG_LSQ_PER_PANEL 32

/* cs_params.flags: evaluate STEP 10 of LIMIT_ALL_SLOPES_P12 (421:9354-9976)
 * in every stage: the min and max over the active interior zones of the 8
 * primitives and of the normalised zone divergence of B, read back with
 * cs_limit_minmax (the V_min_local / V_max_local the reference driver
 * reduces and prints each step, 1000riemann_geomesh_cs_mhd.f:2442-2448,
 * 3149-3179).  Off by default: the reference bypasses it on the GPU; on
 * it costs one reduction over the interior per stage. */
#define CS_FLAG_STEP10 64

/* cs_params.flags: reconstruct with LIMIT_ALL_SLOPES_P2
 * (400riemann_integrate/420limit_all_slopes_p2.f:9), the full third-order
 * WENO-AO the reference driver calls in place of LIMIT_ALL_SLOPES_P12
 * (1000riemann_geomesh_cs_mhd.f:2387-2391, same arguments).  It differs in
 * two steps: STEP 7.a limits the primitives with eight one-sided 9-zone
 * quadratic stencils and the central 18-zone least squares (420:2459-5394,
 * replacing P12's STEPS 7.a and 7.b), and STEP 9.b interpolates E with
 * eight one-sided 10-zone stencils and the central 19-zone least squares
 * (420:8553-12285, replacing STEPS 9.b and 9.c); the entropy slopes and every
 * other step are P12's.  The stencil inverses depend on the geometry only
 * and are resident (built at cs_mesh_build, 5.2 KB (primitives) + 6.4 KB (E)
 * per zone in FP64, shared by the six panels where they are rotations of one
 * another): cs_create rejects the flag together with CS_FLAG_NO_OP_CACHE
 * (CS_ERR_ARG), and cs_mesh_build fails with CS_ERR_NOMEM where the device
 * has no room for them. */
#define CS_FLAG_P2 128

/* Seeded initial-state description (new generator cases of the problem
 * library, built with the reference mechanism of 820init_patch_cube_sphere.f). */
typedef struct cs_init_desc {
  uint64_t seed;
  int32_t kind;         /* 0: surface (config 0), 1: hydrostatic shell (configs 1-2) */
  int32_t lmax;         /* harmonic degree of the seeded sums */
  double rho_amp;       /* density perturbation amplitude */
  double a_amp;         /* vector-potential amplitude */
  double v_amp;         /* solid-body rotation amplitude */
  double p0;            /* background pressure (kind 0) / p_inf (kind 1) */
} cs_init_desc;

typedef struct cs_ctx cs_ctx;

/* Geometry fields readable through cs_geometry_get (component count in ()). */
enum cs_geom_field {
  CS_G_VERT = 0,   /* (3) vertex coordinates            */
  CS_G_XF_QP,      /* (15) x-face quadrature points [c*5+q] (also the B points) */
  CS_G_XF_QW,      /* (5)  x-face area weights (sum 1)  */
  CS_G_XF_N,       /* (3)  x-face unit normal           */
  CS_G_XF_AREA,    /* (1) */
  CS_G_XF_CEN,     /* (3) */
  CS_G_YF_QP, CS_G_YF_QW, CS_G_YF_N, CS_G_YF_AREA, CS_G_YF_CEN,
  CS_G_ZF_QP, CS_G_ZF_QW,
  CS_G_ZF_N,       /* (15) z-face normal per quadrature point [c*5+q] */
  CS_G_ZF_AREA, CS_G_ZF_CEN,
  CS_G_XB_QW, CS_G_YB_QW, CS_G_ZB_QW, /* (5) B-field quadrature weights */
  CS_G_V_SCALE,    /* (1) v_scale_length */
  CS_G_V_VOL,      /* (1) */
  CS_G_V_CEN,      /* (3) */
  CS_G_COEF,       /* (10) Coef_Basis_Moments */
  CS_G_NFIELDS
};

int cs_geom_ncomp(int field);

/* Lifecycle. */
int cs_create(const cs_params* p, cs_ctx** out);
int cs_destroy(cs_ctx* ctx);
const char* cs_last_error(const cs_ctx* ctx);
int cs_box_dims(const cs_ctx* ctx, int32_t* ni, int32_t* nj, int32_t* nk);

/* One-line reason why p is rejected by cs_create, or "" when it is valid. */
const char* cs_params_check(const cs_params* p);

/* Mesh: builds the 6-panel geometry on the host and keeps it resident on the device. */
int cs_mesh_build(cs_ctx* ctx);
/* Mesh shared with another context: ctx (created, no mesh yet) uses the
 * resident mesh of `from` (geometry, ghost-exchange and panel-ownership
 * maps, resident operators) instead of building its own, and allocates only
 * its state.  The parameters that define the mesh (ntp, nr, nghost,
 * radial_mesh, rmin, rmax, radial_ratio, smallnum and the NO_ADP_CACHE,
 * NO_OP_CACHE, NO_PANEL_SYNC, FP32, ADP_PER_PANEL and LSQ_PER_PANEL flags)
 * must be equal, and both
 * contexts on the current device.  The mesh is freed with the last context
 * that uses it.  The reference builds the mesh once per patch and run
 * (MAKE_MESH_GNOMONIC_CS_SECTOR, 201) and has no counterpart for sharing
 * it between solves. */
int cs_mesh_share(cs_ctx* ctx, const cs_ctx* from);
/* Device bytes held by the context's mesh: geometry, mask, stencil,
 * ghost-exchange and panel-ownership maps and the resident operators (ADP
 * factors, least-squares row weights).  Contexts attached to one mesh
 * report the same figure; cs_estimate_device_bytes plans it before a
 * build.  No reference counterpart (the reference does not account device
 * memory). */
int cs_mesh_device_bytes(cs_ctx* ctx, uint64_t* bytes);
/* Host-only mesh build (no device is touched); the geometry, mask and
 * stencil getters below then work without a GPU. */
int cs_mesh_build_host(cs_ctx* ctx);
int cs_geometry_get(cs_ctx* ctx, int field, double* host_out, size_t n_doubles);
int cs_mask_get(cs_ctx* ctx, int32_t* host_out, size_t n);            /* imask_active, per box */
/* Host copy of the ghost-exchange map cs_fill_ghosts applies on the device
 * (the panel-edge exchange of the reference's LOAD_LOCAL_BUFFERS_* /
 * FETCH_BUFFERS_FILL_IN_* routines, 300riemann_module/320-333, written as
 * one list): entry t sets element dst[t] from element src[t], both offsets
 * into a field array of the panel-box layout (for U they include the
 * component), and meta[t] holds the destination field in bits 0-2, the
 * source field in bits 5-7 (0 U, 1 entropy mode 1, 2 Bxf, 3 Byf, 4 Bzf), a
 * negation in bit 3 and, in bit 4, averaging with the destination's value
 * before the exchange.  Every source is read before any destination is
 * written.  Built from the host mesh (cs_mesh_build_host is enough: no
 * device).  With all three arrays null only *n is set; otherwise *n must be
 * the entry count.  A panel split across ranks exchanges the entries whose
 * source and destination panels sit on different ranks. */
int cs_fill_map_get(cs_ctx* ctx, int32_t* src, int32_t* dst, uint8_t* meta, int64_t* n);
/* Host copy of the panel-edge ownership lists the stage applies unless
 * CS_FLAG_NO_PANEL_SYNC is set (the single-device form of the reference's
 * defect exchange, DRV:3200-3461 with 485update_defect_imex_rk.f): every
 * copy of a face or edge that two or three panels compute takes the value
 * of the copy on the lowest-numbered panel.  which = 0: faces on panel
 * edges; dst[t] / src[t] are face offsets (panel * box + point) and
 * dst_kind / src_kind their directions (0 x, 1 y), the copy taking the
 * source's two one-sided flux contributions with the sides exchanged and
 * the negated entropy flux (sign = -1).  which = 1: edges on panel
 * boundaries; offsets as for faces, dst_kind / src_kind the EMF component
 * (0 Ex, 1 Ey, 2 Ez) and sign the factor (+1 or -1, where the two panels
 * run the edge in opposite directions).  No source is a destination.  Built
 * from the host mesh; null arrays and *n as for cs_fill_map_get. */
int cs_sync_map_get(cs_ctx* ctx, int32_t which, int32_t* dst, int32_t* src, int8_t* dst_kind, int8_t* src_kind,
                    int8_t* sign, int64_t* n);
int cs_stencil_get(cs_ctx* ctx, int32_t* host_out, size_t n);         /* istencil, [6][12][2][NJ][NI] */

/* Geometry of one coarse zone cut with stride iscale out of sector isector
 * (1..6) of a ntp_global x ntp_global x nr_global mesh without ghosts: the
 * setting of the reference's quadrature-point test program
 * (_T/_200mesh/004test_quadpoints.f:42-246).  Host only; field as in
 * cs_geometry_get with a box of (ntp_global/iscale + 1)^2 x (nr_global/iscale + 1). */
int cs_geometry_single_zone(int32_t isector, int32_t ntp_global, int32_t nr_global, int32_t iscale,
                            double rmin, double rmax, int32_t radial_mesh, int32_t field,
                            double* host_out, size_t n_doubles);

/* State.  U: 8 components; ent: 1; bxf/byf/bzf: 1 each; all FP64 panel boxes. */
int cs_init_problem(cs_ctx* ctx, const cs_init_desc* d);
/* The same seeded initial state written into host arrays (no device). */
int cs_init_problem_host(cs_ctx* ctx, const cs_init_desc* d, double* U, double* ent,
                         double* bxf, double* byf, double* bzf);
int cs_state_put(cs_ctx* ctx, const double* U, const double* ent,
                 const double* bxf, const double* byf, const double* bzf);
int cs_state_get(cs_ctx* ctx, double* U, double* ent,
                 double* bxf, double* byf, double* bzf);

/* The same state in the reference driver's own module arrays, passed
 * unchanged (300riemann_module_3d.f:495-530, one patch per panel, patch
 * p+1 = panel p, Fortran column-major with their lower bounds):
 *   U_amr(1-G:N+G, 1-G:N+G, 1-G:nr+G, n_cc_components, 6)
 *   entropygr_amr(1-G:N+G, 1-G:N+G, 1-G:nr+G, 6)
 *   Bxf_amr, Byf_amr, Bzf_amr(0-G:N+G, 0-G:N+G, 0-G:nr+G, 6)
 * with G = nghost, N = ntp.  n_cc_components >= 8: the 8 ideal-MHD
 * components are read and written, further ones (passive species) are
 * ignored by put and left untouched by get.  The face arrays' boxes are the
 * panel boxes above; the zone arrays lack the panel box's lower layer
 * (index -G), which put leaves zero. */
int cs_state_put_amr(cs_ctx* ctx, int32_t n_cc_components, const double* U_amr, const double* entropygr_amr,
                     const double* Bxf_amr, const double* Byf_amr, const double* Bzf_amr);
int cs_state_get_amr(cs_ctx* ctx, int32_t n_cc_components, double* U_amr, double* entropygr_amr, double* Bxf_amr,
                     double* Byf_amr, double* Bzf_amr);

/* Whole-stage and whole-step entry points (device resident, on ctx's stream). */
int cs_stage(cs_ctx* ctx, int32_t irk, double dtcur);
int cs_step(cs_ctx* ctx, double dtcur, double* dtcurp1);
/* nsteps steps, each at the time step the previous one chose (the driver's
 * time loop, 1000riemann_geomesh_cs_mhd.f:1738-2908, with dtcur taken from
 * EVALUATE_TIMESTEP after every step); the same results as nsteps calls of
 * cs_step feeding each dtcurp1 into the next.  The time step stays on the
 * device between steps, the step is captured once into a CUDA graph and
 * replayed, and the host synchronises once, at the end, to return the next
 * time step.  (Without the graph while cs_profile_begin is active.) */
int cs_steps(cs_ctx* ctx, int32_t nsteps, double dtcur, double* dtcurp1);
int cs_evaluate_timestep(cs_ctx* ctx, double dtcur, double* dtcurp1);
int cs_synchronize(cs_ctx* ctx);

/* Per-routine entry points with the reference routine names, for
 * step-by-step parity (each runs on the resident state). */
int cs_fill_ghosts(cs_ctx* ctx);
int cs_limit_all_slopes_p12(cs_ctx* ctx);
int cs_make_facial_fluxes(cs_ctx* ctx);
int cs_make_edge_efields_p1(cs_ctx* ctx);
int cs_build_non_stiff_sources(cs_ctx* ctx);
int cs_update_imex_rk_step_p1(cs_ctx* ctx, double dtmove);
int cs_cleanup_after_update(cs_ctx* ctx);

/* Intermediate arrays for parity checks (panel boxes, component-major).
 * which: 0 V (8 comps x 10 modes, comp-major [m*8+c]), 1 entropy modes (4),
 * 2 flattener (1), 3 dU_dt (8), 4 Efx, 5 Efy, 6 Efz, 7 Bxf_quadpts (5),
 * 8 Byf_quadpts (5), 9 Bzf_quadpts (5), 10 E_zc mode-1 (3),
 * 11 face speeds S_L,S_R,S_D,S_U,S_B,S_T (6), 12 entropy fluxes x,y,z (3),
 * 13 positivity record of STEP 7.c per zone (1): 2 x the shrink passes
 * applied (0-15) plus 1 where the zone gave up (440:553-830). */
int cs_debug_get(cs_ctx* ctx, int32_t which, double* host_out, size_t n_doubles);

/* Test hook of the error path of the bounded device waits: the kernels
 * that wait on an mbarrier for a bulk or tensor copy (the ADP substitution,
 * STEP 7.b's row weights) give up after a fixed number of polls and set a
 * per-context device flag, which the next read of the time step turns into
 * CS_ERR_CUDA ("a bounded device wait gave up").  This sets that flag to
 * value from the host (nonzero: as if a wait had given up; 0: clears it),
 * so the path can be tested without making a device wait fail.  No
 * counterpart in the reference. */
int cs_debug_set_wait_error(cs_ctx* ctx, int32_t value);

/* Timing and launch accounting.  cs_get_stream returns the context's
 * cudaStream_t (as void*) so a caller can order its own work and events
 * after the library's.  Between cs_profile_begin and cs_profile_end every
 * kernel launch is bracketed by CUDA events on that stream; cs_profile_end
 * synchronizes and returns, per kernel name (32-byte NUL-padded entries in
 * names), the summed device milliseconds and the launch counts.
 * cs_launch_count returns the kernels this context has launched. */
int cs_get_stream(cs_ctx* ctx, void** stream);
int cs_launch_count(cs_ctx* ctx, int64_t* n);
int cs_profile_begin(cs_ctx* ctx);
int cs_profile_end(cs_ctx* ctx, int32_t max_kernels, char* names, double* total_ms,
                   int64_t* launches, int32_t* n_kernels);

/* CFL time step over caller-owned device arrays, with no device allocation.
 * No counterpart in the reference: it is the EVALUATE_TIMESTEP reduction
 * (490evaluate_timestep.f:121-286, the same result as cs_evaluate_timestep)
 * for callers that cannot let a library allocate device memory, e.g. a host
 * code whose memory pool owns the whole device or whose step loop must not
 * call cudaMalloc.  U (8 components), ent, v_scale and mask are panel boxes
 * of the layout above in device memory; nothing is written to them.  The
 * reduction scratch is a fixed static device array (6 x 2048 layer partials,
 * 96 KB), so nr > 2048 is rejected with CS_ERR_ARG; no slot needs clearing
 * (each is written before it is read).  Every call looks the scratch up
 * with cudaGetSymbolAddress in the current device's context (the first
 * call on a device may load the module), so no address outlives a
 * cudaDeviceReset.  All calls on a device share the scratch: calls that
 * overlap in time (other threads or streams) race, so serialize them.
 * Runs on stream (cudaStream_t, may be null) and synchronizes it to return
 * *dtcurp1 through a copy to host memory, so no call may be made on a
 * stream that is being captured.  FP64 state only: U and ent hold doubles,
 * as in the plain form (not the CS_FLAG_FP32 form's device arrays). */
int cs_cfl_timestep_noalloc(const double* U, const double* ent, const double* v_scale,
                            const int32_t* mask, int32_t ntp, int32_t nr, int32_t nghost,
                            double gamma, double rhofloor, double prsfloor, double cfl_coef,
                            double dtcur, void* stream, double* dtcurp1);

/* Snapshots (checkpoint / resume): the reference's riemann.in (time, dtcur;
 * 1000riemann_geomesh_cs_mhd.f:1798-1804, read under RESTART at :1527-1666)
 * plus its WRITEDATA / READDATA state files, as one binary file: magic
 * "CSB2SNP1", a uint32 length, a JSON header (parameters, time, dtcur, step,
 * array list, FNV-1a 64-bit hash of the payload) and the FP64 arrays U (8),
 * entropy, Bxf, Byf, Bzf in the panel-box layout.  Loading returns
 * CS_ERR_STATE when the file belongs to other mesh / physics parameters and
 * CS_ERR_NUMERIC when the payload does not match its hash; a loaded state
 * continues bit for bit.  The _host forms work on host arrays, no device. */
int cs_snapshot_save(cs_ctx* ctx, const char* path, double time, double dtcur, int64_t step);
int cs_snapshot_load(cs_ctx* ctx, const char* path, double* time, double* dtcur, int64_t* step);
int cs_snapshot_write_host(const char* path, const cs_params* p, const double* U, const double* ent,
                           const double* bxf, const double* byf, const double* bzf,
                           double time, double dtcur, int64_t step);
int cs_snapshot_read_host(const char* path, const cs_params* p, double* U, double* ent,
                          double* bxf, double* byf, double* bzf,
                          double* time, double* dtcur, int64_t* step);

/* Serving (no counterpart in the reference, whose driver runs one solve per
 * job).  A server admits solve requests as they arrive while device memory
 * allows (mem_fraction of the free memory at creation) and runs at most
 * max_active at once, each in its own context and stream driven by its own
 * host thread, so requests that arrive while others run overlap with them
 * on the device.  Meshes stay resident between requests: the first request
 * on a mesh builds it (cs_mesh_build), later requests with the same mesh
 * parameters attach to it (as cs_mesh_share) and allocate only their state;
 * a cached mesh that no running request uses is freed when an admission
 * needs its memory.  A request then runs cs_init_problem, cs_steps and
 * cs_diag; its result does not depend on what else runs (every kernel
 * is deterministic).  Latency is measured from submission to completion.
 * cs_estimate_device_bytes counts a solve's state and its mesh. */
typedef struct cs_server cs_server;
typedef struct cs_request {
  cs_params params;
  cs_init_desc init;
  int32_t steps;
  int32_t reserved;
} cs_request;
typedef struct cs_serve_result {
  int32_t status;       /* cs_status of the request */
  int32_t mesh_reused;  /* 1 when the request ran on a cached resident mesh */
  double latency_s;     /* submission to completion */
  double queue_s;       /* submission to admission */
  double mass, energy, max_divb;  /* cs_diag of the final state */
  double dt_last;       /* the next time step after the last step */
  int64_t zone_updates; /* interior zones x steps */
} cs_serve_result;
size_t cs_estimate_device_bytes(const cs_params* p);
int cs_serve_create(int32_t max_active, double mem_fraction, int32_t keep_state, cs_server** out);
int cs_serve_submit(cs_server* sv, const cs_request* req, int64_t* id);
int cs_serve_wait(cs_server* sv, int64_t id, cs_serve_result* out);   /* blocks; returns the request's status */
int cs_serve_state(cs_server* sv, int64_t id, double* U, double* ent,
                   double* bxf, double* byf, double* bzf);           /* final state, when keep_state */
int cs_serve_stats(cs_server* sv, double* p50_s, double* p99_s, double* zone_updates_per_s, int64_t* completed);
int cs_serve_destroy(cs_server* sv);                                   /* waits for every request */

/* Batched form (no counterpart in the reference): independent solves of
 * different sizes (each its own context, mesh, state and time step, all on
 * the current device) advanced together.  Each member's step is captured
 * once into a CUDA graph (the capture cs_steps uses) and the batch embeds
 * every member's step as an independent child of one graph, so that one
 * graph launch advances every member by one step and the device runs the
 * members side by side.  cs_batch_steps takes and returns one time step per
 * member (dtcur[n], dtcurp1[n]) and gives every member the same results as
 * cs_steps on it alone.  cs_batch_autotune chooses, per size class (members
 * with equal mesh parameters), the share of the SMs each launch's grid is
 * sized for (1, 1/2, 1/4 or 1/8; every kernel strides over its range, so
 * results do not change) by timing trial_steps batch steps per candidate,
 * and restores the members' states afterwards; it returns the best batch
 * step time in ms.  Members must not be stepped elsewhere while in a batch;
 * destroying the batch leaves them to the caller. */
typedef struct cs_batch cs_batch;
int cs_batch_create(cs_ctx* const* members, int32_t n, cs_batch** out);
int cs_batch_steps(cs_batch* b, int32_t nsteps, const double* dtcur, double* dtcurp1);
int cs_batch_autotune(cs_batch* b, int32_t trial_steps, double* best_ms_per_step);
int cs_batch_grid_fraction(const cs_batch* b, int32_t member, double* frac);
const char* cs_batch_last_error(const cs_batch* b);
int cs_batch_destroy(cs_batch* b);

/* Known-answer access to the multidimensional HLL Riemann solvers of the
 * edge EMFs (Two_D_RS_Ez_4State_HLL, 620riemann_2d/630_2d_rs_ez_two_d_rs_ez_4state_hll.f:10;
 * Two_D_RS_Ez_3State_HLL, 631_2d_rs_ez_two_d_rs_ez_3state_hll.f:9), with the
 * single Ez the edge kernels pass for all states: for kind 4, n cases of
 * (S_R, S_L, S_U, S_D, cos_t, sin_t, Ez, Bneta_U, Bneta_D, By_R, By_L); for
 * kind 3, n cases of (S_R1, S_L1, S_R2, S_L2, S_R3, S_L3, Ez, Bneta_1,
 * Bneta_2, Bneta_3).  out[n] = ESSz, evaluated on the current device. */
int cs_twod_rs_ez(int32_t kind, int32_t n, const double* in, double* out);

/* V_min_local / V_max_local of the last LIMIT_ALL_SLOPES_P12 of the context
 * (STEP 10, 421:9354-9976; needs CS_FLAG_STEP10): v_min[0..7] / v_max[0..7]
 * the min / max over the active interior zones of the primitives (rho,
 * v_x, v_y, v_z, p, B_x, B_y, B_z; the zone values the stage reconstructs,
 * B from the ADP solve), v_min[8] / v_max[8] those of the zone's net face
 * flux of B divided by max(|B| on its upper faces, |B| on its lower faces,
 * msonic sqrt(4 x 3.14 x rho)).  After a step these are the last stage's,
 * the values the reference driver prints for that step.  CS_ERR_STATE
 * without the flag or before the first stage. */
int cs_limit_minmax(cs_ctx* ctx, double* v_min, double* v_max);

/* Known-answer access to the pointwise physics of the stage kernels,
 * evaluated on the current device in the state type of the form that
 * p->flags selects (FP64, or FP32 with CS_FLAG_FP32), with the physics
 * constants of p: for kind 0, PRIM_TO_CONS (661pde_3d_prim_to_cons.f:14):
 * n cases of (V[8], ent) -> U[8]; for kind 1, CONS_TO_PRIM
 * (662pde_3d_cons_to_prim.f:14): n cases of (U[8], ent) -> (V[8], ent,
 * floor flag, U[8] after the floors); for kind 2, the HLL solve of
 * OneD_RS_MHD_Ptwise (610_1d_rs_oned_rs_mhd_ptwise.f:100-237) in the face
 * frame: n cases of (V_L[8], V_R[8], ent_L, ent_R) -> (Fluct_L[8],
 * Fluct_R[8], F_L[8], F_R[8], S_L, S_R, entropy flux).  The reference's
 * _T/_660riemann_3d/660pde_3d_test_program.f:58-142 runs kind 0 then 1. */
int cs_pointwise(const cs_params* p, int32_t kind, int32_t n, const double* in, double* out);

/* Measured FP64 fused multiply-add rate of the current device in TFLOP/s
 * (2 flops per FMA): 8 blocks per SM of 256 threads, each running 8
 * independent FMA chains for iters x 16 steps, timed with CUDA events after
 * a warm-up launch.  The denominator of the FP64 roofline; no counterpart
 * in the reference. */
int cs_fp64_fma_rate(int32_t iters, double* tflops);

/* Diagnostics: sums over interior zones of 6 panels of volume-weighted
 * mass, energy and the max |div B| (face-area-weighted, per volume),
 * reduced on the device in FP64 in a fixed order (the same numbers for the
 * same state whatever the launch shapes). */
int cs_diag(cs_ctx* ctx, double* mass, double* energy, double* max_divb);

#ifdef __cplusplus
}
#endif
#endif
