// Host-side description of one resident solve (geometry + state on one
// device, one stream).  Shared by the launch wrappers of every .cu file.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cs_dev.cuh"

namespace cs {

struct FillMap {
  // Gather-then-scatter ghost exchange, one entry per ghost destination:
  // tmp[n] = value(src[n]) (negated when meta bit 3 is set; averaged with
  // the destination's pre-exchange value when bit 4 is set), then
  // field[dst[n]] = tmp[n].  meta bits 0-2 select the destination field
  // and bits 5-7 the source field: 0 U (offsets include the component),
  // 1 ent, 2 Bxf, 3 Byf, 4 Bzf.
  int32_t* d_src = nullptr;
  int32_t* d_dst = nullptr;
  uint8_t* d_meta = nullptr;
  double* d_tmp = nullptr;
  long long n = 0;
};

// Panel-edge ownership maps on the device (see build_sync_maps).
struct PanelSync {
  int32_t *f_dst = nullptr, *f_src = nullptr;
  int8_t *f_ddir = nullptr, *f_sdir = nullptr;
  int32_t *e_dst = nullptr, *e_src = nullptr;
  int8_t *e_df = nullptr, *e_sf = nullptr, *e_sign = nullptr;
  int32_t* e_cls = nullptr;  // ncls + 1 starts: the entries of one edge (its copies but the owner's)
  long long nf = 0, ne = 0, ncls = 0;
};

// Per-kernel device timing with CUDA events recorded on the solve's
// stream between consecutive launches (enabled by cs_profile_begin).
struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> ev;     // ev[0]: start; ev[i]: end of launch i
  std::vector<const char*> name;   // name[i]: launch ending at ev[i]
  int n = 0;                       // events recorded since the last harvest
  std::vector<std::string> keys;   // accumulated per kernel name
  std::vector<double> ms;
  std::vector<long long> count;
};

// What depends on the mesh parameters only: the host geometry, its device
// copy, the ghost-exchange and panel-ownership maps and the resident
// geometry-only operators.  Built once and shared read-only by every solve
// on the same mesh (cs_mesh_share, the serving mesh cache); freed with its
// last user.
struct MeshRes {
  GeomHost host;
  DGeom g{};
  FillMap fill{};       // d_tmp stays null here: the staging buffer is per solve
  PanelSync psync{};
  void* op_m9 = nullptr;   // least-squares inverses in the state's type (FP32 in the precision form)
  void* op_m10 = nullptr;
  void* lsq_map = nullptr;  // LsqPanelMap[6] when row weights are panel 1's only
  bool m9_shared = false, m10_shared = false;  // which of op_m9 / op_m10 are panel 1's only
  void* op_p2v = nullptr;  // CS_FLAG_P2 one-sided stencil inverses (state's type)
  void* op_p2e = nullptr;
  bool p2_shared = false;  // op_p2v / op_p2e are panel 1's only
  void* adp_lu = nullptr;   // FP64 per panel; panel-shared ones in the state's type
  int8_t* adp_piv = nullptr;
  int8_t* adp_pmap = nullptr;  // ADP factors shared by the panels: per panel [unknown map][sign]
  std::vector<void*> allocs;
  size_t bytes = 0;     // device bytes held
  bool on_device = false;
  MeshRes() = default;
  MeshRes(const MeshRes&) = delete;
  MeshRes& operator=(const MeshRes&) = delete;
  ~MeshRes() {
    for (void* q : allocs) cudaFree(q);
  }
};

struct Solve {
  cs_params p{};
  Dims d{};
  PhysC ph{};
  DGeom g{};
  DState st{};                // state of the plain (FP64) form
  DStateT<float> stF{};       // state of the precision (FP32 bulk) form
  bool fp32 = false;          // which of the two this solve uses
  std::shared_ptr<MeshRes> mesh = std::make_shared<MeshRes>();
  std::vector<void*> allocs;  // device allocations owned by the solve
  FillMap fill;
  PanelSync psync;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;  // stream-ordered pool of the solve's own arrays
  unsigned char* init_buf = nullptr;  // seeded harmonic terms of cs_init_problem
  size_t init_buf_bytes = 0;
  double* diag_buf = nullptr;         // cs_diag: result and partial sums
  unsigned long long* step10_keys = nullptr;  // STEP 10 min (9) and max (9) keys, with CS_FLAG_STEP10
  int device = 0;
  int sm_count = 148;
  bool has_mesh = false, has_state = false;
  long long launches = 0;  // kernels launched by this solve
  cudaGraph_t graph = nullptr;           // one step, captured by cs_steps / cs_batch_steps
  cudaGraphExec_t graph_exec = nullptr;  // its executable form
  long long graph_kernels = 0;           // kernels in that graph
  double grid_frac = 1.0;                // share of the SMs a launch's grid is sized for (autotuned in batches)
  Prof prof;
  std::string err;
};

// Attaches a solve (parameters set, no mesh yet) to a resident mesh and
// allocates its own state; builds the mesh first when it is not on the
// device yet.  Defined with the C ABI.
int mesh_attach(Solve& sv, const std::shared_ptr<MeshRes>& m);
// One whole step at the device-resident time step (stages and CFL
// reduction), and its capture into sv.graph / sv.graph_exec (kept until
// drop_graph or the solve's end).  Defined with the C ABI.
int run_step(Solve& sv);
int step_graph(Solve& sv);
void drop_graph(Solve& sv);
// Device-to-host read of the next time step and of the error flags.
int read_dt(Solve& sv, double* out);
int fail(Solve& sv, int code, const std::string& msg);
int cuda_fail(Solve& sv, cudaError_t e, const char* what);
// Device allocation owned by the solve (stream-ordered, zero-filled).
void* solve_alloc(Solve& sv, size_t bytes, cudaError_t& e);
// The seeded initial state built on the device (cs_init_problem).
int init_problem_device(Solve& sv, const cs_init_desc& desc);
// Identity of the mesh a parameter set needs (solves with equal keys can
// share one MeshRes).
std::string mesh_key(const cs_params& p);

// Called after every launch (kernel == false for copies): counts kernel
// launches and, when profiling, records an event on the stream.
void mark(Solve& sv, const char* name, bool kernel = true);
// Records the start event of a profiled sequence (no-op when off).
void prof_start(Solve& sv);

// SMs a launch of this solve sizes its grid for (every kernel loops over
// its range with a grid stride, so the grid size never changes results).
inline int grid_sms(const Solve& sv) {
  const int n = (int)(sv.sm_count * sv.grid_frac + 0.5);
  return n < 1 ? 1 : n;
}

inline int blocks_for(long long n, int threads, int sm_count) {
  long long b = (n + threads - 1) / threads;
  long long cap = (long long)sm_count * 64;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace cs

// The opaque context of the C ABI: one resident solve.
struct cs_ctx {
  cs::Solve sv;
};
