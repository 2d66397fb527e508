// Host-side description of one resident solve (geometry + state on one
// device, one stream).  Shared by the launch wrappers of every .cu file.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
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
  long long nf = 0, ne = 0;
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

struct Solve {
  cs_params p{};
  Dims d{};
  PhysC ph{};
  DGeom g{};
  DState st{};                // state of the plain (FP64) form
  DStateT<float> stF{};       // state of the precision (FP32 bulk) form
  bool fp32 = false;          // which of the two this solve uses
  GeomHost host;             // host geometry (kept for cs_geometry_get)
  std::vector<void*> allocs;  // device allocations owned by the solve
  FillMap fill;
  PanelSync psync;
  cudaStream_t stream = nullptr;
  int device = 0;
  int sm_count = 148;
  bool has_mesh = false, has_state = false;
  long long launches = 0;  // kernels launched by this solve
  Prof prof;
  std::string err;
};

// Called after every launch (kernel == false for copies): counts kernel
// launches and, when profiling, records an event on the stream.
void mark(Solve& sv, const char* name, bool kernel = true);
// Records the start event of a profiled sequence (no-op when off).
void prof_start(Solve& sv);

inline int blocks_for(long long n, int threads, int sm_count) {
  long long b = (n + threads - 1) / threads;
  long long cap = (long long)sm_count * 64;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace cs
