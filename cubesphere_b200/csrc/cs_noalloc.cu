// CFL time step over caller-owned device arrays without any device
// allocation: the reduction's scratch is a file-scope __device__ array.
//
// Same quantity as EVALUATE_TIMESTEP (400riemann_integrate/490evaluate_timestep.f:121-286)
// and cs_evaluate_timestep: min(1.1 dtcur, min over the active interior
// zones of cfl * v_scale / (|v| + c_fast)), with the conserved->primitive
// repair applied in registers only (the arrays are not written).
#include "cs_solve.h"

namespace cs {
namespace {

// One partial minimum per (panel, radial layer); the last slot holds the
// result.  Every slot is written before it is read in the same call, so
// nothing has to start at zero.
constexpr int kMaxLayers = 2048;
constexpr int kSlots = 6 * kMaxLayers + 1;
__device__ __align__(256) double g_cfl_scratch[kSlots];

// Phase 1: block b reduces the N x N zones of layer (panel b / nr, k = b % nr + 1).
__global__ void k_cfl_layers(Dims d, PhysC ph, const double* __restrict__ U, const double* __restrict__ ent,
                             const double* __restrict__ vscale, const int32_t* __restrict__ mask, double* part) {
  const int p = blockIdx.x / d.nr, k = blockIdx.x % d.nr + 1;
  double dtl = 1.0e300;
  for (int t = threadIdx.x; t < d.N * d.N; t += blockDim.x) {
    const int i = t % d.N + 1, j = t / d.N + 1;
    if (mask[(long long)p * d.S + d.idx(i, j, 0)] == 0) continue;
    double Uz[8], V[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) Uz[q] = U[d.at(q, p, i, j, k)];
    double en = ent[d.at(0, p, i, j, k)];
    d_cons_to_prim(ph, en, Uz, V);
    const double b2 = V[5] * V[5] + V[6] * V[6] + V[7] * V[7];
    const double ms = sqrt((ph.gamma * V[4] + ph.ob4pi * b2) / V[0]);
    const double a21 = sqrt(V[1] * V[1] + V[2] * V[2] + V[3] * V[3]) + ms;
    dtl = fmin(dtl, ph.cfl * vscale[d.at(0, p, i, j, k)] / a21);
  }
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_down_sync(0xffffffffu, dtl, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = dtl;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = red[0];
    for (int w = 1; w < (int)(blockDim.x / 32); ++w) m = fmin(m, red[w]);
    part[blockIdx.x] = m;
  }
}

// Phase 2: one block folds the partials into the result slot.
__global__ void k_cfl_final(const double* part, int nparts, double start, double* out) {
  double m = start;
  for (int t = threadIdx.x; t < nparts; t += blockDim.x) m = fmin(m, part[t]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int w = 1; w < (int)(blockDim.x / 32); ++w) r = fmin(r, red[w]);
    *out = r;
  }
}

}  // namespace
}  // namespace cs

extern "C" int cs_cfl_timestep_noalloc(const double* U, const double* ent, const double* v_scale,
                                       const int32_t* mask, int32_t ntp, int32_t nr, int32_t nghost,
                                       double gamma, double rhofloor, double prsfloor, double cfl_coef,
                                       double dtcur, void* stream, double* dtcurp1) {
  if (!U || !ent || !v_scale || !mask || !dtcurp1) return CS_ERR_ARG;
  if (ntp < 1 || nr < 1 || nghost < 1 || !(dtcur > 0.0) || !(gamma > 1.0)) return CS_ERR_ARG;
  if (nr > cs::kMaxLayers) return CS_ERR_ARG;  // scratch holds 6 * 2048 layer partials
  // The scratch's device address in the current device's context, looked
  // up on every call: an address kept from an earlier call would be stale
  // after cudaDeviceReset or under another context.  The first lookup on a
  // device may load the module.
  double* scratch = nullptr;
  if (cudaGetSymbolAddress((void**)&scratch, cs::g_cfl_scratch) != cudaSuccess || !scratch) return CS_ERR_CUDA;
  cs::Dims d;
  d.N = ntp;
  d.nr = nr;
  d.G = nghost;
  d.NI = d.NJ = ntp + 2 * nghost + 1;
  d.NK = nr + 2 * nghost + 1;
  d.S = (long long)d.NI * d.NJ * d.NK;
  cs::PhysC ph{};
  const double pi = 4.0 * std::atan(1.0);
  ph.gamma = gamma;
  ph.rhofloor = rhofloor;
  ph.prsfloor = prsfloor;
  ph.ob4pi = 1.0 / (4.0 * pi);
  ph.ob8pi = 1.0 / (8.0 * pi);
  ph.fourpi = 4.0 * pi;
  ph.cfl = cfl_coef;
  cudaStream_t st = (cudaStream_t)stream;
  const int nparts = 6 * nr;
  cs::k_cfl_layers<<<nparts, 256, 0, st>>>(d, ph, U, ent, v_scale, mask, scratch);
  cs::k_cfl_final<<<1, 1024, 0, st>>>(scratch, nparts, 1.1 * dtcur, scratch + cs::kSlots - 1);
  if (cudaGetLastError() != cudaSuccess) return CS_ERR_CUDA;
  if (cudaMemcpyAsync(dtcurp1, scratch + cs::kSlots - 1, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CS_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return CS_ERR_CUDA;
  return CS_OK;
}
