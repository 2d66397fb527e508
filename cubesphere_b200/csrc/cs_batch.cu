// Batched form: many independent solves of different sizes (their own
// meshes, states and time steps) advanced together.  Each member's step is
// captured once (the same capture cs_steps replays); the batch embeds every
// member's step as an independent child of one CUDA graph, so one graph
// launch advances every member by one step and the device runs the members
// side by side.  The launch shapes are chosen per size class by an
// autotuner that times the whole batch step (cs_batch_autotune).
#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "cs_solve.h"

struct cs_batch {
  std::vector<cs_ctx*> members;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<cudaEvent_t> member_ev;
  std::string err;
};

namespace cs {
namespace {

int bfail(cs_batch* b, int code, const std::string& msg) {
  b->err = msg;
  return code;
}

void drop_batch_graph(cs_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
}

// One graph whose independent children are the members' step graphs.
int build_batch_graph(cs_batch* b) {
  if (b->exec) return CS_OK;
  cudaGraph_t parent = nullptr;
  cudaError_t e = cudaGraphCreate(&parent, 0);
  if (e != cudaSuccess) return bfail(b, CS_ERR_CUDA, std::string("cudaGraphCreate: ") + cudaGetErrorString(e));
  for (cs_ctx* m : b->members) {
    if (int rc = step_graph(m->sv)) {
      cudaGraphDestroy(parent);
      return bfail(b, rc, "member step capture: " + m->sv.err);
    }
    cudaGraphNode_t node;
    e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, m->sv.graph);
    if (e != cudaSuccess) {
      cudaGraphDestroy(parent);
      return bfail(b, CS_ERR_CUDA, std::string("cudaGraphAddChildGraphNode: ") + cudaGetErrorString(e));
    }
  }
  e = cudaGraphInstantiate(&b->exec, parent, 0);
  cudaGraphDestroy(parent);
  if (e != cudaSuccess) {
    b->exec = nullptr;
    return bfail(b, CS_ERR_CUDA, std::string("cudaGraphInstantiate(batch): ") + cudaGetErrorString(e));
  }
  return CS_OK;
}

// Orders the batch stream after the members' streams (time steps set,
// earlier work done) ...
int join_members(cs_batch* b) {
  for (size_t q = 0; q < b->members.size(); ++q) {
    Solve& sv = b->members[q]->sv;
    cudaError_t e = cudaEventRecord(b->member_ev[q], sv.stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->member_ev[q], 0);
    if (e != cudaSuccess) return bfail(b, CS_ERR_CUDA, std::string("member join: ") + cudaGetErrorString(e));
  }
  return CS_OK;
}
// ... and the members' streams after the batch stream.
int release_members(cs_batch* b) {
  cudaError_t e = cudaEventRecord(b->ev, b->stream);
  for (size_t q = 0; e == cudaSuccess && q < b->members.size(); ++q)
    e = cudaStreamWaitEvent(b->members[q]->sv.stream, b->ev, 0);
  if (e != cudaSuccess) return bfail(b, CS_ERR_CUDA, std::string("member release: ") + cudaGetErrorString(e));
  return CS_OK;
}

int run_batch(cs_batch* b, int nsteps, const double* dtcur) {
  for (size_t q = 0; q < b->members.size(); ++q) launch_set_dt(b->members[q]->sv, dtcur[q]);
  if (int rc = join_members(b)) return rc;
  if (int rc = build_batch_graph(b)) return rc;
  for (int n = 0; n < nsteps; ++n) {
    const cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
    if (e != cudaSuccess) return bfail(b, CS_ERR_CUDA, std::string("cudaGraphLaunch(batch): ") + cudaGetErrorString(e));
  }
  for (cs_ctx* m : b->members) m->sv.launches += m->sv.graph_kernels * nsteps;
  return release_members(b);
}

int read_member_dts(cs_batch* b, double* out) {
  for (size_t q = 0; q < b->members.size(); ++q) {
    Solve& sv = b->members[q]->sv;
    if (int rc = read_dt(sv, &out[q])) return bfail(b, rc, "member " + std::to_string(q) + ": " + sv.err);
  }
  return CS_OK;
}

}  // namespace
}  // namespace cs

extern "C" {

int cs_batch_create(cs_ctx* const* members, int32_t n, cs_batch** out) {
  if (!members || n < 1 || !out) return CS_ERR_ARG;
  *out = nullptr;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return CS_ERR_CUDA;
  for (int32_t q = 0; q < n; ++q) {
    const cs_ctx* m = members[q];
    if (!m || !m->sv.has_mesh || !m->sv.has_state || m->sv.device != dev) return CS_ERR_STATE;
    for (int32_t r = 0; r < q; ++r)
      if (members[r] == m) return CS_ERR_ARG;
  }
  cs_batch* b = new cs_batch();
  b->members.assign(members, members + n);
  b->member_ev.resize(n, nullptr);
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) == cudaSuccess;
  for (int32_t q = 0; ok && q < n; ++q)
    ok = cudaEventCreateWithFlags(&b->member_ev[q], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cs_batch_destroy(b);
    return CS_ERR_CUDA;
  }
  *out = b;
  return CS_OK;
}

const char* cs_batch_last_error(const cs_batch* b) { return b ? b->err.c_str() : "null batch"; }

int cs_batch_steps(cs_batch* b, int32_t nsteps, const double* dtcur, double* dtcurp1) {
  if (!b || !dtcur || !dtcurp1 || nsteps < 0) return CS_ERR_ARG;
  const size_t n = b->members.size();
  for (size_t q = 0; q < n; ++q)
    if (!(dtcur[q] > 0.0)) return cs::bfail(b, CS_ERR_ARG, "every dtcur must be > 0");
  if (nsteps == 0) {
    std::copy(dtcur, dtcur + n, dtcurp1);
    return CS_OK;
  }
  if (int rc = cs::run_batch(b, nsteps, dtcur)) return rc;
  return cs::read_member_dts(b, dtcurp1);
}

int cs_batch_autotune(cs_batch* b, int32_t trial_steps, double* best_ms_per_step) {
  if (!b || trial_steps < 1) return CS_ERR_ARG;
  const size_t n = b->members.size();
  // the members' states are restored afterwards: the tuning changes no result
  std::vector<std::vector<double>> keep(n * 5);
  for (size_t q = 0; q < n; ++q) {
    cs::Solve& sv = b->members[q]->sv;
    const size_t S6 = (size_t)6 * sv.d.S;
    keep[5 * q].resize(cs::NVAR * S6);
    for (int a = 1; a < 5; ++a) keep[5 * q + a].resize(S6);
    if (int rc = cs_state_get(b->members[q], keep[5 * q].data(), keep[5 * q + 1].data(), keep[5 * q + 2].data(),
                              keep[5 * q + 3].data(), keep[5 * q + 4].data()))
      return cs::bfail(b, rc, "autotune state save: " + sv.err);
  }
  std::vector<double> dt(n), dtn(n);
  for (size_t q = 0; q < n; ++q)
    if (int rc = cs_evaluate_timestep(b->members[q], 1e30, &dt[q]))
      return cs::bfail(b, rc, "autotune time step: " + b->members[q]->sv.err);
  // size classes: members on the same mesh share their launch shapes
  std::map<std::string, std::vector<size_t>> cls;
  std::map<std::string, double> work;
  for (size_t q = 0; q < n; ++q) {
    const std::string k = cs::mesh_key(b->members[q]->sv.p);
    cls[k].push_back(q);
    work[k] += (double)b->members[q]->sv.d.S;
  }
  std::vector<std::string> order;
  for (auto& kv : cls) order.push_back(kv.first);
  std::sort(order.begin(), order.end(), [&](const std::string& x, const std::string& y) { return work[x] > work[y]; });
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto set_frac = [&](const std::string& k, double f) {
    for (size_t q : cls[k]) {
      cs::Solve& sv = b->members[q]->sv;
      if (sv.grid_frac != f) {
        sv.grid_frac = f;
        cs::drop_graph(sv);
        cs::drop_batch_graph(b);
      }
    }
  };
  auto trial = [&](double& ms) -> int {
    if (int rc = cs::run_batch(b, 1, dt.data())) return rc;  // warm-up (and graph build)
    if (int rc = cs::read_member_dts(b, dtn.data())) return rc;
    dt = dtn;
    cudaEventRecord(t0, b->stream);
    if (int rc = cs::run_batch(b, trial_steps, dt.data())) return rc;
    cudaEventRecord(t1, b->stream);
    if (int rc = cs::read_member_dts(b, dtn.data())) return rc;
    dt = dtn;
    cudaEventSynchronize(t1);
    float f = 0.f;
    cudaEventElapsedTime(&f, t0, t1);
    ms = f / trial_steps;
    return CS_OK;
  };
  const double fracs[4] = {1.0, 0.5, 0.25, 0.125};
  double best_all = 0.0;
  int rc = CS_OK;
  for (const std::string& k : order) {
    double best = 1e300, bestf = 1.0;
    for (double f : fracs) {
      set_frac(k, f);
      double ms = 0.0;
      if ((rc = trial(ms))) break;
      if (ms < best) {
        best = ms;
        bestf = f;
      }
    }
    if (rc) break;
    set_frac(k, bestf);
    best_all = best;
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  for (size_t q = 0; q < n; ++q) {
    const int r2 = cs_state_put(b->members[q], keep[5 * q].data(), keep[5 * q + 1].data(), keep[5 * q + 2].data(),
                                keep[5 * q + 3].data(), keep[5 * q + 4].data());
    if (!rc && r2) rc = cs::bfail(b, r2, "autotune state restore: " + b->members[q]->sv.err);
  }
  if (best_ms_per_step) *best_ms_per_step = best_all;
  return rc;
}

int cs_batch_grid_fraction(const cs_batch* b, int32_t member, double* frac) {
  if (!b || !frac || member < 0 || member >= (int32_t)b->members.size()) return CS_ERR_ARG;
  *frac = b->members[member]->sv.grid_frac;
  return CS_OK;
}

int cs_batch_destroy(cs_batch* b) {
  if (!b) return CS_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  cs::drop_batch_graph(b);
  for (cudaEvent_t e : b->member_ev)
    if (e) cudaEventDestroy(e);
  if (b->ev) cudaEventDestroy(b->ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return CS_OK;
}

}  // extern "C"
