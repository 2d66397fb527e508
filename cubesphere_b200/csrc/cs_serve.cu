// Serving runtime: solves of different sizes arrive as requests, are
// admitted while device memory allows, run concurrently (one context and
// one CUDA stream each, driven by its own host thread) and report their
// latency.  Requests that arrive while others run are admitted as soon as
// a slot and memory free up, so their work overlaps on the device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cs_solve.h"

namespace cs {

// Device bytes of one solve's own state and work arrays, and of the mesh
// resources it shares with other solves on the same mesh (geometry, maps,
// resident operators), with margins for allocation granularity.
size_t state_device_bytes(const cs_params& p) {
  const Box b(p.ntp, p.nr, p.nghost);
  const size_t S6 = (size_t)6 * b.size();
  // words per point of the state's type: U 8 + entropy 4, V 80 + E 30 +
  // E snapshot 3, flattener 3, face contributions 48, entropy fluxes 3,
  // speeds 6, dU/dt 8, U0 8, ent0 1 (IMEX: + 11); FP64 in both forms:
  // face B 3, face-B quadrature 15, EMFs 3, saved faces 3 (IMEX: + 3)
  size_t rwords = 12 + 113 + 3 + 48 + 3 + 6 + 8 + 8 + 1;
  size_t dwords = 3 + 15 + 3 + 3;
  if (p.rk_scheme == CS_IMEX_RK2) {
    rwords += 11;
    dwords += 3;
  }
  const size_t rsize = (p.flags & CS_FLAG_FP32) ? sizeof(float) : sizeof(double);
  size_t bytes = (rwords * rsize + dwords * sizeof(double)) * S6 + S6 * sizeof(int32_t);
  // ghost staging values (one per map entry, see mesh_device_bytes)
  bytes += (size_t)6 * 4 * (p.nghost + 1) * (p.ntp + 2 * p.nghost + 1) * (p.nr + 2 * p.nghost + 1) * 12 * 8;
  const size_t na = (size_t)6 * (p.ntp + 2 * p.nghost - 2) * (p.ntp + 2 * p.nghost - 2) * (p.nr + 2 * p.nghost - 2);
  if (!(p.flags & CS_FLAG_NO_ADP_CACHE)) {
    // ADP right-hand sides: the state's type with panel-shared factors
    const size_t esz = (p.flags & CS_FLAG_ADP_PER_PANEL) ? sizeof(double) : rsize;
    bytes += na * 36 * esz;
  }
  return bytes + ((size_t)64 << 20);
}

size_t mesh_device_bytes(const cs_params& p) {
  const Box b(p.ntp, p.nr, p.nghost);
  const size_t S6 = (size_t)6 * b.size();
  // geometry 126 words, mask and stencil
  size_t bytes = 126 * S6 * sizeof(double) + S6 * sizeof(int32_t) + (size_t)6 * 48 * b.NI * b.NJ;
  // ghost map: per panel 4 strips of G layers, 12 field words per point,
  // 9 bytes per entry (offsets, meta); panel-ownership maps are smaller
  bytes += (size_t)6 * 4 * (p.nghost + 1) * (p.ntp + 2 * p.nghost + 1) * (p.nr + 2 * p.nghost + 1) * 12 * 9 * 2;
  const size_t nl = (size_t)6 * (p.ntp + 2 * p.nghost - 4) * (p.ntp + 2 * p.nghost - 4) * (p.nr + 2 * p.nghost - 4);
  const size_t na = (size_t)6 * (p.ntp + 2 * p.nghost - 2) * (p.ntp + 2 * p.nghost - 2) * (p.nr + 2 * p.nghost - 2);
  if (!(p.flags & CS_FLAG_NO_OP_CACHE)) {
    // row weights shared by the six panels unless per-panel ones are asked
    // for: STEP 9.c's always, STEP 7.b's in the precision form
    const bool f32 = (p.flags & CS_FLAG_FP32) != 0, per = (p.flags & CS_FLAG_LSQ_PER_PANEL) != 0;
    const size_t n9 = (per || !f32) ? nl : nl / 6, n10 = per ? nl : nl / 6;
    bytes += (m9_stride(n9) * 162 + n10 * 190) * (f32 ? sizeof(float) : sizeof(double));
    // CS_FLAG_P2's one-sided stencil inverses, shared like STEP 9.c's
    if (p.flags & CS_FLAG_P2) bytes += n10 * (648 + 800) * (f32 ? sizeof(float) : sizeof(double));
  }
  if (!(p.flags & CS_FLAG_NO_ADP_CACHE)) {
    // factors shared by the six panels (in the state's type) unless
    // per-panel ones (FP64) are asked for
    const bool per = (p.flags & CS_FLAG_ADP_PER_PANEL) != 0;
    const size_t nz = per ? na : na / 6;
    const size_t esz = (per || !(p.flags & CS_FLAG_FP32)) ? sizeof(double) : sizeof(float);
    bytes += (nz + 128) * (1296 * esz + 36);
  }
  return bytes + ((size_t)64 << 20);
}

size_t estimate_device_bytes(const cs_params& p) { return state_device_bytes(p) + mesh_device_bytes(p); }

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  cs_request req{};
  int64_t id = 0;
  Clock::time_point t_submit, t_start, t_done;
  int status = -1;  // -1 pending or running, else the final cs_status
  std::string err;
  double mass = 0, energy = 0, divb = 0, dt_last = 0;
  size_t bytes = 0;      // own state, reserved while it runs
  std::string mesh;      // mesh key
  bool mesh_builder = false;
  bool mesh_reused = false;
  long long zone_updates = 0;
  std::vector<double> U, ent, bx, by, bz;  // final state (when kept)
};

// A resident mesh of the server's cache: built by the first request that
// needs it, then shared by every later request on the same mesh.
struct MeshEntry {
  std::shared_ptr<MeshRes> mesh;  // null while it is being built
  size_t bytes = 0;               // estimated device bytes, reserved while cached
};

}  // namespace
}  // namespace cs

struct cs_server {
  std::mutex mu;
  std::condition_variable cv;
  std::deque<int64_t> pending;
  std::map<int64_t, cs::Request> reqs;
  std::vector<std::thread> workers;
  std::thread sched;
  bool stop = false;
  int max_active = 4;
  int active = 0;
  int keep_state = 0;
  int device = 0;
  size_t budget = 0, reserved = 0;  // reserved: running states + cached meshes
  std::map<std::string, cs::MeshEntry> meshes;
  long long mesh_builds = 0;
  int64_t next_id = 1;
  bool started = false;
  cs::Clock::time_point t0, t_last_done;
  std::vector<double> latencies;
  long long zone_updates = 0;
};

namespace cs {
namespace {

void run_request(cs_server* sv, int64_t id) {
  cudaSetDevice(sv->device);
  Request* r;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    r = &sv->reqs[id];
    r->t_start = Clock::now();
  }
  cs_ctx* ctx = nullptr;
  int rc = cs_create(&r->req.params, &ctx);
  if (!rc && r->mesh_builder) {
    rc = cs_mesh_build(ctx);
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      auto it = sv->meshes.find(r->mesh);
      if (rc) {
        sv->reserved -= it->second.bytes;
        sv->meshes.erase(it);
      } else {
        it->second.mesh = ctx->sv.mesh;
        // account the mesh at what it holds (per-panel operators where the
        // panel-sharing check failed take more than the estimate)
        const size_t held = ctx->sv.mesh->bytes;
        sv->reserved = sv->reserved - it->second.bytes + held;
        it->second.bytes = held;
        sv->mesh_builds += 1;
      }
    }
    sv->cv.notify_all();
  } else if (!rc) {
    std::shared_ptr<MeshRes> m;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->cv.wait(lk, [&] {
        auto it = sv->meshes.find(r->mesh);
        return it == sv->meshes.end() || it->second.mesh != nullptr;
      });
      auto it = sv->meshes.find(r->mesh);
      if (it != sv->meshes.end()) m = it->second.mesh;
    }
    if (!m) {
      rc = cs_mesh_build(ctx);  // its builder failed: build a private mesh
    } else {
      rc = mesh_attach(ctx->sv, m);
      if (!rc) ctx->sv.has_mesh = true;  // on failure cs_destroy below frees what it left
      r->mesh_reused = !rc;
    }
  }
  if (!rc) rc = cs_init_problem(ctx, &r->req.init);
  double dt = 1e30, dtn = 0.0;
  if (!rc) rc = cs_evaluate_timestep(ctx, dt, &dtn);
  dt = dtn;
  if (!rc && r->req.steps > 0) {
    rc = cs_steps(ctx, r->req.steps, dt, &dtn);  // graph replay, one host sync
    dt = dtn;
  }
  double m = 0, e = 0, dv = 0;
  if (!rc) rc = cs_diag(ctx, &m, &e, &dv);
  std::vector<double> U, ent, bx, by, bz;
  if (!rc && sv->keep_state) {
    const Box b(r->req.params.ntp, r->req.params.nr, r->req.params.nghost);
    const size_t S6 = 6 * b.size();
    U.resize(NVAR * S6);
    ent.resize(S6);
    bx.resize(S6);
    by.resize(S6);
    bz.resize(S6);
    rc = cs_state_get(ctx, U.data(), ent.data(), bx.data(), by.data(), bz.data());
  }
  std::string err = (rc && ctx) ? cs_last_error(ctx) : (rc ? "cs_create rejected the parameters" : "");
  if (ctx) cs_destroy(ctx);
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    r->t_done = Clock::now();
    r->status = rc;
    r->err = err;
    r->mass = m;
    r->energy = e;
    r->divb = dv;
    r->dt_last = dt;
    r->U.swap(U);
    r->ent.swap(ent);
    r->bx.swap(bx);
    r->by.swap(by);
    r->bz.swap(bz);
    const Box b(r->req.params.ntp, r->req.params.nr, r->req.params.nghost);
    r->zone_updates = rc ? 0 : 6LL * b.N * b.N * b.nr * r->req.steps;
    if (!rc) {
      sv->latencies.push_back(std::chrono::duration<double>(r->t_done - r->t_submit).count());
      sv->zone_updates += r->zone_updates;
      sv->t_last_done = r->t_done;
    }
    sv->reserved -= r->bytes;
    sv->active -= 1;
  }
  sv->cv.notify_all();
}

// Device bytes a request needs beyond what is reserved already: its own
// state, plus its mesh unless that is cached (or being built).
size_t admission_bytes(cs_server* sv, const Request& r) {
  return r.bytes + (sv->meshes.count(r.mesh) ? 0 : mesh_device_bytes(r.req.params));
}

// Frees cached meshes that no running solve uses, oldest key first, until
// `need` more bytes fit in the budget; returns whether they do.
bool make_room(cs_server* sv, size_t need) {
  for (auto it = sv->meshes.begin(); sv->reserved + need > sv->budget && it != sv->meshes.end();) {
    if (it->second.mesh && it->second.mesh.use_count() == 1) {
      sv->reserved -= it->second.bytes;
      it = sv->meshes.erase(it);
    } else {
      ++it;
    }
  }
  return sv->reserved + need <= sv->budget;
}

// Admission: the oldest pending request starts when a slot is free and its
// estimated device memory (its state, plus its mesh unless the mesh is
// cached) fits in what the running requests and the cached meshes leave of
// the budget; idle cached meshes are freed to make room.  A request larger
// than the whole budget fails at once.
void scheduler(cs_server* sv) {
  cudaSetDevice(sv->device);
  std::unique_lock<std::mutex> lk(sv->mu);
  while (true) {
    sv->cv.wait(lk, [&] {
      if (sv->stop) return true;
      if (sv->pending.empty() || sv->active >= sv->max_active) return false;
      const Request& r = sv->reqs[sv->pending.front()];
      const size_t need = admission_bytes(sv, r);
      return r.bytes + mesh_device_bytes(r.req.params) > sv->budget || make_room(sv, need);
    });
    if (sv->stop) break;
    const int64_t id = sv->pending.front();
    sv->pending.pop_front();
    Request& r = sv->reqs[id];
    if (r.bytes + mesh_device_bytes(r.req.params) > sv->budget) {
      r.status = CS_ERR_NOMEM;
      r.err = "request needs more device memory than the server's budget";
      r.t_start = r.t_done = Clock::now();
      sv->cv.notify_all();
      continue;
    }
    if (!sv->meshes.count(r.mesh)) {
      MeshEntry me;
      me.bytes = mesh_device_bytes(r.req.params);
      sv->reserved += me.bytes;
      sv->meshes[r.mesh] = me;
      r.mesh_builder = true;
    }
    sv->reserved += r.bytes;
    sv->active += 1;
    sv->workers.emplace_back(run_request, sv, id);
  }
}

}  // namespace
}  // namespace cs

extern "C" {

size_t cs_estimate_device_bytes(const cs_params* p) { return p ? cs::estimate_device_bytes(*p) : 0; }

int cs_serve_create(int32_t max_active, double mem_fraction, int32_t keep_state, cs_server** out) {
  if (!out || max_active < 1 || !(mem_fraction > 0.0 && mem_fraction <= 1.0)) return CS_ERR_ARG;
  *out = nullptr;
  cs_server* sv = new cs_server();
  size_t fr = 0, tot = 0;
  if (cudaGetDevice(&sv->device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    delete sv;
    return CS_ERR_CUDA;
  }
  sv->budget = (size_t)(mem_fraction * (double)fr);
  sv->max_active = max_active;
  sv->keep_state = keep_state;
  sv->t0 = cs::Clock::now();
  sv->sched = std::thread(cs::scheduler, sv);
  *out = sv;
  return CS_OK;
}

int cs_serve_submit(cs_server* sv, const cs_request* req, int64_t* id) {
  if (!sv || !req || !id || req->steps < 0) return CS_ERR_ARG;
  cs::Request r;
  r.req = *req;
  r.t_submit = cs::Clock::now();
  r.bytes = cs::state_device_bytes(req->params);
  r.mesh = cs::mesh_key(req->params);
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    r.id = sv->next_id++;
    if (!sv->started) {
      sv->started = true;
      sv->t0 = r.t_submit;
    }
    *id = r.id;
    sv->reqs[r.id] = std::move(r);
    sv->pending.push_back(*id);
  }
  sv->cv.notify_all();
  return CS_OK;
}

int cs_serve_wait(cs_server* sv, int64_t id, cs_serve_result* out) {
  if (!sv || !out) return CS_ERR_ARG;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(id);
  if (it == sv->reqs.end()) return CS_ERR_ARG;
  sv->cv.wait(lk, [&] { return it->second.status >= 0; });
  const cs::Request& r = it->second;
  out->status = r.status;
  out->mesh_reused = r.mesh_reused ? 1 : 0;
  out->latency_s = std::chrono::duration<double>(r.t_done - r.t_submit).count();
  out->queue_s = std::chrono::duration<double>(r.t_start - r.t_submit).count();
  out->mass = r.mass;
  out->energy = r.energy;
  out->max_divb = r.divb;
  out->dt_last = r.dt_last;
  out->zone_updates = r.zone_updates;
  return r.status;
}

int cs_serve_state(cs_server* sv, int64_t id, double* U, double* ent, double* bxf, double* byf, double* bzf) {
  if (!sv || !U || !ent || !bxf || !byf || !bzf) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(id);
  if (it == sv->reqs.end() || it->second.status != 0 || it->second.U.empty()) return CS_ERR_STATE;
  const cs::Request& r = it->second;
  std::memcpy(U, r.U.data(), r.U.size() * sizeof(double));
  std::memcpy(ent, r.ent.data(), r.ent.size() * sizeof(double));
  std::memcpy(bxf, r.bx.data(), r.bx.size() * sizeof(double));
  std::memcpy(byf, r.by.data(), r.by.size() * sizeof(double));
  std::memcpy(bzf, r.bz.data(), r.bz.size() * sizeof(double));
  return CS_OK;
}

int cs_serve_stats(cs_server* sv, double* p50_s, double* p99_s, double* zone_updates_per_s, int64_t* completed) {
  if (!sv || !p50_s || !p99_s || !zone_updates_per_s || !completed) return CS_ERR_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  std::vector<double> l = sv->latencies;
  std::sort(l.begin(), l.end());
  auto pct = [&](double q) {
    if (l.empty()) return 0.0;
    size_t k = (size_t)std::ceil(q * (double)l.size());
    if (k < 1) k = 1;
    return l[std::min(k, l.size()) - 1];
  };
  *p50_s = pct(0.50);
  *p99_s = pct(0.99);
  const double wall = l.empty() ? 0.0 : std::chrono::duration<double>(sv->t_last_done - sv->t0).count();
  *zone_updates_per_s = wall > 0 ? (double)sv->zone_updates / wall : 0.0;
  *completed = (int64_t)l.size();
  return CS_OK;
}

int cs_serve_destroy(cs_server* sv) {
  if (!sv) return CS_OK;
  {
    std::unique_lock<std::mutex> lk(sv->mu);
    sv->cv.wait(lk, [&] { return sv->pending.empty() && sv->active == 0; });
    sv->stop = true;
  }
  sv->cv.notify_all();
  sv->sched.join();
  for (auto& t : sv->workers) t.join();
  delete sv;
  return CS_OK;
}

}  // extern "C"
