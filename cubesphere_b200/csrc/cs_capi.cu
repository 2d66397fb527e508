// C ABI of the B200 stage update (include/cubesphere_b200.h): context
// lifecycle, mesh build and upload, ghost-exchange map construction, state
// transfer, the stage / step sequence and the per-routine entry points.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>


#include "cs_solve.h"

namespace cs {
int fail(Solve& sv, int code, const std::string& msg) {
  sv.err = msg;
  return code;
}

int cuda_fail(Solve& sv, cudaError_t e, const char* what) {
  return fail(sv, CS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// FP64 <-> FP32 copies of the precision form's state at the FP64 boundary.
__global__ void k_narrow(const double* __restrict__ in, float* __restrict__ out, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    out[t] = (float)in[t];
}
__global__ void k_widen(const float* __restrict__ in, double* __restrict__ out, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    out[t] = (double)in[t];
}

namespace {

const int kNbr[6][4] = {{3, 6, 2, 5}, {1, 4, 3, 6}, {2, 5, 1, 4}, {5, 2, 6, 3}, {6, 3, 4, 1}, {4, 1, 5, 2}};

#define CS_CUDA(sv, call)                                   \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cs::cuda_fail(sv, e_, #call); \
  } while (0)

// Stream-ordered pool for the per-solve arrays: allocation and release are
// ordered on the solve's stream and never synchronise the device, so solves
// that start and end while others run (the serving loop, batches) do not
// stall one another.  Freed memory stays in the pool for the next solve and
// goes back to the device when the last solve on it ends.
struct SolvePool {
  std::mutex mu;
  cudaMemPool_t pool = nullptr;
  int live = 0;
};
SolvePool& solve_pool(int dev) {
  static SolvePool pools[64];
  return pools[dev & 63];
}

cudaError_t pool_acquire(Solve& sv) {
  SolvePool& sp = solve_pool(sv.device);
  std::lock_guard<std::mutex> lk(sp.mu);
  if (!sp.pool) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = sv.device;
    cudaError_t e = cudaMemPoolCreate(&sp.pool, &props);
    if (e != cudaSuccess) {
      sp.pool = nullptr;
      return e;
    }
    uint64_t keep = ~0ULL;
    cudaMemPoolSetAttribute(sp.pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  sp.live += 1;
  sv.pool = sp.pool;
  return cudaSuccess;
}

void pool_release(Solve& sv) {
  if (!sv.pool) return;
  SolvePool& sp = solve_pool(sv.device);
  std::lock_guard<std::mutex> lk(sp.mu);
  sp.live -= 1;
  if (sp.live == 0) cudaMemPoolTrimTo(sp.pool, 0);
  sv.pool = nullptr;
}

void* dalloc(Solve& sv, size_t bytes, cudaError_t& e) {
  void* p = nullptr;
  e = cudaMallocFromPoolAsync(&p, bytes, sv.pool, sv.stream);
  if (e != cudaSuccess) return nullptr;
  sv.allocs.push_back(p);
  e = cudaMemsetAsync(p, 0, bytes, sv.stream);
  return p;
}

}  // namespace

void* solve_alloc(Solve& sv, size_t bytes, cudaError_t& e) { return dalloc(sv, bytes, e); }

namespace {

void free_all(Solve& sv) {
  if (sv.stream) cudaStreamSynchronize(sv.stream);
  for (cudaEvent_t e : sv.prof.ev) cudaEventDestroy(e);
  sv.prof.ev.clear();
  sv.prof.name.clear();
  drop_graph(sv);
  for (void* p : sv.allocs) cudaFreeAsync(p, sv.stream);
  sv.allocs.clear();
  if (sv.stream) {
    cudaStreamSynchronize(sv.stream);
    cudaStreamDestroy(sv.stream);
  }
  sv.stream = nullptr;
  pool_release(sv);
  sv.mesh = std::make_shared<MeshRes>();  // drops this solve's share of the mesh
  sv.init_buf = nullptr;
  sv.init_buf_bytes = 0;
  sv.diag_buf = nullptr;
}

// Host construction of the ghost-exchange map.  The strips are visited in
// the order of the reference's fill (x strips of every panel, then y
// strips), a later write to the same destination replaces the earlier
// one, and all sources are read before any destination is written.
struct MapEntry {
  int32_t src, dst;
  uint8_t meta;
};

std::string build_fill_map(const Solve& sv, std::vector<MapEntry>& out) {
  const GeomHost& g = sv.mesh->host;
  const Box& b = g.box;
  const int N = b.N, G = b.G, nr = b.nr;
  const long long S = (long long)b.size();
  const long long S6 = 6 * S;
  if (8 * S6 >= (1LL << 31)) return "solve too large for 32-bit ghost-map offsets";
  std::vector<int32_t> slot[5];
  for (int f = 0; f < 5; ++f) slot[f].assign((size_t)S6, -1);
  std::vector<MapEntry> e;
  std::string err;
  auto off = [&](int p, int i, int j, int k) { return (long long)p * S + (long long)b.idx(i, j, k); };
  // fd / fs: destination / source field (0 U, 1 ent, 2 Bxf, 3 Byf, 4 Bzf).
  auto emit = [&](int fd, int fs, int pd, int i, int j, int k, int ps, int si, int sj, int sk, bool neg, bool avg) {
    const long long d = off(pd, i, j, k), s = off(ps, si, sj, sk);
    const int ncomp = (fd == 0) ? NVAR : 1;
    int32_t& sl = slot[fd][(size_t)d];
    if (sl >= 0 && avg) err = "averaged panel-edge face written twice";
    if (sl < 0) {
      sl = (int32_t)e.size();
      e.resize(e.size() + ncomp);
    }
    for (int c = 0; c < ncomp; ++c) {
      MapEntry& m = e[(size_t)sl + c];
      m.src = (int32_t)(c * S6 + s);
      m.dst = (int32_t)(c * S6 + d);
      m.meta = (uint8_t)(fd | (neg ? 8 : 0) | (avg ? 16 : 0) | (fs << 5));
    }
  };
  auto zone = [&](int pd, int i, int j, int k, int ps, int si, int sj, int sk) {
    emit(0, 0, pd, i, j, k, ps, si, sj, sk, false, false);
    emit(1, 1, pd, i, j, k, ps, si, sj, sk, false, false);
  };
  auto mk = [&](int p, int i, int j) { return g.mask[(size_t)p * S + b.idx(i, j, 0)]; };
  auto xmask = [&](int p, int i, int j) { return mk(p, std::max(i, 1 - G), j) * mk(p, std::min(i + 1, N + G), j); };
  auto ymask = [&](int p, int i, int j) { return mk(p, i, std::max(j, 1 - G)) * mk(p, i, std::min(j + 1, N + G)); };
  // x direction (330fetch_buffers_fill_in_ux.f:220-714 with the index maps of 203:104-163).
  for (int pn = 0; pn < 6; ++pn) {
    const int rt = kNbr[pn][0] - 1, lf = kNbr[pn][1] - 1;
    auto inner = [&](int j, int k) { return j >= 1 && j <= N && k >= 1 && k <= nr; };
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = N + 1; i <= N + G; ++i) zone(pn, i, j, k, rt, j, 2 * N + 1 - i, k);
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = N; i <= N + G; ++i)
          if (xmask(pn, i, j) == 1) emit(2, 3, pn, i, j, k, rt, j, 2 * N - i, k, true, i == N && inner(j, k));
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = -G; j <= N + G; ++j)
        for (int i = N + 1; i <= N + G; ++i) emit(3, 2, pn, i, j, k, rt, j, 2 * N + 1 - i, k, false, false);
    for (int k = -G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = N + 1; i <= N + G; ++i) emit(4, 4, pn, i, j, k, rt, j, 2 * N + 1 - i, k, false, false);
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= 0; ++i) zone(pn, i, j, k, lf, 1 - i, N + 1 - j, k);
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = -G; i <= 0; ++i)
          if (xmask(pn, i, j) == 1) emit(2, 2, pn, i, j, k, lf, -i, N + 1 - j, k, true, i == 0 && inner(j, k));
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = -G; j <= N + G; ++j)
        for (int i = 1 - G; i <= 0; ++i) emit(3, 3, pn, i, j, k, lf, 1 - i, N - j, k, true, false);
    for (int k = -G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= N + G; ++j)
        for (int i = 1 - G; i <= 0; ++i) emit(4, 4, pn, i, j, k, lf, 1 - i, N + 1 - j, k, false, false);
  }
  // y direction (331fetch_buffers_fill_in_uy.f, 332fetch_buffers_fill_in_uy_top.f).
  for (int pn = 0; pn < 6; ++pn) {
    const int up = kNbr[pn][2] - 1, dn = kNbr[pn][3] - 1;
    auto inner = [&](int i, int k) { return i >= 1 && i <= N && k >= 1 && k <= nr; };
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= 0; ++j)
        for (int i = 1 - G; i <= N + G; ++i) zone(pn, i, j, k, dn, N + 1 - i, 1 - j, k);
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = -G; j <= 0; ++j)
        for (int i = 1 - G; i <= N + G; ++i)
          if (ymask(pn, i, j) == 1) emit(3, 3, pn, i, j, k, dn, N + 1 - i, -j, k, true, j == 0 && inner(i, k));
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= 0; ++j)
        for (int i = -G; i <= N + G; ++i) emit(2, 2, pn, i, j, k, dn, N - i, 1 - j, k, true, false);
    for (int k = -G; k <= nr + G; ++k)
      for (int j = 1 - G; j <= 0; ++j)
        for (int i = 1 - G; i <= N + G; ++i) emit(4, 4, pn, i, j, k, dn, N + 1 - i, 1 - j, k, false, false);
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = N + 1; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) zone(pn, i, j, k, up, 2 * N + 1 - j, i, k);
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = N; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i)
          if (ymask(pn, i, j) == 1) emit(3, 2, pn, i, j, k, up, 2 * N - j, i, k, true, j == N && inner(i, k));
    for (int k = 1 - G; k <= nr + G; ++k)
      for (int j = N + 1; j <= N + G; ++j)
        for (int i = -G; i <= N + G; ++i) emit(2, 3, pn, i, j, k, up, 2 * N + 1 - j, i, k, false, false);
    for (int k = -G; k <= nr + G; ++k)
      for (int j = N + 1; j <= N + G; ++j)
        for (int i = 1 - G; i <= N + G; ++i) emit(4, 4, pn, i, j, k, up, 2 * N + 1 - j, i, k, false, false);
  }
  if (!err.empty()) return err;
  // The entries in the order the device applies them: by destination field,
  // then by destination offset (all sources are read before any write, so
  // the order changes no value; it keeps the scatter's writes coalesced).
  // Each (field, point) has one slot, so a scan of the slots gives the order.
  out.clear();
  out.reserve(e.size());
  for (int f = 0; f < 5; ++f)
    for (int c = 0; c < (f == 0 ? NVAR : 1); ++c)
      for (long long d = 0; d < S6; ++d)
        if (slot[f][(size_t)d] >= 0) out.push_back(e[(size_t)slot[f][(size_t)d] + c]);
  return "";
}

}  // namespace
}  // namespace cs

namespace cs {

void mark(Solve& sv, const char* name, bool kernel) {
  if (kernel) ++sv.launches;
  Prof& pf = sv.prof;
  if (!pf.on) return;
  if (pf.n == 0) return;  // no start event: launch outside a profiled sequence
  if ((size_t)pf.n >= pf.ev.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    pf.ev.push_back(e);
    pf.name.push_back(nullptr);
  }
  cudaEventRecord(pf.ev[pf.n], sv.stream);
  pf.name[pf.n] = name;
  ++pf.n;
}

void prof_start(Solve& sv) {
  Prof& pf = sv.prof;
  if (!pf.on || pf.n > 0) return;
  if (pf.ev.empty()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    pf.ev.push_back(e);
    pf.name.push_back(nullptr);
  }
  cudaEventRecord(pf.ev[0], sv.stream);
  pf.n = 1;
}

namespace {

// Adds the recorded intervals to the per-kernel totals (stream must be idle).
void prof_harvest(Solve& sv) {
  Prof& pf = sv.prof;
  for (int i = 1; i < pf.n; ++i) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, pf.ev[i - 1], pf.ev[i]) != cudaSuccess) continue;
    const std::string key = pf.name[i];
    size_t q = 0;
    while (q < pf.keys.size() && pf.keys[q] != key) ++q;
    if (q == pf.keys.size()) {
      pf.keys.push_back(key);
      pf.ms.push_back(0.0);
      pf.count.push_back(0);
    }
    pf.ms[q] += ms;
    pf.count[q] += 1;
  }
  pf.n = 0;
}

// Panel-edge ownership maps.  Faces on panel edges and edges on panel
// boundaries are computed by every panel that holds them (two, or three
// for the radial edges at cube corners); the copies of all panels but the
// lowest-numbered one take that owner's value.  Vertex identity follows the
// ghost-fill index maps: right edge (N, j) ~ right neighbour (j, N), left
// (0, j) ~ (0, N - j), down (i, 0) ~ (N - i, 0), up (i, N) ~ (N, i).
struct SyncMaps {
  std::vector<int32_t> f_dst, f_src;  // face offsets (panel * box + idx)
  std::vector<int8_t> f_ddir, f_sdir;
  std::vector<int32_t> e_dst, e_src;  // edge offsets
  std::vector<int8_t> e_df, e_sf, e_sign;
  std::vector<int32_t> e_cls;  // where each edge's entries start (one or two), then the entry count
};

std::string build_sync_maps(const Solve& sv, SyncMaps& m) {
  const GeomHost& g = sv.mesh->host;
  const Box& b = g.box;
  const int N = b.N, nr = b.nr;
  const long long S = (long long)b.size();
  const int W = N + 1;
  std::vector<int> par((size_t)6 * W * W);
  for (size_t t = 0; t < par.size(); ++t) par[t] = (int)t;
  auto vid = [&](int p, int i, int j) { return (p * W + j) * W + i; };
  auto root = [&](int x) {
    while (par[x] != x) x = par[x] = par[par[x]];
    return x;
  };
  auto unite = [&](int a, int c) {
    a = root(a);
    c = root(c);
    if (a != c) par[std::max(a, c)] = std::min(a, c);
  };
  for (int p = 0; p < 6; ++p) {
    const int rt = kNbr[p][0] - 1, lf = kNbr[p][1] - 1, up = kNbr[p][2] - 1, dn = kNbr[p][3] - 1;
    for (int t = 0; t <= N; ++t) {
      unite(vid(p, N, t), vid(rt, t, N));
      unite(vid(p, 0, t), vid(lf, 0, N - t));
      unite(vid(p, t, 0), vid(dn, N - t, 0));
      unite(vid(p, t, N), vid(up, N, t));
    }
  }
  auto vert = [&](int q, int p, int i, int j) { return g.f[CS_G_VERT][((size_t)q * 6 + p) * S + b.idx(i, j, 0)]; };
  for (int p = 0; p < 6; ++p)
    for (int j = 0; j <= N; ++j)
      for (int i = 0; i <= N; ++i) {
        const int r = root(vid(p, i, j));
        const int rp = r / (W * W), ri = r % W, rj = (r / W) % W;
        double dist = 0.0, mag = 0.0;
        for (int q = 0; q < 3; ++q) {
          dist = std::max(dist, std::fabs(vert(q, p, i, j) - vert(q, rp, ri, rj)));
          mag = std::max(mag, std::fabs(vert(q, p, i, j)));
        }
        if (dist > 1e-9 * mag) return "panel-edge vertex identities do not match the mesh";
      }
  auto off = [&](int p, int i, int j, int k) { return (int32_t)((long long)p * S + (long long)b.idx(i, j, k)); };
  for (int p = 0; p < 6; ++p) {
    const int rt = kNbr[p][0] - 1, lf = kNbr[p][1] - 1, up = kNbr[p][2] - 1, dn = kNbr[p][3] - 1;
    for (int t = 1; t <= N; ++t)
      for (int k = 1; k <= nr; ++k) {
        // (dir, panel, i, j) of this copy, then of the partner copy
        const int c[4][8] = {{0, p, N, t, 1, rt, t, N},
                             {0, p, 0, t, 0, lf, 0, N + 1 - t},
                             {1, p, t, 0, 1, dn, N + 1 - t, 0},
                             {1, p, t, N, 0, up, N, t}};
        for (const auto& e : c) {
          if (e[5] >= e[1]) continue;  // this copy is the owner's
          m.f_ddir.push_back((int8_t)e[0]);
          m.f_dst.push_back(off(e[1], e[2], e[3], k));
          m.f_sdir.push_back((int8_t)e[4]);
          m.f_src.push_back(off(e[5], e[6], e[7], k));
        }
      }
  }
  struct Copy {
    int f, p, i, j, k, a, c;
  };
  std::map<std::tuple<int, int, int>, std::vector<Copy>> cls;
  for (int p = 0; p < 6; ++p) {
    for (int j = 0; j <= N; ++j)
      for (int i = 0; i <= N; ++i) {
        if (!(i == 0 || i == N || j == 0 || j == N)) continue;
        const int r = root(vid(p, i, j));
        for (int k = 1; k <= nr; ++k) cls[std::make_tuple(r, -1, k)].push_back({2, p, i, j, k, r, r});
      }
    for (int k = 0; k <= nr; ++k) {
      for (int i : {0, N})
        for (int j = 1; j <= N; ++j) {
          const int a = root(vid(p, i, j - 1)), c2 = root(vid(p, i, j));
          cls[std::make_tuple(std::min(a, c2), std::max(a, c2), k)].push_back({1, p, i, j, k, a, c2});
        }
      for (int j : {0, N})
        for (int i = 1; i <= N; ++i) {
          const int a = root(vid(p, i - 1, j)), c2 = root(vid(p, i, j));
          cls[std::make_tuple(std::min(a, c2), std::max(a, c2), k)].push_back({0, p, i, j, k, a, c2});
        }
    }
  }
  for (auto& kv : cls) {
    auto& v = kv.second;
    if (v.size() < 2) return "a panel-boundary edge belongs to one panel only";
    std::sort(v.begin(), v.end(), [](const Copy& x, const Copy& y) { return x.p < y.p; });
    const Copy& o = v[0];
    m.e_cls.push_back((int32_t)m.e_dst.size());
    for (size_t q = 1; q < v.size(); ++q) {
      const Copy& x = v[q];
      m.e_df.push_back((int8_t)x.f);
      m.e_dst.push_back(off(x.p, x.i, x.j, x.k));
      m.e_sf.push_back((int8_t)o.f);
      m.e_src.push_back(off(o.p, o.i, o.j, o.k));
      m.e_sign.push_back((int8_t)((x.a == o.a && x.c == o.c) ? 1 : -1));
    }
  }
  m.e_cls.push_back((int32_t)m.e_dst.size());
  return "";
}

bool check_params(const cs_params& p, std::string& why) {
  if (p.ntp < 2 || p.nr < 1) { why = "ntp must be >= 2 and nr >= 1"; return false; }
  if (p.nghost < 3 || p.nghost > p.ntp - 1) { why = "nghost must be in [3, ntp-1]"; return false; }
  if (!(p.gamma > 1.0)) { why = "gamma must be > 1"; return false; }
  if (!(p.rmax > p.rmin) || !(p.rmin > 0.0)) { why = "need 0 < rmin < rmax"; return false; }
  if (p.radial_mesh < 0 || p.radial_mesh > 2) { why = "radial_mesh must be 0, 1 or 2"; return false; }
  if (p.rk_scheme != CS_RK2 && p.rk_scheme != CS_SSPRK3 && p.rk_scheme != CS_IMEX_RK2) {
    why = "rk_scheme must be CS_RK2, CS_SSPRK3 or CS_IMEX_RK2";
    return false;
  }
  if (!(p.smallnum > 0.0) || !(p.rhofloor > 0.0) || !(p.prsfloor > 0.0)) {
    why = "smallnum, rhofloor and prsfloor must be > 0";
    return false;
  }
  if ((p.bc_lower != 2 && p.bc_lower != 0) || (p.bc_upper != 2 && p.bc_upper != 0)) {
    why = "radial boundary codes must be 2 (outflow) or 0 (none)";
    return false;
  }
  if ((p.flags & CS_FLAG_PANEL_AVERAGE) && (p.flags & CS_FLAG_NO_PANEL_SYNC)) {
    why = "CS_FLAG_PANEL_AVERAGE is a rule for the shared copies, which CS_FLAG_NO_PANEL_SYNC leaves alone";
    return false;
  }
  if ((p.flags & CS_FLAG_P2) && (p.flags & CS_FLAG_NO_OP_CACHE)) {
    why = "CS_FLAG_P2 needs the resident stencil operators (not CS_FLAG_NO_OP_CACHE)";
    return false;
  }
  return true;
}

PhysC make_phys(const cs_params& p) {
  PhysC ph;
  const double pi = 4.0 * std::atan(1.0);
  ph.gamma = p.gamma;
  ph.rhofloor = p.rhofloor;
  ph.prsfloor = p.prsfloor;
  ph.smallnum = p.smallnum;
  ph.ob4pi = 1.0 / (4.0 * pi);
  ph.ob8pi = 1.0 / (8.0 * pi);
  ph.fourpi = 4.0 * pi;
  ph.cfl = p.cfl_coef;
  ph.flatten_coef = p.flatten_coef;
  ph.prs_flatten_coef = p.prs_flatten_coef;
  ph.gm = p.gm;
  return ph;
}

int ensure_host_mesh(Solve& sv) {
  if (!sv.mesh->host.f[0].empty()) return CS_OK;
  std::string e = build_geometry(sv.p, sv.mesh->host);
  if (!e.empty()) return fail(sv, CS_ERR_ARG, e);
  return CS_OK;
}

// State and work arrays of the form R (double: the plain form; float: the
// precision form, whose face B, EMFs and operators stay FP64).
template <typename R>
int alloc_state(Solve& sv, DStateT<R>& s) {
  const Dims& d = sv.d;
  const size_t S6 = (size_t)6 * d.S;
  cudaError_t e = cudaSuccess;
  auto A = [&](int ncomp) -> R* { return (R*)dalloc(sv, (size_t)ncomp * S6 * sizeof(R), e); };
  auto D = [&](int ncomp) -> double* { return (double*)dalloc(sv, (size_t)ncomp * S6 * sizeof(double), e); };
  s.U = A(NVAR); s.ent = A(4); s.Bxf = D(1); s.Byf = D(1); s.Bzf = D(1);
  s.V = A(NVAR * NMODE); s.E = A(3 * NMODE); s.Esnap = A(3);
  s.msonic = A(1); s.flatA = A(1); s.flatB = A(1);
  for (int q = 0; q < 3; ++q) { s.Bq[q] = D(NQ); s.fcon[q] = A(2 * NVAR); s.EF[q] = A(1); s.Ef[q] = D(1); s.B0[q] = D(1); }
  for (int q = 0; q < 6; ++q) s.S[q] = A(1);
  s.dUdt = A(NVAR); s.U0 = A(NVAR); s.ent0 = A(1);
  if (sv.p.rk_scheme == CS_IMEX_RK2) {
    s.K1 = A(NVAR);
    for (int q = 0; q < 3; ++q) { s.EF1[q] = A(1); s.Ef1[q] = D(1); }
    if (!s.K1 || !s.EF1[2] || !s.Ef1[2]) return cuda_fail(sv, e, "cudaMalloc(IMEX stage rates)");
  }
  // resident geometry-only operators of the mesh (null until built)
  const MeshRes& m = *sv.mesh;
  s.op_m9 = (R*)m.op_m9;
  s.op_m10 = (R*)m.op_m10;
  s.lsq_map9 = m.m9_shared ? (const LsqPanelMap*)m.lsq_map : nullptr;
  s.lsq_map10 = m.m10_shared ? (const LsqPanelMap*)m.lsq_map : nullptr;
  s.op_p2v = (R*)m.op_p2v;
  s.op_p2e = (R*)m.op_p2e;
  s.p2_map = m.p2_shared ? (const LsqPanelMap*)m.lsq_map : nullptr;
  s.adp_lu = m.adp_lu;
  s.adp_piv = m.adp_piv;
  s.adp_pmap = m.adp_pmap;
  s.adp_rhs = nullptr;
  if (m.adp_lu) {
    const size_t rsz = m.adp_pmap ? sizeof(R) : sizeof(double);  // panel-shared factors: the state's type
    s.adp_rhs = dalloc(sv, (size_t)adp_range_count(d) * 36 * rsz, e);
    if (!s.adp_rhs) return cuda_fail(sv, e, "cudaMalloc(ADP right-hand sides)");
  }
  s.giveup = (int32_t*)dalloc(sv, S6 * sizeof(int32_t), e);
  if (sv.p.flags & CS_FLAG_STEP10) {
    // STEP 10 keys: 9 min keys all ones (no stage yet), 9 max keys zero
    sv.step10_keys = (unsigned long long*)dalloc(sv, 18 * sizeof(unsigned long long), e);
    if (!sv.step10_keys) return cuda_fail(sv, e, "cudaMalloc(STEP 10 keys)");
    e = cudaMemsetAsync(sv.step10_keys, 0xff, 9 * sizeof(unsigned long long), sv.stream);
    if (e != cudaSuccess) return cuda_fail(sv, e, "cudaMemsetAsync(STEP 10 keys)");
  }
  s.err_flag = (int*)dalloc(sv, 64, e);
  if (!s.err_flag) return cuda_fail(sv, e, "cudaMalloc(error flag)");
  s.dtmin = (unsigned long long*)dalloc(sv, 64, e);
  s.dt = (double*)dalloc(sv, 64, e);
  if (!s.dt) return cuda_fail(sv, e, "cudaMalloc(time step)");
  if (e != cudaSuccess || !s.U || !s.V || !s.E || !s.dtmin) return cuda_fail(sv, e, "cudaMalloc(state)");
  for (int q = 0; q < 3; ++q)
    if (!s.Bq[q] || !s.fcon[q] || !s.EF[q] || !s.Ef[q] || !s.B0[q]) return fail(sv, CS_ERR_NOMEM, "cudaMalloc(work)");
  return CS_OK;
}

// Device allocation owned by a mesh (freed with its last user).
void* mdalloc(Solve& sv, MeshRes& m, size_t bytes, cudaError_t& e) {
  void* p = nullptr;
  e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return nullptr;
  m.allocs.push_back(p);
  m.bytes += bytes;
  e = cudaMemsetAsync(p, 0, bytes, sv.stream);
  return p;
}

// Geometry, mask, stencil, ghost-exchange map and panel-ownership maps of
// a mesh that is not on the device yet.
int mesh_upload(Solve& sv, MeshRes& m) {
  cudaError_t e = cudaSuccess;
  for (int f = 0; f < CS_G_NFIELDS; ++f) {
    const size_t bytes = m.host.f[f].size() * sizeof(double);
    double* p = (double*)mdalloc(sv, m, bytes, e);
    if (!p) return cuda_fail(sv, e, "cudaMalloc(geometry)");
    CS_CUDA(sv, cudaMemcpyAsync(p, m.host.f[f].data(), bytes, cudaMemcpyHostToDevice, sv.stream));
    m.g.f[f] = p;
  }
  int32_t* mk = (int32_t*)mdalloc(sv, m, m.host.mask.size() * sizeof(int32_t), e);
  if (!mk) return cuda_fail(sv, e, "cudaMalloc(mask)");
  CS_CUDA(sv, cudaMemcpyAsync(mk, m.host.mask.data(), m.host.mask.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                              sv.stream));
  m.g.mask = mk;
  int32_t* st = (int32_t*)mdalloc(sv, m, m.host.stencil.size() * sizeof(int32_t), e);
  if (!st) return cuda_fail(sv, e, "cudaMalloc(stencil)");
  CS_CUDA(sv, cudaMemcpyAsync(st, m.host.stencil.data(), m.host.stencil.size() * sizeof(int32_t),
                              cudaMemcpyHostToDevice, sv.stream));
  m.g.st = st;
  // Ghost-exchange map.
  std::vector<MapEntry> map;
  std::string why = build_fill_map(sv, map);
  if (!why.empty()) return fail(sv, CS_ERR_ARG, why);
  const size_t n = map.size();
  std::vector<int32_t> hs(n), hd(n);
  std::vector<uint8_t> hm(n);
  for (size_t t = 0; t < n; ++t) { hs[t] = map[t].src; hd[t] = map[t].dst; hm[t] = map[t].meta; }
  FillMap& f = m.fill;
  f.n = (long long)n;
  f.d_src = (int32_t*)mdalloc(sv, m, n * sizeof(int32_t) + 16, e);
  f.d_dst = (int32_t*)mdalloc(sv, m, n * sizeof(int32_t) + 16, e);
  f.d_meta = (uint8_t*)mdalloc(sv, m, n + 16, e);
  if (!f.d_src || !f.d_dst || !f.d_meta) return cuda_fail(sv, e, "cudaMalloc(ghost map)");
  CS_CUDA(sv, cudaMemcpyAsync(f.d_src, hs.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(f.d_dst, hd.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(f.d_meta, hm.data(), n, cudaMemcpyHostToDevice, sv.stream));
  // panel-edge ownership maps
  if (!(sv.p.flags & CS_FLAG_NO_PANEL_SYNC)) {
    SyncMaps sm;
    why = build_sync_maps(sv, sm);
    if (!why.empty()) return fail(sv, CS_ERR_ARG, why);
    PanelSync& ps = m.psync;
    ps.nf = (long long)sm.f_dst.size();
    ps.ne = (long long)sm.e_dst.size();
    ps.ncls = (long long)sm.e_cls.size() - 1;
    auto up32 = [&](const std::vector<int32_t>& v, int32_t*& dptr) -> cudaError_t {
      dptr = (int32_t*)mdalloc(sv, m, v.size() * sizeof(int32_t) + 16, e);
      if (!dptr) return e;
      return cudaMemcpyAsync(dptr, v.data(), v.size() * sizeof(int32_t), cudaMemcpyHostToDevice, sv.stream);
    };
    auto up8 = [&](const std::vector<int8_t>& v, int8_t*& dptr) -> cudaError_t {
      dptr = (int8_t*)mdalloc(sv, m, v.size() + 16, e);
      if (!dptr) return e;
      return cudaMemcpyAsync(dptr, v.data(), v.size(), cudaMemcpyHostToDevice, sv.stream);
    };
    CS_CUDA(sv, up32(sm.f_dst, ps.f_dst));
    CS_CUDA(sv, up32(sm.f_src, ps.f_src));
    CS_CUDA(sv, up8(sm.f_ddir, ps.f_ddir));
    CS_CUDA(sv, up8(sm.f_sdir, ps.f_sdir));
    CS_CUDA(sv, up32(sm.e_dst, ps.e_dst));
    CS_CUDA(sv, up32(sm.e_src, ps.e_src));
    CS_CUDA(sv, up8(sm.e_df, ps.e_df));
    CS_CUDA(sv, up8(sm.e_sf, ps.e_sf));
    CS_CUDA(sv, up8(sm.e_sign, ps.e_sign));
    CS_CUDA(sv, up32(sm.e_cls, ps.e_cls));
    CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  }
  return CS_OK;
}

// The rotation of the cube that carries panel 1 onto panel p, as a signed
// permutation x'_a = s_a x_perm(a) with determinant +1, if the vertices of
// the whole box agree with it to 1e-12 of the largest coordinate (the
// reference's sector construction gives this symmetry); and the map it
// induces on the 30 B-mode unknowns of the ADP system, unknown (c, m) =
// 10 c + m with the basis 1, x, y, z, x^2, y^2, z^2, xy, yz, xz (minus their
// moments): panel p's row entry (c, m) is sgn * panel 1's entry src.
// pmap[p][0][v] = u with src(u) = v, pmap[p][1][v] = sgn(u); identity on
// the 6 multipliers.
// The rotation taking panel 1 to panel p, where the vertices show one: a
// signed permutation with coordinate a of panel p = sg[a] x coordinate
// pm[a] of panel 1 at every vertex (to 1e-12 of the largest coordinate).
bool panel_rotations(const GeomHost& h, int pm[6][3], int sg[6][3]) {
  const size_t S = h.box.size();
  const std::vector<double>& V = h.f[CS_G_VERT];
  double vmax = 0.0;
  for (double x : V) vmax = std::max(vmax, std::fabs(x));
  const double tol = 1e-12 * vmax;
  const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  const int psign[6] = {1, -1, -1, 1, 1, -1};
  for (int p = 0; p < 6; ++p) {
    int found = -1;
    for (int pi = 0; pi < 6 && found < 0; ++pi)
      for (int sm = 0; sm < 8 && found < 0; ++sm) {
        const int s3[3] = {(sm & 1) ? -1 : 1, (sm & 2) ? -1 : 1, (sm & 4) ? -1 : 1};
        if (psign[pi] * s3[0] * s3[1] * s3[2] != 1) continue;
        bool ok = true;
        for (int a = 0; a < 3 && ok; ++a) {
          const double* src = V.data() + ((size_t)perms[pi][a] * 6 + 0) * S;
          const double* dst = V.data() + ((size_t)a * 6 + p) * S;
          for (size_t o = 0; o < S; ++o)
            if (std::fabs(s3[a] * src[o] - dst[o]) > tol) {
              ok = false;
              break;
            }
        }
        if (ok) {
          found = pi;
          for (int a = 0; a < 3; ++a) {
            pm[p][a] = perms[pi][a];
            sg[p][a] = s3[a];
          }
        }
      }
    if (found < 0) return false;
  }
  return true;
}

// Mode mm of a 10-mode polynomial (0 the constant, 1-3 x y z, 4-6 xx yy zz,
// 7-9 xy yz xz) on panel p equals sig x mode mu on panel 1 under the
// rotation (pm, sg).
void rotated_mode(const int* pm, const int* sg, int mm, int& mu, int& sig) {
  auto pair_mode = [](int a, int b) {
    const int lo = std::min(a, b), hi = std::max(a, b);
    return lo == 0 ? (hi == 1 ? 7 : 9) : 8;  // xy 7, yz 8, xz 9
  };
  mu = 0;
  sig = 1;
  if (mm >= 1 && mm <= 3) {
    mu = 1 + pm[mm - 1];
    sig = sg[mm - 1];
  } else if (mm >= 4 && mm <= 6) {
    mu = 4 + pm[mm - 4];
  } else if (mm >= 7) {
    const int a = mm == 8 ? 1 : 0, b = mm == 7 ? 1 : 2;
    mu = pair_mode(pm[a], pm[b]);
    sig = sg[a] * sg[b];
  }
}

// Per panel: the map of the 36 ADP unknowns (30 B modes, 6 multipliers) to
// panel 1's, with signs.  False where the panels are not rotations of
// panel 1.
bool adp_panel_maps(const GeomHost& h, int8_t* pmap) {
  int pm[6][3], sg[6][3];
  if (!panel_rotations(h, pm, sg)) return false;
  for (int p = 0; p < 6; ++p) {
    int8_t* um = pmap + p * 72;
    int8_t* sgm = um + 36;
    for (int c = 0; c < 3; ++c)
      for (int mm = 0; mm < 10; ++mm) {
        int mu, sig;
        rotated_mode(pm[p], sg[p], mm, mu, sig);
        const int u = c * 10 + mm, v = pm[p][c] * 10 + mu;
        um[v] = (int8_t)u;
        sgm[v] = (int8_t)(sg[p][c] * sig);
      }
    for (int v = 30; v < 36; ++v) {
      um[v] = (int8_t)v;
      sgm[v] = 1;
    }
  }
  return true;
}

// Per panel: which of panel 1's least-squares modes (and sign) each mode
// reads.  Besides the rotation, the rows need the same neighbours in the
// same order: every panel's stencil table and mask must equal panel 1's.
bool lsq_panel_maps(const GeomHost& h, LsqPanelMap* q) {
  int pm[6][3], sg[6][3];
  if (!panel_rotations(h, pm, sg)) return false;
  const size_t ns = h.stencil.size() / 6, nm = h.mask.size() / 6;
  for (int p = 1; p < 6; ++p) {
    if (!std::equal(h.stencil.begin() + p * ns, h.stencil.begin() + (p + 1) * ns, h.stencil.begin())) return false;
    if (!std::equal(h.mask.begin() + p * nm, h.mask.begin() + (p + 1) * nm, h.mask.begin())) return false;
  }
  for (int p = 0; p < 6; ++p) {
    q[p].src = 0;
    q[p].neg = 0;
    q[p].pad = 0;
    for (int mm = 0; mm < 10; ++mm) {
      int mu, sig;
      rotated_mode(pm[p], sg[p], mm, mu, sig);
      q[p].src |= (unsigned long long)mu << (4 * mm);
      if (sig < 0) q[p].neg |= 1u << mm;
    }
  }
  return true;
}

// Resident geometry-only operators of a new mesh, where the device has room
// for them after the first solve's state, computed by that solve's stream.
template <typename R>
int mesh_operators(Solve& sv, MeshRes& m, DStateT<R>& s) {
  const Dims& d = sv.d;
  const size_t S6 = (size_t)6 * d.S;
  cudaError_t e = cudaSuccess;
  // ADP: the KKT matrix of every zone depends on the geometry only, so its
  // factors are computed once here and each stage only substitutes.  They
  // take 10.4 KB per zone per panel (1.7 KB shared by the panels); without
  // room for them (or with CS_FLAG_NO_ADP_CACHE) every stage assembles and
  // factors in place.  The least-squares solution operators of STEPS
  // 7.b / 9.c are geometry-only as well: the row weights Minv A_row^T
  // (2.8 KB per zone in FP64 per panel, 1.55 KB with STEP 9.c's shared).
  if (!(sv.p.flags & CS_FLAG_NO_OP_CACHE)) {
    // Panel-shared row weights where the mesh allows: STEP 9.c's always,
    // STEP 7.b's in the precision form only (the FP64 k_weno7b, at its
    // register limit, measured slower with them).
    LsqPanelMap qmap[6];
    const bool shared = !(sv.p.flags & CS_FLAG_LSQ_PER_PANEL) && lsq_panel_maps(m.host, qmap);
    m.m10_shared = shared;
    m.m9_shared = shared && sizeof(R) == 4;
    const long long nl = lsq_range_count(d);
    const long long n9 = m.m9_shared ? nl / 6 : nl, n10 = m.m10_shared ? nl / 6 : nl;
    size_t fr = 0, tot = 0;
    const size_t bytes = (size_t)(m9_stride(n9) * 162 + n10 * 190) * sizeof(R);
    // room left after them as for the ADP factors below
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess && bytes + (size_t)8 * S6 + ((size_t)2 << 30) < fr) {
      m.op_m9 = mdalloc(sv, m, (size_t)m9_stride(n9) * 162 * sizeof(R), e);
      m.op_m10 = m.op_m9 ? mdalloc(sv, m, (size_t)n10 * 190 * sizeof(R), e) : nullptr;
      if (!m.op_m9 || !m.op_m10) return cuda_fail(sv, e, "cudaMalloc(least-squares operators)");
      if (shared) {
        m.lsq_map = mdalloc(sv, m, sizeof qmap, e);
        if (!m.lsq_map) return cuda_fail(sv, e, "cudaMalloc(least-squares panel maps)");
        CS_CUDA(sv, cudaMemcpyAsync(m.lsq_map, qmap, sizeof qmap, cudaMemcpyHostToDevice, sv.stream));
        CS_CUDA(sv, cudaStreamSynchronize(sv.stream));  // qmap is a stack array
      }
    }
    // CS_FLAG_P2: the inverses of the eight one-sided stencils of STEPS 7.a
    // (9 x 9) and 9.b (10 x 10) of every zone, with the same panel maps as
    // the row weights.  P2 has no in-stage rebuild, so no room is an error.
    if (sv.p.flags & CS_FLAG_P2) {
      if (!m.op_m10) return fail(sv, CS_ERR_NOMEM, "no device room for the least-squares operators CS_FLAG_P2 needs");
      m.p2_shared = shared;
      const long long np = shared ? nl / 6 : nl;
      const size_t pb = (size_t)np * (648 + 800) * sizeof(R);
      if (cudaMemGetInfo(&fr, &tot) != cudaSuccess || pb + (size_t)8 * S6 + ((size_t)2 << 30) >= fr)
        return fail(sv, CS_ERR_NOMEM, "no device room for the CS_FLAG_P2 stencil inverses");
      m.op_p2v = mdalloc(sv, m, (size_t)np * 648 * sizeof(R), e);
      m.op_p2e = m.op_p2v ? mdalloc(sv, m, (size_t)np * 800 * sizeof(R), e) : nullptr;
      if (!m.op_p2v || !m.op_p2e) return cuda_fail(sv, e, "cudaMalloc(P2 stencil inverses)");
    }
  }
  if (!(sv.p.flags & CS_FLAG_NO_ADP_CACHE)) {
    int8_t pmap[6 * 72];
    const bool shared = !(sv.p.flags & CS_FLAG_ADP_PER_PANEL) && adp_panel_maps(m.host, pmap);
    // panel-shared factors and right-hand sides in the state's type (the
    // precision form substitutes in FP32), per-panel ones in FP64
    const size_t esz = shared ? sizeof(R) : sizeof(double);
    const long long nf = adp_factor_doubles(d, shared);
    const size_t lu_bytes = (size_t)nf * esz, pv_bytes = (size_t)nf / 36;
    const size_t rhs_bytes = (size_t)adp_range_count(d) * 36 * esz;
    size_t fr = 0, tot = 0;
    // room left after them and their right-hand sides: the FP32 form's state
    // staging (one FP64 word per point, cs_state_put / cs_state_get) and 2 GB
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess &&
        lu_bytes + pv_bytes + rhs_bytes + (size_t)8 * S6 + ((size_t)2 << 30) < fr) {
      m.adp_lu = mdalloc(sv, m, lu_bytes, e);
      m.adp_piv = m.adp_lu ? (int8_t*)mdalloc(sv, m, pv_bytes, e) : nullptr;
      s.adp_rhs = m.adp_piv ? dalloc(sv, (size_t)adp_range_count(d) * 36 * esz, e) : nullptr;
      if (!m.adp_lu || !m.adp_piv || !s.adp_rhs) return cuda_fail(sv, e, "cudaMalloc(ADP factors)");
      if (shared) {
        m.adp_pmap = (int8_t*)mdalloc(sv, m, sizeof pmap, e);
        if (!m.adp_pmap) return cuda_fail(sv, e, "cudaMalloc(ADP panel maps)");
        CS_CUDA(sv, cudaMemcpyAsync(m.adp_pmap, pmap, sizeof pmap, cudaMemcpyHostToDevice, sv.stream));
        CS_CUDA(sv, cudaStreamSynchronize(sv.stream));  // pmap is a stack array
      }
    }
  }
  s.adp_pmap = m.adp_pmap;
  s.op_m9 = (R*)m.op_m9;
  s.op_m10 = (R*)m.op_m10;
  s.lsq_map9 = m.m9_shared ? (const LsqPanelMap*)m.lsq_map : nullptr;
  s.lsq_map10 = m.m10_shared ? (const LsqPanelMap*)m.lsq_map : nullptr;
  s.op_p2v = (R*)m.op_p2v;
  s.op_p2e = (R*)m.op_p2e;
  s.p2_map = m.p2_shared ? (const LsqPanelMap*)m.lsq_map : nullptr;
  s.adp_lu = m.adp_lu;
  s.adp_piv = m.adp_piv;
  launch_ops_build(sv);
  if (m.adp_lu) launch_adp_factor(sv);
  CS_CUDA(sv, cudaGetLastError());
  return CS_OK;
}

}  // namespace

std::string mesh_key(const cs_params& p) {
  char b[320];
  std::snprintf(b, sizeof b, "%d/%d/%d/%d/%.17g/%.17g/%.17g/%.17g/%d", p.ntp, p.nr, p.nghost, p.radial_mesh, p.rmin,
                p.rmax, p.radial_ratio, p.smallnum,
                p.flags & (CS_FLAG_NO_ADP_CACHE | CS_FLAG_NO_OP_CACHE | CS_FLAG_NO_PANEL_SYNC | CS_FLAG_FP32 |
                           CS_FLAG_ADP_PER_PANEL | CS_FLAG_LSQ_PER_PANEL | CS_FLAG_P2));
  return b;
}

int mesh_attach(Solve& sv, const std::shared_ptr<MeshRes>& mp) {
  sv.mesh = mp;
  MeshRes& m = *mp;
  if (m.host.f[0].empty()) {
    std::string why = build_geometry(sv.p, m.host);
    if (!why.empty()) return fail(sv, CS_ERR_ARG, why);
  }
  const Box& b = m.host.box;
  Dims& d = sv.d;
  d.N = b.N; d.nr = b.nr; d.G = b.G; d.NI = b.NI; d.NJ = b.NJ; d.NK = b.NK;
  d.S = (long long)b.size();
  CS_CUDA(sv, cudaGetDevice(&sv.device));
  CS_CUDA(sv, cudaDeviceGetAttribute(&sv.sm_count, cudaDevAttrMultiProcessorCount, sv.device));
  CS_CUDA(sv, cudaStreamCreateWithFlags(&sv.stream, cudaStreamNonBlocking));
  CS_CUDA(sv, pool_acquire(sv));
  set_adp_smem_limits();
  const bool fresh = !m.on_device;
  if (fresh)
    if (int rc = mesh_upload(sv, m)) return rc;
  sv.g = m.g;
  sv.psync = m.psync;
  sv.fill = m.fill;
  cudaError_t e = cudaSuccess;
  sv.fill.d_tmp = (double*)dalloc(sv, (size_t)sv.fill.n * sizeof(double) + 16, e);
  if (!sv.fill.d_tmp) return cuda_fail(sv, e, "cudaMalloc(ghost staging)");
  // State and work arrays.
  sv.fp32 = (sv.p.flags & CS_FLAG_FP32) != 0;
  if (int rc = sv.fp32 ? alloc_state(sv, sv.stF) : alloc_state(sv, sv.st)) return rc;
  if (fresh)
    if (int rc = sv.fp32 ? mesh_operators(sv, m, sv.stF) : mesh_operators(sv, m, sv.st)) return rc;
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  m.on_device = true;
  return CS_OK;
}

namespace {

int launch_check(Solve& sv, const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(sv, e, what);
  return CS_OK;
}

int need(Solve& sv, bool state) {
  if (!sv.has_mesh) return fail(sv, CS_ERR_STATE, "cs_mesh_build has not run");
  if (state && !sv.has_state) return fail(sv, CS_ERR_STATE, "no state: call cs_init_problem or cs_state_put");
  return CS_OK;
}

void limit_all(Solve& sv) {
  launch_prim_and_masks(sv);
  launch_flattener(sv);
  launch_weno(sv);
  launch_positivity(sv);
  launch_faceB_adp(sv);
  launch_step10(sv);
  launch_efield(sv);
}

// The state with the first stage's rates in place of the current ones.
template <typename R>
DStateT<R> first_stage_rates(const DStateT<R>& st) {
  DStateT<R> s1 = st;
  s1.dUdt = st.K1;
  for (int q = 0; q < 3; ++q) {
    s1.EF[q] = st.EF1[q];
    s1.Ef[q] = st.Ef1[q];
  }
  return s1;
}

// IMEX-RK2: ARS(2,2,2) (Ascher, Ruuth & Spiteri 1997) with the fluxes, the
// entropy transport and CT explicit and the point-mass gravity implicit,
// gamma = 1 - 1/sqrt(2), delta = 1 - 1/(2 gamma):
//   stage 1: U* = U^n + gamma dt F(U^n);          U2 = U* + gamma dt S(U2)
//   stage 2: U* = U^n + delta dt F(U^n) + (1-delta) dt F(U2) + (1-gamma) dt S(U2)
//            U^{n+1} = U* + gamma dt S(U^{n+1})
// with face B and the entropy advanced by the same explicit weights.
int run_stage_imex(Solve& sv, int irk) {
  const double gam = 1.0 - 1.0 / std::sqrt(2.0), del = 1.0 - 1.0 / (2.0 * gam);
  prof_start(sv);
  launch_fill_ghosts(sv);
  limit_all(sv);
  launch_fluxes(sv);
  launch_edges(sv);
  if (irk == 1) {
    launch_save_stage0(sv);
    launch_save_stage1_rates(sv);
    launch_update(sv, gam);
  } else {
    launch_add_gravity(sv, (1.0 - gam) / (1.0 - del));
    launch_restore_stage0(sv);
    if (sv.fp32)
      launch_update_with(sv, first_stage_rates(sv.stF), del);
    else
      launch_update_with(sv, first_stage_rates(sv.st), del);
    launch_update(sv, 1.0 - del);
  }
  launch_gravity_implicit(sv, gam);
  launch_cleanup(sv);
  return launch_check(sv, "stage launch");
}

// One RK stage of the scheme at the device-resident time step.
int run_stage(Solve& sv, int irk) {
  const int ns = sv.p.rk_scheme == CS_SSPRK3 ? 3 : 2;
  if (irk < 1 || irk > ns) return fail(sv, CS_ERR_ARG, "irk out of range for the RK scheme");
  if (sv.p.rk_scheme == CS_IMEX_RK2) return run_stage_imex(sv, irk);
  double dtmove = 1.0, a0 = 0.0;  // dtmove: fraction of the step
  int kind = 0;
  if (sv.p.rk_scheme == CS_SSPRK3) {
    kind = 1;
    if (irk == 2) { a0 = 0.75; dtmove = 0.25; }
    if (irk == 3) { a0 = 1.0 / 3.0; dtmove = 2.0 / 3.0; }
  } else if (irk == 2) {
    dtmove = 0.5;
  }
  prof_start(sv);
  launch_fill_ghosts(sv);
  limit_all(sv);
  launch_fluxes(sv);
  launch_edges(sv);
  launch_sources(sv);
  if (irk == 1) launch_save_stage0(sv);
  else launch_combine(sv, a0, kind);
  launch_update(sv, dtmove);
  launch_cleanup(sv);
  return launch_check(sv, "stage launch");
}

}  // namespace

// One whole step at the device-resident time step: the stages, then the
// CFL reduction that leaves the next step on the device.
int run_step(Solve& sv) {
  const int ns = sv.p.rk_scheme == CS_SSPRK3 ? 3 : 2;
  for (int irk = 1; irk <= ns; ++irk)
    if (int rc = run_stage(sv, irk)) return rc;
  prof_start(sv);
  launch_timestep(sv);
  return launch_check(sv, "timestep launch");
}

// The launches of run_step captured once into a CUDA graph on the solve's
// stream (its buffers never move), so that a run of steps is one graph
// launch per step and one host synchronisation at the end.
int step_graph(Solve& sv) {
  if (sv.graph_exec) return CS_OK;
  const long long l0 = sv.launches;
  cudaGraph_t g = nullptr;
  CS_CUDA(sv, cudaStreamBeginCapture(sv.stream, cudaStreamCaptureModeThreadLocal));
  const int rc = run_step(sv);
  const cudaError_t e = cudaStreamEndCapture(sv.stream, &g);
  sv.graph_kernels = sv.launches - l0;
  sv.launches = l0;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(sv, e, "cudaStreamEndCapture(step)");
  const cudaError_t ei = cudaGraphInstantiate(&sv.graph_exec, g, 0);
  if (ei != cudaSuccess) {
    cudaGraphDestroy(g);
    sv.graph_exec = nullptr;
    return cuda_fail(sv, ei, "cudaGraphInstantiate(step)");
  }
  sv.graph = g;
  return CS_OK;
}

void drop_graph(Solve& sv) {
  if (sv.graph_exec) cudaGraphExecDestroy(sv.graph_exec);
  if (sv.graph) cudaGraphDestroy(sv.graph);
  sv.graph_exec = nullptr;
  sv.graph = nullptr;
}

int read_dt(Solve& sv, double* out) {
  unsigned long long bits = 0;
  int flag = 0;
  const unsigned long long* dtmin = sv.fp32 ? sv.stF.dtmin : sv.st.dtmin;
  const int* err_flag = sv.fp32 ? sv.stF.err_flag : sv.st.err_flag;
  CS_CUDA(sv, cudaMemcpyAsync(&bits, dtmin, sizeof(bits), cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(&flag, err_flag, sizeof(flag), cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  if (flag) return fail(sv, CS_ERR_CUDA, "a bounded device wait gave up (bulk copy did not complete)");
  if (sv.prof.on) prof_harvest(sv);
  std::memcpy(out, &bits, sizeof(bits));
  return CS_OK;
}

namespace {

// Device-to-host copy of one debug array; arrays of the state's type R
// are widened to double on the host.
template <typename R>
cudaError_t debug_copy(Solve& sv, const DStateT<R>& s, int which, size_t nc, double* host_out) {
  const size_t S6 = (size_t)6 * sv.d.S;
  std::vector<R> tmp;
  auto cp = [&](double* dst, const R* src, size_t n) -> cudaError_t {
    tmp.resize(n);
    cudaError_t e = cudaMemcpyAsync(tmp.data(), src, n * sizeof(R), cudaMemcpyDeviceToHost, sv.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sv.stream);
    for (size_t t = 0; e == cudaSuccess && t < n; ++t) dst[t] = (double)tmp[t];
    return e;
  };
  auto cpd = [&](double* dst, const double* src, size_t n) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, sv.stream);
    return e == cudaSuccess ? cudaStreamSynchronize(sv.stream) : e;
  };
  cudaError_t e = cudaSuccess;
  switch (which) {
    case 0: e = cp(host_out, s.V, nc * S6); break;
    case 1: e = cp(host_out, s.ent, nc * S6); break;
    case 2: e = cp(host_out, s.flatA, S6); break;
    case 3: e = cp(host_out, s.dUdt, nc * S6); break;
    case 4: case 5: case 6: e = cpd(host_out, s.Ef[which - 4], S6); break;
    case 7: case 8: case 9: e = cpd(host_out, s.Bq[which - 7], nc * S6); break;
    case 10: e = cp(host_out, s.E, 3 * S6); break;
    case 11:
      for (int q = 0; q < 6 && e == cudaSuccess; ++q) e = cp(host_out + q * S6, s.S[q], S6);
      break;
    case 12:
      for (int q = 0; q < 3 && e == cudaSuccess; ++q) e = cp(host_out + q * S6, s.EF[q], S6);
      break;
    case 13: {
      std::vector<int32_t> flags(S6);
      e = cudaMemcpyAsync(flags.data(), s.giveup, S6 * sizeof(int32_t), cudaMemcpyDeviceToHost, sv.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(sv.stream);
      for (size_t t = 0; e == cudaSuccess && t < S6; ++t) host_out[t] = (double)flags[t];
      break;
    }
  }
  return e;
}

size_t field_ncomp_debug(int which) {
  static const int nc[14] = {NVAR * NMODE, 4, 1, NVAR, 1, 1, 1, NQ, NQ, NQ, 3, 6, 3, 1};
  return (which < 0 || which > 13) ? 0 : (size_t)nc[which];
}

// Known-answer access to the pointwise physics the stage kernels call: one
// thread per case, in the state type R of the form (see cs_pointwise).
template <typename R>
__global__ void k_pointwise(PhysC ph, int kind, int n, const double* in, double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (kind == 0) {
    const double* a = in + (long long)t * 9;
    R V[8], U[8];
    for (int c = 0; c < 8; ++c) V[c] = (R)a[c];
    d_prim_to_cons(ph, (R)a[8], U, V);
    for (int c = 0; c < 8; ++c) out[(long long)t * 8 + c] = (double)U[c];
  } else if (kind == 1) {
    const double* a = in + (long long)t * 9;
    R V[8], U[8];
    for (int c = 0; c < 8; ++c) U[c] = (R)a[c];
    R ent = (R)a[8];
    const int flag = d_cons_to_prim(ph, ent, U, V);
    double* o = out + (long long)t * 18;
    for (int c = 0; c < 8; ++c) o[c] = (double)V[c];
    o[8] = (double)ent;
    o[9] = (double)flag;
    for (int c = 0; c < 8; ++c) o[10 + c] = (double)U[c];
  } else {
    const double* a = in + (long long)t * 18;
    R VL[8], VR[8], FlL[8], FlR[8], FL[8], FR[8], SL, SR, entF;
    for (int c = 0; c < 8; ++c) {
      VL[c] = (R)a[c];
      VR[c] = (R)a[8 + c];
    }
    d_hll(ph, VL, VR, (R)a[16], (R)a[17], FlL, FlR, FL, FR, SL, SR, entF);
    double* o = out + (long long)t * 35;
    for (int c = 0; c < 8; ++c) {
      o[c] = (double)FlL[c];
      o[8 + c] = (double)FlR[c];
      o[16 + c] = (double)FL[c];
      o[24 + c] = (double)FR[c];
    }
    o[32] = (double)SL;
    o[33] = (double)SR;
    o[34] = (double)entF;
  }
}

}  // namespace
}  // namespace cs

using cs::Solve;

extern "C" {

int cs_geom_ncomp(int field) { return cs::geom_ncomp(field); }

int cs_create(const cs_params* p, cs_ctx** out) {
  if (!p || !out) return CS_ERR_ARG;
  *out = nullptr;
  cs_ctx* c = new (std::nothrow) cs_ctx();
  if (!c) return CS_ERR_NOMEM;
  std::string why;
  if (!cs::check_params(*p, why)) {
    delete c;
    return CS_ERR_ARG;
  }
  c->sv.p = *p;
  c->sv.ph = cs::make_phys(*p);
  const cs::Box b(p->ntp, p->nr, p->nghost);
  c->sv.d.N = b.N; c->sv.d.nr = b.nr; c->sv.d.G = b.G; c->sv.d.NI = b.NI; c->sv.d.NJ = b.NJ; c->sv.d.NK = b.NK;
  c->sv.d.S = (long long)b.size();
  *out = c;
  return CS_OK;
}

const char* cs_params_check(const cs_params* p) {
  static thread_local std::string why;
  why.clear();
  if (!p) return "null params";
  cs::check_params(*p, why);
  return why.c_str();
}

int cs_destroy(cs_ctx* ctx) {
  if (!ctx) return CS_OK;
  cs::free_all(ctx->sv);
  delete ctx;
  return CS_OK;
}

const char* cs_last_error(const cs_ctx* ctx) { return ctx ? ctx->sv.err.c_str() : "null context"; }

int cs_box_dims(const cs_ctx* ctx, int32_t* ni, int32_t* nj, int32_t* nk) {
  if (!ctx || !ni || !nj || !nk) return CS_ERR_ARG;
  *ni = ctx->sv.d.NI;
  *nj = ctx->sv.d.NJ;
  *nk = ctx->sv.d.NK;
  return CS_OK;
}

int cs_mesh_build_host(cs_ctx* ctx) {
  if (!ctx) return CS_ERR_ARG;
  return cs::ensure_host_mesh(ctx->sv);
}

int cs_mesh_build(cs_ctx* ctx) {
  if (!ctx) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (sv.has_mesh) return cs::fail(sv, CS_ERR_STATE, "mesh already built on this context");
  int rc = cs::ensure_host_mesh(sv);
  if (rc) return rc;
  rc = cs::mesh_attach(sv, sv.mesh);
  if (rc) {
    cs::free_all(sv);
    return rc;
  }
  sv.has_mesh = true;
  return CS_OK;
}

int cs_mesh_share(cs_ctx* ctx, const cs_ctx* from) {
  if (!ctx || !from) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (sv.has_mesh) return cs::fail(sv, CS_ERR_STATE, "mesh already built on this context");
  if (!from->sv.has_mesh) return cs::fail(sv, CS_ERR_STATE, "the source context has no device mesh");
  if (cs::mesh_key(sv.p) != cs::mesh_key(from->sv.p))
    return cs::fail(sv, CS_ERR_ARG, "the two contexts' mesh parameters differ");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != from->sv.device)
    return cs::fail(sv, CS_ERR_ARG, "the source context lives on another device");
  const int rc = cs::mesh_attach(sv, from->sv.mesh);
  if (rc) {
    cs::free_all(sv);
    return rc;
  }
  sv.has_mesh = true;
  return CS_OK;
}

int cs_geometry_get(cs_ctx* ctx, int field, double* host_out, size_t n) {
  if (!ctx || !host_out || field < 0 || field >= CS_G_NFIELDS) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (sv.mesh->host.f[0].empty()) return cs::fail(sv, CS_ERR_STATE, "no mesh: call cs_mesh_build or cs_mesh_build_host");
  const std::vector<double>& v = sv.mesh->host.f[field];
  if (n != v.size()) return cs::fail(sv, CS_ERR_ARG, "geometry buffer size mismatch");
  std::memcpy(host_out, v.data(), n * sizeof(double));
  return CS_OK;
}

int cs_fill_map_get(cs_ctx* ctx, int32_t* src, int32_t* dst, uint8_t* meta, int64_t* n) {
  if (!ctx || !n) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::ensure_host_mesh(sv)) return rc;
  std::vector<cs::MapEntry> map;
  const std::string why = cs::build_fill_map(sv, map);
  if (!why.empty()) return cs::fail(sv, CS_ERR_ARG, why);
  if (src || dst || meta) {
    if (!src || !dst || !meta) return cs::fail(sv, CS_ERR_ARG, "src, dst and meta are all given or all null");
    if (*n != (int64_t)map.size()) return cs::fail(sv, CS_ERR_ARG, "fill map buffer size mismatch");
    for (size_t t = 0; t < map.size(); ++t) {
      src[t] = map[t].src;
      dst[t] = map[t].dst;
      meta[t] = map[t].meta;
    }
  }
  *n = (int64_t)map.size();
  return CS_OK;
}

int cs_sync_map_get(cs_ctx* ctx, int32_t which, int32_t* dst, int32_t* src, int8_t* dst_kind, int8_t* src_kind,
                    int8_t* sign, int64_t* n) {
  if (!ctx || !n || (which != 0 && which != 1)) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::ensure_host_mesh(sv)) return rc;
  cs::SyncMaps m;
  const std::string why = cs::build_sync_maps(sv, m);
  if (!why.empty()) return cs::fail(sv, CS_ERR_ARG, why);
  const size_t cnt = which == 0 ? m.f_dst.size() : m.e_dst.size();
  if (dst || src || dst_kind || src_kind || sign) {
    if (!dst || !src || !dst_kind || !src_kind || !sign)
      return cs::fail(sv, CS_ERR_ARG, "dst, src, dst_kind, src_kind and sign are all given or all null");
    if (*n != (int64_t)cnt) return cs::fail(sv, CS_ERR_ARG, "sync map buffer size mismatch");
    for (size_t t = 0; t < cnt; ++t) {
      dst[t] = which == 0 ? m.f_dst[t] : m.e_dst[t];
      src[t] = which == 0 ? m.f_src[t] : m.e_src[t];
      dst_kind[t] = which == 0 ? m.f_ddir[t] : m.e_df[t];
      src_kind[t] = which == 0 ? m.f_sdir[t] : m.e_sf[t];
      sign[t] = which == 0 ? (int8_t)-1 : m.e_sign[t];
    }
  }
  *n = (int64_t)cnt;
  return CS_OK;
}

int cs_mask_get(cs_ctx* ctx, int32_t* host_out, size_t n) {
  if (!ctx || !host_out) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (sv.mesh->host.mask.empty()) return cs::fail(sv, CS_ERR_STATE, "no mesh");
  if (n != sv.mesh->host.mask.size()) return cs::fail(sv, CS_ERR_ARG, "mask buffer size mismatch");
  std::memcpy(host_out, sv.mesh->host.mask.data(), n * sizeof(int32_t));
  return CS_OK;
}

int cs_stencil_get(cs_ctx* ctx, int32_t* host_out, size_t n) {
  if (!ctx || !host_out) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (sv.mesh->host.stencil.empty()) return cs::fail(sv, CS_ERR_STATE, "no mesh");
  if (n != sv.mesh->host.stencil.size()) return cs::fail(sv, CS_ERR_ARG, "stencil buffer size mismatch");
  std::memcpy(host_out, sv.mesh->host.stencil.data(), n * sizeof(int32_t));
  return CS_OK;
}

int cs_geometry_single_zone(int32_t isector, int32_t ntp_global, int32_t nr_global, int32_t iscale, double rmin,
                            double rmax, int32_t radial_mesh, int32_t field, double* host_out, size_t n) {
  if (!host_out || field < 0 || field >= CS_G_NFIELDS || isector < 1 || isector > 6 || iscale < 1 ||
      ntp_global < 1 || nr_global < 1 || ntp_global % iscale || nr_global % iscale)
    return CS_ERR_ARG;
  cs::GeomHost g;
  std::string e = cs::build_geometry_single_zone(isector, ntp_global, nr_global, iscale, rmin, rmax, radial_mesh, g);
  if (!e.empty()) return CS_ERR_ARG;
  const std::vector<double>& v = g.f[field];
  if (n != v.size()) return CS_ERR_ARG;
  std::memcpy(host_out, v.data(), n * sizeof(double));
  return CS_OK;
}

int cs_init_problem_host(cs_ctx* ctx, const cs_init_desc* d, double* U, double* ent, double* bxf, double* byf,
                         double* bzf) {
  if (!ctx || !d || !U || !ent || !bxf || !byf || !bzf) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  int rc = cs::ensure_host_mesh(sv);
  if (rc) return rc;
  std::string e = cs::init_problem_host(sv.p, *d, sv.mesh->host, U, ent, bxf, byf, bzf);
  if (!e.empty()) return cs::fail(sv, CS_ERR_ARG, e);
  return CS_OK;
}

int cs_state_put(cs_ctx* ctx, const double* U, const double* ent, const double* bxf, const double* byf,
                 const double* bzf) {
  if (!ctx || !U || !ent || !bxf || !byf || !bzf) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, false)) return rc;
  const size_t S6 = (size_t)6 * sv.d.S;
  if (sv.fp32) {
    // The precision form keeps U and the entropy in FP32 on the device: the
    // FP64 host values go through a stream-ordered staging buffer of one
    // component and are rounded on the device, component by component.
    double* stage = nullptr;
    CS_CUDA(sv, cudaMallocFromPoolAsync((void**)&stage, S6 * sizeof(double), sv.pool, sv.stream));
    for (int c = 0; c <= cs::NVAR; ++c) {
      const double* src = c < cs::NVAR ? U + (size_t)c * S6 : ent;
      float* dst = c < cs::NVAR ? sv.stF.U + (size_t)c * S6 : sv.stF.ent;
      CS_CUDA(sv, cudaMemcpyAsync(stage, src, S6 * sizeof(double), cudaMemcpyHostToDevice, sv.stream));
      cs::k_narrow<<<cs::blocks_for((long long)S6, 256, sv.sm_count), 256, 0, sv.stream>>>(stage, dst, (long long)S6);
    }
    CS_CUDA(sv, cudaGetLastError());
    CS_CUDA(sv, cudaFreeAsync(stage, sv.stream));
    CS_CUDA(sv, cudaMemcpyAsync(sv.stF.Bxf, bxf, S6 * sizeof(double), cudaMemcpyHostToDevice, sv.stream));
    CS_CUDA(sv, cudaMemcpyAsync(sv.stF.Byf, byf, S6 * sizeof(double), cudaMemcpyHostToDevice, sv.stream));
    CS_CUDA(sv, cudaMemcpyAsync(sv.stF.Bzf, bzf, S6 * sizeof(double), cudaMemcpyHostToDevice, sv.stream));
    CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
    sv.has_state = true;
    return CS_OK;
  }
  const size_t B = S6 * sizeof(double);
  CS_CUDA(sv, cudaMemcpyAsync(sv.st.U, U, cs::NVAR * B, cudaMemcpyHostToDevice, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(sv.st.ent, ent, B, cudaMemcpyHostToDevice, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(sv.st.Bxf, bxf, B, cudaMemcpyHostToDevice, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(sv.st.Byf, byf, B, cudaMemcpyHostToDevice, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(sv.st.Bzf, bzf, B, cudaMemcpyHostToDevice, sv.stream));
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  sv.has_state = true;
  return CS_OK;
}

int cs_state_get(cs_ctx* ctx, double* U, double* ent, double* bxf, double* byf, double* bzf) {
  if (!ctx || !U || !ent || !bxf || !byf || !bzf) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  const size_t S6 = (size_t)6 * sv.d.S;
  if (sv.fp32) {
    // widened to FP64 on the device, component by component, through a
    // stream-ordered staging buffer of one component
    double* stage = nullptr;
    CS_CUDA(sv, cudaMallocFromPoolAsync((void**)&stage, S6 * sizeof(double), sv.pool, sv.stream));
    for (int c = 0; c <= cs::NVAR; ++c) {
      const float* src = c < cs::NVAR ? sv.stF.U + (size_t)c * S6 : sv.stF.ent;
      double* dst = c < cs::NVAR ? U + (size_t)c * S6 : ent;
      cs::k_widen<<<cs::blocks_for((long long)S6, 256, sv.sm_count), 256, 0, sv.stream>>>(src, stage, (long long)S6);
      CS_CUDA(sv, cudaMemcpyAsync(dst, stage, S6 * sizeof(double), cudaMemcpyDeviceToHost, sv.stream));
    }
    CS_CUDA(sv, cudaGetLastError());
    CS_CUDA(sv, cudaFreeAsync(stage, sv.stream));
    CS_CUDA(sv, cudaMemcpyAsync(bxf, sv.stF.Bxf, S6 * sizeof(double), cudaMemcpyDeviceToHost, sv.stream));
    CS_CUDA(sv, cudaMemcpyAsync(byf, sv.stF.Byf, S6 * sizeof(double), cudaMemcpyDeviceToHost, sv.stream));
    CS_CUDA(sv, cudaMemcpyAsync(bzf, sv.stF.Bzf, S6 * sizeof(double), cudaMemcpyDeviceToHost, sv.stream));
    CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
    return CS_OK;
  }
  const size_t B = S6 * sizeof(double);
  CS_CUDA(sv, cudaMemcpyAsync(U, sv.st.U, cs::NVAR * B, cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(ent, sv.st.ent, B, cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(bxf, sv.st.Bxf, B, cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(byf, sv.st.Byf, B, cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaMemcpyAsync(bzf, sv.st.Bzf, B, cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  return CS_OK;
}

int cs_init_problem(cs_ctx* ctx, const cs_init_desc* d) {
  if (!ctx || !d) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, false)) return rc;
  if (int rc = cs::init_problem_device(sv, *d)) return rc;
  sv.has_state = true;
  return CS_OK;
}

int cs_stage(cs_ctx* ctx, int32_t irk, double dtcur) {
  if (!ctx) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  if (!(dtcur > 0.0)) return cs::fail(sv, CS_ERR_ARG, "dtcur must be > 0");
  cs::launch_set_dt(sv, dtcur);
  return cs::run_stage(sv, irk);
}

int cs_evaluate_timestep(cs_ctx* ctx, double dtcur, double* dtcurp1) {
  if (!ctx || !dtcurp1) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  if (!(dtcur > 0.0)) return cs::fail(sv, CS_ERR_ARG, "dtcur must be > 0");
  cs::prof_start(sv);
  cs::launch_set_dt(sv, dtcur);
  cs::launch_timestep(sv);
  if (int rc = cs::launch_check(sv, "timestep launch")) return rc;
  return cs::read_dt(sv, dtcurp1);
}

int cs_step(cs_ctx* ctx, double dtcur, double* dtcurp1) {
  if (!ctx || !dtcurp1) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  if (!(dtcur > 0.0)) return cs::fail(sv, CS_ERR_ARG, "dtcur must be > 0");
  cs::launch_set_dt(sv, dtcur);
  if (int rc = cs::run_step(sv)) return rc;
  return cs::read_dt(sv, dtcurp1);
}

int cs_steps(cs_ctx* ctx, int32_t nsteps, double dtcur, double* dtcurp1) {
  if (!ctx || !dtcurp1 || nsteps < 0) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  if (!(dtcur > 0.0)) return cs::fail(sv, CS_ERR_ARG, "dtcur must be > 0");
  if (nsteps == 0) {
    *dtcurp1 = dtcur;
    return CS_OK;
  }
  cs::launch_set_dt(sv, dtcur);
  if (sv.prof.on) {
    // profiled: the same launches one by one, so each can be timed
    for (int n = 0; n < nsteps; ++n)
      if (int rc = cs::run_step(sv)) return rc;
  } else {
    if (int rc = cs::step_graph(sv)) return rc;
    for (int n = 0; n < nsteps; ++n) CS_CUDA(sv, cudaGraphLaunch(sv.graph_exec, sv.stream));
    sv.launches += sv.graph_kernels * nsteps;
  }
  return cs::read_dt(sv, dtcurp1);
}

int cs_synchronize(cs_ctx* ctx) {
  if (!ctx) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (!sv.stream) return CS_OK;
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  if (sv.prof.on) cs::prof_harvest(sv);
  return CS_OK;
}

int cs_get_stream(cs_ctx* ctx, void** stream) {
  if (!ctx || !stream) return CS_ERR_ARG;
  if (int rc = cs::need(ctx->sv, false)) return rc;
  *stream = (void*)ctx->sv.stream;
  return CS_OK;
}

int cs_mesh_device_bytes(cs_ctx* ctx, uint64_t* bytes) {
  if (!ctx || !bytes) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, false)) return rc;
  *bytes = (uint64_t)sv.mesh->bytes;
  return CS_OK;
}

int cs_launch_count(cs_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return CS_ERR_ARG;
  *n = ctx->sv.launches;
  return CS_OK;
}

int cs_profile_begin(cs_ctx* ctx) {
  if (!ctx) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, false)) return rc;
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  sv.prof.keys.clear();
  sv.prof.ms.clear();
  sv.prof.count.clear();
  sv.prof.n = 0;
  sv.prof.on = true;
  return CS_OK;
}

int cs_profile_end(cs_ctx* ctx, int32_t max_kernels, char* names, double* total_ms, int64_t* launches,
                   int32_t* n_kernels) {
  if (!ctx || !names || !total_ms || !launches || !n_kernels || max_kernels < 0) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, false)) return rc;
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  cs::prof_harvest(sv);
  sv.prof.on = false;
  const int n = (int)sv.prof.keys.size();
  *n_kernels = n;
  for (int q = 0; q < n && q < max_kernels; ++q) {
    std::memset(names + 32 * q, 0, 32);
    std::strncpy(names + 32 * q, sv.prof.keys[q].c_str(), 31);
    total_ms[q] = sv.prof.ms[q];
    launches[q] = sv.prof.count[q];
  }
  return n > max_kernels ? cs::fail(sv, CS_ERR_ARG, "more kernels than max_kernels") : CS_OK;
}

#define CS_ROUTINE(name, body)                       \
  int name(cs_ctx* ctx) {                            \
    if (!ctx) return CS_ERR_ARG;                     \
    Solve& sv = ctx->sv;                             \
    if (int rc = cs::need(sv, true)) return rc;      \
    body;                                            \
    return cs::launch_check(sv, #name);              \
  }

CS_ROUTINE(cs_fill_ghosts, cs::launch_fill_ghosts(sv))
CS_ROUTINE(cs_limit_all_slopes_p12, cs::limit_all(sv))
CS_ROUTINE(cs_make_facial_fluxes, cs::launch_fluxes(sv))
CS_ROUTINE(cs_make_edge_efields_p1, cs::launch_edges(sv))
CS_ROUTINE(cs_build_non_stiff_sources, cs::launch_sources(sv))
CS_ROUTINE(cs_cleanup_after_update, cs::launch_cleanup(sv))

int cs_update_imex_rk_step_p1(cs_ctx* ctx, double dtmove) {
  if (!ctx) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  cs::launch_set_dt(sv, dtmove);
  cs::launch_update(sv, 1.0);
  return cs::launch_check(sv, "cs_update_imex_rk_step_p1");
}

int cs_debug_get(cs_ctx* ctx, int32_t which, double* host_out, size_t n) {
  if (!ctx || !host_out) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  const size_t nc = cs::field_ncomp_debug(which);
  const size_t S6 = (size_t)6 * sv.d.S;
  if (nc == 0) return cs::fail(sv, CS_ERR_ARG, "unknown debug array");
  if (n != nc * S6) return cs::fail(sv, CS_ERR_ARG, "debug buffer size mismatch");
  const cudaError_t e = sv.fp32 ? cs::debug_copy(sv, sv.stF, which, nc, host_out)
                                 : cs::debug_copy(sv, sv.st, which, nc, host_out);
  if (e != cudaSuccess) return cs::cuda_fail(sv, e, "cs_debug_get copy");
  return CS_OK;
}

namespace {
// The driver's module zone arrays, U_amr(1-G:N+G, 1-G:N+G, 1-G:nr+G, ncomp,
// patch) and entropygr_amr(1-G:N+G, 1-G:N+G, 1-G:nr+G, patch), Fortran
// column-major: offset of zone (i, j, k), component c, patch p.
struct AmrZones {
  long long ni, nj, nk;
  int G, ncomp;
  AmrZones(const cs::Dims& d, int nc) : ni(d.N + 2 * d.G), nj(d.N + 2 * d.G), nk(d.nr + 2 * d.G), G(d.G), ncomp(nc) {}
  long long off(int c, int p, int i, int j, int k) const {
    return (((long long)p * ncomp + c) * nk + (k + G - 1)) * nj * ni + (long long)(j + G - 1) * ni + (i + G - 1);
  }
  long long off1(int p, int i, int j, int k) const {  // one component per patch
    return ((long long)p * nk + (k + G - 1)) * nj * ni + (long long)(j + G - 1) * ni + (i + G - 1);
  }
};

// Panel-box (U, ent) <-> module-array (U_amr, entropygr_amr) copies of the
// zones 1-G .. N+G; the panel box's extra lower layer (index -G) is zero.
void amr_to_box(const cs::Dims& d, int ncomp, const double* U_amr, const double* ent_amr, double* U, double* ent) {
  const AmrZones a(d, ncomp);
  const long long S = d.S;
#pragma omp parallel for collapse(2) schedule(static)
  for (int p = 0; p < 6; ++p)
    for (int k = -d.G; k <= d.nr + d.G; ++k)
      for (int j = -d.G; j <= d.N + d.G; ++j)
        for (int i = -d.G; i <= d.N + d.G; ++i) {
          const long long o = d.idx(i, j, k);
          const bool in = i > -d.G && j > -d.G && k > -d.G;
          for (int c = 0; c < cs::NVAR; ++c) U[((long long)c * 6 + p) * S + o] = in ? U_amr[a.off(c, p, i, j, k)] : 0.0;
          ent[(long long)p * S + o] = in ? ent_amr[a.off1(p, i, j, k)] : 0.0;
        }
}
void box_to_amr(const cs::Dims& d, int ncomp, const double* U, const double* ent, double* U_amr, double* ent_amr) {
  const AmrZones a(d, ncomp);
  const long long S = d.S;
#pragma omp parallel for collapse(2) schedule(static)
  for (int p = 0; p < 6; ++p)
    for (int k = 1 - d.G; k <= d.nr + d.G; ++k)
      for (int j = 1 - d.G; j <= d.N + d.G; ++j)
        for (int i = 1 - d.G; i <= d.N + d.G; ++i) {
          const long long o = d.idx(i, j, k);
          for (int c = 0; c < cs::NVAR; ++c) U_amr[a.off(c, p, i, j, k)] = U[((long long)c * 6 + p) * S + o];
          ent_amr[a.off1(p, i, j, k)] = ent[(long long)p * S + o];
        }
}
}  // namespace

int cs_state_put_amr(cs_ctx* ctx, int32_t n_cc_components, const double* U_amr, const double* entropygr_amr,
                     const double* Bxf_amr, const double* Byf_amr, const double* Bzf_amr) {
  if (!ctx || !U_amr || !entropygr_amr || !Bxf_amr || !Byf_amr || !Bzf_amr) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (n_cc_components < cs::NVAR) return cs::fail(sv, CS_ERR_ARG, "n_cc_components must be >= 8 (ideal MHD)");
  if (int rc = cs::need(sv, false)) return rc;
  const size_t S6 = (size_t)6 * sv.d.S;
  std::vector<double> U(cs::NVAR * S6), ent(S6);
  amr_to_box(sv.d, n_cc_components, U_amr, entropygr_amr, U.data(), ent.data());
  // the face arrays' box (0-G:N+G)^2 x (0-G:nr+G) per patch is the panel box
  return cs_state_put(ctx, U.data(), ent.data(), Bxf_amr, Byf_amr, Bzf_amr);
}

int cs_state_get_amr(cs_ctx* ctx, int32_t n_cc_components, double* U_amr, double* entropygr_amr, double* Bxf_amr,
                     double* Byf_amr, double* Bzf_amr) {
  if (!ctx || !U_amr || !entropygr_amr || !Bxf_amr || !Byf_amr || !Bzf_amr) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (n_cc_components < cs::NVAR) return cs::fail(sv, CS_ERR_ARG, "n_cc_components must be >= 8 (ideal MHD)");
  if (int rc = cs::need(sv, true)) return rc;
  const size_t S6 = (size_t)6 * sv.d.S;
  std::vector<double> U(cs::NVAR * S6), ent(S6);
  if (int rc = cs_state_get(ctx, U.data(), ent.data(), Bxf_amr, Byf_amr, Bzf_amr)) return rc;
  box_to_amr(sv.d, n_cc_components, U.data(), ent.data(), U_amr, entropygr_amr);
  return CS_OK;
}

int cs_debug_set_wait_error(cs_ctx* ctx, int32_t value) {
  if (!ctx) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, false)) return rc;
  int* flag = sv.fp32 ? sv.stF.err_flag : sv.st.err_flag;
  const int v = value;
  CS_CUDA(sv, cudaMemcpyAsync(flag, &v, sizeof v, cudaMemcpyHostToDevice, sv.stream));
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  return CS_OK;
}

int cs_limit_minmax(cs_ctx* ctx, double* v_min, double* v_max) {
  if (!ctx || !v_min || !v_max) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  if (!sv.step10_keys) return cs::fail(sv, CS_ERR_STATE, "STEP 10 is evaluated only with CS_FLAG_STEP10");
  unsigned long long keys[18];
  CS_CUDA(sv, cudaMemcpyAsync(keys, sv.step10_keys, sizeof keys, cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  if (keys[0] == ~0ULL) return cs::fail(sv, CS_ERR_STATE, "no LIMIT_ALL_SLOPES_P12 has run yet");
  for (int q = 0; q < 18; ++q) {
    const unsigned long long k = keys[q];
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
    double v;
    std::memcpy(&v, &b, sizeof v);
    (q < 9 ? v_min[q] : v_max[q - 9]) = v;
  }
  return CS_OK;
}

int cs_pointwise(const cs_params* p, int32_t kind, int32_t n, const double* in, double* out) {
  if (!p || kind < 0 || kind > 2 || n < 0 || (n > 0 && (!in || !out))) return CS_ERR_ARG;
  std::string why;
  if (!cs::check_params(*p, why)) return CS_ERR_ARG;
  if (n == 0) return CS_OK;
  static const int nin[3] = {9, 9, 18}, nout[3] = {8, 18, 35};
  const size_t bi = (size_t)n * nin[kind] * sizeof(double), bo = (size_t)n * nout[kind] * sizeof(double);
  double *din = nullptr, *dout = nullptr;
  if (cudaMalloc(&din, bi) != cudaSuccess) return CS_ERR_CUDA;
  if (cudaMalloc(&dout, bo) != cudaSuccess) {
    cudaFree(din);
    return CS_ERR_CUDA;
  }
  const cs::PhysC ph = cs::make_phys(*p);
  cudaError_t e = cudaMemcpy(din, in, bi, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    if (p->flags & CS_FLAG_FP32)
      cs::k_pointwise<float><<<(n + 127) / 128, 128>>>(ph, kind, n, din, dout);
    else
      cs::k_pointwise<double><<<(n + 127) / 128, 128>>>(ph, kind, n, din, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, bo, cudaMemcpyDeviceToHost);
  cudaFree(din);
  cudaFree(dout);
  return e == cudaSuccess ? CS_OK : CS_ERR_CUDA;
}

int cs_snapshot_save(cs_ctx* ctx, const char* path, double time, double dtcur, int64_t step) {
  if (!ctx || !path) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  const size_t S6 = (size_t)6 * sv.d.S;
  std::vector<double> U(cs::NVAR * S6), ent(S6), bx(S6), by(S6), bz(S6);
  if (int rc = cs_state_get(ctx, U.data(), ent.data(), bx.data(), by.data(), bz.data())) return rc;
  const int rc = cs_snapshot_write_host(path, &sv.p, U.data(), ent.data(), bx.data(), by.data(), bz.data(), time,
                                        dtcur, step);
  if (rc) return cs::fail(sv, rc, std::string("cannot write snapshot ") + path);
  return CS_OK;
}

int cs_snapshot_load(cs_ctx* ctx, const char* path, double* time, double* dtcur, int64_t* step) {
  if (!ctx || !path || !time || !dtcur || !step) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, false)) return rc;
  const size_t S6 = (size_t)6 * sv.d.S;
  std::vector<double> U(cs::NVAR * S6), ent(S6), bx(S6), by(S6), bz(S6);
  const int rc = cs_snapshot_read_host(path, &sv.p, U.data(), ent.data(), bx.data(), by.data(), bz.data(), time,
                                       dtcur, step);
  if (rc == CS_ERR_STATE) return cs::fail(sv, rc, "snapshot belongs to another mesh or physics");
  if (rc == CS_ERR_NUMERIC) return cs::fail(sv, rc, "snapshot payload does not match its hash");
  if (rc) return cs::fail(sv, rc, std::string("cannot read snapshot ") + path);
  return cs_state_put(ctx, U.data(), ent.data(), bx.data(), by.data(), bz.data());
}

int cs_diag(cs_ctx* ctx, double* mass, double* energy, double* max_divb) {
  if (!ctx || !mass || !energy || !max_divb) return CS_ERR_ARG;
  Solve& sv = ctx->sv;
  if (int rc = cs::need(sv, true)) return rc;
  if (!sv.diag_buf) {
    cudaError_t e = cudaSuccess;
    sv.diag_buf = (double*)cs::solve_alloc(sv, cs::diag_scratch_doubles() * sizeof(double), e);
    if (!sv.diag_buf) return cs::cuda_fail(sv, e, "cudaMalloc(diagnostics)");
  }
  double* part = sv.diag_buf + 4;
  cs::launch_diag(sv, part, sv.diag_buf);
  double out[3];
  CS_CUDA(sv, cudaMemcpyAsync(out, sv.diag_buf, sizeof out, cudaMemcpyDeviceToHost, sv.stream));
  CS_CUDA(sv, cudaStreamSynchronize(sv.stream));
  *mass = out[0];
  *energy = out[1];
  *max_divb = out[2];
  return CS_OK;
}

}  // extern "C"
