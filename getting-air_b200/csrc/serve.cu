// Serving form: a request loop with HBM-budget admission and continuous
// batching of resident solves.
//
// The server owns ONE device arena of `budget` bytes, allocated at creation.
// A request (a dense lbm_config plus a step count) is admitted when its
// state -- two f buffers, the mac field and its force scratch -- fits in the
// arena (first fit, FIFO order); until then it waits in the queue. Every
// tick advances all resident requests together: per step, one persistent
// launch per lattice (D2Q9, D3Q19, D3Q27) walks a tile list covering every
// resident domain and applies the same per-cell update as a dense session
// (cell3 / cell2), so a request's result is bit-identical whether it runs
// alone or in a mix. A tick ends when the soonest request completes; finished
// requests are retired (force read back, memory returned to the arena) and
// queued ones admitted into the freed space before the next tick.
//
// A request may also be a 3D two-level AMR solve (lbm_server_submit_amr3d):
// its hierarchy is built inside its share of the arena
// (lbm_amr3d_create_in), it advances on a stream of its own -- graph-launched
// macro-steps that overlap the persistent dense launches -- and it is the
// same solve, bit for bit, as an lbm_amr3d session of the same config.
//
// The reference has no serving form (one page steps one domain).

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lbm.h"
#include "cell_update.cuh"
#include "dense.cuh"
#include "host_params.cuh"

namespace lbm {
namespace {

constexpr int kServeThreads = 256;
constexpr int kServeCpt = 4;  // cells per thread per tile
constexpr int kCellsPerTile = kServeThreads * kServeCpt;

// Per-domain descriptor: the dense StepParams plus the domain's own buffers.
struct ServeDom {
  StepParams p;
  const void *fa;  // current f at the start of the tick
  void *fb;        // the other buffer
  float *mac;
};

template <int Q, typename S>
__global__ void __launch_bounds__(kServeThreads)
    serve_step(const ServeDom *__restrict__ doms, const int2 *__restrict__ tiles, int ntiles, int parity,
               int write_mac) {
  __shared__ __align__(16) unsigned char raw[sizeof(ServeDom)];
  ServeDom &d = *reinterpret_cast<ServeDom *>(raw);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int2 td = __ldg(&tiles[t]);
    const int *src = reinterpret_cast<const int *>(doms + td.x);
    int *dst = reinterpret_cast<int *>(raw);
    for (int k = threadIdx.x; k < (int)(sizeof(ServeDom) / 4); k += kServeThreads) dst[k] = __ldg(src + k);
    __syncthreads();
    if (threadIdx.x == 0) d.p.write_mac = write_mac;
    __syncthreads();
    const S *fin = (const S *)(parity ? d.fb : d.fa);
    S *fout = (S *)(parity ? const_cast<void *>(d.fa) : d.fb);
    const int nx = d.p.nx, ny = d.p.ny;
    const int ncell = nx * ny * d.p.nz;
    const int end = min(td.y + kCellsPerTile, ncell);
    const int lt = t - d.p.tile0;
    const bool region = d.p.force_on && lt >= d.p.ft0 && lt < d.p.ft1;
    ForceAcc acc;
    for (int c = td.y + threadIdx.x; c < end; c += kServeThreads) {
      const int x = c % nx, r = c / nx;
      CellForce cf;
      if constexpr (Q == 9) {
        cell2<S>(fin, fout, d.mac, d.p, x, r, region, cf);
      } else {
        cell3<Q, S>(fin, fout, d.mac, d.p, x, r % ny, r / ny, region, cf);
      }
      if (region) acc.add(cf);
    }
    if (region)
      reduce_force<kServeThreads>(acc, d.p.partials, d.p.counter, d.p.ft1 - d.p.ft0, lt - d.p.ft0, d.p.force_out);
    __syncthreads();
  }
}

cudaError_t launch_serve(int q, int storage, int grid, cudaStream_t st, const ServeDom *doms, const int2 *tiles,
                         int ntiles, int parity, int write_mac) {
#define SERVE_CASE(QQ, SS)                                                                          \
  serve_step<QQ, SS><<<grid, kServeThreads, 0, st>>>(doms, tiles, ntiles, parity, write_mac);       \
  break;
  switch (q * 4 + storage) {
    case 9 * 4 + 0: SERVE_CASE(9, float)
    case 9 * 4 + 1: SERVE_CASE(9, __half)
    case 9 * 4 + 2: SERVE_CASE(9, __nv_bfloat16)
    case 19 * 4 + 0: SERVE_CASE(19, float)
    case 19 * 4 + 1: SERVE_CASE(19, __half)
    case 19 * 4 + 2: SERVE_CASE(19, __nv_bfloat16)
    case 27 * 4 + 0: SERVE_CASE(27, float)
    case 27 * 4 + 1: SERVE_CASE(27, __half)
    case 27 * 4 + 2: SERVE_CASE(27, __nv_bfloat16)
    default: return cudaErrorInvalidValue;
  }
#undef SERVE_CASE
  return cudaGetLastError();
}

// First-fit allocator over [0, size) with 256-byte granules.
struct Arena {
  int64_t size = 0;
  std::map<int64_t, int64_t> free_;  // offset -> length
  void reset(int64_t n) {
    size = n;
    free_.clear();
    free_[0] = n;
  }
  int64_t alloc(int64_t n) {
    n = (n + 255) & ~int64_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const int64_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > n) free_[off + n] = len - n;
      return off;
    }
    return -1;
  }
  void release(int64_t off, int64_t n) {
    n = (n + 255) & ~int64_t(255);
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  int64_t free_bytes() const {
    int64_t s = 0;
    for (auto &kv : free_) s += kv.second;
    return s;
  }
};

struct Request {
  int64_t id = 0;
  lbm_config cfg{};
  std::vector<float> mac_seed;  // empty: uniform freestream at sponge_u
  int steps = 0, done = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  int64_t off = -1, bytes = 0;
  char *base = nullptr;  // arena pointer
  void *f[2] = {nullptr, nullptr};
  int cur = 0;
  float *mac = nullptr;
  double *partials = nullptr;
  unsigned *counter = nullptr;
  double *force_out = nullptr;
  int nparts = 0;
  int state = 0;  // 0 queued, 1 resident, 2 finished (resident until released)
  double force[8] = {};
  // a 3D two-level AMR solve (kind 1): its hierarchy and stream
  int kind = 0;
  lbm_amr3d_config acfg{};
  lbm_amr3d *amr = nullptr;
  cudaStream_t amr_stream = nullptr;
};

// Lattice cells of a request's domain (L0 for an AMR solve).
int64_t request_cells(const Request &r) { return (int64_t)r.cfg.nx * r.cfg.ny * r.cfg.nz; }

int64_t request_bytes(const lbm_config &c, int nparts) {
  const int64_t n = (int64_t)c.nx * c.ny * c.nz;
  const int elem = c.storage == LBM_STORE_FP32 ? 4 : 2;
  auto up = [](int64_t b) { return (b + 255) & ~int64_t(255); };
  return 2 * up((int64_t)c.q * n * elem) + up(n * 16) + up((int64_t)nparts * kForceSlots * 8) + 256 + up(kForceSlots * 8);
}

// Force-region tiles [ft0, ft1) of a domain tiled by kCellsPerTile.
int force_tiles(const lbm_config &c, StepParams &p) {
  int box[6];
  p.force_on = force_cell_box(c, p, box) ? 1 : 0;
  if (!p.force_on) {
    p.ft0 = p.ft1 = 0;
    return 0;
  }
  const int64_t first = ((int64_t)box[4] * c.ny + box[2]) * c.nx + box[0];
  const int64_t last = ((int64_t)box[5] * c.ny + box[3]) * c.nx + box[1];
  p.ft0 = (int)(first / kCellsPerTile);
  p.ft1 = (int)(last / kCellsPerTile) + 1;
  return p.ft1 - p.ft0;
}

}  // namespace
}  // namespace lbm

using namespace lbm;

struct lbm_server {
  int64_t budget = 0;
  char *arena_ptr = nullptr;
  Arena arena;
  std::map<int64_t, Request> reqs;   // by id
  std::deque<int64_t> queue;         // FIFO of queued ids
  cudaStream_t stream = nullptr;
  ServeDom *d_doms = nullptr;
  int2 *d_tiles = nullptr;
  int cap_doms = 0, cap_tiles = 0;
  ServeDom *h_doms = nullptr;        // pinned staging
  int2 *h_tiles = nullptr;
  int sms = 148;
  int policy = 0;                    // 0 FIFO, 1 shortest work first
  int64_t max_resident_cells = 0;    // 0: no cap besides the budget
  std::chrono::steady_clock::time_point t0;
  int64_t lattice_updates = 0;
  std::string err;
};

namespace {

thread_local std::string g_server_error;

int sfail(lbm_server *s, int code, const std::string &m) {
  if (s) s->err = m; else g_server_error = m;
  return code;
}

#define SCK(s, call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return sfail(s, e_ == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA,        \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

double now_s(const lbm_server *s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

int ensure_staging(lbm_server *s, int ndoms, int ntiles) {
  if (ndoms > s->cap_doms) {
    cudaFree(s->d_doms);
    cudaFreeHost(s->h_doms);
    s->d_doms = nullptr;
    s->h_doms = nullptr;
    const int cap = std::max(ndoms, 2 * s->cap_doms);
    SCK(s, cudaMalloc(&s->d_doms, cap * sizeof(ServeDom)));
    SCK(s, cudaMallocHost(&s->h_doms, cap * sizeof(ServeDom)));
    s->cap_doms = cap;
  }
  if (ntiles > s->cap_tiles) {
    cudaFree(s->d_tiles);
    cudaFreeHost(s->h_tiles);
    s->d_tiles = nullptr;
    s->h_tiles = nullptr;
    const int cap = std::max(ntiles, 2 * s->cap_tiles);
    SCK(s, cudaMalloc(&s->d_tiles, (size_t)cap * sizeof(int2)));
    SCK(s, cudaMallocHost(&s->h_tiles, (size_t)cap * sizeof(int2)));
    s->cap_tiles = cap;
  }
  return LBM_OK;
}

// Places a queued request into the arena and seeds it; false when it does
// not fit right now.
int admit_amr(lbm_server *s, Request &r, bool &ok) {
  ok = false;
  int64_t bytes = 0;
  int rc = lbm_amr3d_device_bytes(&r.acfg, nullptr, &bytes);
  if (rc) return sfail(s, rc, lbm_amr3d_last_error(nullptr));
  const int64_t off = s->arena.alloc(bytes);
  if (off < 0) return LBM_OK;
  r.off = off;
  r.bytes = bytes;
  rc = lbm_amr3d_create_in(&r.acfg, nullptr, s->arena_ptr + off, bytes, &r.amr);
  if (rc) {
    s->arena.release(off, bytes);
    return sfail(s, rc, lbm_amr3d_last_error(nullptr));
  }
  SCK(s, cudaStreamCreateWithFlags(&r.amr_stream, cudaStreamNonBlocking));
  lbm_amr3d_set_stream(r.amr, r.amr_stream);
  const int64_t n = request_cells(r);
  std::vector<float> seed;
  const float *src = r.mac_seed.empty() ? nullptr : r.mac_seed.data();
  if (!src) {
    const lbm_config &c = r.cfg;
    const float ux = c.sponge_u[0], uy = c.sponge_u[1], uz = c.sponge_u[2];
    const float rho = 1.0f - (ux * ux + uy * uy + uz * uz) * 1.5f;
    seed.resize(4 * n);
    for (int64_t k = 0; k < n; ++k) {
      seed[4 * k] = rho; seed[4 * k + 1] = ux; seed[4 * k + 2] = uy; seed[4 * k + 3] = uz;
    }
    src = seed.data();
  }
  rc = lbm_amr3d_init_macro(r.amr, src);
  if (rc) return sfail(s, rc, lbm_amr3d_last_error(r.amr));
  r.mac_seed.clear();
  r.mac_seed.shrink_to_fit();
  r.state = 1;
  r.t_admit = now_s(s);
  ok = true;
  return LBM_OK;
}

int admit(lbm_server *s, Request &r, bool &ok) {
  if (r.kind == 1) return admit_amr(s, r, ok);
  ok = false;
  StepParams tmp{};
  fill_step_params(r.cfg, 1, 0, tmp);
  const int nparts = force_tiles(r.cfg, tmp);
  const int64_t bytes = request_bytes(r.cfg, nparts);
  const int64_t off = s->arena.alloc(bytes);
  if (off < 0) return LBM_OK;
  r.off = off;
  r.bytes = bytes;
  r.nparts = nparts;
  char *p = s->arena_ptr + off;
  const int64_t n = (int64_t)r.cfg.nx * r.cfg.ny * r.cfg.nz;
  const int elem = r.cfg.storage == LBM_STORE_FP32 ? 4 : 2;
  auto up = [](int64_t b) { return (b + 255) & ~int64_t(255); };
  const int64_t fb = up((int64_t)r.cfg.q * n * elem);
  r.f[0] = p; p += fb;
  r.f[1] = p; p += fb;
  r.mac = (float *)p; p += up(n * 16);
  r.partials = (double *)p; p += up((int64_t)nparts * kForceSlots * 8);
  r.counter = (unsigned *)p; p += 256;
  r.force_out = (double *)p;
  r.cur = 0;
  // Seed: the caller's macroscopic field, else the uniform freestream at
  // sponge_u with rho = 1 - |u|^2 / (2 cs^2) (d3-scenarios.mjs seedMacro3).
  std::vector<float> seed;
  const float *src = r.mac_seed.empty() ? nullptr : r.mac_seed.data();
  if (!src) {
    const float ux = r.cfg.sponge_u[0], uy = r.cfg.sponge_u[1], uz = r.cfg.q == 9 ? 0.f : r.cfg.sponge_u[2];
    const float rho = 1.0f - (ux * ux + uy * uy + uz * uz) * 1.5f;
    seed.resize(4 * n);
    for (int64_t k = 0; k < n; ++k) {
      seed[4 * k] = rho; seed[4 * k + 1] = ux; seed[4 * k + 2] = uy; seed[4 * k + 3] = uz;
    }
    src = seed.data();
  }
  SCK(s, cudaMemcpyAsync(r.mac, src, n * 16, cudaMemcpyHostToDevice, s->stream));
  SCK(s, launch_init_eq(r.cfg.q, r.cfg.storage, r.mac, r.f[0], n, make_pack(r.cfg), s->stream));
  SCK(s, cudaMemsetAsync(r.counter, 0, 4, s->stream));
  SCK(s, cudaMemsetAsync(r.force_out, 0, kForceSlots * 8, s->stream));
  // The seed must be on the device before `seed` goes out of scope.
  SCK(s, cudaStreamSynchronize(s->stream));
  r.mac_seed.clear();
  r.mac_seed.shrink_to_fit();
  r.state = 1;
  r.t_admit = now_s(s);
  ok = true;
  return LBM_OK;
}

// Runs `k` steps of every resident, unfinished request.
int run_steps(lbm_server *s, const std::vector<Request *> &act, int k) {
  // the AMR solves first: k macro-steps each, queued on their own streams
  for (Request *r : act) {
    if (r->kind != 1) continue;
    const int rc = lbm_amr3d_step(r->amr, k);
    if (rc) return sfail(s, rc, lbm_amr3d_last_error(r->amr));
  }
  for (int q : {9, 19, 27})
    for (int st = 0; st <= 2; ++st) {
      std::vector<Request *> group;
      for (Request *r : act)
        if (r->kind == 0 && r->cfg.q == q && r->cfg.storage == st) group.push_back(r);
      if (group.empty()) continue;
      int ntiles = 0;
      for (Request *r : group) {
        const int64_t n = (int64_t)r->cfg.nx * r->cfg.ny * r->cfg.nz;
        ntiles += (int)((n + kCellsPerTile - 1) / kCellsPerTile);
      }
      int rc = ensure_staging(s, (int)group.size(), ntiles);
      if (rc) return rc;
      int t = 0;
      for (size_t d = 0; d < group.size(); ++d) {
        Request &r = *group[d];
        const int64_t n = (int64_t)r.cfg.nx * r.cfg.ny * r.cfg.nz;
        ServeDom &sd = s->h_doms[d];
        std::memset(&sd, 0, sizeof(sd));
        fill_step_params(r.cfg, n, 0, sd.p);
        force_tiles(r.cfg, sd.p);
        sd.p.tile0 = t;
        sd.p.partials = r.partials;
        sd.p.counter = r.counter;
        sd.p.force_out = r.force_out;
        sd.fa = r.f[r.cur];
        sd.fb = r.f[1 - r.cur];
        sd.mac = r.mac;
        const int nt = (int)((n + kCellsPerTile - 1) / kCellsPerTile);
        for (int j = 0; j < nt; ++j) s->h_tiles[t++] = make_int2((int)d, j * kCellsPerTile);
      }
      SCK(s, cudaMemcpyAsync(s->d_doms, s->h_doms, group.size() * sizeof(ServeDom), cudaMemcpyHostToDevice,
                             s->stream));
      SCK(s, cudaMemcpyAsync(s->d_tiles, s->h_tiles, (size_t)t * sizeof(int2), cudaMemcpyHostToDevice, s->stream));
      const int grid = std::min(t, 8 * s->sms);
      for (int j = 0; j < k; ++j) SCK(s, launch_serve(q, st, grid, s->stream, s->d_doms, s->d_tiles, t, j & 1, j == k - 1));
      for (Request *r : group) {
        r->done += k;
        if (k & 1) r->cur = 1 - r->cur;
        s->lattice_updates += (int64_t)k * r->cfg.nx * r->cfg.ny * r->cfg.nz;
      }
      // The staging buffers are rewritten by the next group: wait for the copies.
      SCK(s, cudaStreamSynchronize(s->stream));
    }
  for (Request *r : act) {
    if (r->kind != 1) continue;
    SCK(s, cudaStreamSynchronize(r->amr_stream));
    r->done += k;
    s->lattice_updates += (int64_t)k * lbm_amr3d_cell_updates(r->amr);
  }
  return LBM_OK;
}

void drop_amr(Request &r) {
  if (r.amr) lbm_amr3d_destroy(r.amr);
  if (r.amr_stream) cudaStreamDestroy(r.amr_stream);
  r.amr = nullptr;
  r.amr_stream = nullptr;
}

}  // namespace

extern "C" {

int lbm_server_create(int64_t budget_bytes, lbm_server **out) {
  if (!out) return sfail(nullptr, LBM_EINVAL, "out is NULL");
  *out = nullptr;
  if (budget_bytes < (1 << 20)) return sfail(nullptr, LBM_EINVAL, "budget must be at least 1 MiB");
  lbm_server *s = new lbm_server();
  s->budget = budget_bytes;
  cudaError_t e = cudaMalloc(&s->arena_ptr, budget_bytes);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaFree(s->arena_ptr);
    delete s;
    return sfail(nullptr, e == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA,
                 std::string("server arena: ") + cudaGetErrorString(e));
  }
  s->arena.reset(budget_bytes);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, dev);
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return LBM_OK;
}

void lbm_server_destroy(lbm_server *s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto &kv : s->reqs) drop_amr(kv.second);
  cudaFree(s->arena_ptr);
  cudaFree(s->d_doms);
  cudaFree(s->d_tiles);
  if (s->h_doms) cudaFreeHost(s->h_doms);
  if (s->h_tiles) cudaFreeHost(s->h_tiles);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

const char *lbm_server_last_error(const lbm_server *s) { return s ? s->err.c_str() : g_server_error.c_str(); }

int lbm_server_submit(lbm_server *s, int64_t id, const lbm_config *cfg, const float *mac, int steps) {
  if (!s) return LBM_EINVAL;
  std::string why;
  if (validate_config(cfg, why)) return sfail(s, LBM_EINVAL, why);
  if (cfg->window[0] || cfg->window[1] || cfg->window[2])
    return sfail(s, LBM_ENOTSUP, "the moving window runs in dense sessions and 3D AMR");
  if (steps < 1) return sfail(s, LBM_EINVAL, "steps must be >= 1");
  if (s->reqs.count(id)) return sfail(s, LBM_EINVAL, "request id already in use");
  StepParams tmp{};
  fill_step_params(*cfg, 1, 0, tmp);
  const int64_t bytes = request_bytes(*cfg, force_tiles(*cfg, tmp));
  if (bytes > s->budget)
    return sfail(s, LBM_ENOSPC, "request needs " + std::to_string(bytes) + " bytes, more than the whole budget");
  Request r;
  r.id = id;
  r.cfg = *cfg;
  r.steps = steps;
  r.t_submit = now_s(s);
  if (mac) r.mac_seed.assign(mac, mac + 4 * (int64_t)cfg->nx * cfg->ny * cfg->nz);
  s->reqs.emplace(id, std::move(r));
  s->queue.push_back(id);
  return LBM_OK;
}

int lbm_server_set_policy(lbm_server *s, int policy, int64_t max_resident_cells) {
  if (!s) return LBM_EINVAL;
  if (policy != 0 && policy != 1) return sfail(s, LBM_EINVAL, "policy must be 0 (FIFO) or 1 (shortest work first)");
  if (max_resident_cells < 0) return sfail(s, LBM_EINVAL, "max_resident_cells must be >= 0");
  s->policy = policy;
  s->max_resident_cells = max_resident_cells;
  return LBM_OK;
}

int lbm_server_submit_amr3d(lbm_server *s, int64_t id, const lbm_amr3d_config *cfg, const float *mac, int steps) {
  if (!s) return LBM_EINVAL;
  if (!cfg) return sfail(s, LBM_EINVAL, "config is NULL");
  if (cfg->refine == LBM_REFINE_LIST) return sfail(s, LBM_EINVAL, "a served hierarchy is refined by a rule, not a list");
  int64_t bytes = 0;
  const int rc = lbm_amr3d_device_bytes(cfg, nullptr, &bytes);
  if (rc) return sfail(s, rc, lbm_amr3d_last_error(nullptr));
  if (steps < 1) return sfail(s, LBM_EINVAL, "steps must be >= 1");
  if (s->reqs.count(id)) return sfail(s, LBM_EINVAL, "request id already in use");
  if (bytes > s->budget)
    return sfail(s, LBM_ENOSPC, "request needs " + std::to_string(bytes) + " bytes, more than the whole budget");
  Request r;
  r.id = id;
  r.kind = 1;
  r.acfg = *cfg;
  r.cfg = cfg->root;
  r.steps = steps;
  r.t_submit = now_s(s);
  if (mac) r.mac_seed.assign(mac, mac + 4 * request_cells(r));
  s->reqs.emplace(id, std::move(r));
  s->queue.push_back(id);
  return LBM_OK;
}

int lbm_server_poll(lbm_server *s, int max_steps, lbm_result *done, int max_done, int *n_done) {
  if (!s || max_steps < 1) return s ? sfail(s, LBM_EINVAL, "max_steps must be >= 1") : LBM_EINVAL;
  if (n_done) *n_done = 0;
  // 1. admit: FIFO while the head fits, or the least total work first;
  // the resident-cell cap keeps the GPU busy without making every request
  // share it (continuous batching's latency cost)
  int64_t resident = 0;
  for (auto &kv : s->reqs)
    if (kv.second.state == 1) resident += request_cells(kv.second);
  auto capped = [&](const Request &r) {
    return s->max_resident_cells > 0 && resident > 0 && resident + request_cells(r) > s->max_resident_cells;
  };
  if (s->policy == 1) {
    std::stable_sort(s->queue.begin(), s->queue.end(), [&](int64_t x, int64_t y) {
      const Request &a = s->reqs[x], &b = s->reqs[y];
      return request_cells(a) * a.steps < request_cells(b) * b.steps;
    });
  }
  while (!s->queue.empty()) {
    Request &r = s->reqs[s->queue.front()];
    if (capped(r)) break;
    bool ok = false;
    int rc = admit(s, r, ok);
    if (rc) return rc;
    if (!ok) break;
    resident += request_cells(r);
    s->queue.pop_front();
  }
  // 2. one tick: every resident unfinished request, up to the soonest finish
  std::vector<Request *> act;
  int k = max_steps;
  for (auto &kv : s->reqs)
    if (kv.second.state == 1) {
      act.push_back(&kv.second);
      k = std::min(k, kv.second.steps - kv.second.done);
    }
  if (!act.empty()) {
    int rc = run_steps(s, act, k);
    if (rc) return rc;
  }
  // 3. retire the finished ones
  int nd = 0;
  for (Request *r : act) {
    if (r->done < r->steps) continue;
    if (done && nd >= max_done) break;  // the rest retire on the next poll
    if (r->kind == 1) {
      const int rc = lbm_amr3d_forces(r->amr, r->force);
      if (rc) return sfail(s, rc, lbm_amr3d_last_error(r->amr));
    } else {
      SCK(s, cudaMemcpy(r->force, r->force_out, kForceSlots * 8, cudaMemcpyDeviceToHost));
    }
    r->state = 2;
    r->t_done = now_s(s);
    if (done && nd < max_done) {
      lbm_result &o = done[nd];
      o.id = r->id;
      o.status = 0;
      o.steps = r->done;
      for (int j = 0; j < 6; ++j) o.forces[j] = r->force[j];
      o.submit_s = r->t_submit;
      o.admit_s = r->t_admit;
      o.done_s = r->t_done;
    }
    ++nd;
  }
  if (n_done) *n_done = std::min(nd, max_done);
  return LBM_OK;
}

int lbm_server_read(lbm_server *s, int64_t id, float *f, float *mac) {
  if (!s) return LBM_EINVAL;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end() || it->second.state != 2) return sfail(s, LBM_ESTATE, "request is not finished");
  Request &r = it->second;
  const int64_t n = (int64_t)r.cfg.nx * r.cfg.ny * r.cfg.nz;
  if (r.kind == 1) {
    // the L0 level: f of the current time level and the mac
    const int64_t qn = (int64_t)r.cfg.q * n;
    std::vector<float> fb(f ? 0 : qn), mb(mac ? 0 : 4 * n);
    const int rc = lbm_amr3d_read_coarse(r.amr, f ? f : fb.data(), mac ? mac : mb.data());
    if (rc) return sfail(s, rc, lbm_amr3d_last_error(r.amr));
    return LBM_OK;
  }
  if (f) {
    if (r.cfg.storage == LBM_STORE_FP32) {
      SCK(s, cudaMemcpyAsync(f, r.f[r.cur], (size_t)r.cfg.q * n * 4, cudaMemcpyDeviceToHost, s->stream));
    } else {
      // Unpack into the spare buffer's space (as f32 it may not fit): unpack
      // plane groups through the mac field, which is overwritten by it.
      return sfail(s, LBM_ENOTSUP, "reading packed-storage f from the server is not supported; read mac");
    }
  }
  if (mac) SCK(s, cudaMemcpyAsync(mac, r.mac, n * 16, cudaMemcpyDeviceToHost, s->stream));
  SCK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int lbm_server_release(lbm_server *s, int64_t id) {
  if (!s) return LBM_EINVAL;
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sfail(s, LBM_EINVAL, "unknown request id");
  if (it->second.state == 1) return sfail(s, LBM_ESTATE, "request is still running");
  if (it->second.state == 0) {
    s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), id), s->queue.end());
  } else {
    drop_amr(it->second);
    s->arena.release(it->second.off, it->second.bytes);
  }
  s->reqs.erase(it);
  return LBM_OK;
}

int lbm_server_stats(lbm_server *s, int64_t out[6]) {
  if (!s || !out) return LBM_EINVAL;
  int64_t q = 0, res = 0, fin = 0;
  for (auto &kv : s->reqs) {
    if (kv.second.state == 0) ++q;
    else if (kv.second.state == 1) ++res;
    else ++fin;
  }
  out[0] = q;
  out[1] = res;
  out[2] = fin;
  out[3] = s->budget - s->arena.free_bytes();
  out[4] = s->budget;
  out[5] = s->lattice_updates;
  return LBM_OK;
}

}  // extern "C"
