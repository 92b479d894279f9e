// Serving form: a request loop with HBM-budget admission and continuous
// batching of resident solves.
//
// The server owns ONE device arena of `budget` bytes, allocated at creation.
// A request (a dense lbm_config plus a step count) is admitted when its
// state -- two f buffers, the mac field and its force scratch -- fits in the
// arena (first fit; FIFO or least work first); until then it waits in the
// queue. A tick advances every resident request by the same number of steps:
// per step, one persistent launch per (lattice, storage) walks a tile list
// covering every resident domain of that kind and applies the same per-cell
// update as a dense session (cell3 / cell2), so a request's result is
// bit-identical whether it runs alone or in a mix. A tick ends when the
// soonest request completes.
//
// Dense requests of at least kStreamCells cells do not join the tile
// launches: each runs the dense session's own step (launch_step, the same
// kernels and force sums as an lbm_session) on a stream of its own, so a
// large domain gets the tuned dense kernel and the small ones share the
// tile launches; all of them, the AMR solves included, overlap on the GPU.
//
// Ticks are pipelined: lbm_server_poll enqueues the next tick (two tick
// slots, each with its own staging buffers and completion events) before
// it waits for the oldest one, so the GPU always has a tick queued while
// the host retires finished requests (completion by CUDA event, the force
// read back by an asynchronous copy into pinned memory queued behind the
// request's last step) and admits new ones (a uniform seed is built on the
// device; a caller's seed goes up on a separate upload stream). Nothing in
// a tick waits on the host.
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
// Dense requests from this size up step on their own stream with the dense
// session's kernels (64^3 cells: where one domain fills the GPU's launch).
constexpr int64_t kStreamCells = int64_t(1) << 18;

// Per-domain descriptor: the dense StepParams plus the domain's own buffers.
struct ServeDom {
  StepParams p;
  const void *fa;  // current f at the start of the tick
  void *fb;        // the other buffer
  float *mac;
};

template <int Q, typename S, bool TRT>
__global__ void __launch_bounds__(kServeThreads, 2)
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
    CellWalk w(td.y + threadIdx.x, kServeThreads, nx, ny);
    for (int c = td.y + threadIdx.x; c < end; c += kServeThreads) {
      CellForce cf;
      if constexpr (Q == 9) {
        cell2<S>(fin, fout, d.mac, d.p, w.x, w.y, region, cf);
      } else {
        cell3<Q, S, TRT>(fin, fout, d.mac, d.p, w.x, w.y, w.z, region, cf);
      }
      if (region) acc.add(cf);
      w.advance();
    }
    if (region)
      reduce_force<kServeThreads>(acc, d.p.partials, d.p.counter, d.p.ft1 - d.p.ft0, lt - d.p.ft0, d.p.force_out);
    __syncthreads();
  }
}

cudaError_t launch_serve(int q, int storage, bool trt, int grid, cudaStream_t st, const ServeDom *doms,
                         const int2 *tiles, int ntiles, int parity, int write_mac) {
#define SERVE_CASE(QQ, SS)                                                                                   \
  if (trt && QQ != 9)                                                                                         \
    serve_step<QQ, SS, true><<<grid, kServeThreads, 0, st>>>(doms, tiles, ntiles, parity, write_mac);        \
  else                                                                                                        \
    serve_step<QQ, SS, false><<<grid, kServeThreads, 0, st>>>(doms, tiles, ntiles, parity, write_mac);       \
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
  int steps = 0;
  int enq = 0;                  // steps enqueued (complete once retired)
  double t_submit = 0, t_admit = 0, t_done = 0;
  int64_t off = -1, bytes = 0;
  void *f[2] = {nullptr, nullptr};
  int cur = 0;                  // f buffer current after the enqueued steps
  float *mac = nullptr;
  double *partials = nullptr;
  unsigned *counter = nullptr;
  double *force_out = nullptr;
  int nparts = 0;
  int state = 0;  // 0 queued, 1 resident, 2 finished (resident until released)
  double force[8] = {};
  // kind 0: a dense solve in the tile launches; kind 1: a 3D two-level AMR
  // solve (its hierarchy); kind 2: a dense solve stepped by the dense
  // session's kernels (its StepParams, and the group sums of its force
  // partials, two sets of dparts). Kinds 1 and 2 run on their own stream,
  // with one completion event per tick slot.
  int kind = 0;
  lbm_amr3d_config acfg{};
  lbm_amr3d *amr = nullptr;
  StepParams sp{};
  double *groups = nullptr;
  int dparts = 0;
  cudaStream_t own = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
};

// One tick in flight: its staging (pinned host and device copies of the
// domain descriptors and tiles), the requests whose last step it holds, the
// AMR requests it stepped (their ev[slot]), and its event on the server
// stream (after the dense launches and the force copies).
struct TickSlot {
  bool busy = false;
  int64_t seq = 0;
  cudaEvent_t ev = nullptr;
  std::vector<std::pair<int64_t, int>> finishing;  // (id, its row of h_force or -1)
  std::vector<int64_t> streams;                    // kind 1 and 2 requests stepped
  ServeDom *h_doms = nullptr, *d_doms = nullptr;
  int2 *h_tiles = nullptr, *d_tiles = nullptr;
  int cap_doms = 0, cap_tiles = 0;
  double *h_force = nullptr;  // pinned, kForceSlots per finishing dense request
  int cap_force = 0;
};

// Lattice cells of a request's domain (L0 for an AMR solve).
int64_t request_cells(const Request &r) { return (int64_t)r.cfg.nx * r.cfg.ny * r.cfg.nz; }

int64_t request_bytes(const lbm_config &c, int nparts) {
  const int64_t n = (int64_t)c.nx * c.ny * c.nz;
  const int elem = c.storage == LBM_STORE_FP32 ? 4 : 2;
  auto up = [](int64_t b) { return (b + 255) & ~int64_t(255); };
  return 2 * up((int64_t)c.q * n * elem) + up(n * 16) + up((int64_t)nparts * kForceSlots * 8) + 256 + up(kForceSlots * 8);
}

// The dense session's step parameters of a kind-2 request (its reach box and
// force region set as a session sets them) and its number of force partials.
int streamed_params(const lbm_config &c, StepParams &sp) {
  fill_step_params(c, (int64_t)c.nx * c.ny * c.nz, 0, sp);
  return set_body_regions(c, sp, true) ? force_parts(c.q, sp) : 0;
}

// A kind-2 request: two f buffers, the mac field, two sets of force
// partials (consecutive steps alternate), their group sums, the ticket and
// the force.
int64_t streamed_bytes(const lbm_config &c, int dparts) {
  const int64_t n = (int64_t)c.nx * c.ny * c.nz;
  const int elem = c.storage == LBM_STORE_FP32 ? 4 : 2;
  auto up = [](int64_t b) { return (b + 255) & ~int64_t(255); };
  return 2 * up((int64_t)c.q * n * elem) + up(n * 16) + up((int64_t)2 * dparts * kForceSlots * 8) +
         up((int64_t)sum_groups(dparts) * kForceSlots * 8) + 256 + up(kForceSlots * 8);
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
  std::deque<int64_t> queue;         // queued ids, in admission order
  std::deque<int64_t> ready;         // retired, not yet reported by a poll
  cudaStream_t stream = nullptr;     // the dense ticks
  cudaStream_t upload = nullptr;     // callers' seeds
  TickSlot slot[2];
  int64_t tick_seq = 0;
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

template <typename T> int grow_pair(lbm_server *s, T **h, T **d, int &cap, int need) {
  if (need <= cap) return LBM_OK;
  const int c = std::max({need, 2 * cap, 64});
  cudaFree(*d);
  if (*h) cudaFreeHost(*h);
  *d = nullptr;
  *h = nullptr;
  cap = 0;
  SCK(s, cudaMalloc(d, (size_t)c * sizeof(T)));
  SCK(s, cudaMallocHost(h, (size_t)c * sizeof(T)));
  cap = c;
  return LBM_OK;
}

int ensure_staging(lbm_server *s, TickSlot &t, int ndoms, int ntiles, int nforce) {
  int rc = grow_pair(s, &t.h_doms, &t.d_doms, t.cap_doms, ndoms);
  if (!rc) rc = grow_pair(s, &t.h_tiles, &t.d_tiles, t.cap_tiles, ntiles);
  if (rc) return rc;
  if (nforce > t.cap_force) {
    const int c = std::max({nforce, 2 * t.cap_force, 16});
    if (t.h_force) cudaFreeHost(t.h_force);
    t.h_force = nullptr;
    t.cap_force = 0;
    SCK(s, cudaMallocHost(&t.h_force, (size_t)c * kForceSlots * sizeof(double)));
    t.cap_force = c;
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
  SCK(s, cudaStreamCreateWithFlags(&r.own, cudaStreamNonBlocking));
  for (int k = 0; k < 2; ++k) SCK(s, cudaEventCreateWithFlags(&r.ev[k], cudaEventDisableTiming));
  lbm_amr3d_set_stream(r.amr, r.own);
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
  const int64_t n = request_cells(r);
  int nparts = 0;
  int64_t bytes = 0;
  if (r.kind == 2) {
    r.dparts = streamed_params(r.cfg, r.sp);
    bytes = streamed_bytes(r.cfg, r.dparts);
  } else {
    StepParams tmp{};
    fill_step_params(r.cfg, 1, 0, tmp);
    nparts = force_tiles(r.cfg, tmp);
    bytes = request_bytes(r.cfg, nparts);
  }
  const int64_t off = s->arena.alloc(bytes);
  if (off < 0) return LBM_OK;
  r.off = off;
  r.bytes = bytes;
  r.nparts = nparts;
  char *p = s->arena_ptr + off;
  const int elem = r.cfg.storage == LBM_STORE_FP32 ? 4 : 2;
  auto up = [](int64_t b) { return (b + 255) & ~int64_t(255); };
  const int64_t fb = up((int64_t)r.cfg.q * n * elem);
  r.f[0] = p; p += fb;
  r.f[1] = p; p += fb;
  r.mac = (float *)p; p += up(n * 16);
  if (r.kind == 2) {
    r.partials = (double *)p; p += up((int64_t)2 * r.dparts * kForceSlots * 8);
    r.groups = (double *)p; p += up((int64_t)sum_groups(r.dparts) * kForceSlots * 8);
  } else {
    r.partials = (double *)p; p += up((int64_t)nparts * kForceSlots * 8);
  }
  r.counter = (unsigned *)p; p += 256;
  r.force_out = (double *)p;
  r.cur = 0;
  cudaStream_t st = s->stream;
  if (r.kind == 2) {
    SCK(s, cudaStreamCreateWithFlags(&r.own, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) SCK(s, cudaEventCreateWithFlags(&r.ev[k], cudaEventDisableTiming));
    r.sp.partials = r.partials;
    r.sp.groups = r.groups;
    r.sp.counter = r.counter;
    r.sp.force_out = r.force_out;
    st = r.own;
  }
  // Seed: the caller's macroscopic field, else the uniform freestream at
  // sponge_u with rho = 1 - |u|^2 / (2 cs^2) (d3-scenarios.mjs seedMacro3),
  // built on the device. A caller's field goes up on a stream no tick uses
  // (the upload stream, which the server stream then waits for, or the
  // request's own): a pageable copy waits for its stream and returns once
  // the host buffer is staged, so neither waits for a tick in flight.
  const Pack pk = make_pack(r.cfg);
  if (!r.mac_seed.empty()) {
    cudaStream_t us = r.kind == 2 ? r.own : s->upload;
    cudaError_t e = cudaMemcpyAsync(r.mac, r.mac_seed.data(), n * 16, cudaMemcpyHostToDevice, us);
    if (!e) e = launch_init_eq(r.cfg.q, r.cfg.storage, r.mac, r.f[0], n, pk, us);
    if (!e && r.kind != 2) {
      cudaEvent_t upe = nullptr;
      e = cudaEventCreateWithFlags(&upe, cudaEventDisableTiming);
      if (!e) e = cudaEventRecord(upe, s->upload);
      if (!e) e = cudaStreamWaitEvent(s->stream, upe, 0);
      if (upe) cudaEventDestroy(upe);
    }
    if (e) return sfail(s, LBM_ECUDA, std::string("seed: ") + cudaGetErrorString(e));
  } else {
    const float ux = r.cfg.sponge_u[0], uy = r.cfg.sponge_u[1], uz = r.cfg.q == 9 ? 0.f : r.cfg.sponge_u[2];
    const float rho_u[4] = {1.0f - (ux * ux + uy * uy + uz * uz) * 1.5f, ux, uy, uz};
    SCK(s, launch_init_uniform(r.cfg.q, r.cfg.storage, rho_u, r.mac, r.f[0], n, pk, st));
  }
  SCK(s, cudaMemsetAsync(r.counter, 0, 4, st));
  SCK(s, cudaMemsetAsync(r.force_out, 0, kForceSlots * 8, st));
  r.mac_seed.clear();
  r.mac_seed.shrink_to_fit();
  r.state = 1;
  r.t_admit = now_s(s);
  ok = true;
  return LBM_OK;
}

// k steps of a kind-2 request on its own stream: lbm_step's sequence (each
// step's force partials summed by the next step's first blocks, the last
// step's by the sum launch after it).
int step_streamed(lbm_server *s, Request &r, int k) {
  const int64_t half = (int64_t)r.dparts * kForceSlots;
  const int parts = r.sp.force_on ? r.dparts : 0;
  for (int j = 0; j < k; ++j) {
    StepParams &sp = r.sp;
    sp.write_mac = (j == k - 1);
    sp.partials = r.partials + (j & 1) * half;
    sp.defer_force = j < k - 1;
    sp.prev_parts = j > 0 ? parts : 0;
    sp.prev_partials = r.partials + ((j + 1) & 1) * half;
    SCK(s, launch_step(r.cfg.q, r.cfg.storage, r.f[r.cur], r.f[1 - r.cur], r.mac, sp, r.own));
    r.cur = 1 - r.cur;
  }
  r.sp.partials = r.partials;
  r.sp.defer_force = 0;
  r.sp.prev_parts = 0;
  return LBM_OK;
}

// Enqueues one tick into slot `si`: k steps of every resident request with
// steps left, k = the fewest left (at most max_steps). Returns with nothing
// enqueued when no request has steps left.
int enqueue_tick(lbm_server *s, int si, int max_steps) {
  TickSlot &t = s->slot[si];
  std::vector<Request *> act;
  int k = max_steps;
  for (auto &kv : s->reqs)
    if (kv.second.state == 1 && kv.second.enq < kv.second.steps) {
      act.push_back(&kv.second);
      k = std::min(k, kv.second.steps - kv.second.enq);
    }
  if (act.empty()) return LBM_OK;
  t.finishing.clear();
  t.streams.clear();
  int ndoms = 0, ntiles = 0, nforce = 0;
  for (Request *r : act) {
    if (r->kind == 0) {
      ++ndoms;
      ntiles += (int)((request_cells(*r) + kCellsPerTile - 1) / kCellsPerTile);
    }
    nforce += r->kind != 1 && r->enq + k == r->steps;
  }
  int rc = ensure_staging(s, t, ndoms, ntiles, nforce);
  if (rc) return rc;
  int fi = 0;
  // the solves on their own streams: AMR macro-steps, or the dense step
  for (Request *r : act) {
    if (r->kind == 0) continue;
    if (r->kind == 1) {
      rc = lbm_amr3d_step(r->amr, k);
      if (rc) return sfail(s, rc, lbm_amr3d_last_error(r->amr));
    } else {
      rc = step_streamed(s, *r, k);
      if (rc) return rc;
    }
    if (r->enq + k == r->steps) {
      int row = -1;
      if (r->kind == 2) {
        row = fi++;
        SCK(s, cudaMemcpyAsync(t.h_force + (size_t)kForceSlots * row, r->force_out, kForceSlots * sizeof(double),
                               cudaMemcpyDeviceToHost, r->own));
      }
      t.finishing.emplace_back(r->id, row);
    }
    SCK(s, cudaEventRecord(r->ev[si], r->own));
    t.streams.push_back(r->id);
  }
  // the tile launches: one descriptor and tile list per (lattice, storage,
  // collision) group, all groups staged together and uploaded once
  struct Group { int q, st; bool trt; int dom0, ndom, tile0, ntile; };
  std::vector<Group> groups;
  int d = 0, tt = 0;
  for (int q : {9, 19, 27})
    for (int st = 0; st <= 2; ++st)
      for (int trt = 0; trt <= 1; ++trt) {
        Group g{q, st, trt == 1, d, 0, tt, 0};
        for (Request *r : act) {
          if (r->kind != 0 || r->cfg.q != q || r->cfg.storage != st || (r->cfg.trt != 0) != (trt == 1)) continue;
          const int64_t n = request_cells(*r);
          ServeDom &sd = t.h_doms[d];
          std::memset(&sd, 0, sizeof(sd));
          fill_step_params(r->cfg, n, 0, sd.p);
          force_tiles(r->cfg, sd.p);
          sd.p.tile0 = tt - g.tile0;
          sd.p.partials = r->partials;
          sd.p.counter = r->counter;
          sd.p.force_out = r->force_out;
          sd.fa = r->f[r->cur];
          sd.fb = r->f[1 - r->cur];
          sd.mac = r->mac;
          const int nt = (int)((n + kCellsPerTile - 1) / kCellsPerTile);
          for (int j = 0; j < nt; ++j) t.h_tiles[tt++] = make_int2(d - g.dom0, j * kCellsPerTile);
          ++d;
        }
        g.ndom = d - g.dom0;
        g.ntile = tt - g.tile0;
        if (g.ndom) groups.push_back(g);
      }
  if (ndoms) {
    SCK(s, cudaMemcpyAsync(t.d_doms, t.h_doms, (size_t)ndoms * sizeof(ServeDom), cudaMemcpyHostToDevice, s->stream));
    SCK(s, cudaMemcpyAsync(t.d_tiles, t.h_tiles, (size_t)ntiles * sizeof(int2), cudaMemcpyHostToDevice, s->stream));
  }
  for (int j = 0; j < k; ++j)
    for (const Group &g : groups)
      SCK(s, launch_serve(g.q, g.st, g.trt, std::min(g.ntile, 8 * s->sms), s->stream, t.d_doms + g.dom0,
                          t.d_tiles + g.tile0, g.ntile, j & 1, j == k - 1));
  // the last step's force of each tile request that finishes in this tick
  for (Request *r : act) {
    if (r->kind != 0 || r->enq + k != r->steps) continue;
    const int row = fi++;
    SCK(s, cudaMemcpyAsync(t.h_force + (size_t)kForceSlots * row, r->force_out, kForceSlots * sizeof(double),
                           cudaMemcpyDeviceToHost, s->stream));
    t.finishing.emplace_back(r->id, row);
  }
  SCK(s, cudaEventRecord(t.ev, s->stream));
  for (Request *r : act) {
    r->enq += k;
    if (r->kind == 0) {
      if (k & 1) r->cur = 1 - r->cur;
      s->lattice_updates += (int64_t)k * request_cells(*r);
    } else if (r->kind == 2) {
      s->lattice_updates += (int64_t)k * request_cells(*r);  // step_streamed moved cur
    } else {
      s->lattice_updates += (int64_t)k * lbm_amr3d_cell_updates(r->amr);
    }
  }
  t.busy = true;
  t.seq = ++s->tick_seq;
  return LBM_OK;
}

// Whether slot si's tick has finished (block: wait for it).
int tick_done(lbm_server *s, int si, bool block, bool &done) {
  TickSlot &t = s->slot[si];
  done = false;
  std::vector<cudaEvent_t> evs{t.ev};
  for (int64_t id : t.streams) evs.push_back(s->reqs[id].ev[si]);
  for (cudaEvent_t e : evs) {
    const cudaError_t r = block ? cudaEventSynchronize(e) : cudaEventQuery(e);
    if (r == cudaErrorNotReady) return LBM_OK;
    if (r != cudaSuccess) return sfail(s, LBM_ECUDA, std::string("tick: ") + cudaGetErrorString(r));
  }
  done = true;
  return LBM_OK;
}

// Retires the requests whose last step slot si's (finished) tick held.
int retire_tick(lbm_server *s, int si) {
  TickSlot &t = s->slot[si];
  for (const auto &fr : t.finishing) {
    Request &r = s->reqs[fr.first];
    if (r.kind == 1) {
      const int rc = lbm_amr3d_forces(r.amr, r.force);
      if (rc) return sfail(s, rc, lbm_amr3d_last_error(r.amr));
    } else {
      std::memcpy(r.force, t.h_force + (size_t)kForceSlots * fr.second, kForceSlots * sizeof(double));
    }
    r.state = 2;
    r.t_done = now_s(s);
    s->ready.push_back(fr.first);
  }
  t.finishing.clear();
  t.streams.clear();
  t.busy = false;
  return LBM_OK;
}

// Finishes the busy ticks, oldest first: those already done, or (block)
// the oldest one whatever its state.
int complete_ticks(lbm_server *s, bool block_oldest) {
  for (int pass = 0; pass < 2; ++pass) {
    int si = -1;
    for (int k = 0; k < 2; ++k)
      if (s->slot[k].busy && (si < 0 || s->slot[k].seq < s->slot[si].seq)) si = k;
    if (si < 0) return LBM_OK;
    bool done = false;
    int rc = tick_done(s, si, block_oldest && pass == 0, done);
    if (rc) return rc;
    if (!done) return LBM_OK;
    rc = retire_tick(s, si);
    if (rc) return rc;
  }
  return LBM_OK;
}

// Releases what a request holds outside the arena: an AMR hierarchy's
// handle, its own stream and events.
void drop_amr(Request &r) {
  if (r.amr) lbm_amr3d_destroy(r.amr);
  if (r.own) {
    cudaStreamSynchronize(r.own);
    cudaStreamDestroy(r.own);
  }
  for (cudaEvent_t &e : r.ev)
    if (e) {
      cudaEventDestroy(e);
      e = nullptr;
    }
  r.amr = nullptr;
  r.own = nullptr;
}

void free_slot(TickSlot &t) {
  cudaFree(t.d_doms);
  cudaFree(t.d_tiles);
  if (t.h_doms) cudaFreeHost(t.h_doms);
  if (t.h_tiles) cudaFreeHost(t.h_tiles);
  if (t.h_force) cudaFreeHost(t.h_force);
  if (t.ev) cudaEventDestroy(t.ev);
  t = TickSlot{};
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
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking);
  for (int k = 0; k < 2 && e == cudaSuccess; ++k) e = cudaEventCreateWithFlags(&s->slot[k].ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cudaFree(s->arena_ptr);
    for (TickSlot &t : s->slot) free_slot(t);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->upload) cudaStreamDestroy(s->upload);
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
  if (s->upload) cudaStreamSynchronize(s->upload);
  for (auto &kv : s->reqs) drop_amr(kv.second);
  cudaFree(s->arena_ptr);
  for (TickSlot &t : s->slot) free_slot(t);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->upload) cudaStreamDestroy(s->upload);
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
  const int kind = (int64_t)cfg->nx * cfg->ny * cfg->nz >= kStreamCells ? 2 : 0;
  int64_t bytes = 0;
  if (kind == 2) {
    StepParams sp{};
    bytes = streamed_bytes(*cfg, streamed_params(*cfg, sp));
  } else {
    StepParams tmp{};
    fill_step_params(*cfg, 1, 0, tmp);
    bytes = request_bytes(*cfg, force_tiles(*cfg, tmp));
  }
  if (bytes > s->budget)
    return sfail(s, LBM_ENOSPC, "request needs " + std::to_string(bytes) + " bytes, more than the whole budget");
  Request r;
  r.id = id;
  r.kind = kind;
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
  // 1. retire what the finished ticks completed (no waiting)
  int rc = complete_ticks(s, false);
  if (rc) return rc;
  // 2. admit: FIFO while the head fits, or the least total work first;
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
    rc = admit(s, r, ok);
    if (rc) return rc;
    if (!ok) break;
    resident += request_cells(r);
    s->queue.pop_front();
  }
  // 3. fill the free tick slots (oldest first), so that a tick is queued
  // behind the one the host is about to wait for
  for (int n = 0; n < 2; ++n) {
    int si = -1;
    for (int k = 0; k < 2; ++k)
      if (!s->slot[k].busy) si = k;
    if (si < 0) break;
    const int64_t before = s->tick_seq;
    rc = enqueue_tick(s, si, max_steps);
    if (rc) return rc;
    if (s->tick_seq == before) break;  // nothing left to step
  }
  // 4. nothing to report yet: wait for the oldest tick in flight
  if (s->ready.empty()) {
    rc = complete_ticks(s, true);
    if (rc) return rc;
  }
  int nd = 0;
  while (!s->ready.empty() && done && nd < max_done) {
    const Request &r = s->reqs[s->ready.front()];
    s->ready.pop_front();
    lbm_result &o = done[nd++];
    o.id = r.id;
    o.status = 0;
    o.steps = r.enq;
    for (int j = 0; j < 6; ++j) o.forces[j] = r.force[j];
    o.submit_s = r.t_submit;
    o.admit_s = r.t_admit;
    o.done_s = r.t_done;
  }
  if (n_done) *n_done = nd;
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
  // a retired request's work is complete; its own stream (kind 2) is idle
  cudaStream_t st = r.kind == 2 ? r.own : s->stream;
  if (f) {
    if (r.cfg.storage != LBM_STORE_FP32)
      return sfail(s, LBM_ENOTSUP, "reading packed-storage f from the server is not supported; read mac");
    SCK(s, cudaMemcpyAsync(f, r.f[r.cur], (size_t)r.cfg.q * n * 4, cudaMemcpyDeviceToHost, st));
  }
  if (mac) SCK(s, cudaMemcpyAsync(mac, r.mac, n * 16, cudaMemcpyDeviceToHost, st));
  SCK(s, cudaStreamSynchronize(st));
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
    // retired: its last tick is complete, no queued work reads its memory
    drop_amr(it->second);
    s->arena.release(it->second.off, it->second.bytes);
    s->ready.erase(std::remove(s->ready.begin(), s->ready.end(), id), s->ready.end());
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
