// Batched form: many independent domains of uneven sizes advanced by ONE
// persistent launch per step, replayed from a CUDA graph.
//
// All domains of a batch share one arena of Q planes (plane stride = total
// cells), each domain a contiguous run of cells at its own base. The work is
// a list of equal tiles (domain, first cell) of THREADS * cpt cells; a grid
// of ctas_per_sm * SMs CTAs walks the list round-robin, loads the tile's
// domain constants into shared memory and runs the same per-cell update the
// dense solver uses (cell3 / cell2), so a domain stepped in a batch is
// bit-identical to the same domain stepped alone. Body forces are reduced
// per domain over the contiguous tile range that can see the body, with the
// same deterministic last-block finish as the dense step.
//
// The tile shape (THREADS, cells per thread, CTAs per SM) is picked by a
// small autotuner that times each candidate on the batch itself, stepping
// from the current state into the spare buffer so the state is unchanged.
//
// Reference: the reference has no batched form; every domain it steps is
// one page with its own dispatches (main-3d.js encodeSteps).

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lbm.h"
#include "cell_update.cuh"
#include "dense.cuh"
#include "host_params.cuh"

namespace lbm {

namespace {

// Register budget for 768 resident threads per SM (85 per thread): the
// loop over a tile's cells is latency-bound, and occupancy is what hides it.
// The CTA's share of the tiles: positions k0 .. k1-1 of `order` (tile
// indices; the identity when NULL), round-robin over the grid.
template <int Q, typename S, int THREADS>
__global__ void __launch_bounds__(THREADS, 768 / THREADS)
    batch_step(const S *__restrict__ fin, S *__restrict__ fout, float *__restrict__ mac,
               const StepParams *__restrict__ doms, const int2 *__restrict__ tiles, const int *__restrict__ order,
               int k0, int k1, int cells_per_tile, int write_mac) {
  __shared__ __align__(16) unsigned char sp_raw[sizeof(StepParams)];
  StepParams &sp = *reinterpret_cast<StepParams *>(sp_raw);
  for (int k = k0 + (int)blockIdx.x; k < k1; k += gridDim.x) {
    const int t = order ? __ldg(order + k) : k;
    const int2 td = __ldg(&tiles[t]);
    const int *src = reinterpret_cast<const int *>(doms + td.x);
    int *dst = reinterpret_cast<int *>(sp_raw);
    for (int k = threadIdx.x; k < (int)(sizeof(StepParams) / 4); k += THREADS) dst[k] = __ldg(src + k);
    __syncthreads();
    if (threadIdx.x == 0) sp.write_mac = write_mac;
    __syncthreads();
    const int nx = sp.nx, ny = sp.ny;
    const int ncell = nx * ny * sp.nz;
    const int end = min(td.y + cells_per_tile, ncell);
    const int lt = t - sp.tile0;
    const bool region = sp.force_on && lt >= sp.ft0 && lt < sp.ft1;
    ForceAcc acc;
    if constexpr (Q == 9) {
      // two cells per pass, both gathers issued before either update, so a
      // thread keeps 18 loads in flight
      for (int c = td.y + threadIdx.x; c < end; c += 2 * THREADS) {
        const int c2 = c + THREADS;
        const bool two = c2 < end;
        const int x = c % nx, r = c / nx;
        const int x2 = two ? c2 % nx : 0, r2 = two ? c2 / nx : 0;
        float f[9], g[9];
        gather2<S>(fin + sp.base, sp, x, r, f);
        if (two) gather2<S>(fin + sp.base, sp, x2, r2, g);
        CellForce cf;
        cell2_core<S>(fin, f, fout, mac, sp, x, r, region, cf);
        if (region) acc.add(cf);
        if (two) {
          CellForce cf2;
          cell2_core<S>(fin, g, fout, mac, sp, x2, r2, region, cf2);
          if (region) acc.add(cf2);
        }
      }
    } else {
      for (int c = td.y + threadIdx.x; c < end; c += THREADS) {
        const int x = c % nx, r = c / nx;
        CellForce cf;
        cell3_any<Q, S>(fin, fout, mac, sp, x, r % ny, r / ny, region, cf);
        if (region) acc.add(cf);
      }
    }
    if (region)
      reduce_force<THREADS>(acc, sp.partials, sp.counter, sp.ft1 - sp.ft0, lt - sp.ft0, sp.force_out);
    __syncthreads();
  }
}

// One D2Q9 cell of a domain with no body and outside any force region:
// cell2_core with the tests that cannot fire taken out (no solid link,
// chi = 0 and u_s = 0, so the Guo force is the body force) and only the
// moving-wall patch of a wall row kept, the same arithmetic in the same
// order, so the same bits.
template <typename S>
__device__ __forceinline__ void cell2_fluid(const S *__restrict__ fin, float (&f)[9], S *__restrict__ fout,
                                            float *__restrict__ mac, const StepParams &p, int x, int y) {
  using L = Lattice<9>;
  const int W = p.nx, H = p.ny;
  const int cell = y * W + x;
  if (p.wall_y && (y == 0 || y == H - 1)) {
    const S *fi = fin + p.base;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const int ex = L::ex(i), ey = L::ey(i), o = L::opp(i);
      const int ysrc = y - ey;
      if (ysrc < 0 || ysrc >= H) {
        const float wu = ysrc < 0 ? p.wall_u0 : p.wall_u1;
        const float corr = 2.f * L::w(i) * (float)ex * wu * kInvCS2;
        f[i] = Codec<S>::ld(fi + (int64_t)o * p.n + cell, o, p.pk) + corr;
      }
    }
  }
  float rho, mxs, mys, mzs;
  moments<L, 9>(f, rho, mxs, mys, mzs);
  const float rhoDen = fmaxf(rho, 1e-6f);
  const float inv = 1.0f / rhoDen;
  const float uxs = mxs * inv, uys = mys * inv;
  const float chi = 0.f, usx = 0.f, usy = 0.f;
  const float Fx = rho * chi * (usx - uxs) + p.fx;
  const float Fy = rho * chi * (usy - uys) + p.fy;
  const float hinv = 0.5f * inv;
  const float ux = fmaf(Fx, hinv, uxs);
  const float uy = fmaf(Fy, hinv, uys);
  float spw = 0.f;
  if (p.sponge_w > 0.f) {
    const float dx = fminf((float)x, (float)(W - 1 - x));
    const float dy = fminf((float)y, (float)(H - 1 - y));
    spw = sponge_weight_inv(fminf(dx, dy), p.sponge_inv);
  }
  MemSink<S> sink{fout + p.base, p.n, cell, p.pk};
  collide_store<L, 9>(f, rho, ux, uy, 0.f, Fx, Fy, 0.f, p.omega, spw, p.ftarget, sink);
  if (p.write_mac) reinterpret_cast<float4 *>(mac + 4 * p.base)[cell] = make_float4(rho, ux, uy, 0.f);
}

// The fluid tiles of a D2Q9 batch (cell2_fluid). Without the bounce-back
// and force code the update fits 64 registers, and 1024 resident
// threads per SM keep more loads in flight: the loop is memory-latency
// bound (measured on B200 for the 512-domain workload: 0.53 ms per step
// with every tile on the general kernel, 0.48 ms with the lean one).
// (16-bit storage decodes and encodes each population: it keeps 80
// registers, 768 threads per SM, where 64 would spill.)
template <typename S, int THREADS>
__global__ void __launch_bounds__(THREADS, (sizeof(S) == 4 ? 1024 : 768) / THREADS)
    batch_step_fluid2(const S *__restrict__ fin, S *__restrict__ fout, float *__restrict__ mac,
                      const StepParams *__restrict__ doms, const int2 *__restrict__ tiles,
                      const int *__restrict__ order, int k0, int k1, int cells_per_tile, int write_mac) {
  __shared__ __align__(16) unsigned char sp_raw[sizeof(StepParams)];
  StepParams &sp = *reinterpret_cast<StepParams *>(sp_raw);
  for (int k = k0 + (int)blockIdx.x; k < k1; k += gridDim.x) {
    const int2 td = __ldg(&tiles[__ldg(order + k)]);
    const int *src = reinterpret_cast<const int *>(doms + td.x);
    int *dst = reinterpret_cast<int *>(sp_raw);
    for (int j = threadIdx.x; j < (int)(sizeof(StepParams) / 4); j += THREADS) dst[j] = __ldg(src + j);
    __syncthreads();
    if (threadIdx.x == 0) sp.write_mac = write_mac;
    __syncthreads();
    const int nx = sp.nx;
    const int end = min(td.y + cells_per_tile, nx * sp.ny);
    // two cells per pass, both gathers issued before either update
    for (int c = td.y + threadIdx.x; c < end; c += 2 * THREADS) {
      const int c2 = c + THREADS;
      const bool two = c2 < end;
      const int x = c % nx, r = c / nx;
      const int x2 = two ? c2 % nx : 0, r2 = two ? c2 / nx : 0;
      float f[9], g[9];
      gather2<S>(fin + sp.base, sp, x, r, f);
      if (two) gather2<S>(fin + sp.base, sp, x2, r2, g);
      cell2_fluid<S>(fin, f, fout, mac, sp, x, r);
      if (two) cell2_fluid<S>(fin, g, fout, mac, sp, x2, r2);
    }
    __syncthreads();
  }
}

using BatchFn = void (*)(const void *, void *, float *, const StepParams *, const int2 *, int, int, int);

template <int Q, typename S, int T>
void launch_batch(dim3 g, cudaStream_t st, const void *fin, void *fout, float *mac, const StepParams *d,
                  const int2 *tiles, const int *order, int k0, int k1, int cpt, int wm, bool fluid) {
  if constexpr (Q == 9) {
    if (fluid) {
      batch_step_fluid2<S, T><<<g, T, 0, st>>>((const S *)fin, (S *)fout, mac, d, tiles, order, k0, k1, cpt, wm);
      return;
    }
  }
  batch_step<Q, S, T><<<g, T, 0, st>>>((const S *)fin, (S *)fout, mac, d, tiles, order, k0, k1, cpt, wm);
}

template <int T>
cudaError_t launch_any(int q, int storage, dim3 g, cudaStream_t st, const void *fin, void *fout, float *mac,
                       const StepParams *d, const int2 *tiles, const int *order, int k0, int k1, int cpt, int wm,
                       bool fluid) {
  switch (q * 4 + storage) {
    case 9 * 4 + 0: launch_batch<9, float, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, fluid); break;
    case 9 * 4 + 1: launch_batch<9, __half, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, fluid); break;
    case 9 * 4 + 2:
      launch_batch<9, __nv_bfloat16, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, fluid);
      break;
    case 19 * 4 + 0: launch_batch<19, float, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, false); break;
    case 19 * 4 + 1: launch_batch<19, __half, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, false); break;
    case 19 * 4 + 2:
      launch_batch<19, __nv_bfloat16, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, false);
      break;
    case 27 * 4 + 0: launch_batch<27, float, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, false); break;
    case 27 * 4 + 1: launch_batch<27, __half, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, false); break;
    case 27 * 4 + 2:
      launch_batch<27, __nv_bfloat16, T>(g, st, fin, fout, mac, d, tiles, order, k0, k1, cpt, wm, false);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

// One launch over tile positions k0 .. k1-1 of `order`; `fluid` picks the
// lean D2Q9 kernel for tiles the host classified as fluid.
cudaError_t launch_batch_step(int q, int storage, int threads, int ctas, cudaStream_t st, const void *fin,
                              void *fout, float *mac, const StepParams *doms, const int2 *tiles, const int *order,
                              int k0, int k1, int cells_per_tile, int write_mac, bool fluid) {
  dim3 g(ctas);
  if (k1 <= k0) return cudaSuccess;
  if (threads == 128)
    return launch_any<128>(q, storage, g, st, fin, fout, mac, doms, tiles, order, k0, k1, cells_per_tile, write_mac,
                           fluid);
  if (threads == 256)
    return launch_any<256>(q, storage, g, st, fin, fout, mac, doms, tiles, order, k0, k1, cells_per_tile, write_mac,
                           fluid);
  return cudaErrorInvalidValue;
}

}  // namespace lbm

// ---- C ABI ---------------------------------------------------------------------

using namespace lbm;

struct lbm_batch {
  int q = 0, storage = 0, elem = 4, ndom = 0;
  std::vector<lbm_config> cfg;
  std::vector<int64_t> base;     // arena index of each domain's cell 0
  std::vector<int64_t> ncell;
  int64_t total = 0;
  void *f[2] = {nullptr, nullptr};
  int cur = 0;
  float *mac = nullptr;
  StepParams *d_doms = nullptr;
  std::vector<StepParams> h_doms;
  int2 *d_tiles = nullptr;
  int ntiles = 0;
  int *d_order = nullptr;        // tile indices: the general tiles, then the fluid ones
  int ngeneral = 0;
  double *partials = nullptr;
  int64_t npartials = 0;
  unsigned int *counters = nullptr;
  double *force_out = nullptr;
  double *tot_partials = nullptr;
  unsigned int *tot_counter = nullptr;
  double *tot_out = nullptr;
  double *host = nullptr;        // pinned readback scratch
  int threads = 256, cpt = 4, ctas_per_sm = 4, sms = 148;
  cudaStream_t own = nullptr, stream = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // kGraphSteps steps from buffer 0 / 1, no mac
  std::string err;
  int64_t bytes = 0;
};

namespace {

constexpr int kGraphSteps = 16;

int bfail(lbm_batch *b, int code, const std::string &m) {
  if (b) b->err = m;
  return code;
}

#define BCK(b, call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return bfail(b, e_ == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA,        \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

thread_local std::string g_batch_error;

void drop_graphs(lbm_batch *b) {
  for (auto &g : b->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

// (Re)builds the tile list and the per-domain force tile ranges for the
// current tiling, and uploads the domain descriptors.
int retile(lbm_batch *b) {
  drop_graphs(b);
  const int cells_per_tile = b->threads * b->cpt;
  std::vector<int2> tiles;
  int64_t parts = 0;
  std::vector<int64_t> part_off(b->ndom, 0);
  for (int d = 0; d < b->ndom; ++d) {
    StepParams &p = b->h_doms[d];
    const int nt = (int)((b->ncell[d] + cells_per_tile - 1) / cells_per_tile);
    p.tile0 = (int)tiles.size();
    for (int k = 0; k < nt; ++k) tiles.push_back(make_int2(d, k * cells_per_tile));
    int box[6];
    p.force_on = force_cell_box(b->cfg[d], p, box) ? 1 : 0;
    if (p.force_on) {
      const int64_t first = ((int64_t)box[4] * p.ny + box[2]) * p.nx + box[0];
      const int64_t last = ((int64_t)box[5] * p.ny + box[3]) * p.nx + box[1];
      p.ft0 = (int)(first / cells_per_tile);
      p.ft1 = (int)(last / cells_per_tile) + 1;
      part_off[d] = parts;
      parts += p.ft1 - p.ft0;
    } else {
      p.ft0 = p.ft1 = 0;
    }
  }
  if (tiles.size() > 0x7fffffff) return bfail(b, LBM_EINVAL, "too many tiles");
  // D2Q9 tiles that need none of the bounce-back and force code run the
  // lean kernel: no body, no force region (walls it handles).
  std::vector<int> general, fluid;
  for (int t = 0; t < (int)tiles.size(); ++t) {
    const StepParams &p = b->h_doms[tiles[t].x];
    (b->q == 9 && !p.has_body && !p.force_on ? fluid : general).push_back(t);
  }
  b->ngeneral = (int)general.size();
  general.insert(general.end(), fluid.begin(), fluid.end());
  cudaFree(b->d_order);
  b->d_order = nullptr;
  BCK(b, cudaMalloc(&b->d_order, general.size() * sizeof(int)));
  BCK(b, cudaMemcpy(b->d_order, general.data(), general.size() * sizeof(int), cudaMemcpyHostToDevice));
  cudaFree(b->d_tiles);
  b->d_tiles = nullptr;
  BCK(b, cudaMalloc(&b->d_tiles, tiles.size() * sizeof(int2)));
  BCK(b, cudaMemcpy(b->d_tiles, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
  b->ntiles = (int)tiles.size();
  if (parts > b->npartials) {
    cudaFree(b->partials);
    b->partials = nullptr;
    BCK(b, cudaMalloc(&b->partials, (size_t)parts * kForceSlots * sizeof(double)));
    b->npartials = parts;
  }
  for (int d = 0; d < b->ndom; ++d) {
    StepParams &p = b->h_doms[d];
    p.partials = b->partials + part_off[d] * kForceSlots;
    p.counter = b->counters + d;
    p.force_out = b->force_out + (int64_t)d * kForceSlots;
  }
  BCK(b, cudaMemcpy(b->d_doms, b->h_doms.data(), b->ndom * sizeof(StepParams), cudaMemcpyHostToDevice));
  return LBM_OK;
}

// A step: the general tiles, then the fluid ones (their cells are disjoint;
// both read the step's input buffer and write its output).
cudaError_t one_step(lbm_batch *b, cudaStream_t st, int from, int write_mac) {
  const int ctas = b->ctas_per_sm * b->sms, cpt = b->threads * b->cpt;
  cudaError_t e = launch_batch_step(b->q, b->storage, b->threads, ctas, st, b->f[from], b->f[1 - from], b->mac,
                                    b->d_doms, b->d_tiles, b->d_order, 0, b->ngeneral, cpt, write_mac, false);
  if (e != cudaSuccess) return e;
  return launch_batch_step(b->q, b->storage, b->threads, ctas, st, b->f[from], b->f[1 - from], b->mac, b->d_doms,
                           b->d_tiles, b->d_order, b->ngeneral, b->ntiles, cpt, write_mac, true);
}

int build_graph(lbm_batch *b, int from) {
  cudaStream_t cs;
  BCK(b, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  int k = 0;
  for (; e == cudaSuccess && k < kGraphSteps; ++k) e = one_step(b, cs, (from + k) & 1, 0);
  cudaError_t e2 = cudaStreamEndCapture(cs, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph[from], g, 0);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) return bfail(b, LBM_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  return LBM_OK;
}

void release_batch(lbm_batch *b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  cudaFree(b->f[0]);
  cudaFree(b->f[1]);
  cudaFree(b->mac);
  cudaFree(b->d_doms);
  cudaFree(b->d_tiles);
  cudaFree(b->d_order);
  cudaFree(b->partials);
  cudaFree(b->counters);
  cudaFree(b->force_out);
  cudaFree(b->tot_partials);
  cudaFree(b->tot_counter);
  cudaFree(b->tot_out);
  if (b->host) cudaFreeHost(b->host);
  if (b->own) cudaStreamDestroy(b->own);
}

bool dom_ok(lbm_batch *b, int d) { return b && d >= 0 && d < b->ndom; }

}  // namespace

extern "C" {

int lbm_batch_create(const lbm_config *doms, int ndomains, lbm_batch **out) {
  if (!out) return LBM_EINVAL;
  *out = nullptr;
  if (!doms || ndomains <= 0) {
    g_batch_error = "need at least one domain";
    return LBM_EINVAL;
  }
  for (int d = 0; d < ndomains; ++d) {
    std::string why;
    if (validate_config(&doms[d], why)) {
      g_batch_error = "domain " + std::to_string(d) + ": " + why;
      return LBM_EINVAL;
    }
    if (doms[d].window[0] || doms[d].window[1] || doms[d].window[2]) {
      g_batch_error = "domain " + std::to_string(d) + ": the moving window runs in dense sessions and 3D AMR";
      return LBM_ENOTSUP;
    }
    if (doms[d].q != doms[0].q || doms[d].storage != doms[0].storage) {
      g_batch_error = "all domains of a batch must share q and storage";
      return LBM_EINVAL;
    }
  }
  lbm_batch *b = new lbm_batch();
  b->q = doms[0].q;
  b->storage = doms[0].storage;
  b->elem = b->storage == LBM_STORE_FP32 ? 4 : 2;
  b->ndom = ndomains;
  b->cfg.assign(doms, doms + ndomains);
  for (int d = 0; d < ndomains; ++d) {
    const int64_t n = (int64_t)doms[d].nx * doms[d].ny * doms[d].nz;
    b->base.push_back(b->total);
    b->ncell.push_back(n);
    b->total += n;
  }
  auto bail = [&](int code) {
    g_batch_error = b->err;
    release_batch(b);
    delete b;
    return code;
  };
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e;
  auto need = [&](cudaError_t r, const char *what) {
    if (r != cudaSuccess) b->err = std::string(what) + ": " + cudaGetErrorString(r);
    return r;
  };
  const size_t fbytes = (size_t)b->q * b->total * b->elem;
  if ((e = need(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking), "stream")) ||
      (e = need(cudaMalloc(&b->f[0], fbytes), "cudaMalloc f[0]")) ||
      (e = need(cudaMalloc(&b->f[1], fbytes), "cudaMalloc f[1]")) ||
      (e = need(cudaMalloc(&b->mac, (size_t)b->total * 16), "cudaMalloc mac")) ||
      (e = need(cudaMalloc(&b->d_doms, ndomains * sizeof(StepParams)), "cudaMalloc domains")) ||
      (e = need(cudaMalloc(&b->counters, ndomains * sizeof(unsigned int)), "cudaMalloc counters")) ||
      (e = need(cudaMalloc(&b->force_out, (size_t)ndomains * kForceSlots * sizeof(double)), "cudaMalloc force")) ||
      (e = need(cudaMalloc(&b->tot_partials, (size_t)totals_blocks() * kTotalsSlots * sizeof(double)), "cudaMalloc totals")) ||
      (e = need(cudaMalloc(&b->tot_counter, sizeof(unsigned int)), "cudaMalloc counter")) ||
      (e = need(cudaMalloc(&b->tot_out, kTotalsSlots * sizeof(double)), "cudaMalloc totals")) ||
      (e = need(cudaMallocHost(&b->host, (size_t)std::max(16, 8 * ndomains) * sizeof(double)), "cudaMallocHost")))
    return bail(e == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA);
  b->stream = b->own;
  cudaMemset(b->counters, 0, ndomains * sizeof(unsigned int));
  cudaMemset(b->tot_counter, 0, sizeof(unsigned int));
  cudaMemset(b->force_out, 0, (size_t)ndomains * kForceSlots * sizeof(double));
  cudaMemset(b->f[0], 0, fbytes);
  cudaMemset(b->mac, 0, (size_t)b->total * 16);
  b->h_doms.resize(ndomains);
  for (int d = 0; d < ndomains; ++d) fill_step_params(b->cfg[d], b->total, b->base[d], b->h_doms[d]);
  if (retile(b)) return bail(LBM_ECUDA);
  b->bytes = 2 * (int64_t)fbytes + b->total * 16;
  *out = b;
  return LBM_OK;
}

void lbm_batch_destroy(lbm_batch *b) {
  release_batch(b);
  delete b;
}

const char *lbm_batch_last_error(const lbm_batch *b) { return b ? b->err.c_str() : g_batch_error.c_str(); }

int lbm_batch_set_stream(lbm_batch *b, void *stream) {
  if (!b) return LBM_EINVAL;
  BCK(b, cudaStreamSynchronize(b->stream));
  b->stream = stream ? (cudaStream_t)stream : b->own;
  return LBM_OK;
}

int lbm_batch_domains(const lbm_batch *b) { return b ? b->ndom : 0; }
int64_t lbm_batch_cells(const lbm_batch *b) { return b ? b->total : 0; }

int lbm_batch_init_macro(lbm_batch *b, int d, const float *mac) {
  if (!dom_ok(b, d) || !mac) return b ? bfail(b, LBM_EINVAL, "bad domain or NULL mac") : LBM_EINVAL;
  float *m = b->mac + 4 * b->base[d];
  BCK(b, cudaMemcpyAsync(m, mac, (size_t)b->ncell[d] * 16, cudaMemcpyHostToDevice, b->stream));
  // Seed into a domain-sized view of the current buffer: plane stride is the
  // arena's, so seed each plane through the equilibrium kernel on a
  // temporary and scatter (domain planes are not contiguous in the arena).
  const size_t fb = (size_t)b->q * b->ncell[d] * b->elem;
  void *tmp = nullptr;
  BCK(b, cudaMallocAsync(&tmp, fb, b->stream));
  cudaError_t e = launch_init_eq(b->q, b->storage, m, tmp, b->ncell[d], b->h_doms[d].pk, b->stream);
  for (int i = 0; e == cudaSuccess && i < b->q; ++i)
    e = cudaMemcpyAsync((char *)b->f[b->cur] + ((size_t)i * b->total + b->base[d]) * b->elem,
                        (char *)tmp + (size_t)i * b->ncell[d] * b->elem, (size_t)b->ncell[d] * b->elem,
                        cudaMemcpyDeviceToDevice, b->stream);
  cudaFreeAsync(tmp, b->stream);
  if (e) return bfail(b, LBM_ECUDA, std::string("init: ") + cudaGetErrorString(e));
  BCK(b, cudaStreamSynchronize(b->stream));
  return LBM_OK;
}

int lbm_batch_write_f(lbm_batch *b, int d, const float *f) {
  if (!dom_ok(b, d) || !f) return b ? bfail(b, LBM_EINVAL, "bad domain or NULL f") : LBM_EINVAL;
  const int64_t n = b->ncell[d];
  void *tmp = nullptr;
  float *t32 = nullptr;
  BCK(b, cudaMallocAsync(&t32, (size_t)b->q * n * 4, b->stream));
  BCK(b, cudaMallocAsync(&tmp, (size_t)b->q * n * b->elem, b->stream));
  cudaError_t e = cudaMemcpyAsync(t32, f, (size_t)b->q * n * 4, cudaMemcpyHostToDevice, b->stream);
  if (!e) e = launch_pack(b->q, b->storage, t32, tmp, n, b->h_doms[d].pk, b->stream);
  for (int i = 0; e == cudaSuccess && i < b->q; ++i)
    e = cudaMemcpyAsync((char *)b->f[b->cur] + ((size_t)i * b->total + b->base[d]) * b->elem,
                        (char *)tmp + (size_t)i * n * b->elem, (size_t)n * b->elem, cudaMemcpyDeviceToDevice,
                        b->stream);
  cudaFreeAsync(t32, b->stream);
  cudaFreeAsync(tmp, b->stream);
  if (e) return bfail(b, LBM_ECUDA, std::string("write_f: ") + cudaGetErrorString(e));
  BCK(b, cudaStreamSynchronize(b->stream));
  return LBM_OK;
}

int lbm_batch_read_f(lbm_batch *b, int d, float *f) {
  if (!dom_ok(b, d) || !f) return b ? bfail(b, LBM_EINVAL, "bad domain or NULL f") : LBM_EINVAL;
  const int64_t n = b->ncell[d];
  void *tmp = nullptr;
  float *t32 = nullptr;
  BCK(b, cudaMallocAsync(&t32, (size_t)b->q * n * 4, b->stream));
  BCK(b, cudaMallocAsync(&tmp, (size_t)b->q * n * b->elem, b->stream));
  cudaError_t e = cudaSuccess;
  for (int i = 0; e == cudaSuccess && i < b->q; ++i)
    e = cudaMemcpyAsync((char *)tmp + (size_t)i * n * b->elem,
                        (char *)b->f[b->cur] + ((size_t)i * b->total + b->base[d]) * b->elem, (size_t)n * b->elem,
                        cudaMemcpyDeviceToDevice, b->stream);
  if (!e) e = launch_unpack(b->q, b->storage, tmp, t32, n, b->h_doms[d].pk, b->stream);
  if (!e) e = cudaMemcpyAsync(f, t32, (size_t)b->q * n * 4, cudaMemcpyDeviceToHost, b->stream);
  cudaFreeAsync(t32, b->stream);
  cudaFreeAsync(tmp, b->stream);
  if (e) return bfail(b, LBM_ECUDA, std::string("read_f: ") + cudaGetErrorString(e));
  BCK(b, cudaStreamSynchronize(b->stream));
  return LBM_OK;
}

int lbm_batch_read_mac(lbm_batch *b, int d, float *mac) {
  if (!dom_ok(b, d) || !mac) return b ? bfail(b, LBM_EINVAL, "bad domain or NULL mac") : LBM_EINVAL;
  BCK(b, cudaMemcpyAsync(mac, b->mac + 4 * b->base[d], (size_t)b->ncell[d] * 16, cudaMemcpyDeviceToHost,
                         b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  return LBM_OK;
}

int lbm_batch_step(lbm_batch *b, int n) {
  if (!b) return LBM_EINVAL;
  if (n < 0) return bfail(b, LBM_EINVAL, "step count must be >= 0");
  int left = n;
  // All but the last step run without the mac write, kGraphSteps at a time
  // from a captured graph; the last step writes mac.
  while (left > kGraphSteps) {
    if (!b->graph[b->cur]) {
      int rc = build_graph(b, b->cur);
      if (rc) return rc;
    }
    BCK(b, cudaGraphLaunch(b->graph[b->cur], b->stream));
    left -= kGraphSteps;  // kGraphSteps is even: parity unchanged
  }
  for (; left > 0; --left) {
    BCK(b, one_step(b, b->stream, b->cur, left == 1));
    b->cur = 1 - b->cur;
  }
  return LBM_OK;
}

int lbm_batch_set_tiling(lbm_batch *b, int threads, int cells_per_thread, int ctas_per_sm) {
  if (!b) return LBM_EINVAL;
  if ((threads != 128 && threads != 256) || cells_per_thread < 1 || cells_per_thread > 64 || ctas_per_sm < 1 ||
      ctas_per_sm > 32)
    return bfail(b, LBM_EINVAL, "tiling: threads 128|256, cells_per_thread 1..64, ctas_per_sm 1..32");
  BCK(b, cudaStreamSynchronize(b->stream));
  b->threads = threads;
  b->cpt = cells_per_thread;
  b->ctas_per_sm = ctas_per_sm;
  return retile(b);
}

int lbm_batch_get_tiling(const lbm_batch *b, int *threads, int *cells_per_thread, int *ctas_per_sm) {
  if (!b) return LBM_EINVAL;
  if (threads) *threads = b->threads;
  if (cells_per_thread) *cells_per_thread = b->cpt;
  if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
  return LBM_OK;
}

// Times every candidate tiling for `trials` steps from the current state into
// the spare buffer (the state and the step count do not change) and keeps
// the fastest. `best_ms` receives its time per step.
int lbm_batch_autotune(lbm_batch *b, int trials, float *best_ms) {
  if (!b) return LBM_EINVAL;
  if (trials < 1) trials = 3;
  const int thr[] = {128, 256};
  const int cpts[] = {1, 2, 4, 8, 16};
  const int ctas[] = {2, 4, 8, 16};
  cudaEvent_t a, z;
  BCK(b, cudaEventCreate(&a));
  BCK(b, cudaEventCreate(&z));
  float best = 1e30f;
  int bt = b->threads, bc = b->cpt, bs = b->ctas_per_sm;
  for (int t : thr)
    for (int c : cpts)
      for (int k : ctas) {
        b->threads = t;
        b->cpt = c;
        b->ctas_per_sm = k;
        int rc = retile(b);
        if (rc) return rc;
        BCK(b, one_step(b, b->stream, b->cur, 0));  // warm
        BCK(b, cudaEventRecord(a, b->stream));
        for (int r = 0; r < trials; ++r) BCK(b, one_step(b, b->stream, b->cur, 0));
        BCK(b, cudaEventRecord(z, b->stream));
        BCK(b, cudaEventSynchronize(z));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, z);
        ms /= trials;
        if (ms < best) { best = ms; bt = t; bc = c; bs = k; }
      }
  cudaEventDestroy(a);
  cudaEventDestroy(z);
  b->threads = bt;
  b->cpt = bc;
  b->ctas_per_sm = bs;
  if (best_ms) *best_ms = best;
  return retile(b);
}

int lbm_batch_forces(lbm_batch *b, double *out) {
  if (!b || !out) return b ? bfail(b, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  BCK(b, cudaMemcpyAsync(b->host, b->force_out, (size_t)b->ndom * kForceSlots * sizeof(double),
                         cudaMemcpyDeviceToHost, b->stream));
  BCK(b, cudaStreamSynchronize(b->stream));
  for (int d = 0; d < b->ndom; ++d)
    for (int k = 0; k < 6; ++k) out[6 * d + k] = b->h_doms[d].force_on ? b->host[kForceSlots * d + k] : 0.0;
  return LBM_OK;
}

int lbm_batch_sync(lbm_batch *b) {
  if (!b) return LBM_EINVAL;
  BCK(b, cudaStreamSynchronize(b->stream));
  return LBM_OK;
}

}  // extern "C"
