// The reference's AMR host rules (amr2d.mjs, card-params.mjs) as pure C
// functions: level tau chain, the non-equilibrium transfer factors, the
// deterministic free-list grant/release order, the active-slot list and the
// 2:1 cascade closure. The device manager (amr2d.cu) applies the same grant
// and release order; these are the specification it is tested against.
// The cascade closure also runs on the device (lbm_cascade21_device), as the
// reference's amr_cascade.wgsl does, and is tested against the host rule.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lbm.h"

namespace {

// amr_cascade.wgsl:114-129 completeQuads: a wanted block at level m >= 2
// wants its whole quad (tiles are granted in quads). Every write is "= 1",
// so threads writing the same byte agree and the order does not matter.
__global__ void cascade_complete_quads(uint8_t *__restrict__ want, int nbx, int nby) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbx * nby || !want[b]) return;
  const int bx = b % nbx, by = b / nbx;
  const int qx0 = bx & ~1, qy0 = by & ~1;
  for (int k = 0; k < 4; ++k) want[(qy0 + (k >> 1)) * nbx + qx0 + (k & 1)] = 1;
}

// amr_cascade.wgsl:138-157 balance: a wanted block at level m wants the
// parents of itself and of its 8 periodic neighbours at level m - 1 (a
// different array, so the pass has no read/write hazard).
__global__ void cascade_balance(const uint8_t *__restrict__ want, uint8_t *__restrict__ parent, int nbx, int nby) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbx * nby || !want[b]) return;
  const int bx = b % nbx, by = b / nbx;
  const int pbx = nbx >> 1;
  for (int k = 0; k < 9; ++k) {
    const int nx = (bx + nbx + k % 3 - 1) % nbx, ny = (by + nby + k / 3 - 1) % nby;
    parent[(ny >> 1) * pbx + (nx >> 1)] = 1;
  }
}

}  // namespace

extern "C" {

double lbm_tau_at_level(double tau0, int m) {
  double t = tau0;
  for (int i = 0; i < m; ++i) t = 2.0 * t - 0.5;
  return t;
}

double lbm_trt_tau_minus(double tau_plus, double lambda) { return 0.5 + lambda / (tau_plus - 0.5); }

double lbm_trt_lambda(double tau_plus, double tau_minus) { return (tau_plus - 0.5) * (tau_minus - 0.5); }

double lbm_dc_rescale_c2f(double tau_coarse, double tau_fine) {
  return 0.5 * (tau_fine - 1.0) / (tau_coarse - 1.0);
}

double lbm_dc_rescale_f2c(double tau_coarse, double tau_fine) {
  return 2.0 * (tau_coarse - 1.0) / (tau_fine - 1.0);
}

int lbm_tau_chain_singularity(double tau0, int levels, double band) {
  for (int m = 0; m < levels; ++m)
    if (std::fabs(lbm_tau_at_level(tau0, m) - 1.0) < band) return m;
  return -1;
}

int lbm_grant_assignment(const int32_t *candidates, int n, int free_count, int32_t *granted_ids,
                         int32_t *granted_free_index, int32_t *n_granted) {
  std::vector<int32_t> ids(candidates, candidates + (n > 0 ? n : 0));
  std::sort(ids.begin(), ids.end());
  int count = free_count, g = 0;
  for (size_t k = 0; k < ids.size(); ++k) {
    if (granted_ids) granted_ids[k] = ids[k];
    if (count <= 0) {
      if (granted_free_index) granted_free_index[k] = -1;
      continue;
    }
    count -= 1;
    if (granted_free_index) granted_free_index[k] = count;
    ++g;
  }
  if (n_granted) *n_granted = g;
  return count;
}

int lbm_release_assignment(const int32_t *releases, int n, int free_count, int32_t *ids, int32_t *free_index) {
  std::vector<int32_t> r(releases, releases + (n > 0 ? n : 0));
  std::sort(r.begin(), r.end());
  for (size_t j = 0; j < r.size(); ++j) {
    if (ids) ids[j] = r[j];
    if (free_index) free_index[j] = free_count + (int32_t)j;
  }
  return free_count + (int)r.size();
}

int lbm_active_slot_list(const int32_t *slot_to_block, int nslots, int32_t *out) {
  int k = 0;
  for (int s = 0; s < nslots; ++s)
    if (slot_to_block[s] >= 0) out[k++] = s;
  return k;
}

int lbm_cascade21(uint8_t **want, int levels, int nbx1, int nby1) {
  if (!want || levels < 2 || nbx1 <= 0 || nby1 <= 0) return LBM_EINVAL;
  int added = 0;
  auto nbx = [&](int m) { return nbx1 << (m - 1); };
  auto nby = [&](int m) { return nby1 << (m - 1); };
  // ensure(m, b): mark block b at level m, and at m >= 2 its three siblings
  // too (quads are granted whole).
  auto ensure = [&](int m, int bx, int by) {
    if (m < 1) return;
    const int px = bx >> 1, py = by >> 1;
    const int n = m >= 2 ? 4 : 1;
    for (int k = 0; k < n; ++k) {
      const int cx = m >= 2 ? px * 2 + (k & 1) : bx;
      const int cy = m >= 2 ? py * 2 + ((k >> 1) & 1) : by;
      uint8_t &w = want[m][cy * nbx(m) + cx];
      if (!w) {
        w = 1;
        ++added;
      }
    }
  };
  for (int m = levels - 1; m >= 2; --m) {
    const int W = nbx(m), H = nby(m);
    std::vector<int> wanted;
    for (int i = 0; i < W * H; ++i)
      if (want[m][i]) wanted.push_back(i);
    for (int id : wanted) ensure(m, id % W, id / W);
    for (int id = 0; id < W * H; ++id) {
      if (!want[m][id]) continue;
      const int bx = id % W, by = id / W;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int nx = ((bx + dx) % W + W) % W, ny = ((by + dy) % H + H) % H;
          ensure(m - 1, nx >> 1, ny >> 1);
        }
    }
  }
  return added;
}

int lbm_cascade21_device(uint8_t **want, int levels, int nbx1, int nby1, void *cuda_stream) {
  if (!want || levels < 2 || nbx1 <= 0 || nby1 <= 0) return LBM_EINVAL;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  std::vector<size_t> off(levels + 1, 0);
  for (int m = 1; m < levels; ++m) {
    if (!want[m]) return LBM_EINVAL;
    off[m + 1] = off[m] + (size_t)(nbx1 << (m - 1)) * (size_t)(nby1 << (m - 1));
  }
  const size_t total = off[levels];
  uint8_t *d = nullptr;
  if (cudaMallocAsync((void **)&d, total, st) != cudaSuccess) return LBM_ENOMEM;
  cudaError_t e = cudaSuccess;
  for (int m = 1; m < levels && !e; ++m)
    e = cudaMemcpyAsync(d + off[m], want[m], off[m + 1] - off[m], cudaMemcpyHostToDevice, st);
  // one sweep, deepest first (amr_cascade.wgsl: the rule only propagates
  // down the levels, so this is the fixed point)
  for (int m = levels - 1; m >= 2 && !e; --m) {
    const int W = nbx1 << (m - 1), H = nby1 << (m - 1);
    const int grid = (W * H + 127) / 128;
    cascade_complete_quads<<<grid, 128, 0, st>>>(d + off[m], W, H);
    cascade_balance<<<grid, 128, 0, st>>>(d + off[m], d + off[m - 1], W, H);
    e = cudaGetLastError();
  }
  std::vector<uint8_t> out(total);
  if (!e) e = cudaMemcpyAsync(out.data(), d, total, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (!e) e = cudaStreamSynchronize(st);
  if (e) return LBM_ECUDA;
  int added = 0;
  for (int m = 1; m < levels; ++m)
    for (size_t i = 0; i < off[m + 1] - off[m]; ++i) {
      const uint8_t v = out[off[m] + i] ? 1 : 0;
      added += v && !want[m][i];
      want[m][i] = v;
    }
  return added;
}

}  // extern "C"
