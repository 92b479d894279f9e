// The reference's AMR host rules (amr2d.mjs, card-params.mjs) as pure C
// functions: level tau chain, the non-equilibrium transfer factors, the
// deterministic free-list grant/release order, the active-slot list and the
// 2:1 cascade closure. The device manager (amr2d.cu) applies the same grant
// and release order; these are the specification it is tested against.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/lbm.h"

extern "C" {

double lbm_tau_at_level(double tau0, int m) {
  double t = tau0;
  for (int i = 0; i < m; ++i) t = 2.0 * t - 0.5;
  return t;
}

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

}  // extern "C"
