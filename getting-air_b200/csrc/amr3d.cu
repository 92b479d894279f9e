// 3D block-structured AMR, two levels, on the device: the kernels of one
// macro-step and the session behind lbm_amr3d_*.
//
// One macro-step (main-3d.js:3219-3341, ?interface=explode):
//   amr3_force     pool force on the tiles at time t (FP64, deterministic)
//   amr3_explode   L0 (time t) -> every tile's ring, Chen et al. 2006: the
//                  populations of an unrefined L0 cell V whose target V + e_i
//                  is covered, moved unchanged into V's eight fine cells
//                  (plus the linear term orthogonal to e_i), and the
//                  in-orphans of a convex edge; common_d3_amr_explode.wgsl
//   amr3_substep x2  the tiles, A then B: DIRECT_GHOST pull (a source past
//                  the interior comes from the refined neighbour's interior,
//                  else from the ring), BGK + Guo at tau_f = 2 tau - 1/2; the
//                  ring advects without colliding; common_d3_amr_step1.wgsl
//   amr3_coalesce  the tiles -> the covered L0 cells of the time-t buffer
//                  (the mean of the eight fine cells that will be pulled),
//                  the covered cells' mac, and the out/in orphan balance of
//                  unrefined cells at a seam; common_d3_amr_coalesce.wgsl
//   amr3_coarse    the dense step on L0, skipping covered blocks
//                  (common_d3_step.wgsl:110 coveredByFiner)
// All but the last macro-step of a call run from one CUDA graph per L0
// parity; the last is launched directly with the mac writes switched on.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lbm.h"
#include "amr3d.cuh"
#include "cell_update.cuh"
#include "host_params.cuh"
#include "scan.cuh"
#include "sample.cuh"

namespace lbm {

namespace {

// Periodic wrap of an index at most one period outside [0, n) -- every index
// here is a cell, block or fine coordinate a step or two past an edge --
// without an integer division.
__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ bool covered(const Amr3Params &p, int x, int y, int z) {
  x = wrapi(x, p.nx); y = wrapi(y, p.ny); z = wrapi(z, p.nz);
  return p.block_slot[((z / p.rb) * p.nby + y / p.rb) * p.nbx + x / p.rb] >= 0;
}

__device__ __forceinline__ int64_t ccell(const Amr3Params &p, int x, int y, int z) {
  return ((int64_t)wrapi(z, p.nz) * p.ny + wrapi(y, p.ny)) * p.nx + wrapi(x, p.nx);
}

__device__ __forceinline__ float f2c(int j, int origin) { return (float)origin - 0.25f + 0.5f * (float)(j - kAmrGhost); }

__device__ __forceinline__ bool interior(const Amr3Params &p, int j) { return j >= kAmrGhost && j < kAmrGhost + p.RB2; }

struct TileCell {
  int slot, bx, by, bz, fx, fy, fz;
  int64_t cell;
  int k;  // position in the tile's cell list (cell-list kernels)
};

// Tile kernels run one CTA per (fz, slot) with an FB x FB thread block, so a
// thread's tile coordinates need no division.
__device__ __forceinline__ bool tile_cell(const Amr3Params &p, TileCell &t) {
  t.slot = blockIdx.y;
  const int id = p.slot_to_block[t.slot];
  if (id < 0) return false;
  t.bx = id % p.nbx; t.by = (id / p.nbx) % p.nby; t.bz = id / (p.nbx * p.nby);
  t.fx = threadIdx.x; t.fy = threadIdx.y; t.fz = blockIdx.x;
  t.cell = (int64_t)t.slot * p.T3 + (t.fz * p.FB + t.fy) * p.FB + t.fx;
  return true;
}

// The D3Q27 directions (D3Q19 their first 19), as a table in constant
// memory for loops over a runtime direction index.
struct DirTable {
  signed char ex[27], ey[27], ez[27];
};
constexpr DirTable make_dirs() {
  DirTable t{};
  for (int i = 0; i < 27; ++i) {
    t.ex[i] = (signed char)detail::ex27(i);
    t.ey[i] = (signed char)detail::ey27(i);
    t.ez[i] = (signed char)detail::ez27(i);
  }
  return t;
}
__constant__ DirTable c_dirs = make_dirs();

// Cell-list kernels: one CTA of kListThreads per (chunk, slot) walking a
// per-session list of the tile's cells -- the interior first, then the
// ring -- so that a warp holds interior cells or ring cells, not both, and
// a ring-only pass launches no interior threads. Sets up the CTA's
// neighbour table; false for a thread with no cell (after the barrier).
constexpr int kListThreads = 128;

__device__ __forceinline__ bool list_tile(const Amr3Params &p, int *nb27, TileCell &t, bool as_base) {
  t.slot = blockIdx.y;
  const int id = p.slot_to_block[t.slot];
  if (id < 0) return false;  // the whole CTA: a free slot
  t.bx = id % p.nbx; t.by = (id / p.nbx) % p.nby; t.bz = id / (p.nbx * p.nby);
  if (threadIdx.x < 27) {
    const int k = threadIdx.x, dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
    const int ns = k == 13 ? t.slot
                           : p.block_slot[(wrapi(t.bz + dz, p.nbz) * p.nby + wrapi(t.by + dy, p.nby)) * p.nbx +
                                          wrapi(t.bx + dx, p.nbx)];
    // as_base: the slot's first pool cell (slot * T3 < P < 2^31)
    nb27[k] = as_base && ns >= 0 ? ns * p.T3 : ns;
  }
  __syncthreads();
  return true;
}

// The cell at list position pos of the CTA's tile.
__device__ __forceinline__ void list_at(const Amr3Params &p, const uint32_t *__restrict__ cells, int pos,
                                        TileCell &t) {
  t.k = pos;
  const uint32_t c = __ldg(cells + pos);
  t.fx = c & 0xff; t.fy = (c >> 8) & 0xff; t.fz = c >> 16;
  t.cell = (int64_t)t.slot * p.T3 + (t.fz * p.FB + t.fy) * p.FB + t.fx;
}

__device__ __forceinline__ bool list_cell(const Amr3Params &p, const uint32_t *__restrict__ cells, int first,
                                          int count, int *nb27, TileCell &t, bool as_base = false) {
  if (!list_tile(p, nb27, t, as_base)) return false;
  const int k = blockIdx.x * kListThreads + threadIdx.x;
  if (k >= count) return false;
  list_at(p, cells, first + k, t);
  return true;
}

// Is L0 cell (x, y, z) -- within one L0 cell of block b's 3 x 3 x 3
// neighbourhood -- under a refined block? From the CTA's neighbour table.
__device__ __forceinline__ bool covered_near(const Amr3Params &p, const int *nb27, const int b[3], int x, int y,
                                             int z) {
  const int r[3] = {x - b[0] * p.rb, y - b[1] * p.rb, z - b[2] * p.rb};
  int k[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) k[a] = r[a] < 0 ? 0 : (r[a] >= p.rb ? 2 : 1);
  return nb27[k[2] * 9 + k[1] * 3 + k[0]] >= 0;
}

template <int Q>
__device__ __forceinline__ float feq3(int i, float rho, float ux, float uy, float uz) {
  using L = Lattice<Q>;
  const float eu = (float)L::ex(i) * ux + (float)L::ey(i) * uy + (float)L::ez(i) * uz;
  const float usq = ux * ux + uy * uy + uz * uz;
  return L::w(i) * rho * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * usq);
}

// ---- seed / fill: trilinear interpolation of L0 into a tile ----------------
// interpCoarseToFine3: rho and u interpolated, f = feq(rho, u) + DC-rescaled
// interpolated fneq (common_d3_pool.wgsl:192-220).
template <int Q>
__global__ void __launch_bounds__(kTileMaxThreads)
    amr3_interp(const float *__restrict__ fc, float *__restrict__ fp, const __grid_constant__ Amr3Params p,
                int ring_only, const unsigned char *__restrict__ only_new) {
  using L = Lattice<Q>;
  TileCell t;
  if (!tile_cell(p, t)) return;
  if (only_new && !only_new[t.slot]) return;
  if (ring_only && interior(p, t.fx) && interior(p, t.fy) && interior(p, t.fz)) return;
  const float pos[3] = {f2c(t.fx, t.bx * p.rb), f2c(t.fy, t.by * p.rb), f2c(t.fz, t.bz * p.rb)};
  int c0[3];
  float tt[3];
  for (int a = 0; a < 3; ++a) {
    c0[a] = (int)floorf(pos[a]);
    tt[a] = pos[a] - (float)c0[a];
  }
  float rho = 0.f, ux = 0.f, uy = 0.f, uz = 0.f, fneq[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) fneq[i] = 0.f;
  for (int k = 0; k < 8; ++k) {
    const int di = k & 1, dj = (k >> 1) & 1, dk = (k >> 2) & 1;
    const float w = (di ? tt[0] : 1.f - tt[0]) * (dj ? tt[1] : 1.f - tt[1]) * (dk ? tt[2] : 1.f - tt[2]);
    const int64_t cc = ccell(p, c0[0] + di, c0[1] + dj, c0[2] + dk);
    float f[Q], r, mx, my, mz;
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = __ldg(fc + (int64_t)i * p.N + cc);
    moments<L, Q>(f, r, mx, my, mz);
    const float den = fmaxf(r, 1e-6f);
    const float u0 = mx / den, u1 = my / den, u2 = mz / den;
    rho += w * r;
    ux += w * u0; uy += w * u1; uz += w * u2;
#pragma unroll
    for (int i = 0; i < Q; ++i) fneq[i] += w * (f[i] - feq3<Q>(i, r, u0, u1, u2));
  }
#pragma unroll
  for (int i = 0; i < Q; ++i) fp[(int64_t)i * p.P + t.cell] = feq3<Q>(i, rho, ux, uy, uz) + p.rescale_c2f * fneq[i];
}

// common_d3_moments.wgsl: the tiles' mac from their f.
template <int Q>
__global__ void __launch_bounds__(kTileMaxThreads)
    amr3_moments(const float *__restrict__ fp, float4 *__restrict__ macp, const __grid_constant__ Amr3Params p) {
  using L = Lattice<Q>;
  TileCell t;
  if (!tile_cell(p, t)) return;
  float f[Q], rho, mx, my, mz;
#pragma unroll
  for (int i = 0; i < Q; ++i) f[i] = __ldg(fp + (int64_t)i * p.P + t.cell);
  moments<L, Q>(f, rho, mx, my, mz);
  const float den = fmaxf(rho, 1e-6f);
  macp[t.cell] = make_float4(rho, mx / den, my / den, mz / den);
}

// ---- bounce-back link table -------------------------------------------------
// With bounce-back, a pool cell's treatment of the body depends only on its
// position and the body's pose: whether it lies inside (phi < 0), whether a
// fine link from it can end inside (phi < 1: a fine link is sqrt(3)/2 L0
// units long and phi is 1-Lipschitz), and which of its Q pull sources do.
// Deciding the sources costs Q - 1 distance evaluations per near cell (a
// rotation and a box distance for a rounded box), which dominated the
// substeps of a large hierarchy. Between changes of the body (lbm_amr3d_set_body)
// and of the tiles (the manager), the codes are constant, so they are kept
// in a table of one word per pool cell and rebuilt on those events: bits
// 0 .. Q-1 the solid sources, kLinkNear, kLinkSolid. The table and the
// direct evaluation share link_code, so a step reads the same bits either way.
constexpr uint32_t kLinkNear = 1u << 29;
constexpr uint32_t kLinkSolid = 1u << 30;

template <int Q>
__device__ __forceinline__ uint32_t link_code(const Amr3Params &p, const TileCell &t, float phi) {
  uint32_t code = phi < 0.f ? kLinkSolid : 0u;
  if (phi < 1.0f) {
    code |= kLinkNear;
    if (phi < -0.87f) {
      // deeper than a link's length plus rounding: every source is solid
      code |= (1u << Q) - 1u;
    } else {
      // the rest direction's source is the cell itself; for a ring cell its
      // regular pull would read the neighbour tile, so it is decided like
      // any other link. One rolled loop: one out-of-line SDF call site.
      code |= phi < 0.f ? 1u : 0u;
#pragma unroll 1
      for (int i = 1; i < Q; ++i) {
        const V3 sp = {f2c(t.fx - c_dirs.ex[i], t.bx * p.rb), f2c(t.fy - c_dirs.ey[i], t.by * p.rb),
                       f2c(t.fz - c_dirs.ez[i], t.bz * p.rb)};
        if (phi3(sp, p.c.body, p.c.win) < 0.f) code |= 1u << i;
      }
    }
  }
  return code;
}

__device__ __forceinline__ V3 tile_pos(const Amr3Params &p, const TileCell &t) {
  return {f2c(t.fx, t.bx * p.rb), f2c(t.fy, t.by * p.rb), f2c(t.fz, t.bz * p.rb)};
}

// Every cell (ring included) of every live tile, or of the tiles flagged in
// only_new (the manager's grants).
template <int Q>
__global__ void __launch_bounds__(kListThreads)
    amr3_links(const __grid_constant__ Amr3Params p, uint32_t *__restrict__ links, const uint32_t *__restrict__ cells,
               const unsigned char *__restrict__ only_new) {
  TileCell t;
  __shared__ int nb27[27];
  if (!list_cell(p, cells, 0, p.T3, nb27, t)) return;
  if (only_new && !only_new[t.slot]) return;
  links[t.cell] = link_code<Q>(p, t, phi3(tile_pos(p, t), p.c.body, p.c.win));
}

// ---- explode ------------------------------------------------------------
// Which of block b's 3 x 3 x 3 neighbours an L0 coordinate r (relative to
// b's first cell, one axis) lies in: 0, 1 or 2.
__device__ __forceinline__ int nb_side(int r, int rb) { return r < 0 ? 0 : (r >= rb ? 2 : 1); }

template <int Q>
__global__ void __launch_bounds__(kListThreads)
    amr3_explode(const float *__restrict__ fc, float *__restrict__ fp, const __grid_constant__ Amr3Params p,
                 const uint32_t *__restrict__ cells, int first, int count) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a no-op unless launched by launch_pdl
  using L = Lattice<Q>;
  TileCell t;
  // the ring cells only; coverage of the L0 cells around the tile from the
  // neighbour table
  __shared__ int nb27[27];
  if (!list_cell(p, cells, first, count, nb27, t)) return;
  const int b[3] = {t.bx, t.by, t.bz};
  const int fi[3] = {t.fx, t.fy, t.fz};
  const int nf[3] = {2 * p.nx, 2 * p.ny, 2 * p.nz};
  // Per axis: g the fine coordinate (wrapped), v its L0 cell; fr the fine
  // coordinate from the block's first fine cell and rv = fr / 2 (rounded
  // down) its L0 cell from the block's first L0 cell. side packs, for
  // e = -1, 0, +1, the neighbour side (nb_side) of L0 cell rv + e (bits
  // 2(e+1)) and of the L0 cell holding fine cell fr + e (bits 6 + 2(e+1)).
  int g[3], v[3], side[3];
  for (int a = 0; a < 3; ++a) {
    const int fr = fi[a] - kAmrGhost;
    g[a] = wrapi(b[a] * p.RB2 + fr, nf[a]);
    v[a] = g[a] / 2;
    const int rv = fr >> 1;
    side[a] = 0;
    for (int k = 0; k < 3; ++k)
      side[a] |= nb_side(rv + k - 1, p.rb) << (2 * k) | nb_side((fr + k - 1) >> 1, p.rb) << (6 + 2 * k);
  }
  auto sd = [&](int a, int e) { return (side[a] >> (2 * (e + 1))) & 3; };
  auto sf = [&](int a, int e) { return (side[a] >> (6 + 2 * (e + 1))) & 3; };
  // A ring cell inside a covered L0 cell is never read (DIRECT_GHOST).
  if (nb27[sd(2, 0) * 9 + sd(1, 0) * 3 + sd(0, 0)] >= 0) return;
  // L0 cells as 32-bit offsets (N < 2^31)
  const int vc = (int)ccell(p, v[0], v[1], v[2]);
  bool ok[3];
  int vm[3], vp[3];
  for (int a = 0; a < 3; ++a) {
    int k0[3] = {sd(0, 0), sd(1, 0), sd(2, 0)}, k1[3] = {sd(0, 0), sd(1, 0), sd(2, 0)};
    k0[a] = sd(a, -1);
    k1[a] = sd(a, 1);
    ok[a] = nb27[k0[2] * 9 + k0[1] * 3 + k0[0]] < 0 && nb27[k1[2] * 9 + k1[1] * 3 + k1[0]] < 0;
    int m[3] = {v[0], v[1], v[2]}, q[3] = {v[0], v[1], v[2]};
    m[a] -= 1;
    q[a] += 1;
    vm[a] = (int)ccell(p, m[0], m[1], m[2]);
    vp[a] = (int)ccell(p, q[0], q[1], q[2]);
  }
  float d[3];
  for (int a = 0; a < 3; ++a) d[a] = ((float)(g[a] - 2 * v[a]) - 0.5f) * 0.5f;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const int e[3] = {L::ex(i), L::ey(i), L::ez(i)};
    const float *plane = fc + (int64_t)i * p.N;
    float out;
    if (nb27[sd(2, e[2]) * 9 + sd(1, e[1]) * 3 + sd(0, e[0])] < 0) {
      // in-orphan: this child's own one-step destination is in this tile
      // (its L0 cell covered, and the wrapped fine cell in this block)
      bool own = true;
      for (int a = 0; a < 3; ++a) {
        const int dg = wrapi(g[a] + e[a], nf[a]);
        own = own && dg >= b[a] * p.RB2 && dg < (b[a] + 1) * p.RB2;
      }
      const bool into = nb27[sf(2, e[2]) * 9 + sf(1, e[1]) * 3 + sf(0, e[0])] >= 0 && own;
      out = into ? __ldg(plane + vc) : 0.f;
    } else {
      const float f = __ldg(plane + vc);
      if (!p.linear) {
        out = f;
      } else {
        float G[3];
        for (int a = 0; a < 3; ++a) G[a] = ok[a] ? 0.5f * (__ldg(plane + vp[a]) - __ldg(plane + vm[a])) : 0.f;
        // projected orthogonal to e_i, so the two substeps see one state
        const float ee = (float)(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        const float gd = (G[0] * (float)e[0] + G[1] * (float)e[1] + G[2] * (float)e[2]) / ee;
        for (int a = 0; a < 3; ++a) G[a] -= (float)e[a] * gd;
        out = f + (d[0] * G[0] + d[1] * G[1] + d[2] * G[2]);
      }
    }
    fp[(int64_t)i * p.P + t.cell] = out;
  }
}

// ---- one pool substep ----------------------------------------------------
// Population index i * P + cell, in 32 bits when every index of the pool
// fits (W32: Q * P < 2^31, the usual case), so that an address is one
// multiply-add from the buffer's base instead of 64-bit arithmetic.
template <bool W32> using PoolIdx = std::conditional_t<W32, int, int64_t>;

template <bool W32> struct PoolSink {
  float *fo;
  PoolIdx<W32> n;
  int cell;  // < P < 2^31
  __device__ __forceinline__ void put(int i, float v) { fo[(PoolIdx<W32>)i * n + cell] = v; }
};

template <int Q, bool W32>
__device__ __forceinline__ void substep_cell(const float *__restrict__ fin, float *__restrict__ fout,
                                             float4 *__restrict__ macp, const Amr3Params &p, const int *nbase,
                                             const TileCell &t) {
  using L = Lattice<Q>;
  using I = PoolIdx<W32>;
  const I P = (I)p.P;
  const int cell = (int)t.cell;  // < P < 2^31
  const StepParams &c = p.c;
  const V3 pos = tile_pos(p, t);
  const bool bb = c.has_body && c.bb;
  float phi = 1e30f;  // the penalty's chi reads it; bounce-back reads the link code
  V3 us = {0.f, 0.f, 0.f};
  uint32_t code = 0;
  if (c.has_body) {
    if (!bb) phi = phi3(pos, c.body, c.win);
    else code = p.links ? __ldg(p.links + t.cell) : link_code<Q>(p, t, phi3(pos, c.body, c.win));
    us = body_velocity3(pos, c.body, c.win);
  }
  const bool in_tile = interior(p, t.fx) && interior(p, t.fy) && interior(p, t.fz);
  // A cell that collides inside the body (SOLID_EQ) is held at feq(1, u_body),
  // whatever it pulls: write that and skip the pull.
  if ((in_tile || p.collide_ring) && c.solid_eq && (code & kLinkSolid)) {
    const float ussq = us.x * us.x + us.y * us.y + us.z * us.z;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const float eu = (float)L::ex(i) * us.x + (float)L::ey(i) * us.y + (float)L::ez(i) * us.z;
      fout[(I)i * P + cell] = L::w(i) * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * ussq);
    }
    if (p.write_mac) macp[t.cell] = make_float4(1.f, us.x, us.y, us.z);
    return;
  }
  const bool near = code & kLinkNear;
  float rhoW = 1.f;
  if (near && c.rho_w_local) {
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < Q; ++i) s += __ldg(fin + (I)i * P + cell);
    rhoW = s;
  }
  const uint32_t solid_links = code & ((1u << Q) - 1u);
  // The Q pull loads, addressed from the pull table (four directions per
  // 128-bit load of it) as 32-bit cell offsets from each plane's base, all
  // in flight together. A solid link then takes the cell's own opposite
  // population instead (those loads hit the lines the rho_w sum just read).
  const int own = nbase[13];
  constexpr int kW = pull_words(Q);
  const uint4 *pw = reinterpret_cast<const uint4 *>(p.pulls) + (size_t)t.k * (kW / 4);
  float f[Q];
#pragma unroll
  for (int j = 0; j < kW / 4; ++j) {
    const uint4 w4 = __ldg(pw + j);
    const uint32_t w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = 4 * j + u;
      if (i < Q) {
        const int nb = nbase[w[u] & 31u];
        const int off = nb >= 0 ? nb + (int)((w[u] >> 5) & 0x1fffu) : own + (int)(w[u] >> 18);
        f[i] = __ldg(fin + (I)i * P + off);
      }
    }
  }
  if (solid_links) {
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      if ((solid_links >> i) & 1u) {
        const float corr = 2.f * L::w(i) * rhoW *
                           ((float)L::ex(i) * us.x + (float)L::ey(i) * us.y + (float)L::ez(i) * us.z) * kInvCS2;
        f[i] = __ldg(fin + (I)L::opp(i) * P + cell) + corr;
      }
    }
  }
  float rho, mx, my, mz;
  moments<L, Q>(f, rho, mx, my, mz);
  const float den = fmaxf(rho, 1e-6f);
  const float inv = 1.f / den;
  const float uxs = mx * inv, uys = my * inv, uzs = mz * inv;
  const float chi = (c.has_body && !c.bb) ? chi_from_phi(phi, p.chi_eps_f) : 0.f;
  const float rc = rho * chi;
  const float Fx = rc * (us.x - uxs) + c.fx, Fy = rc * (us.y - uys) + c.fy, Fz = rc * (us.z - uzs) + c.fz;
  const float hinv = 0.5f * inv;
  const float ux = fmaf(Fx, hinv, uxs), uy = fmaf(Fy, hinv, uys), uz = fmaf(Fz, hinv, uzs);
  PoolSink<W32> sink{fout, P, cell};
  if (!in_tile && !p.collide_ring) {
    // explode/coalesce: the ring advects and does not collide (COLLIDE_RING = 0)
    if (p.write_mac) macp[t.cell] = make_float4(rho, ux, uy, uz);
#pragma unroll
    for (int i = 0; i < Q; ++i) fout[(I)i * P + cell] = f[i];
    return;
  }
  float spw = 0.f;
  if (c.sponge_w > 0.f) {
    // L0 units, window coordinates (common_d3_amr_step1.wgsl:356-366)
    V3 wp = pos;
    if (c.win.on) {
      wp.x = win_coord1(pos.x, win_offset1(c.body.cx, c.win.anchor[0], c.win.n[0]), c.win.n[0]);
      wp.y = win_coord1(pos.y, win_offset1(c.body.cy, c.win.anchor[1], c.win.n[1]), c.win.n[1]);
      wp.z = win_coord1(pos.z, win_offset1(c.body.cz, c.win.anchor[2], c.win.n[2]), c.win.n[2]);
    }
    const float dx = c.sax ? fminf(wp.x, (float)(p.nx - 1) - wp.x) : 1e30f;
    const float dy = c.say ? fminf(wp.y, (float)(p.ny - 1) - wp.y) : 1e30f;
    const float dz = c.saz ? fminf(wp.z, (float)(p.nz - 1) - wp.z) : 1e30f;
    spw = sponge_weight_inv(fminf(dx, fminf(dy, dz)), c.sponge_inv);
  }
  collide_store<L, Q>(f, rho, ux, uy, uz, Fx, Fy, Fz, p.omega_f, spw, c.ftarget, sink);
  if (p.write_mac) macp[t.cell] = make_float4(rho, ux, uy, uz);
}

// One thread per tile cell: CTAs of kListThreads over chunks of the tile's
// cell list. (A CTA walking several chunks, so that the tile set-up is paid
// once, held more registers and ran slower: other CTAs hide the set-up.)
template <int Q, bool W32>
__global__ void __launch_bounds__(kListThreads, Q == 19 ? (W32 ? 9 : 8) : 6)
    amr3_substep(const float *__restrict__ fin, float *__restrict__ fout, float4 *__restrict__ macp,
                 const __grid_constant__ Amr3Params p, const uint32_t *__restrict__ cells, int count) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a no-op unless launched by launch_pdl
  TileCell t;
  // the tile's 26 same-level neighbours as pool cell bases, once per CTA
  __shared__ int nbase[27];
  if (!list_cell(p, cells, 0, count, nbase, t, true)) return;
  substep_cell<Q, W32>(fin, fout, macp, p, nbase, t);
}

// ---- coalesce -------------------------------------------------------------
// One thread per L0 cell of the interface blocks (covered blocks and the
// blocks touching one). Each thread writes only its own L0 cell.
__device__ __forceinline__ int local_in_tile(const Amr3Params &p, int g, int b, int nfine) {
  int d = g - b * p.RB2;
  if (d < -nfine / 2) d += nfine;
  if (d > nfine / 2) d -= nfine;
  return d + kAmrGhost;
}

// One CTA per interface block, SUBS threads per L0 cell of it (rb^3 * SUBS
// threads, adjacent lanes sharing a cell), each taking every SUBS-th
// direction. The directions of a cell are independent, and a seam cell's
// out/in-orphan balance walks 8 children per direction, too long a chain
// for one thread when a few hundred blocks cannot fill the device; with
// thousands of blocks one thread per cell (SUBS = 1) keeps its restriction
// loop unrolled. The 3 x 3 x 3 neighbour blocks' slots come from a shared
// table, so no coverage or slot lookup goes to global memory or divides.
__device__ __forceinline__ int rel_block(int q, int b, int nb) {
  int d = q - b;
  if (d > 1) d -= nb;
  if (d < -1) d += nb;
  return d;
}

template <int Q, int SUBS>
__global__ void __launch_bounds__(kMaxAmrRb * kMaxAmrRb * kMaxAmrRb)
    amr3_coalesce(const float *__restrict__ fp, float *__restrict__ fc, float4 *__restrict__ macc,
                  const float4 *__restrict__ macp, const __grid_constant__ Amr3Params p) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a no-op unless launched by launch_pdl
  using L = Lattice<Q>;
  const int id = p.iface ? p.iface[blockIdx.x] : (int)blockIdx.x;
  if (!p.iface && !p.iface_flag[id]) return;  // the whole CTA
  const int b[3] = {id % p.nbx, (id / p.nbx) % p.nby, id / (p.nbx * p.nby)};
  __shared__ int nb27[27];
  __shared__ signed char dir[3][27];
  for (int k = threadIdx.x; k < 27; k += blockDim.x) {
    const int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
    nb27[k] = p.block_slot[(wrapi(b[2] + dz, p.nbz) * p.nby + wrapi(b[1] + dy, p.nby)) * p.nbx +
                           wrapi(b[0] + dx, p.nbx)];
    dir[0][k] = (signed char)L::ex(k < Q ? k : 0);
    dir[1][k] = (signed char)L::ey(k < Q ? k : 0);
    dir[2][k] = (signed char)L::ez(k < Q ? k : 0);
  }
  __syncthreads();
  const int l = threadIdx.x / SUBS, sub = threadIdx.x % SUBS;
  // the cell's position within its block, per axis
  const int lc[3] = {l % p.rb, (l / p.rb) % p.rb, l / (p.rb * p.rb)};
  const int x = b[0] * p.rb + lc[0], y = b[1] * p.rb + lc[1], z = b[2] * p.rb + lc[2];
  const int64_t cell = ccell(p, x, y, z);
  const int slot = nb27[13];
  if (slot < 0) {
    // out-orphans (half-step exits no coarse bucket absorbs) against
    // in-orphans (what explode injected into this cell's own children)
    bool nearc = false;
#pragma unroll
    for (int i = 1; i < Q; ++i) nearc = nearc || covered_near(p, nb27, b, x + L::ex(i), y + L::ey(i), z + L::ez(i));
    if (!nearc) return;
#pragma unroll 1
    for (int i = 1 + sub; i < Q; i += SUBS) {
      const int e[3] = {dir[0][i], dir[1][i], dir[2][i]};
      const int tc[3] = {x + e[0], y + e[1], z + e[2]};
      if (covered_near(p, nb27, b, tc[0], tc[1], tc[2])) continue;
      // Child o of the target tc = cell + e, per axis relative to block b
      // (the neighbour table is b's): its fine source 2 l + e + o (one fine
      // step upstream, from b's first fine cell) picks the source's block,
      // the child's coordinate in that tile is the source's plus e, and
      // the cell's own child o shifted by e lies in L0 cell l + (o + e) / 2
      // (rounded down), covered or not.
      float sacc = 0.f, nin = 0.f;
      for (int q = 0; q < 8; ++q) {
        int ks = 0, kc = 0, loc[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int o = (q >> a) & 1, m = a == 0 ? 1 : (a == 1 ? 3 : 9);
          const int d = 2 * lc[a] + e[a] + o;
          const int rel = d < 0 ? -1 : (d >= p.RB2 ? 1 : 0);
          ks += (rel + 1) * m;
          loc[a] = d + e[a] - rel * p.RB2 + kAmrGhost;
          const int r = lc[a] + ((o + e[a]) >> 1);
          kc += (r < 0 ? 0 : (r >= p.rb ? 2 : 1)) * m;
        }
        const int qs = nb27[ks];
        if (qs >= 0)
          sacc += __ldg(fp + (int64_t)i * p.P + (int64_t)qs * p.T3 + (loc[2] * p.FB + loc[1]) * p.FB + loc[0]);
        if (nb27[kc] >= 0) nin += 1.f;
      }
      const float own = fc[(int64_t)i * p.N + cell];
      const float net = sacc - nin * own;
      if (net != 0.f) fc[(int64_t)i * p.N + cell] = own + net * 0.125f;
    }
    return;
  }
  const int lx0 = kAmrGhost + 2 * (x - b[0] * p.rb), ly0 = kAmrGhost + 2 * (y - b[1] * p.rb),
            lz0 = kAmrGhost + 2 * (z - b[2] * p.rb);
  if (p.write_mac && sub == 0) {
    float rs = 0.f, m0 = 0.f, m1 = 0.f, m2 = 0.f;
    for (int q = 0; q < 8; ++q) {
      const float4 m = macp[(int64_t)slot * p.T3 + ((lz0 + ((q >> 2) & 1)) * p.FB + ly0 + ((q >> 1) & 1)) * p.FB +
                            lx0 + (q & 1)];
      rs += m.x;
      m0 += m.x * m.y; m1 += m.x * m.z; m2 += m.x * m.w;
    }
    const float inv = 1.f / fmaxf(rs, 1e-6f);
    macc[cell] = make_float4(rs * 0.125f, m0 * inv, m1 * inv, m2 * inv);
  }
#pragma unroll
  for (int i = sub; i < Q; i += SUBS) {
    const int e[3] = {SUBS == 1 ? L::ex(i) : dir[0][i], SUBS == 1 ? L::ey(i) : dir[1][i],
                      SUBS == 1 ? L::ez(i) : dir[2][i]};
    const int tc[3] = {x + e[0], y + e[1], z + e[2]};
    if (covered_near(p, nb27, b, tc[0], tc[1], tc[2])) continue;
    // the children of tc, in this tile's coordinates (tc is next to the block)
    const int c0[3] = {2 * (lc[0] + e[0]) + kAmrGhost, 2 * (lc[1] + e[1]) + kAmrGhost, 2 * (lc[2] + e[2]) + kAmrGhost};
    float sacc = 0.f;
    for (int q = 0; q < 8; ++q) {
      const int lx = c0[0] + (q & 1), ly = c0[1] + ((q >> 1) & 1), lz = c0[2] + ((q >> 2) & 1);
      sacc += __ldg(fp + (int64_t)i * p.P + (int64_t)slot * p.T3 + (lz * p.FB + ly) * p.FB + lx);
    }
    fc[(int64_t)i * p.N + cell] = sacc * 0.125f;
  }
}

// ---- flux correction of the interp interface -------------------------------
// (common_d3_amr_flux.wgsl, common_d3_amr_reflux.wgsl; opt-in, as the
// reference's ?reflux=1.) Seam cells: unrefined L0 cells whose block touches
// a refined block on the side (face, edge or corner) the cell sits at.
__device__ __forceinline__ bool seam_cell(const Amr3Params &p, int x, int y, int z, int id) {
  if (p.block_slot[id] >= 0) return false;
  const int c3[3] = {x, y, z}, b[3] = {x / p.rb, y / p.rb, z / p.rb}, nb[3] = {p.nbx, p.nby, p.nbz};
  int off[3];
  for (int a = 0; a < 3; ++a) off[a] = c3[a] % p.rb == 0 ? -1 : ((c3[a] + 1) % p.rb == 0 ? 1 : 0);
  for (int k = 1; k < 8; ++k) {
    int q[3];
    for (int a = 0; a < 3; ++a) q[a] = wrapi(b[a] + ((k >> a) & 1) * off[a], nb[a]);
    if (p.block_slot[(q[2] * p.nby + q[1]) * p.nbx + q[0]] >= 0) return true;
  }
  return false;
}

// Thread -> L0 cell of an interface block; false when there is none.
__device__ __forceinline__ bool iface_cell(const Amr3Params &p, int &x, int &y, int &z, int &id) {
  const int rb3 = p.rb * p.rb * p.rb;
  const int k = blockIdx.x * kTileThreads + threadIdx.x;
  if (k >= p.n_iface * rb3) return false;
  id = p.iface ? p.iface[k / rb3] : k / rb3;
  if (!p.iface && !p.iface_flag[id]) return false;
  const int l = k % rb3;
  x = (id % p.nbx) * p.rb + l % p.rb;
  y = ((id / p.nbx) % p.nby) * p.rb + (l / p.rb) % p.rb;
  z = (id / (p.nbx * p.nby)) * p.rb + l / (p.rb * p.rb);
  return true;
}

// The mass and momentum the fine level moves across the seam into each seam
// cell during one substep (the buffer that substep streams), 1/8 per fine cell.
template <int Q>
__global__ void __launch_bounds__(kTileThreads)
    amr3_flux(const float *__restrict__ fp, float4 *__restrict__ acc, const __grid_constant__ Amr3Params p,
              int accumulate) {
  using L = Lattice<Q>;
  int x, y, z, id;
  if (!iface_cell(p, x, y, z, id) || !seam_cell(p, x, y, z, id)) return;
  const int nf[3] = {2 * p.nx, 2 * p.ny, 2 * p.nz};
  float dm = 0.f, dp0 = 0.f, dp1 = 0.f, dp2 = 0.f;
  for (int oc = 0; oc < 8; ++oc) {
    const int pp[3] = {2 * x + (oc & 1), 2 * y + ((oc >> 1) & 1), 2 * z + ((oc >> 2) & 1)};
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const int e[3] = {L::ex(i), L::ey(i), L::ez(i)};
      int q[3], t[3];
      for (int a = 0; a < 3; ++a) {
        q[a] = wrapi(pp[a] - e[a], nf[a]);
        t[a] = wrapi(pp[a] + e[a], nf[a]);
      }
      const int so = p.block_slot[((q[2] / p.RB2) * p.nby + q[1] / p.RB2) * p.nbx + q[0] / p.RB2];
      if (so >= 0) {
        const int lx = local_in_tile(p, q[0], q[0] / p.RB2, nf[0]), ly = local_in_tile(p, q[1], q[1] / p.RB2, nf[1]),
                  lz = local_in_tile(p, q[2], q[2] / p.RB2, nf[2]);
        const float f = __ldg(fp + (int64_t)i * p.P + (int64_t)so * p.T3 + (lz * p.FB + ly) * p.FB + lx);
        dm += f; dp0 += f * (float)e[0]; dp1 += f * (float)e[1]; dp2 += f * (float)e[2];
      }
      const int si = p.block_slot[((t[2] / p.RB2) * p.nby + t[1] / p.RB2) * p.nbx + t[0] / p.RB2];
      if (si >= 0) {
        const int lx = local_in_tile(p, pp[0], t[0] / p.RB2, nf[0]), ly = local_in_tile(p, pp[1], t[1] / p.RB2, nf[1]),
                  lz = local_in_tile(p, pp[2], t[2] / p.RB2, nf[2]);
        const float f = __ldg(fp + (int64_t)i * p.P + (int64_t)si * p.T3 + (lz * p.FB + ly) * p.FB + lx);
        dm -= f; dp0 -= f * (float)e[0]; dp1 -= f * (float)e[1]; dp2 -= f * (float)e[2];
      }
    }
  }
  const int64_t cell = ccell(p, x, y, z);
  float4 v = make_float4(dm * 0.125f, dp0 * 0.125f, dp1 * 0.125f, dp2 * 0.125f);
  if (accumulate) {
    const float4 o = acc[cell];
    v = make_float4(o.x + v.x, o.y + v.y, o.z + v.z, o.w + v.w);
  }
  acc[cell] = v;
}

// The fine flux less the one L0 computed across the same faces, added to the
// new L0 populations as w_i (dm + 3 e_i . dp); cells within 2 of the body
// are left alone. Rewrites the seam cells' mac.
template <int Q>
__global__ void __launch_bounds__(kTileThreads)
    amr3_reflux(const float *__restrict__ fin, float *__restrict__ fout, float4 *__restrict__ macc,
                float4 *__restrict__ acc, const __grid_constant__ Amr3Params p) {
  using L = Lattice<Q>;
  int x, y, z, id;
  if (!iface_cell(p, x, y, z, id) || !seam_cell(p, x, y, z, id)) return;
  const StepParams &c = p.c;
  if (c.has_body && phi3({(float)x, (float)y, (float)z}, c.body, c.win) < 2.0f) return;
  const int64_t cell = ccell(p, x, y, z);
  const float4 a0 = acc[cell];
  float dm = a0.x, dp0 = a0.y, dp1 = a0.z, dp2 = a0.w;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const int e[3] = {L::ex(i), L::ey(i), L::ez(i)};
    if (covered(p, x - e[0], y - e[1], z - e[2])) {
      const float v = __ldg(fin + (int64_t)i * p.N + ccell(p, x - e[0], y - e[1], z - e[2]));
      dm -= v; dp0 -= v * (float)e[0]; dp1 -= v * (float)e[1]; dp2 -= v * (float)e[2];
    }
    if (covered(p, x + e[0], y + e[1], z + e[2])) {
      const float v = __ldg(fin + (int64_t)i * p.N + cell);
      dm += v; dp0 += v * (float)e[0]; dp1 += v * (float)e[1]; dp2 += v * (float)e[2];
    }
  }
  acc[cell] = make_float4(dm, dp0, dp1, dp2);
  float rho = 0.f, m0 = 0.f, m1 = 0.f, m2 = 0.f;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const float ex = (float)L::ex(i), ey = (float)L::ey(i), ez = (float)L::ez(i);
    const float fo = fout[(int64_t)i * p.N + cell] + L::w(i) * (dm + 3.f * (ex * dp0 + ey * dp1 + ez * dp2));
    fout[(int64_t)i * p.N + cell] = fo;
    rho += fo;
    m0 += fo * ex; m1 += fo * ey; m2 += fo * ez;
  }
  const float den = fmaxf(rho, 1e-6f);
  macc[cell] = make_float4(rho, m0 / den + c.fx / (2.f * den), m1 / den + c.fy / (2.f * den),
                           m2 / den + c.fz / (2.f * den));
}

// ---- L0 step, skipping covered blocks ------------------------------------
template <int Q>
__global__ void __launch_bounds__(kStepThreads, Q == 27 ? (kStepMinBlocks * 3) / 4 : kStepMinBlocks)
    amr3_coarse(const float *__restrict__ fin, float *__restrict__ fout, float *__restrict__ mac,
                const __grid_constant__ StepParams sp, const int *__restrict__ block_slot, int rb, int nbx, int nby) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a no-op unless launched by launch_pdl
  const int x = blockIdx.x * kStepThreads + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= sp.nx) return;
  if (block_slot[((z / rb) * nby + y / rb) * nbx + x / rb] >= 0) return;
  CellForce cf;
  cell3<Q, float>(fin, fout, mac, sp, x, y, z, false, cf);
}

// ---- pool force (common_d3_force_pool.wgsl) -------------------------------
// Interior cells of every tile at time t: momentum exchange with local rho_w
// weighted by dx^2 = 1/4, the swept-cell term by dx^3 = 1/8, or the chi
// penalty with a tile-clamped gather; FP64 partial per CTA, last-CTA sum.
template <int Q>
__global__ void __launch_bounds__(kTileThreads)
    amr3_force(const float *__restrict__ fp, const __grid_constant__ Amr3Params p, const uint32_t *__restrict__ cells) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a no-op unless launched by launch_pdl
  using L = Lattice<Q>;
  const StepParams &c = p.c;
  const int r3 = p.RB2 * p.RB2 * p.RB2;
  const int k = blockIdx.x * kTileThreads + threadIdx.x;
  CellForce cf;
  const int slot = blockIdx.y;
  const int id = p.slot_to_block[slot];
  if (k < r3 && id >= 0) {
    const int b[3] = {id % p.nbx, (id / p.nbx) % p.nby, id / (p.nbx * p.nby)};
    // interior cell k (the cell list holds the interior first, z-, y-, x-major)
    const uint32_t cl = __ldg(cells + k);
    const int fx = cl & 0xff, fy = (cl >> 8) & 0xff, fz = cl >> 16;
    const int64_t cell = (int64_t)slot * p.T3 + (fz * p.FB + fy) * p.FB + fx;
    const V3 pos = {f2c(fx, b[0] * p.rb), f2c(fy, b[1] * p.rb), f2c(fz, b[2] * p.rb)};
    // With the link table and no swept-cell term, the cell's code says all
    // the bounce-back force needs (0 <= phi < 1: near and not solid) and
    // the distance is not evaluated.
    const bool coded = c.bb && p.links && !c.swept;
    const uint32_t code = coded ? __ldg(p.links + cell) : 0u;
    const float phi = coded ? 0.5f : phi3(pos, c.body, c.win);
    const V3 us = body_velocity3(pos, c.body, c.win);
    float fbx = 0.f, fby = 0.f, fbz = 0.f, fsx = 0.f, fsy = 0.f, fsz = 0.f;
    if (c.bb) {
      if (coded ? (code & (kLinkNear | kLinkSolid)) == kLinkNear : (phi >= 0.f && phi < 1.0f)) {
        float rhoW = 1.f;
        if (c.rho_w_local && phi < 2.f) {
          float s = 0.f;
#pragma unroll
          for (int i = 0; i < Q; ++i) s += __ldg(fp + (int64_t)i * p.P + cell);
          rhoW = s;
        }
        // the solid sources (the cell itself, phi >= 0 here, is not one)
        uint32_t solid;
        if (coded) {
          solid = code & ((1u << Q) - 2u);
        } else if (p.links) {
          solid = __ldg(p.links + cell) & ((1u << Q) - 2u);
        } else {
          const TileCell t = {slot, b[0], b[1], b[2], fx, fy, fz, cell};
          solid = link_code<Q>(p, t, phi) & ((1u << Q) - 2u);
        }
#pragma unroll
        for (int i = 0; i < Q; ++i) {
          if (solid & (1u << i)) {
            const float fo = __ldg(fp + (int64_t)L::opp(i) * p.P + cell);
            const float corr =
                2.f * L::w(i) * rhoW * ((float)L::ex(i) * us.x + (float)L::ey(i) * us.y + (float)L::ez(i) * us.z) * kInvCS2;
            const float m = 2.f * fo + corr;
            fbx += -(float)L::ex(i) * m;
            fby += -(float)L::ey(i) * m;
            fbz += -(float)L::ez(i) * m;
          }
        }
      }
      if (c.swept && fabsf(phi) < c.swept_band) {
        const bool now = phi < 0.f;
        if (now != (phi3_ahead(pos, c.body, 1.f, c.win) < 0.f)) {
          float mcx = 0.f, mcy = 0.f, mcz = 0.f;
#pragma unroll
          for (int i = 0; i < Q; ++i) {
            const float v = __ldg(fp + (int64_t)i * p.P + cell);
            mcx += v * (float)L::ex(i); mcy += v * (float)L::ey(i); mcz += v * (float)L::ez(i);
          }
          if (!now) { fsx = mcx; fsy = mcy; fsz = mcz; }
          else { fsx = -mcx; fsy = -mcy; fsz = -mcz; }
        }
      }
    } else {
      const float chi = chi_from_phi(phi, p.chi_eps_f);
      if (chi >= 1e-6f) {
        float rho = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
          const int sx = min(max(fx - L::ex(i), 0), p.FB - 1), sy = min(max(fy - L::ey(i), 0), p.FB - 1),
                    sz = min(max(fz - L::ez(i), 0), p.FB - 1);
          const float v = __ldg(fp + (int64_t)i * p.P + (int64_t)slot * p.T3 + (sz * p.FB + sy) * p.FB + sx);
          rho += v;
          mx += v * (float)L::ex(i); my += v * (float)L::ey(i); mz += v * (float)L::ez(i);
        }
        const float den = fmaxf(rho, 1e-6f);
        fbx = -(rho * chi * (us.x - mx / den));
        fby = -(rho * chi * (us.y - my / den));
        fbz = -(rho * chi * (us.z - mz / den));
      }
    }
    const float tx = fbx * 0.25f + fsx * 0.125f, ty = fby * 0.25f + fsy * 0.125f, tz = fbz * 0.25f + fsz * 0.125f;
    const V3 r = body_delta(pos, c.body, c.win);
    const float rx = r.x, ry = r.y, rz = r.z;
    cf.fx = tx; cf.fy = ty; cf.fz = tz;
    cf.tx = ry * tz - rz * ty;
    cf.ty = rz * tx - rx * tz;
    cf.tz = rx * ty - ry * tx;
  }
  ForceAcc acc;
  acc.add(cf);
  publish_force<kTileThreads>(acc, p.partials, blockIdx.y * gridDim.x + blockIdx.x);
}

// The pool force's partials summed in a fixed order (groups of kSumGroup,
// then the groups), deterministic; a launch of its own, so that the force
// CTAs publish their partials without a ticket and its fence.
__global__ void __launch_bounds__(kSumGroup)
    amr3_force_sum(const double *__restrict__ partials, int nparts, double *__restrict__ groups,
                   unsigned int *__restrict__ counter, double *__restrict__ out) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a no-op unless launched by launch_pdl
  sum_partials_grouped<kSumGroup>(partials, nparts, groups, counter, out, blockIdx.x);
}

// ---- the refinement manager (common_d3_manage.wgsl) ------------------------

// blockWanted: does any point of the block come within margin + lead of the
// body? One SDF evaluation brackets the minimum over a box of half-edge h as
// phi(c) - h sqrt(3) <= min <= phi(c); undecided boxes split into octants,
// three levels deep, accepting at the bottom. sqrt(3) rounded up.
__device__ __noinline__ bool box_near_body(const lbm_body &b, const Win &w, float cx, float cy, float cz, float h0,
                                           float reach) {
  const float S3 = 1.7320509f;
  float R0 = h0 * S3;
  const float p0 = phi3({cx, cy, cz}, b, w);
  if (p0 - R0 > reach) return false;
  if (p0 <= reach) return true;
  const float h1 = h0 * 0.5f, R1 = R0 * 0.5f;
  for (int i = 0; i < 8; ++i) {
    const float c1x = cx + ((i & 1) ? h1 : -h1), c1y = cy + ((i & 2) ? h1 : -h1), c1z = cz + ((i & 4) ? h1 : -h1);
    const float p1 = phi3({c1x, c1y, c1z}, b, w);
    if (p1 - R1 > reach) continue;
    if (p1 <= reach) return true;
    const float h2 = h1 * 0.5f, R2 = R1 * 0.5f;
    for (int j = 0; j < 8; ++j) {
      const float c2x = c1x + ((j & 1) ? h2 : -h2), c2y = c1y + ((j & 2) ? h2 : -h2), c2z = c1z + ((j & 4) ? h2 : -h2);
      const float p2 = phi3({c2x, c2y, c2z}, b, w);
      if (p2 - R2 > reach) continue;
      if (p2 <= reach) return true;
      const float h3 = h2 * 0.5f, R3 = R2 * 0.5f;
      for (int k = 0; k < 8; ++k) {
        const float c3x = c2x + ((k & 1) ? h3 : -h3), c3y = c2y + ((k & 2) ? h3 : -h3),
                    c3z = c2z + ((k & 4) ? h3 : -h3);
        if (phi3({c3x, c3y, c3z}, b, w) - R3 <= reach) return true;
      }
    }
  }
  return false;
}

// The field half of the decision (common_d3_criterion.wgsl reduceQ): per
// block, the max over the L0 cells of its box dilated by `lead` (floor /
// ceil, so the box contains the region) of Q = 1/2 (|Omega|^2 - |S|^2), from
// centred differences of the L0 velocity over the six face neighbours,
// periodic. Products and sums are rounded one by one (no contraction), so
// the value is the plain f32 arithmetic of the formula.
__device__ __forceinline__ float3 mac_u(const float4 *__restrict__ mac, const Amr3Params &p, int x, int y, int z) {
  x %= p.nx; x += x < 0 ? p.nx : 0;
  y %= p.ny; y += y < 0 ? p.ny : 0;
  z %= p.nz; z += z < 0 ? p.nz : 0;
  const float4 m = __ldg(mac + ((int64_t)z * p.ny + y) * p.nx + x);
  return make_float3(m.y, m.z, m.w);
}

__device__ float q_at(const float4 *__restrict__ mac, const Amr3Params &p, int x, int y, int z) {
  float J[3][3];  // J[j][i] = du_i / dx_j
  const float3 xp = mac_u(mac, p, x + 1, y, z), xm = mac_u(mac, p, x - 1, y, z);
  const float3 yp = mac_u(mac, p, x, y + 1, z), ym = mac_u(mac, p, x, y - 1, z);
  const float3 zp = mac_u(mac, p, x, y, z + 1), zm = mac_u(mac, p, x, y, z - 1);
  J[0][0] = __fmul_rn(__fsub_rn(xp.x, xm.x), 0.5f); J[0][1] = __fmul_rn(__fsub_rn(xp.y, xm.y), 0.5f);
  J[0][2] = __fmul_rn(__fsub_rn(xp.z, xm.z), 0.5f);
  J[1][0] = __fmul_rn(__fsub_rn(yp.x, ym.x), 0.5f); J[1][1] = __fmul_rn(__fsub_rn(yp.y, ym.y), 0.5f);
  J[1][2] = __fmul_rn(__fsub_rn(yp.z, ym.z), 0.5f);
  J[2][0] = __fmul_rn(__fsub_rn(zp.x, zm.x), 0.5f); J[2][1] = __fmul_rn(__fsub_rn(zp.y, zm.y), 0.5f);
  J[2][2] = __fmul_rn(__fsub_rn(zp.z, zm.z), 0.5f);
  float s2 = 0.f, om2 = 0.f;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float a = J[j][i], b = J[i][j];
      const float S = __fmul_rn(0.5f, __fadd_rn(a, b)), O = __fmul_rn(0.5f, __fsub_rn(a, b));
      s2 = __fadd_rn(s2, __fmul_rn(S, S));
      om2 = __fadd_rn(om2, __fmul_rn(O, O));
    }
  return __fmul_rn(0.5f, __fsub_rn(om2, s2));
}

constexpr int kCritThreads = 128;

__global__ void __launch_bounds__(kCritThreads)
    amr3_criterion(const float4 *__restrict__ mac, float *__restrict__ block_q, const __grid_constant__ Amr3Params p,
                   float lead) {
  const int id = blockIdx.x;
  const int b[3] = {id % p.nbx, (id / p.nbx) % p.nby, id / (p.nbx * p.nby)};
  int i0[3], n[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float lo = (float)b[a] * (float)p.rb - lead;
    const float hi = lo + (float)p.rb + 2.f * lead;
    i0[a] = (int)floorf(lo);
    n[a] = max((int)ceilf(hi) - i0[a], 0);
  }
  const int total = n[0] * n[1] * n[2];
  float best = -1e30f;
  for (int k = threadIdx.x; k < total; k += kCritThreads)
    best = fmaxf(best, q_at(mac, p, i0[0] + k % n[0], i0[1] + (k / n[0]) % n[1], i0[2] + k / (n[0] * n[1])));
#pragma unroll
  for (int o = 16; o; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ float wq[kCritThreads / 32];
  if ((threadIdx.x & 31) == 0) wq[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = wq[0];
#pragma unroll
    for (int w = 1; w < kCritThreads / 32; ++w) m = fmaxf(m, wq[w]);
    block_q[id] = m;
  }
}

// decide (common_d3_manage.wgsl): the union of the geometry test and, with
// block_q, the field test -- max Q at or above q_refine for a block not yet
// refined, at or above the one-band-lower q_hold for a block that holds a
// tile (the refine / coarsen ladders of common_refine.wgsl at one level:
// 1/2 log2 max(Q, 1e-30) >= 1/2 log2 Q_abs, minus the hysteresis band when
// held, compared here in Q itself, which is monotone in the same quantity).
__global__ void amr3_decide(const __grid_constant__ Amr3Params p, unsigned char *__restrict__ want, float reach,
                            const float *__restrict__ block_q, float q_refine, float q_hold) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= p.nbx * p.nby * p.nbz) return;
  const int bx = id % p.nbx, by = (id / p.nbx) % p.nby, bz = id / (p.nbx * p.nby);
  const float half = 0.5f * (float)p.rb;
  bool w = box_near_body(p.c.body, p.c.win, (float)(bx * p.rb) + half, (float)(by * p.rb) + half, (float)(bz * p.rb) + half,
                         half, reach);
  if (!w && block_q) w = fmaxf(block_q[id], 1e-30f) >= (p.block_slot[id] >= 0 ? q_hold : q_refine);
  want[id] = w ? 1 : 0;
}

// drain (common_d3_amr_average.wgsl, DYING_ONLY): a tile about to be freed
// restricts into its L0 cells at time t -- feq of the children's mean rho
// and mass-weighted u plus the F2C-rescaled mean fneq, 2 (tau_c - 1)/(tau_f - 1).
template <int Q>
__global__ void __launch_bounds__(kTileThreads)
    amr3_drain(const float *__restrict__ fp, float *__restrict__ fc, float4 *__restrict__ macc,
               const __grid_constant__ Amr3Params p, const unsigned char *__restrict__ want, float rescale_f2c) {
  using L = Lattice<Q>;
  const int rb3 = p.rb * p.rb * p.rb;
  const int k = blockIdx.x * kTileThreads + threadIdx.x;
  if (k >= rb3) return;
  const int slot = blockIdx.y;
  const int id = p.slot_to_block[slot];
  if (id < 0 || (want && want[id])) return;
  const int lc[3] = {k % p.rb, (k / p.rb) % p.rb, k / (p.rb * p.rb)};
  const int b[3] = {id % p.nbx, (id / p.nbx) % p.nby, id / (p.nbx * p.nby)};
  float rs = 0.f, ms0 = 0.f, ms1 = 0.f, ms2 = 0.f, fneq[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) fneq[i] = 0.f;
  for (int c = 0; c < 8; ++c) {
    const int64_t cell = (int64_t)slot * p.T3 +
                         ((kAmrGhost + 2 * lc[2] + ((c >> 2) & 1)) * p.FB + kAmrGhost + 2 * lc[1] + ((c >> 1) & 1)) * p.FB +
                         kAmrGhost + 2 * lc[0] + (c & 1);
    float f[Q], r, mx, my, mz;
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] = __ldg(fp + (int64_t)i * p.P + cell);
    moments<L, Q>(f, r, mx, my, mz);
    const float den = fmaxf(r, 1e-6f);
    const float u0 = mx / den, u1 = my / den, u2 = mz / den;
    rs += r;
    ms0 += r * u0; ms1 += r * u1; ms2 += r * u2;
#pragma unroll
    for (int i = 0; i < Q; ++i) fneq[i] += f[i] - feq3<Q>(i, r, u0, u1, u2);
  }
  const float ra = rs * 0.125f, inv = 1.f / fmaxf(rs, 1e-6f);
  const float ua = ms0 * inv, va = ms1 * inv, wa = ms2 * inv;
  const int64_t dst = ccell(p, b[0] * p.rb + lc[0], b[1] * p.rb + lc[1], b[2] * p.rb + lc[2]);
#pragma unroll
  for (int i = 0; i < Q; ++i) fc[(int64_t)i * p.N + dst] = feq3<Q>(i, ra, ua, va, wa) + rescale_f2c * (fneq[i] * 0.125f);
  macc[dst] = make_float4(ra, ua, va, wa);
}

constexpr int kManageThreads = 1024;

// coarsen + refine in one CTA, deterministic: dying blocks push their slots
// on the free stack in ascending block id, then newly wanted blocks pop
// slots in ascending block id (the stack top first); a block the pool cannot
// hold stays coarse and is counted. Then the coalesce's interface flags.
// counts = {free, refusals, lowest free, decisions}.
__global__ void __launch_bounds__(kManageThreads)
    amr3_manage(int *block_slot, int *slot_to_block, int *free_list, int *counts, unsigned char *slot_new,
                unsigned char *iface_flag, const unsigned char *__restrict__ want, int nbx, int nby, int nbz,
                int capacity) {
  __shared__ int sm[64];
  const int nb = nbx * nby * nbz;
  for (int s = threadIdx.x; s < capacity; s += kManageThreads) slot_new[s] = 0;
  int fc = counts[0];
  __syncthreads();
  for (int base = 0; base < nb; base += kManageThreads) {
    const int id = base + threadIdx.x;
    const int slot = id < nb ? block_slot[id] : -1;
    const int dying = (slot >= 0 && !want[id]) ? 1 : 0;
    int total;
    const int r = block_scan(dying, sm, total);
    if (dying) {
      free_list[fc + r] = slot;
      block_slot[id] = -1;
      slot_to_block[slot] = -1;
    }
    fc += total;
    __syncthreads();
  }
  int refused = 0;
  for (int base = 0; base < nb; base += kManageThreads) {
    const int id = base + threadIdx.x;
    const int born = (id < nb && block_slot[id] < 0 && want[id]) ? 1 : 0;
    int total;
    const int r = block_scan(born, sm, total);
    if (born && r < fc) {
      const int slot = free_list[fc - 1 - r];
      block_slot[id] = slot;
      slot_to_block[slot] = id;
      slot_new[slot] = 1;
    }
    refused += total > fc ? total - fc : 0;
    fc = total > fc ? 0 : fc - total;
    __syncthreads();
  }
  for (int id = threadIdx.x; id < nb; id += kManageThreads) {
    const int bx = id % nbx, by = (id / nbx) % nby, bz = id / (nbx * nby);
    unsigned char f = 0;
    for (int d = 0; d < 27 && !f; ++d) {
      const int x = (bx + d % 3 - 1 + nbx) % nbx, y = (by + (d / 3) % 3 - 1 + nby) % nby, z = (bz + d / 9 - 1 + nbz) % nbz;
      f = block_slot[(z * nby + y) * nbx + x] >= 0;
    }
    iface_flag[id] = f;
  }
  if (threadIdx.x == 0) {
    counts[0] = fc;
    counts[1] += refused;
    counts[2] = min(counts[2], fc);
    counts[3] += 1;
  }
}

// ---- totals over the L0 mac ------------------------------------------------
constexpr int kTotThreads = 256;
__global__ void __launch_bounds__(kTotThreads)
    amr3_totals(const float4 *__restrict__ mac, int64_t n, double *partials, unsigned int *counter, double *out) {
  __shared__ double sm[4 * (kTotThreads / 32)];
  double v[4] = {0, 0, 0, 0};
  for (int64_t c = (int64_t)blockIdx.x * kTotThreads + threadIdx.x; c < n; c += (int64_t)gridDim.x * kTotThreads) {
    const float4 m = mac[c];
    v[0] += (double)m.x - 1.0;
    v[1] += (double)m.x * m.y;
    v[2] += (double)m.x * m.z;
    v[3] += (double)m.x * m.w;
  }
  block_sum<4, kTotThreads>(v, sm);
  finish_sum<4, kTotThreads>(v, partials, counter, gridDim.x, blockIdx.x, out, sm);
}

#define AMR3_DISPATCH(q, ...)                                    \
  switch (q) {                                                   \
    case 19: { constexpr int Q = 19; __VA_ARGS__; } break;       \
    case 27: { constexpr int Q = 27; __VA_ARGS__; } break;       \
    default: return cudaErrorInvalidValue;                       \
  }                                                              \
  return cudaGetLastError();

}  // namespace

}  // namespace lbm

using namespace lbm;

struct lbm_amr3d {
  lbm_amr3d_config cfg{};
  int q = 19;
  Amr3Params p{};
  StepParams sp{};  // L0 step
  float *fc[2] = {nullptr, nullptr};
  float *fp[2] = {nullptr, nullptr};
  float *macc = nullptr;
  float4 *macp = nullptr;
  int *d_block_slot = nullptr, *d_slot_to_block = nullptr, *d_iface = nullptr;
  std::vector<int> block_slot, slot_to_block, iface;
  double *partials = nullptr, *force_out = nullptr, *tot_partials = nullptr, *tot_out = nullptr;
  double *force_groups = nullptr;  // the force partials' group sums
  unsigned int *counter = nullptr, *tot_counter = nullptr;
  double *host_out = nullptr;
  int force_parts = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  int cp = 0;
  bool seeded = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // dynamic refinement
  bool dynamic = false;
  int capacity = 0, initial = 0;
  int64_t step_count = 0;
  unsigned char *d_want = nullptr, *d_slot_new = nullptr, *d_iface_flag = nullptr;
  int *d_free_list = nullptr, *d_counts = nullptr;
  cudaGraphExec_t manage_graph[2] = {nullptr, nullptr};
  bool carved = false;          // device memory carved from a caller's block
  uint32_t *d_cells = nullptr;  // tile cells: interior (RB2^3) then ring, packed x | y << 8 | z << 16
  uint32_t *d_links = nullptr;  // bounce-back link code per pool cell (bounce-back bodies only)
  uint32_t *d_pulls = nullptr;  // substep pull sources per (direction, cell list position)
  int coalesce_subs = 1;        // threads per L0 cell in the coalesce
  float *d_block_q = nullptr;   // field criterion: per-block max Q (NULL = off)
  float q_refine = 0.f, q_hold = 0.f;
  float4 *flux = nullptr;  // reflux: per L0 cell {dm, dp}
  std::string err;
};

namespace {

thread_local std::string g_amr3_error;

int afail(lbm_amr3d *a, int code, const std::string &m) {
  if (a) a->err = m; else g_amr3_error = m;
  return code;
}

#define ACK(a, call)                                                                                       \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess)                                                                                 \
      return afail(a, e_ == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA,                            \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                                    \
  } while (0)

dim3 tile_grid(const lbm_amr3d *a) { return dim3(a->p.FB, a->p.slots); }
dim3 tile_block(const lbm_amr3d *a) { return dim3(a->p.FB, a->p.FB); }

cudaError_t launch_interp(lbm_amr3d *a, const float *fc, int ring_only, const unsigned char *only_new) {
  if (!a->p.slots) return cudaSuccess;
  const dim3 g = tile_grid(a);
  AMR3_DISPATCH(a->q,
                amr3_interp<Q><<<g, tile_block(a), 0, a->stream>>>(fc, a->fp[0], a->p, ring_only, only_new));
}

// The link table of every live tile, or of the tiles in only_new; nothing
// when the table is off.
cudaError_t launch_links(lbm_amr3d *a, const unsigned char *only_new) {
  if (!a->p.slots || !a->p.links) return cudaSuccess;
  const dim3 gl((a->p.T3 + kListThreads - 1) / kListThreads, a->p.slots);
  AMR3_DISPATCH(a->q, amr3_links<Q><<<gl, kListThreads, 0, a->stream>>>(a->p, a->d_links, a->d_cells, only_new));
}

// One decision of the manager before the macro-step from L0 parity `cp`
// (main-3d.js:3247-3317): decide, drain the dying tiles into the time-t L0
// buffer, free and grant slots, fill the new tiles from that buffer.
cudaError_t launch_manage(lbm_amr3d *a, int cp) {
  const Amr3Params &p = a->p;
  const lbm_body &b = p.c.body;
  const float rc = body_circumradius(b);
  const float lead = (float)a->cfg.manage_every *
                     (sqrtf(b.vx * b.vx + b.vy * b.vy + b.vz * b.vz) + sqrtf(b.wx * b.wx + b.wy * b.wy + b.wz * b.wz) * rc);
  const int nb = p.nbx * p.nby * p.nbz;
  cudaStream_t st = a->stream;
  if (a->d_block_q) {
    amr3_criterion<<<nb, kCritThreads, 0, st>>>((const float4 *)a->macc, a->d_block_q, p, a->cfg.q_lead);
    amr3_decide<<<(nb + 127) / 128, 128, 0, st>>>(p, a->d_want, a->cfg.margin + lead, a->d_block_q, a->q_refine,
                                                  a->q_hold);
  } else {
    amr3_decide<<<(nb + 127) / 128, 128, 0, st>>>(p, a->d_want, a->cfg.margin + lead, nullptr, 0.f, 0.f);
  }
  const float tc = a->cfg.root.tau, tf = 2.f * tc - 0.5f;
  const float f2c_rescale = 2.f * (tc - 1.f) / (tf - 1.f);
  const int rb3 = p.rb * p.rb * p.rb;
  const dim3 gd((rb3 + kTileThreads - 1) / kTileThreads, p.slots);
  cudaError_t e = cudaSuccess;
  {
    auto drain = [&]() -> cudaError_t {
      AMR3_DISPATCH(a->q, amr3_drain<Q><<<gd, kTileThreads, 0, st>>>(a->fp[0], a->fc[cp], (float4 *)a->macc, p,
                                                                      a->d_want, f2c_rescale));
    };
    if ((e = drain()) != cudaSuccess) return e;
  }
  amr3_manage<<<1, kManageThreads, 0, st>>>(a->d_block_slot, a->d_slot_to_block, a->d_free_list, a->d_counts,
                                           a->d_slot_new, a->d_iface_flag, a->d_want, p.nbx, p.nby, p.nbz,
                                           a->capacity);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = launch_links(a, a->d_slot_new)) != cudaSuccess) return e;
  return launch_interp(a, a->fc[cp], 0, a->d_slot_new);
}

cudaError_t launch_moments(lbm_amr3d *a) {
  if (!a->p.slots) return cudaSuccess;
  const dim3 g = tile_grid(a);
  AMR3_DISPATCH(a->q, amr3_moments<Q><<<g, tile_block(a), 0, a->stream>>>(a->fp[0], a->macp, a->p));
}

// Threads per L0 cell in the coalesce: doubled up to 8 while the interface
// blocks' threads still fit the device's resident threads and a CTA's 512.
int coalesce_subs(const Amr3Params &p, int sms) {
  const int rb3 = p.rb * p.rb * p.rb;
  const int64_t resident = (int64_t)sms * 2048;
  int subs = 1;
  while (subs < 8 && rb3 * subs * 2 <= kMaxAmrRb * kMaxAmrRb * kMaxAmrRb &&
         (int64_t)p.n_iface * rb3 * subs * 2 <= resident)
    subs *= 2;
  return subs;
}

// A launch that may begin while the previous kernel on the stream drains
// (programmatic dependent launch; in a graph, a programmatic edge): the
// macro-step's kernels wait at their first instruction (griddepcontrol.wait)
// until the previous one has completed and its writes are visible, so the
// order is the stream's; the new grid's launch overlaps the old one's tail.
template <typename... K, typename... A>
void launch_pdl(dim3 g, dim3 b, cudaStream_t st, void (*k)(K...), A &&...args) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = g;
  lc.blockDim = b;
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  cudaLaunchKernelEx(&lc, k, std::forward<A>(args)...);
}

template <int Q>
void launch_coalesce(cudaStream_t st, const float *fp, float *fc, float4 *macc, const float4 *macp,
                     const Amr3Params &p, int subs) {
  const int t = p.rb * p.rb * p.rb * subs;
  switch (subs) {
    case 8: launch_pdl(dim3(p.n_iface), dim3(t), st, amr3_coalesce<Q, 8>, fp, fc, macc, macp, p); break;
    case 4: launch_pdl(dim3(p.n_iface), dim3(t), st, amr3_coalesce<Q, 4>, fp, fc, macc, macp, p); break;
    case 2: launch_pdl(dim3(p.n_iface), dim3(t), st, amr3_coalesce<Q, 2>, fp, fc, macc, macp, p); break;
    default: launch_pdl(dim3(p.n_iface), dim3(t), st, amr3_coalesce<Q, 1>, fp, fc, macc, macp, p); break;
  }
}

// A pool substep, with 32-bit population indices when the pool allows.
template <int Q>
void launch_substep(dim3 gl, cudaStream_t st, const float *fin, float *fout, float4 *macp, const Amr3Params &p,
                    const uint32_t *cells) {
  if ((int64_t)Q * p.P <= INT32_MAX)
    launch_pdl(gl, dim3(kListThreads), st, amr3_substep<Q, true>, fin, fout, macp, p, cells, p.T3);
  else
    launch_pdl(gl, dim3(kListThreads), st, amr3_substep<Q, false>, fin, fout, macp, p, cells, p.T3);
}

// The pool force at time t and its deterministic sum.
template <int Q>
void launch_pool_force(lbm_amr3d *a, const Amr3Params &p, cudaStream_t st) {
  const int r3 = p.RB2 * p.RB2 * p.RB2;
  const dim3 gf((r3 + kTileThreads - 1) / kTileThreads, p.slots);
  launch_pdl(gf, dim3(kTileThreads), st, amr3_force<Q>, (const float *)a->fp[0], p, (const uint32_t *)a->d_cells);
  const int parts = gf.x * gf.y;
  launch_pdl(dim3(sum_groups(parts)), dim3(kSumGroup), st, amr3_force_sum, (const double *)a->partials, parts,
             a->force_groups, a->counter, a->force_out);
}

// One macro-step from L0 parity `cp`.
cudaError_t launch_macro(lbm_amr3d *a, int cp, bool write_mac) {
  Amr3Params p = a->p;
  p.write_mac = write_mac ? 1 : 0;
  const int q = a->q;
  cudaStream_t st = a->stream;
  cudaError_t e = cudaSuccess;
  if (p.slots && a->cfg.iface == 1) {
    // ?interface=interp (main-3d.js:3343-3356): the L0 step first, then the
    // ring interpolated from L0 at t, two substeps with the ring collided,
    // and every tile restricted into L0's new buffer.
    StepParams sp = a->sp;
    sp.write_mac = write_mac ? 1 : 0;
    const dim3 gs((p.nx + kStepThreads - 1) / kStepThreads, p.ny, p.nz);
    const dim3 g = tile_grid(a);
    const dim3 gl((p.T3 + kListThreads - 1) / kListThreads, p.slots);
    const int rb3 = p.rb * p.rb * p.rb;
    const dim3 gd((rb3 + kTileThreads - 1) / kTileThreads, p.slots);
    const int r3 = p.RB2 * p.RB2 * p.RB2;
    const dim3 gf((r3 + kTileThreads - 1) / kTileThreads, p.slots);
    const float tc = a->cfg.root.tau, tf = 2.f * tc - 0.5f;
    const float f2c_rescale = 2.f * (tc - 1.f) / (tf - 1.f);
    AMR3_DISPATCH(q, {
      if (p.c.has_body) launch_pool_force<Q>(a, p, st);
      amr3_coarse<Q><<<gs, kStepThreads, 0, st>>>(a->fc[cp], a->fc[1 - cp], a->macc, sp, a->d_block_slot, p.rb,
                                                   p.nbx, p.nby);
      amr3_interp<Q><<<g, tile_block(a), 0, st>>>(a->fc[cp], a->fp[0], p, 1, nullptr);
      Amr3Params pa = p;
      pa.write_mac = 0;
      const int gc = (p.n_iface * rb3 + kTileThreads - 1) / kTileThreads;
      if (a->flux && gc) amr3_flux<Q><<<gc, kTileThreads, 0, st>>>(a->fp[0], a->flux, p, 0);
      launch_substep<Q>(gl, st, a->fp[0], a->fp[1], a->macp, pa, a->d_cells);
      if (a->flux && gc) amr3_flux<Q><<<gc, kTileThreads, 0, st>>>(a->fp[1], a->flux, p, 1);
      launch_substep<Q>(gl, st, a->fp[1], a->fp[0], a->macp, p, a->d_cells);
      amr3_drain<Q><<<gd, kTileThreads, 0, st>>>(a->fp[0], a->fc[1 - cp], (float4 *)a->macc, p, nullptr,
                                                 f2c_rescale);
      if (a->flux && gc)
        amr3_reflux<Q><<<gc, kTileThreads, 0, st>>>(a->fc[cp], a->fc[1 - cp], (float4 *)a->macc, a->flux, p);
    });
  }
  if (p.slots) {
    const dim3 gl((p.T3 + kListThreads - 1) / kListThreads, p.slots);
    auto body = [&]() -> cudaError_t {
      AMR3_DISPATCH(q, {
        if (p.c.has_body) launch_pool_force<Q>(a, p, st);
        const int r3i = p.RB2 * p.RB2 * p.RB2, nring = p.T3 - r3i;
        const dim3 gr((nring + kListThreads - 1) / kListThreads, p.slots);
        launch_pdl(gr, dim3(kListThreads), st, amr3_explode<Q>, (const float *)a->fc[cp], a->fp[0], p,
                   (const uint32_t *)a->d_cells, r3i, nring);
        Amr3Params pa = p;
        pa.write_mac = 0;
        launch_substep<Q>(gl, st, a->fp[0], a->fp[1], a->macp, pa, a->d_cells);
        launch_substep<Q>(gl, st, a->fp[1], a->fp[0], a->macp, p, a->d_cells);
        if (p.n_iface)
          launch_coalesce<Q>(st, a->fp[0], a->fc[cp], (float4 *)a->macc, a->macp, p, a->coalesce_subs);
      });
    };
    e = body();
    if (e != cudaSuccess) return e;
  }
  StepParams sp = a->sp;
  sp.write_mac = write_mac ? 1 : 0;
  const dim3 gs((p.nx + kStepThreads - 1) / kStepThreads, p.ny, p.nz);
  AMR3_DISPATCH(q, launch_pdl(gs, dim3(kStepThreads), st, amr3_coarse<Q>, (const float *)a->fc[cp], a->fc[1 - cp],
                              a->macc, sp, (const int *)a->d_block_slot, p.rb, p.nbx, p.nby));
}

void destroy_graphs(lbm_amr3d *a) {
  for (auto &g : a->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto &g : a->manage_graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

template <class F> int capture(lbm_amr3d *a, cudaGraphExec_t *out, F &&launches) {
  cudaGraph_t g = nullptr;
  ACK(a, cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = launches();
  cudaError_t e2 = cudaStreamEndCapture(a->stream, &g);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return afail(a, LBM_ECUDA, std::string("capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  ACK(a, e);
  return LBM_OK;
}

int build_graphs(lbm_amr3d *a) {
  for (int cp = 0; cp < 2; ++cp) {
    int rc = capture(a, &a->graph[cp], [&] { return launch_macro(a, cp, false); });
    if (rc) return rc;
    if (a->dynamic) {
      rc = capture(a, &a->manage_graph[cp], [&] { return launch_manage(a, cp); });
      if (rc) return rc;
    }
  }
  return LBM_OK;
}

// Device memory of a hierarchy: its own allocations, or carved in order
// from a caller's block (256-byte granules); `measure` only adds up the bytes.
struct DevCarve {
  char *base = nullptr;
  size_t cap = 0, used = 0;
  bool measure = false;
  template <class T> cudaError_t take(T **ptr, size_t bytes) {
    const size_t b = (bytes + 255) & ~size_t(255);
    if (measure) { *ptr = nullptr; used += b; return cudaSuccess; }
    if (!base) return cudaMalloc(ptr, bytes);
    if (used + b > cap) return cudaErrorMemoryAllocation;
    *ptr = reinterpret_cast<T *>(base + used);
    used += b;
    return cudaSuccess;
  }
};

void release(lbm_amr3d *a) {
  if (a->stream) cudaStreamSynchronize(a->stream);
  destroy_graphs(a);
  for (auto *ptr : {(void *)a->fc[0], (void *)a->fc[1], (void *)a->fp[0], (void *)a->fp[1], (void *)a->macc,
                    (void *)a->macp, (void *)a->d_block_slot, (void *)a->d_slot_to_block, (void *)a->d_iface,
                    (void *)a->partials, (void *)a->force_out, (void *)a->tot_partials, (void *)a->tot_out,
                    (void *)a->counter, (void *)a->tot_counter, (void *)a->d_want, (void *)a->d_slot_new,
                    (void *)a->d_iface_flag, (void *)a->d_free_list, (void *)a->d_counts, (void *)a->flux,
                    (void *)a->d_block_q, (void *)a->d_cells, (void *)a->d_links, (void *)a->d_pulls,
                    (void *)a->force_groups})
    if (!a->carved) cudaFree(ptr);
  if (a->host_out) cudaFreeHost(a->host_out);
  if (a->own) cudaStreamDestroy(a->own);

}

constexpr int kTotBlocks = 296;

}  // namespace

extern "C" {

int lbm_amr3d_config_default(lbm_amr3d_config *c, int q, int nx, int ny, int nz) {
  if (!c) return LBM_EINVAL;
  *c = lbm_amr3d_config{};
  int rc = lbm_config_default(&c->root, q, nx, ny, nz);
  if (rc) return rc;
  c->levels = 2;
  c->rb = 4;
  c->refine = LBM_REFINE_BODY;
  c->margin = 2.0f;
  c->boxfrac = 0.5f;
  c->explode_linear = 1;
  return LBM_OK;
}

const char *lbm_amr3d_last_error(const lbm_amr3d *a) { return a ? a->err.c_str() : g_amr3_error.c_str(); }

}  // extern "C"

namespace {

// The substep's pull sources, the same for every tile: per cell list
// position k, pull_words(q) words (Q rounded up to a multiple of 4, so a
// thread reads its row with 128-bit loads); word i, for direction i, holds
// the neighbour the source lies in (its index in the CTA's 3 x 3 x 3 table,
// 13 = this tile) in bits 0-4, the source cell in that tile in bits 5-17,
// and the cell of this tile it clamps to when that neighbour is not refined
// in bits 18-30 (T3 <= 20^3 < 2^13). DIRECT_GHOST
// (common_d3_amr_step1.wgsl): a source past the interior, toward the tile
// edge the cell sits at, is read from the refined neighbour's interior, else
// from this tile's ring.
std::vector<uint32_t> pull_table(int q, int FB, int RB2, const std::vector<uint32_t> &cl) {
  const int G = kAmrGhost, n = (int)cl.size(), kw = pull_words(q);
  std::vector<uint32_t> t((size_t)kw * n, 0u);
  for (int k = 0; k < n; ++k) {
    const int fi[3] = {(int)(cl[k] & 0xff), (int)((cl[k] >> 8) & 0xff), (int)(cl[k] >> 16)};
    for (int i = 0; i < q; ++i) {
      const int e[3] = {detail::ex27(i), detail::ey27(i), detail::ez27(i)};
      int o[3], sh[3], sc[3];
      for (int a = 0; a < 3; ++a) {
        const int edge = fi[a] <= G ? -1 : (fi[a] + 1 >= G + RB2 ? 1 : 0);
        const int sa = fi[a] - e[a];
        o[a] = (sa < G || sa >= G + RB2) ? edge : 0;
        sh[a] = sa - o[a] * RB2;
        sc[a] = std::min(std::max(sa, 0), FB - 1);
      }
      const uint32_t nb = (uint32_t)((o[2] + 1) * 9 + (o[1] + 1) * 3 + (o[0] + 1));
      const uint32_t ls = (uint32_t)((sh[2] * FB + sh[1]) * FB + sh[0]);
      const uint32_t lc = (uint32_t)((sc[2] * FB + sc[1]) * FB + sc[0]);
      t[(size_t)k * kw + i] = nb | ls << 5 | lc << 18;
    }
  }
  return t;
}

// Builds the hierarchy with its device memory from `mem`; with mem.measure
// nothing touches the GPU and *bytes receives the device bytes it needs.
int amr3_create_impl(const lbm_amr3d_config *c, const uint8_t *block_want, DevCarve &mem, lbm_amr3d **out,
                     size_t *bytes) {
  if (!out) return afail(nullptr, LBM_EINVAL, "out is NULL");
  *out = nullptr;
  std::string why;
  int rc = amr3_validate(c, why);
  if (rc) return afail(nullptr, rc, why);
  if (validate_config(&c->root, why)) return afail(nullptr, LBM_EINVAL, why);
  // the pool's transfers rescale one relaxation time (plans/TRT.md sec 8.0(4)
  // splits them per parity): the hierarchy stays BGK
  if (c->root.trt) return afail(nullptr, LBM_ENOTSUP, "the TRT collision runs in dense, batched and served domains, not in AMR hierarchies");
  if (c->refine == LBM_REFINE_LIST && !block_want) return afail(nullptr, LBM_EINVAL, "refine = list needs block flags");
  auto *a = new lbm_amr3d();
  a->cfg = *c;
  a->q = c->root.q;
  Amr3Params &p = a->p;
  const lbm_config &r = c->root;
  p.nx = r.nx; p.ny = r.ny; p.nz = r.nz; p.rb = c->rb;
  p.nbx = r.nx / c->rb; p.nby = r.ny / c->rb; p.nbz = r.nz / c->rb;
  p.FB = 2 * c->rb + 2 * kAmrGhost;
  p.RB2 = 2 * c->rb;
  p.T3 = p.FB * p.FB * p.FB;
  p.N = (int64_t)r.nx * r.ny * r.nz;
  std::vector<uint8_t> want;
  amr3_want(*c, block_want, want);
  const int nb = p.nbx * p.nby * p.nbz;
  a->block_slot.assign(nb, -1);
  for (int id = 0; id < nb; ++id)
    if (want[id]) {
      a->block_slot[id] = (int)a->slot_to_block.size();
      a->slot_to_block.push_back(id);
    }
  a->initial = (int)a->slot_to_block.size();
  a->dynamic = c->dynamic != 0;
  if (a->dynamic && c->refine != LBM_REFINE_BODY) {
    delete a;
    return afail(nullptr, LBM_ENOTSUP, "dynamic refinement decides by the body's geometry: refine must be body");
  }
  if (a->dynamic && c->manage_every < 1) {
    delete a;
    return afail(nullptr, LBM_EINVAL, "manage_every must be >= 1");
  }
  {
    int cap = a->initial;
    if (c->max_slots > 0) cap = std::max(c->max_slots, a->initial);
    else if (a->dynamic) cap = (int)std::ceil(a->initial * (double)std::max(1.0f, c->slot_headroom));
    a->capacity = std::max(1, std::min(cap, nb));
  }
  a->slot_to_block.resize(a->capacity, -1);
  p.slots = a->capacity;
  p.P = (int64_t)a->capacity * p.T3;
  if (p.N > INT32_MAX) {
    // L0 cells are addressed with 32-bit offsets (2^31 cells of Q >= 19
    // populations would be 150+ GB per buffer)
    delete a;
    return afail(nullptr, LBM_ENOMEM, "L0 grid of more than 2^31 cells");
  }
  if (p.P > INT32_MAX) {
    // the substep addresses pool cells with 32-bit offsets (2^31 cells of
    // Q >= 19 populations would be 150+ GB per buffer)
    delete a;
    return afail(nullptr, LBM_ENOMEM, "pool of more than 2^31 cells");
  }
  // interface blocks: covered, or a covered block among the 26 neighbours
  for (int id = 0; id < nb; ++id) {
    const int bx = id % p.nbx, by = (id / p.nbx) % p.nby, bz = id / (p.nbx * p.nby);
    bool keep = false;
    for (int d = 0; d < 27 && !keep; ++d) {
      const int nx_ = ((bx + d % 3 - 1) % p.nbx + p.nbx) % p.nbx, ny_ = ((by + (d / 3) % 3 - 1) % p.nby + p.nby) % p.nby,
                nz_ = ((bz + d / 9 - 1) % p.nbz + p.nbz) % p.nbz;
      keep = a->block_slot[(nz_ * p.nby + ny_) * p.nbx + nx_] >= 0;
    }
    if (keep) a->iface.push_back(id);
  }
  p.n_iface = (int)a->iface.size();
  if (a->dynamic) p.n_iface = nb;  // every block, filtered by the device's interface flags
  const float tc = r.tau, tf = 2.f * tc - 0.5f;
  p.omega_f = 1.f / tf;
  p.rescale_c2f = 0.5f * (tf - 1.f) / (tc - 1.f);
  p.chi_eps_f = r.chi_eps * 0.5f;
  p.linear = c->explode_linear ? 1 : 0;
  p.collide_ring = c->iface == 1 ? 1 : 0;
  fill_step_params(r, p.N, 0, a->sp);
  a->sp.force_on = 0;
  {
    StepParams tmp = a->sp;
    int box[6];
    force_cell_box(r, tmp, box);  // swept-cell switch and band for the pool force
    a->sp.swept = tmp.swept;
    a->sp.swept_band = tmp.swept_band;
  }
  p.c = a->sp;
  auto bail = [&](cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    release(a);
    delete a;
    return afail(nullptr, e == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA, m);
  };
  cudaError_t e;
  const bool live = !mem.measure;
  a->carved = mem.base != nullptr;
  const size_t fcb = (size_t)a->q * p.N * sizeof(float), fpb = (size_t)a->q * p.P * sizeof(float);
  const int nfree = a->capacity - a->initial;
  const size_t nfl = (size_t)std::max(1, a->capacity);
  // every device allocation, in one order for measuring and for carving
  {
    for (int k = 0; k < 2; ++k) {
      if ((e = mem.take(&a->fc[k], fcb))) return bail(e, "L0 f");
      if ((e = mem.take(&a->fp[k], fpb))) return bail(e, "pool f");
    }
    if ((e = mem.take(&a->macc, (size_t)p.N * 16))) return bail(e, "L0 mac");
    if (c->reflux && (e = mem.take(&a->flux, (size_t)p.N * 16))) return bail(e, "flux");
    if ((e = mem.take(&a->macp, (size_t)p.P * 16))) return bail(e, "pool mac");
    if ((e = mem.take(&a->d_block_slot, nb * sizeof(int)))) return bail(e, "block_slot");
    if ((e = mem.take(&a->d_slot_to_block, a->capacity * sizeof(int)))) return bail(e, "slots");
    if ((e = mem.take(&a->d_iface, std::max(p.n_iface, 1) * sizeof(int)))) return bail(e, "iface");
    if ((e = mem.take(&a->d_cells, (size_t)p.T3 * sizeof(uint32_t)))) return bail(e, "cell list");
    if ((e = mem.take(&a->d_pulls, (size_t)pull_words(a->q) * p.T3 * sizeof(uint32_t)))) return bail(e, "pull table");
    if (r.has_body && r.use_bounceback && (e = mem.take(&a->d_links, (size_t)p.P * sizeof(uint32_t))))
      return bail(e, "link table");
    if (a->dynamic) {
      if ((e = mem.take(&a->d_want, nb))) return bail(e, "want");
      if ((e = mem.take(&a->d_iface_flag, nb))) return bail(e, "flags");
      if ((e = mem.take(&a->d_slot_new, a->capacity))) return bail(e, "new");
      if ((e = mem.take(&a->d_free_list, nfl * sizeof(int)))) return bail(e, "free list");
      if ((e = mem.take(&a->d_counts, 4 * sizeof(int)))) return bail(e, "counts");
      if (c->q_abs > 0 && (e = mem.take(&a->d_block_q, nb * sizeof(float)))) return bail(e, "block Q");
    }
    const int r3 = p.RB2 * p.RB2 * p.RB2;
    a->force_parts = std::max(1, ((r3 + kTileThreads - 1) / kTileThreads) * p.slots);
    if ((e = mem.take(&a->partials, (size_t)a->force_parts * kForceSlots * sizeof(double)))) return bail(e, "partials");
    if ((e = mem.take(&a->force_out, kForceSlots * sizeof(double)))) return bail(e, "force");
    if ((e = mem.take(&a->force_groups, (size_t)sum_groups(a->force_parts) * kForceSlots * sizeof(double))))
      return bail(e, "force");
    if ((e = mem.take(&a->counter, sizeof(unsigned int)))) return bail(e, "counter");
    if ((e = mem.take(&a->tot_partials, (size_t)kTotBlocks * 4 * sizeof(double)))) return bail(e, "totals");
    if ((e = mem.take(&a->tot_out, 4 * sizeof(double)))) return bail(e, "totals");
    if ((e = mem.take(&a->tot_counter, sizeof(unsigned int)))) return bail(e, "totals");
  }
  if (!live) {
    *bytes = mem.used;
    delete a;
    return LBM_OK;
  }
  if ((e = cudaStreamCreateWithFlags(&a->own, cudaStreamNonBlocking))) return bail(e, "stream");

  a->stream = a->own;
  for (int k = 0; k < 2; ++k)
    if ((e = cudaMemsetAsync(a->fp[k], 0, fpb, a->own))) return bail(e, "memset pool f");
  if (a->flux && (e = cudaMemsetAsync(a->flux, 0, (size_t)p.N * 16, a->own))) return bail(e, "memset flux");
  if ((e = cudaMemsetAsync(a->macp, 0, (size_t)p.P * 16, a->own))) return bail(e, "memset pool mac");
  cudaMemcpyAsync(a->d_block_slot, a->block_slot.data(), nb * sizeof(int), cudaMemcpyHostToDevice, a->own);
  cudaMemcpyAsync(a->d_slot_to_block, a->slot_to_block.data(), a->capacity * sizeof(int), cudaMemcpyHostToDevice,
                  a->own);
  {
    std::vector<uint32_t> cl;
    cl.reserve(p.T3);
    for (int pass = 0; pass < 2; ++pass)
      for (int z = 0; z < p.FB; ++z)
        for (int y = 0; y < p.FB; ++y)
          for (int x = 0; x < p.FB; ++x) {
            auto in = [&](int j) { return j >= kAmrGhost && j < kAmrGhost + p.RB2; };
            if ((in(x) && in(y) && in(z)) == (pass == 0)) cl.push_back(x | (y << 8) | (z << 16));
          }
    cudaMemcpyAsync(a->d_cells, cl.data(), cl.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, a->own);
    const std::vector<uint32_t> pt = pull_table(a->q, p.FB, p.RB2, cl);
    cudaMemcpyAsync(a->d_pulls, pt.data(), pt.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, a->own);
  }
  if (a->dynamic) {
    std::vector<unsigned char> flag(nb, 0);
    for (int id : a->iface) flag[id] = 1;
    cudaMemcpyAsync(a->d_iface_flag, flag.data(), nb, cudaMemcpyHostToDevice, a->own);
    std::vector<int> fl(nfl, 0);
    for (int i = 0; i < nfree; ++i) fl[i] = a->initial + i;
    const int counts[4] = {nfree, 0, nfree, 0};
    cudaMemsetAsync(a->d_want, 0, nb, a->own);
    cudaMemsetAsync(a->d_slot_new, 0, a->capacity, a->own);
    cudaMemcpyAsync(a->d_free_list, fl.data(), fl.size() * sizeof(int), cudaMemcpyHostToDevice, a->own);
    cudaMemcpyAsync(a->d_counts, counts, sizeof(counts), cudaMemcpyHostToDevice, a->own);
    if (c->q_abs > 0) {
      // main-3d.js: REFINE_THRESH = 1/2 log2 max(Q_ABS, 1e-30), COARSEN_THRESH
      // one hysteresis band lower, both as thresholds on Q itself
      const double qr = std::max((double)c->q_abs, 1e-30);
      a->q_refine = (float)qr;
      a->q_hold = (float)(qr * std::exp2(-2.0 * (double)c->q_hyst));
    }
  }
  if (p.n_iface)
    cudaMemcpyAsync(a->d_iface, a->iface.data(), p.n_iface * sizeof(int), cudaMemcpyHostToDevice, a->own);
  if ((e = cudaMemsetAsync(a->counter, 0, sizeof(unsigned int), a->own))) return bail(e, "counter");
  if ((e = cudaMemsetAsync(a->force_out, 0, kForceSlots * sizeof(double), a->own))) return bail(e, "force");
  if ((e = cudaMemsetAsync(a->tot_counter, 0, sizeof(unsigned int), a->own))) return bail(e, "totals");
  if ((e = cudaMallocHost(&a->host_out, 16 * sizeof(double)))) return bail(e, "cudaMallocHost");
  // set-up is ordered on the hierarchy's own stream: it waits for nothing
  // else on the device (a server admits hierarchies while ticks run)
  if ((e = cudaStreamSynchronize(a->own))) return bail(e, "set-up");
  p.block_slot = a->d_block_slot;
  p.slot_to_block = a->d_slot_to_block;
  p.iface = a->dynamic ? nullptr : a->d_iface;
  p.iface_flag = a->d_iface_flag;
  p.partials = a->partials;
  p.counter = a->counter;
  p.force_out = a->force_out;
  p.links = a->d_links;  // filled when the hierarchy is seeded
  p.pulls = a->d_pulls;
  {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    a->coalesce_subs = coalesce_subs(p, std::max(sms, 1));
  }
  *out = a;
  return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_amr3d_create(const lbm_amr3d_config *c, const uint8_t *block_want, lbm_amr3d **out) {
  DevCarve mem;
  return amr3_create_impl(c, block_want, mem, out, nullptr);
}

int lbm_amr3d_device_bytes(const lbm_amr3d_config *c, const uint8_t *block_want, int64_t *bytes) {
  if (!bytes) return LBM_EINVAL;
  DevCarve mem;
  mem.measure = true;
  lbm_amr3d *a = nullptr;
  size_t b = 0;
  const int rc = amr3_create_impl(c, block_want, mem, &a, &b);
  if (rc) return rc;
  *bytes = (int64_t)b;
  return LBM_OK;
}

int lbm_amr3d_create_in(const lbm_amr3d_config *c, const uint8_t *block_want, void *device_base, int64_t capacity,
                        lbm_amr3d **out) {
  if (!device_base || capacity <= 0) return afail(nullptr, LBM_EINVAL, "device block is NULL or empty");
  if ((uintptr_t)device_base % 256) return afail(nullptr, LBM_EINVAL, "device block must be 256-byte aligned");
  DevCarve mem;
  mem.base = (char *)device_base;
  mem.cap = (size_t)capacity;
  return amr3_create_impl(c, block_want, mem, out, nullptr);
}

void lbm_amr3d_destroy(lbm_amr3d *a) {
  if (!a) return;
  release(a);
  delete a;
}

int lbm_amr3d_set_stream(lbm_amr3d *a, void *cuda_stream) {
  if (!a) return LBM_EINVAL;
  cudaStreamSynchronize(a->stream);
  a->stream = cuda_stream ? (cudaStream_t)cuda_stream : a->own;
  destroy_graphs(a);
  return LBM_OK;
}

int lbm_amr3d_init_macro(lbm_amr3d *a, const float *mac) {
  if (!a || !mac) return a ? afail(a, LBM_EINVAL, "mac is NULL") : LBM_EINVAL;
  const size_t bytes = (size_t)a->p.N * 16;
  ACK(a, cudaMemcpyAsync(a->macc, mac, bytes, cudaMemcpyHostToDevice, a->stream));
  for (int k = 0; k < 2; ++k)
    ACK(a, launch_init_eq(a->q, LBM_STORE_FP32, a->macc, a->fc[k], a->p.N, a->sp.pk, a->stream));
  ACK(a, launch_interp(a, a->fc[0], 0, nullptr));
  ACK(a, launch_links(a, nullptr));
  ACK(a, launch_moments(a));
  ACK(a, cudaStreamSynchronize(a->stream));
  a->cp = 0;
  a->step_count = 0;
  a->seeded = true;
  return LBM_OK;
}

int lbm_amr3d_step(lbm_amr3d *a, int n) {
  if (!a) return LBM_EINVAL;
  if (n < 0) return afail(a, LBM_EINVAL, "step count must be >= 0");
  if (!a->seeded) return afail(a, LBM_EINVAL, "call lbm_amr3d_init_macro first");
  if ((n > 1 || a->dynamic) && !a->graph[0]) {
    int rc = build_graphs(a);
    if (rc) return rc;
  }
  const lbm_amr3d_config &c = a->cfg;
  auto manages = [&](int64_t s) {
    return a->dynamic && s >= c.manage_start && (s - c.manage_start) % c.manage_every == 0;
  };
  for (int k = 0; k < n; ++k) {
    if (manages(a->step_count)) ACK(a, cudaGraphLaunch(a->manage_graph[a->cp], a->stream));
    // the field criterion reads the L0 velocity of the macro-step before it
    if (a->d_block_q && manages(a->step_count + 1)) ACK(a, launch_macro(a, a->cp, true));
    else if (k < n - 1) ACK(a, cudaGraphLaunch(a->graph[a->cp], a->stream));
    else ACK(a, launch_macro(a, a->cp, true));
    a->cp = 1 - a->cp;
    a->step_count += 1;
  }
  return LBM_OK;
}

int lbm_amr3d_manage_now(lbm_amr3d *a) {
  if (!a) return LBM_EINVAL;
  if (!a->dynamic) return afail(a, LBM_EINVAL, "the hierarchy is static (dynamic = 0)");
  if (!a->seeded) return afail(a, LBM_EINVAL, "call lbm_amr3d_init_macro first");
  if (!a->graph[0]) {
    int rc = build_graphs(a);
    if (rc) return rc;
  }
  ACK(a, cudaGraphLaunch(a->manage_graph[a->cp], a->stream));
  return LBM_OK;
}

int lbm_amr3d_set_body(lbm_amr3d *a, const lbm_body *body) {
  if (!a || !body) return a ? afail(a, LBM_EINVAL, "body is NULL") : LBM_EINVAL;
  if (!a->cfg.root.has_body) return afail(a, LBM_EINVAL, "the hierarchy has no body");
  lbm_config r = a->cfg.root;
  r.body = *body;
  std::string why;
  if (validate_config(&r, why)) return afail(a, LBM_EINVAL, why);
  ACK(a, cudaStreamSynchronize(a->stream));
  a->cfg.root = r;
  a->sp.body = *body;
  StepParams tmp = a->sp;
  int box[6];
  force_cell_box(r, tmp, box);
  a->sp.swept = tmp.swept;
  a->sp.swept_band = tmp.swept_band;
  a->p.c = a->sp;
  destroy_graphs(a);
  if (a->seeded) ACK(a, launch_links(a, nullptr));
  return LBM_OK;
}

int lbm_amr3d_set_links(lbm_amr3d *a, int on) {
  if (!a) return LBM_EINVAL;
  ACK(a, cudaStreamSynchronize(a->stream));
  destroy_graphs(a);
  a->p.links = on ? a->d_links : nullptr;
  if (a->seeded) ACK(a, launch_links(a, nullptr));
  return LBM_OK;
}

int lbm_amr3d_links(const lbm_amr3d *a) { return a && a->p.links ? 1 : 0; }

int lbm_amr3d_block_q(lbm_amr3d *a, float lead, float *block_q) {
  if (!a || !block_q) return a ? afail(a, LBM_EINVAL, "block_q is NULL") : LBM_EINVAL;
  if (!std::isfinite(lead) || lead < 0) return afail(a, LBM_EINVAL, "lead must be finite and >= 0");
  const int nb = a->p.nbx * a->p.nby * a->p.nbz;
  float *d = a->d_block_q;
  if (!d) ACK(a, cudaMallocAsync(&d, nb * sizeof(float), a->stream));
  amr3_criterion<<<nb, kCritThreads, 0, a->stream>>>((const float4 *)a->macc, d, a->p, lead);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(block_q, d, nb * sizeof(float), cudaMemcpyDeviceToHost, a->stream);
  if (d != a->d_block_q) cudaFreeAsync(d, a->stream);
  ACK(a, e);
  ACK(a, cudaStreamSynchronize(a->stream));
  return LBM_OK;
}

int lbm_amr3d_resample(lbm_amr3d *a, const lbm_volume_spec *spec, void *out, uint8_t *level) {
  if (!a) return LBM_EINVAL;
  std::string why;
  if (validate_volume(spec, why)) return afail(a, LBM_EINVAL, why);
  if (!out) return afail(a, LBM_EINVAL, "out is NULL");
  const Amr3Params &p = a->p;
  const TreeView t{(const float4 *)a->macc, p.nx, p.ny, p.nz, p.slots ? 1 : 0, (const float4 *)a->macp,
                   a->d_block_slot, p.rb, p.FB, p.T3};
  ACK(a, run_resample(t, *spec, out, level, a->stream));
  return LBM_OK;
}

int lbm_amr3d_render_slice(lbm_amr3d *a, const lbm_slice_spec *spec, uint8_t *rgba) {
  if (!a) return LBM_EINVAL;
  const Amr3Params &p = a->p;
  std::string why;
  if (validate_slice(spec, p.nx, p.ny, p.nz, why)) return afail(a, LBM_EINVAL, why);
  if (!rgba) return afail(a, LBM_EINVAL, "rgba is NULL");
  const lbm_config &c = a->cfg.root;
  ViewOffset off{{0.f, 0.f, 0.f}};
  const float ctr[3] = {c.body.cx, c.body.cy, c.body.cz};
  for (int k = 0; k < 3; ++k)
    if (c.window[k]) off.v[k] = ctr[k] - (float)c.win_anchor[k];
  const TreeView t{(const float4 *)a->macc, p.nx, p.ny, p.nz, p.slots ? 1 : 0, (const float4 *)a->macp,
                   a->d_block_slot, p.rb, p.FB, p.T3};
  ACK(a, run_slice(t, *spec, off, rgba, a->stream));
  return LBM_OK;
}

int lbm_amr3d_pool_stats(lbm_amr3d *a, int32_t out[4]) {
  if (!a || !out) return a ? afail(a, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  if (!a->dynamic) {
    out[0] = a->initial; out[1] = 0; out[2] = a->capacity - a->initial; out[3] = 0;
    return LBM_OK;
  }
  int counts[4];
  ACK(a, cudaMemcpyAsync(counts, a->d_counts, sizeof(counts), cudaMemcpyDeviceToHost, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  out[0] = a->capacity - counts[0];
  out[1] = counts[1];
  out[2] = counts[2];
  out[3] = counts[3];
  return LBM_OK;
}

int lbm_amr3d_forces(lbm_amr3d *a, double out[6]) {
  if (!a || !out) return a ? afail(a, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  ACK(a, cudaMemcpyAsync(a->host_out, a->force_out, 6 * sizeof(double), cudaMemcpyDeviceToHost, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  for (int k = 0; k < 6; ++k) out[k] = a->host_out[k];
  return LBM_OK;
}

int lbm_amr3d_totals(lbm_amr3d *a, double out[4]) {
  if (!a || !out) return a ? afail(a, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  const int64_t nb = (a->p.N + kTotThreads - 1) / kTotThreads;
  const int grid = (int)std::min<int64_t>(kTotBlocks, nb);
  amr3_totals<<<grid, kTotThreads, 0, a->stream>>>((const float4 *)a->macc, a->p.N, a->tot_partials, a->tot_counter,
                                                  a->tot_out);
  ACK(a, cudaGetLastError());
  ACK(a, cudaMemcpyAsync(a->host_out, a->tot_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  for (int k = 0; k < 4; ++k) out[k] = a->host_out[k];
  return LBM_OK;
}

int lbm_amr3d_read_coarse(lbm_amr3d *a, float *f, float *mac) {
  if (!a) return LBM_EINVAL;
  if (f) ACK(a, cudaMemcpyAsync(f, a->fc[a->cp], (size_t)a->q * a->p.N * 4, cudaMemcpyDeviceToHost, a->stream));
  if (mac) ACK(a, cudaMemcpyAsync(mac, a->macc, (size_t)a->p.N * 16, cudaMemcpyDeviceToHost, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  return LBM_OK;
}

int lbm_amr3d_read_pool(lbm_amr3d *a, float *f, float *mac) {
  if (!a) return LBM_EINVAL;
  const int64_t used = (int64_t)a->p.slots * a->p.T3;
  if (f)
    for (int i = 0; i < a->q; ++i)
      ACK(a, cudaMemcpyAsync(f + i * used, a->fp[0] + (int64_t)i * a->p.P, used * 4, cudaMemcpyDeviceToHost, a->stream));
  if (mac) ACK(a, cudaMemcpyAsync(mac, a->macp, used * 16, cudaMemcpyDeviceToHost, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  return LBM_OK;
}

int lbm_amr3d_topology(lbm_amr3d *a, int32_t *block_slot, int32_t *slot_to_block, int32_t counts[3]) {
  if (!a) return LBM_EINVAL;
  if (a->dynamic) {
    ACK(a, cudaMemcpyAsync(a->block_slot.data(), a->d_block_slot, a->block_slot.size() * sizeof(int),
                           cudaMemcpyDeviceToHost, a->stream));
    ACK(a, cudaMemcpyAsync(a->slot_to_block.data(), a->d_slot_to_block, a->capacity * sizeof(int),
                           cudaMemcpyDeviceToHost, a->stream));
    ACK(a, cudaStreamSynchronize(a->stream));
  }
  if (block_slot) std::memcpy(block_slot, a->block_slot.data(), a->block_slot.size() * sizeof(int32_t));
  if (slot_to_block) std::memcpy(slot_to_block, a->slot_to_block.data(), a->capacity * sizeof(int32_t));
  if (counts) { counts[0] = a->capacity; counts[1] = a->p.FB; counts[2] = (int32_t)a->block_slot.size(); }
  return LBM_OK;
}

int64_t lbm_amr3d_cell_updates(lbm_amr3d *a) {
  if (!a) return 0;
  int32_t st[4];
  if (lbm_amr3d_pool_stats(a, st)) return 0;
  const int64_t rb3 = (int64_t)a->p.rb * a->p.rb * a->p.rb, fine = (int64_t)a->p.RB2 * a->p.RB2 * a->p.RB2;
  return a->p.N - (int64_t)st[0] * rb3 + 2 * (int64_t)st[0] * fine;
}

int lbm_amr3d_sync(lbm_amr3d *a) {
  if (!a) return LBM_EINVAL;
  ACK(a, cudaStreamSynchronize(a->stream));
  return LBM_OK;
}

}  // extern "C"
