// 2D block-structured AMR (D2Q9, root + one pool level) on the device.
//
// Layout in HBM:
//   root      dense W x H, 9 planes, two buffers; mac float4 per cell (the
//             root velocity the criterion reads).
//   pool      S tiles of FB x FB cells (FB = 2 RB + 4: one block of RB x RB
//             root cells refined 2:1, plus a 2-cell ring), 9 planes of S*FB^2,
//             two buffers (a/b), slot-major `slot*FB^2 + fy*FB + fx` (the
//             reference's pool layout, amr2d.mjs:220 makePool).
//   topology  blockSlot[NBX*NBY], slotToBlock[S], parentSlot[S],
//             freeList[S/4] (quads), counts {free quads, active slots},
//             activeList[S], want/criterion[NBX*NBY], newly[S].
//
// One macro-step (main-cylinder-amr.js:1831 dispatchMacroStep, `interp`
// interface of amr2d-gpu.mjs:1120 S_Advance):
//   [every refine_every: criterion -> decide -> coarsen/refine (serial,
//    deterministic) -> active list -> whole-tile fill of new tiles]
//   force on the pool (FP64, deterministic)   amr_force1.wgsl
//   ring fill from neighbour or root          common_interp_kernel.wgsl GHOST_ONLY
//   root step (dense d2 kernel, writes mac)   amr_step1.wgsl NO_PARENT
//   pool substep a->b, b->a at tau_f          amr_step1.wgsl stepCell
//   restriction of the pool into the root     common_average.wgsl
// Every pool kernel runs one CTA per slot of the active list (count read on
// the device), so the non-refine macro-step is topology-independent and is
// replayed from a CUDA graph.

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lbm.h"
#include "cell_update.cuh"
#include "scan.cuh"
#include "dense.cuh"
#include "host_params.cuh"

namespace lbm {
namespace {

constexpr int kPoolThreads = 256;
// Cell-parallel tile kernels (substep, fill, explode): one CTA per
// (active tile, chunk of kChunk cells), so that a few tiles still spread
// over every SM.
constexpr int kChunk = 128;

struct AmrParams {
  int W, H, RB, G, FB, RB2, NBX, NBY, PNX, PNY, S;
  int64_t N0, N1;
  float tau_c, tau_f, omega_f, eps_f, sponge_w, sux, suy, fx, fy, margin, lookahead;
  float resc_c2f, resc_f2c;
  double thr;
  int vort_on, bb, solid_eq;
  int explode, linear;  // explode/coalesce interface; its linear explosion
  float ftarget[9];
  lbm_body body;
  int *blockSlot, *slotToBlock, *parentSlot, *freeList, *counts, *activeList;
  unsigned *want, *newly;
  float *crit;
  double *partials;
  unsigned *counter;
  double *force_out;
};

using L9 = Lattice<9>;

__device__ __forceinline__ float feq9(float rho, float ux, float uy, int i) {
  const float eu = (float)L9::ex(i) * ux + (float)L9::ey(i) * uy;
  return L9::w(i) * rho * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * (ux * ux + uy * uy));
}

__device__ __forceinline__ float pool_pos(const AmrParams &p, int b, int f) {
  return (float)(b * p.RB) - 0.25f + 0.5f * (float)(f - p.G);
}

__device__ __forceinline__ int64_t pcell(const AmrParams &p, int slot, int fx, int fy) {
  return (int64_t)slot * p.FB * p.FB + (int64_t)fy * p.FB + fx;
}

// ---- refine round ------------------------------------------------------------

// Max |discrete curl| of the root velocity over each level-1 block's RB x RB
// root cells (amr_criterion_pool.wgsl, GHOST == 0 branch). Every operation is
// rounded on its own so the value is reproducible bit for bit.
__global__ void amr_criterion(const float4 *__restrict__ mac, const __grid_constant__ AmrParams p) {
  const int b = blockIdx.x;
  const int bx = b % p.NBX, by = b / p.NBX;
  float m = 0.f;
  for (int k = threadIdx.x; k < p.RB * p.RB; k += blockDim.x) {
    const int x = bx * p.RB + k % p.RB, y = by * p.RB + k / p.RB;
    const int xp = x + 1 == p.W ? 0 : x + 1, xm = x == 0 ? p.W - 1 : x - 1;
    const int yp = y + 1 == p.H ? 0 : y + 1, ym = y == 0 ? p.H - 1 : y - 1;
    const float a = mac[(int64_t)y * p.W + xp].z, bb = mac[(int64_t)y * p.W + xm].z;
    const float c = mac[(int64_t)yp * p.W + x].y, d = mac[(int64_t)ym * p.W + x].y;
    const float om = __fsub_rn(__fmul_rn(__fsub_rn(a, bb), 0.5f), __fmul_rn(__fsub_rn(c, d), 0.5f));
    m = fmaxf(m, fabsf(om));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ float sm[32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float r = 0.f;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) r = fmaxf(r, sm[w]);
    p.crit[b] = r;
  }
}

// nearBodyBox (common_geometry.wgsl:230-290): branch and bound on a
// 1-Lipschitz distance, conservative at every depth.
__device__ bool near_body_box(const AmrParams &p, float cx, float cy, float half) {
  const float SQRT2_UP = 1.4142136f;
  lbm_body fut = p.body;
  fut.theta = __fadd_rn(p.body.theta, __fmul_rn(p.body.wz, p.lookahead));
  float sx[16], sy[16], sh[16];
  int sd[16];
  int sp = 0;
  sx[0] = cx; sy[0] = cy; sh[0] = half; sd[0] = 3; sp = 1;
  const float Wf = (float)p.W, Hf = (float)p.H;
  while (sp > 0) {
    --sp;
    const float x = sx[sp], y = sy[sp], h = sh[sp];
    const int d = sd[sp];
    const float now = phi2(x, y, p.body, Wf, Hf);
    const float fu = phi2(__fsub_rn(x, __fmul_rn(p.body.vx, p.lookahead)),
                          __fsub_rn(y, __fmul_rn(p.body.vy, p.lookahead)), fut, Wf, Hf);
    const float phi = fminf(now, fu);
    if (__fsub_rn(phi, __fmul_rn(h, SQRT2_UP)) > p.margin) continue;
    if (phi <= p.margin) return true;
    if (d == 0) return true;
    const float hh = __fmul_rn(h, 0.5f);
    for (int i = 0; i < 4; ++i) {
      sx[sp] = __fadd_rn(x, (i & 1) ? hh : -hh);
      sy[sp] = __fadd_rn(y, (i & 2) ? hh : -hh);
      sh[sp] = hh;
      sd[sp] = d - 1;
      ++sp;
    }
  }
  return false;
}

// decide (amr_manage_pool.wgsl): per root block, want all four children if
// the body is within the margin of the block (now or lookahead steps on) or
// the block's vorticity reaches the refine threshold.
__global__ void amr_decide(const __grid_constant__ AmrParams p) {
  const int pb = blockIdx.x * blockDim.x + threadIdx.x;
  if (pb >= p.PNX * p.PNY) return;
  const int bxP = pb % p.PNX, byP = pb / p.PNX;
  float mc = 0.f;
  for (int q = 0; q < 4; ++q) mc = fmaxf(mc, p.crit[(byP * 2 + (q >> 1)) * p.NBX + bxP * 2 + (q & 1)]);
  const bool vort = p.vort_on && fmax((double)mc, 1e-6) >= p.thr;
  const float half = (float)p.RB;
  const float cx = (float)(bxP * p.RB2) + half - 0.5f, cy = (float)(byP * p.RB2) + half - 0.5f;
  const bool w = vort || near_body_box(p, cx, cy, half);
  for (int q = 0; q < 4; ++q) p.want[(byP * 2 + (q >> 1)) * p.NBX + bxP * 2 + (q & 1)] = w ? 1u : 0u;
}

// Coarsen then refine in the deterministic serial order of DET_SLOTS
// (amr_manage_pool.wgsl coarsen/refine), then compact the active list
// (amr_active_list.wgsl).
// One CTA of kManageThreads, the serial order kept exactly: dying quads
// pushed on the free stack in ascending slot order, parents wanting
// refinement served in ascending parent id from the top of the stack (the
// rest refused), then the active list compacted in ascending slot order --
// each a block-wide prefix sum over the candidates.
constexpr int kManageThreads = 1024;

__global__ void __launch_bounds__(kManageThreads) amr_coarsen_refine(const __grid_constant__ AmrParams p) {
  __shared__ int sm[64];
  int count = p.counts[0];
  // coarsen: quads whose first block is no longer wanted
  const int nquads = p.S / 4;
  for (int base = 0; base < nquads; base += kManageThreads) {
    const int q = base + threadIdx.x;
    int dying = 0;
    if (q < nquads) {
      const int b = p.slotToBlock[4 * q];
      dying = (b >= 0 && !p.want[b]) ? 1 : 0;
    }
    int total;
    const int r = block_scan(dying, sm, total);
    if (dying) {
      p.freeList[count + r] = q;
      for (int k = 0; k < 4; ++k) {
        const int bb = p.slotToBlock[4 * q + k];
        if (bb >= 0) p.blockSlot[bb] = -1;
        p.slotToBlock[4 * q + k] = -1;
      }
    }
    count += total;
  }
  __syncthreads();
  // refine: parents whose first child is unrefined and wanted
  const int np = p.PNX * p.PNY;
  for (int base = 0; base < np; base += kManageThreads) {
    const int ps = base + threadIdx.x;
    int need = 0, bxP = 0, byP = 0;
    if (ps < np) {
      bxP = ps % p.PNX;
      byP = ps / p.PNX;
      const int b0 = (byP * 2) * p.NBX + bxP * 2;
      need = (p.blockSlot[b0] < 0 && p.want[b0]) ? 1 : 0;
    }
    int total;
    const int r = block_scan(need, sm, total);
    if (need && r < count) {
      const int quad = p.freeList[count - 1 - r];
      for (int qy = 0; qy < 2; ++qy)
        for (int qx = 0; qx < 2; ++qx) {
          const int slot = quad * 4 + qx + 2 * qy;
          const int bid = (byP * 2 + qy) * p.NBX + bxP * 2 + qx;
          p.blockSlot[bid] = slot;
          p.slotToBlock[slot] = bid;
          p.parentSlot[slot] = ps;
          p.newly[slot] = 1u;
        }
    }
    count -= min(total, count);
    __syncthreads();
  }
  if (threadIdx.x == 0) p.counts[0] = count;
  // the active list
  int n = 0;
  for (int base = 0; base < p.S; base += kManageThreads) {
    const int s = base + threadIdx.x;
    const int act = (s < p.S && p.slotToBlock[s] >= 0) ? 1 : 0;
    int total;
    const int r = block_scan(act, sm, total);
    if (act) p.activeList[n + r] = s;
    n += total;
  }
  if (threadIdx.x == 0) p.counts[1] = n;
}

// ---- transfers ------------------------------------------------------------------

struct Sample {
  float rho, ux, uy, fneq[9];
};

__device__ __forceinline__ void sample_root(const AmrParams &p, const float *__restrict__ f0, int gx, int gy,
                                            Sample &s) {
  gx = ((gx % p.W) + p.W) % p.W;
  gy = ((gy % p.H) + p.H) % p.H;
  const int64_t cell = (int64_t)gy * p.W + gx;
  float f[9], rho = 0.f, ux = 0.f, uy = 0.f;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    f[i] = __ldg(f0 + i * p.N0 + cell);
    rho += f[i];
    ux += f[i] * (float)L9::ex(i);
    uy += f[i] * (float)L9::ey(i);
  }
  ux /= fmaxf(rho, 1e-6f);
  uy /= fmaxf(rho, 1e-6f);
  s.rho = rho; s.ux = ux; s.uy = uy;
#pragma unroll
  for (int i = 0; i < 9; ++i) s.fneq[i] = f[i] - feq9(rho, ux, uy, i);
}

// Bilinear rho, u, fneq from the four root cells around the pool cell,
// f = feq + 0.5 (tf-1)/(tc-1) fneq (common_interp.wgsl interpCoarseToFine).
__device__ void interp_cell(const AmrParams &p, const float *__restrict__ f0, float *__restrict__ f1, int slot,
                            int bx, int by, int fx, int fy) {
  const float px = pool_pos(p, bx, fx), py = pool_pos(p, by, fy);
  const int x0 = (int)floorf(px), y0 = (int)floorf(py);
  const float tx = px - (float)x0, ty = py - (float)y0;
  Sample s00, s10, s01, s11;
  sample_root(p, f0, x0, y0, s00);
  sample_root(p, f0, x0 + 1, y0, s10);
  sample_root(p, f0, x0, y0 + 1, s01);
  sample_root(p, f0, x0 + 1, y0 + 1, s11);
  const float w00 = (1.f - tx) * (1.f - ty), w10 = tx * (1.f - ty), w01 = (1.f - tx) * ty, w11 = tx * ty;
  const float rho = w00 * s00.rho + w10 * s10.rho + w01 * s01.rho + w11 * s11.rho;
  const float ux = w00 * s00.ux + w10 * s10.ux + w01 * s01.ux + w11 * s11.ux;
  const float uy = w00 * s00.uy + w10 * s10.uy + w01 * s01.uy + w11 * s11.uy;
  const int64_t cell = pcell(p, slot, fx, fy);
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const float fneq = w00 * s00.fneq[i] + w10 * s10.fneq[i] + w01 * s01.fneq[i] + w11 * s11.fneq[i];
    f1[i * p.N1 + cell] = feq9(rho, ux, uy, i) + p.resc_c2f * fneq;
  }
}

// One ring cell of tile `s` (block bx, by): the same-level neighbour's
// interior cell when that neighbour is refined, else root interpolation.
__device__ __forceinline__ void fill_ring_cell(const AmrParams &p, const float *__restrict__ f0,
                                               float *__restrict__ f1, int s, int bx, int by, int fx, int fy) {
  const int bxm = (bx + p.NBX - 1) % p.NBX, bxp = (bx + 1) % p.NBX;
  const int bym = (by + p.NBY - 1) % p.NBY, byp = (by + 1) % p.NBY;
  const int G = p.G, RB2 = p.RB2;
  const bool inX = fx >= G && fx < G + RB2, inY = fy >= G && fy < G + RB2;
  int ns, nfx = fx, nfy = fy;
  if (inY && fx < G) { ns = p.blockSlot[by * p.NBX + bxm]; nfx = fx + RB2; }
  else if (inY && fx >= G + RB2) { ns = p.blockSlot[by * p.NBX + bxp]; nfx = fx - RB2; }
  else if (inX && fy < G) { ns = p.blockSlot[bym * p.NBX + bx]; nfy = fy + RB2; }
  else if (inX && fy >= G + RB2) { ns = p.blockSlot[byp * p.NBX + bx]; nfy = fy - RB2; }
  else if (fx < G && fy < G) { ns = p.blockSlot[bym * p.NBX + bxm]; nfx = fx + RB2; nfy = fy + RB2; }
  else if (fx >= G + RB2 && fy < G) { ns = p.blockSlot[bym * p.NBX + bxp]; nfx = fx - RB2; nfy = fy + RB2; }
  else if (fx < G && fy >= G + RB2) { ns = p.blockSlot[byp * p.NBX + bxm]; nfx = fx + RB2; nfy = fy - RB2; }
  else { ns = p.blockSlot[byp * p.NBX + bxp]; nfx = fx - RB2; nfy = fy - RB2; }
  if (ns >= 0) {
    const int64_t dst = pcell(p, s, fx, fy), src = pcell(p, ns, nfx, nfy);
#pragma unroll
    for (int i = 0; i < 9; ++i) f1[i * p.N1 + dst] = f1[i * p.N1 + src];
  } else {
    interp_cell(p, f0, f1, s, bx, by, fx, fy);
  }
}

// mode 0: ring of every active tile (same-level neighbour copy, else root
// interpolation); mode 1: every cell of the tiles activated this round.
__global__ void __launch_bounds__(kChunk)
    amr_fill(const float *__restrict__ f0, float *__restrict__ f1, int mode, const __grid_constant__ AmrParams p) {
  const int n = p.counts[1];
  const int FB2 = p.FB * p.FB, nch = (FB2 + kChunk - 1) / kChunk;
  for (int w = blockIdx.x; w < n * nch; w += gridDim.x) {
    const int k = w / nch, c0 = (w % nch) * kChunk, c1 = min(c0 + kChunk, FB2);
    const int s = p.activeList[k];
    if (mode == 1 && !p.newly[s]) continue;
    const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
    const int G = p.G, RB2 = p.RB2, FB = p.FB;
    for (int c = c0 + threadIdx.x; c < c1; c += kChunk) {
      const int fx = c % FB, fy = c / FB;
      const bool inX = fx >= G && fx < G + RB2, inY = fy >= G && fy < G + RB2;
      if (mode == 1) {
        interp_cell(p, f0, f1, s, bx, by, fx, fy);
        continue;
      }
      if (inX && inY) continue;
      fill_ring_cell(p, f0, f1, s, bx, by, fx, fy);
    }
  }
}

// One pool substep (amr_step1.wgsl stepCell): DIRECT_GHOST pull (a source
// past the tile interior comes from the same-level neighbour's interior when
// that neighbour is refined, else from this tile's ring), BGK + Guo at
// tau_f with the chi penalty on this level's band, sponge, SOLID_EQ. Every
// cell of the tile, ring included, collides (COLLIDE_RING = 1).
__device__ __forceinline__ void substep_cell(const AmrParams &p, const float *__restrict__ fin,
                                             float *__restrict__ fout, float2 *__restrict__ vel1, int s, int bx,
                                             int by, int fx, int fy) {
  const float Wf = (float)p.W, Hf = (float)p.H;
  const int bxm = (bx + p.NBX - 1) % p.NBX, bxp = (bx + 1) % p.NBX;
  const int bym = (by + p.NBY - 1) % p.NBY, byp = (by + 1) % p.NBY;
  const int G = p.G, RB2 = p.RB2, FB = p.FB;
  const int offX = fx <= G ? -1 : (fx + 1 >= G + RB2 ? 1 : 0);
  const int offY = fy <= G ? -1 : (fy + 1 >= G + RB2 ? 1 : 0);
  const int cxb = offX > 0 ? bxp : (offX < 0 ? bxm : bx);
  const int cyb = offY > 0 ? byp : (offY < 0 ? bym : by);
  const int nbrX = offX ? p.blockSlot[by * p.NBX + cxb] : -1;
  const int nbrY = offY ? p.blockSlot[cyb * p.NBX + bx] : -1;
  const int nbrXY = (offX && offY) ? p.blockSlot[cyb * p.NBX + cxb] : -1;
  const int64_t cell = pcell(p, s, fx, fy);
  const float px = pool_pos(p, bx, fx), py = pool_pos(p, by, fy);
  float wx = fmodf(px, Wf); if (wx < 0.f) wx += Wf;
  float wy = fmodf(py, Hf); if (wy < 0.f) wy += Hf;
  const float rx = wrap_delta(px - p.body.cx, Wf), ry = wrap_delta(py - p.body.cy, Hf);
  const float usx = p.body.vx - p.body.wz * ry, usy = p.body.vy + p.body.wz * rx;
  const float phi = phi2(px, py, p.body, Wf, Hf);
  const bool near = p.bb && phi < 2.0f;  // a link is at most sqrt(2)/2 root cells long here
  float f[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int ex = L9::ex(i), ey = L9::ey(i);
    if (near && phi2(pool_pos(p, bx, fx - ex), pool_pos(p, by, fy - ey), p.body, Wf, Hf) < 0.f) {
      const float corr = 2.f * L9::w(i) * ((float)ex * usx + (float)ey * usy) * kInvCS2;
      f[i] = __ldg(fin + L9::opp(i) * p.N1 + cell) + corr;
      continue;
    }
    int sx = fx - ex, sy = fy - ey, src = s;
    const int ox = (sx < G || sx >= G + RB2) ? offX : 0;
    const int oy = (sy < G || sy >= G + RB2) ? offY : 0;
    const int ns = (ox && oy) ? nbrXY : (ox ? nbrX : (oy ? nbrY : -1));
    if (ns >= 0) { src = ns; sx -= ox * RB2; sy -= oy * RB2; }
    sx = min(max(sx, 0), FB - 1);
    sy = min(max(sy, 0), FB - 1);
    f[i] = __ldg(fin + i * p.N1 + pcell(p, src, sx, sy));
  }
  float rho = 0.f, uxs = 0.f, uys = 0.f;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    rho += f[i];
    uxs += f[i] * (float)L9::ex(i);
    uys += f[i] * (float)L9::ey(i);
  }
  const float den = fmaxf(rho, 1e-6f);
  uxs /= den;
  uys /= den;
  const float chi = p.bb ? 0.f : chi_from_phi(phi, p.eps_f);
  const float Fx = rho * chi * (usx - uxs) + p.fx;
  const float Fy = rho * chi * (usy - uys) + p.fy;
  const float ux = uxs + Fx / (2.0f * den), uy = uys + Fy / (2.0f * den);
  const float usq = ux * ux + uy * uy;
  vel1[cell] = make_float2(ux, uy);
  if (p.explode && !(fx >= G && fx < G + RB2 && fy >= G && fy < G + RB2)) {
    // explode/coalesce: the ring advects without colliding (COLLIDE_RING = 0)
#pragma unroll
    for (int i = 0; i < 9; ++i) fout[i * p.N1 + cell] = f[i];
    return;
  }
  const float dx = fminf(wx, Wf - 1.0f - wx), dy = fminf(wy, Hf - 1.0f - wy);
  const float sw = sponge_weight(fminf(dx, dy), p.sponge_w);
  const bool solid = p.solid_eq && p.bb && phi < 0.f;
  const float omg = p.omega_f, sfac = 1.0f - 0.5f * omg;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const float exf = (float)L9::ex(i), eyf = (float)L9::ey(i), w = L9::w(i);
    float o;
    if (solid) {
      o = feq9(1.0f, usx, usy, i);
    } else {
      const float eu = exf * ux + eyf * uy;
      const float fe = w * rho * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * usq);
      const float t2 = (exf * ux + eyf * uy) * 9.0f;
      const float Si = sfac * w * (((exf - ux) * 3.0f + t2 * exf) * Fx + ((eyf - uy) * 3.0f + t2 * eyf) * Fy);
      const float fc = f[i] - omg * (f[i] - fe) + Si;
      o = fc * (1.0f - sw) + p.ftarget[i] * sw;
    }
    fout[i * p.N1 + cell] = o;
  }
}

__global__ void __launch_bounds__(kChunk)
    amr_substep(const float *__restrict__ fin, float *__restrict__ fout, float2 *__restrict__ vel1,
                const __grid_constant__ AmrParams p) {
  const int n = p.counts[1];
  const int FB2 = p.FB * p.FB, nch = (FB2 + kChunk - 1) / kChunk;
  for (int w = blockIdx.x; w < n * nch; w += gridDim.x) {
    const int k = w / nch, c0 = (w % nch) * kChunk, c1 = min(c0 + kChunk, FB2);
    const int s = p.activeList[k];
    const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
    for (int c = c0 + threadIdx.x; c < c1; c += kChunk) substep_cell(p, fin, fout, vel1, s, bx, by, c % p.FB, c / p.FB);
  }
}

// 4-child restriction into the root (common_average.wgsl averageCell): root
// cell c (of RB x RB) of tile s's block.
__device__ __forceinline__ void average_cell(const AmrParams &p, const float *__restrict__ f1, float *__restrict__ f0,
                                             int s, int bx, int by, int c) {
  const int lx = c % p.RB, ly = c / p.RB;
  const int fx0 = p.G + 2 * lx, fy0 = p.G + 2 * ly;
  const int64_t ch[4] = {pcell(p, s, fx0, fy0), pcell(p, s, fx0 + 1, fy0), pcell(p, s, fx0, fy0 + 1),
                         pcell(p, s, fx0 + 1, fy0 + 1)};
  float fneq_sum[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) fneq_sum[i] = 0.f;
  float rs = 0.f, rxs = 0.f, rys = 0.f;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float f[9], rho = 0.f, ux = 0.f, uy = 0.f;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      f[i] = __ldg(f1 + i * p.N1 + ch[q]);
      rho += f[i];
      ux += f[i] * (float)L9::ex(i);
      uy += f[i] * (float)L9::ey(i);
    }
    ux /= fmaxf(rho, 1e-6f);
    uy /= fmaxf(rho, 1e-6f);
    rs += rho;
    rxs += rho * ux;
    rys += rho * uy;
#pragma unroll
    for (int i = 0; i < 9; ++i) fneq_sum[i] += f[i] - feq9(rho, ux, uy, i);
  }
  const float ra = rs * 0.25f, den = fmaxf(rs, 1e-6f);
  const float uxa = rxs / den, uya = rys / den;
  const int64_t pc = (int64_t)(by * p.RB + ly) * p.W + (bx * p.RB + lx);
#pragma unroll
  for (int i = 0; i < 9; ++i) f0[i * p.N0 + pc] = feq9(ra, uxa, uya, i) + p.resc_f2c * (fneq_sum[i] * 0.25f);
}

__global__ void __launch_bounds__(64)
    amr_average(const float *__restrict__ f1, float *__restrict__ f0, const __grid_constant__ AmrParams p) {
  const int n = p.counts[1];
  for (int k = blockIdx.x; k < n; k += gridDim.x) {
    const int s = p.activeList[k];
    const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
    for (int c = threadIdx.x; c < p.RB * p.RB; c += 64) average_cell(p, f1, f0, s, bx, by, c);
  }
}

// Finest-level force (amr_force1.wgsl forceCell): this thread's share of
// the interior cells of tile s (cells threadIdx.x, + kPoolThreads, ...),
// momentum exchange or penalty weighted by dx = 1/2.
__device__ __forceinline__ void force_tile_acc(const AmrParams &p, const float *__restrict__ f1, int s, int bx, int by,
                                               ForceAcc &acc) {
  const float Wf = (float)p.W, Hf = (float)p.H;
  for (int c = threadIdx.x; c < p.RB2 * p.RB2; c += kPoolThreads) {
    const int fx = p.G + c % p.RB2, fy = p.G + c / p.RB2;
    const float px = pool_pos(p, bx, fx), py = pool_pos(p, by, fy);
    const float phi = phi2(px, py, p.body, Wf, Hf);
    const int64_t cell = pcell(p, s, fx, fy);
    const float rx = wrap_delta(px - p.body.cx, Wf), ry = wrap_delta(py - p.body.cy, Hf);
    const float usx = p.body.vx - p.body.wz * ry, usy = p.body.vy + p.body.wz * rx;
    float fxb = 0.f, fyb = 0.f, tz = 0.f;
    if (p.bb) {
      if (phi >= 0.f && phi < 2.0f) {
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          const int ex = L9::ex(i), ey = L9::ey(i);
          if (phi2(pool_pos(p, bx, fx - ex), pool_pos(p, by, fy - ey), p.body, Wf, Hf) < 0.f) {
            const float fo = __ldg(f1 + L9::opp(i) * p.N1 + cell);
            const float corr = 2.f * L9::w(i) * ((float)ex * usx + (float)ey * usy) * kInvCS2;
            fxb += -(float)ex * (2.f * fo + corr) * 0.5f;
            fyb += -(float)ey * (2.f * fo + corr) * 0.5f;
          }
        }
        tz = rx * fyb - ry * fxb;
      }
    } else {
      const float chi = chi_from_phi(phi, p.eps_f);
      if (chi >= 1e-6f) {
        float rho = 0.f, ux = 0.f, uy = 0.f;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
          const int sx0 = fx - L9::ex(i), sy0 = fy - L9::ey(i);
          const int sx = min(max(sx0, 0), p.FB - 1), sy = min(max(sy0, 0), p.FB - 1);
          int64_t src = pcell(p, s, sx, sy);
          if (p.explode) {
            // RING_FREE_FORCE: sources past the interior resolve as the step's do
            const int ox = sx0 >= p.G + p.RB2 ? 1 : (sx0 < p.G ? -1 : 0);
            const int oy = sy0 >= p.G + p.RB2 ? 1 : (sy0 < p.G ? -1 : 0);
            if (ox || oy) {
              const int ns = p.blockSlot[((by + oy + p.NBY) % p.NBY) * p.NBX + (bx + ox + p.NBX) % p.NBX];
              if (ns >= 0) src = pcell(p, ns, sx0 - ox * p.RB2, sy0 - oy * p.RB2);
            }
          }
          const float v = __ldg(f1 + i * p.N1 + src);
          rho += v;
          ux += v * (float)L9::ex(i);
          uy += v * (float)L9::ey(i);
        }
        ux /= fmaxf(rho, 1e-6f);
        uy /= fmaxf(rho, 1e-6f);
        const float Fx = rho * chi * (usx - ux), Fy = rho * chi * (usy - uy);
        fxb = -Fx * 0.5f;
        fyb = -Fy * 0.5f;
        tz = rx * fyb - ry * fxb;
      }
    }
    CellForce cf;
    cf.fx = fxb;
    cf.fy = fyb;
    cf.tz = tz;
    acc.add(cf);
  }
}

// The force of every active tile: one FP64 partial per tile and a
// deterministic last-block sum.
__global__ void __launch_bounds__(kPoolThreads)
    amr_force(const float *__restrict__ f1, const __grid_constant__ AmrParams p) {
  const int n = p.counts[1];
  if (n == 0) {
    if (blockIdx.x == 0 && threadIdx.x < 4) p.force_out[threadIdx.x] = 0.0;
    return;
  }
  for (int k = blockIdx.x; k < n; k += gridDim.x) {
    const int s = p.activeList[k];
    const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
    ForceAcc acc;
    force_tile_acc(p, f1, s, bx, by, acc);
    reduce_force<kPoolThreads>(acc, p.partials, p.counter, n, k, p.force_out);
    __syncthreads();
  }
}

// ---- the interp macro-step as one cooperative launch -----------------------
// The six launches of a macro-step (force, ring fill, root step, two
// substeps, restriction) are latency-bound: 64 tiles are 25,600 pool cells,
// and each launch mostly waits on a chain of dependent loads and on its own
// start and drain. Here one launch of resident blocks runs them as phases
// separated by grid barriers:
//   0  force partials of every tile | ring fill | root step   (independent)
//   1  force sum (block 0) | substep a -> b
//   2  substep b -> a
//   3  restriction into the root
// Every cell goes through the same device function as in the separate
// kernels (fill_ring_cell, cell2, substep_cell, average_cell,
// force_tile_acc, the same block tree and fixed-order partial sum), so the
// result is theirs to the bit. 256-thread blocks: the force tree must see
// amr_force's thread mapping.

struct MacroArgs {
  const float *f0in;
  float *f0out;
  float *mac;
  float *f1a, *f1b;
  float2 *vel1;
  unsigned *bar;  // arrivals, generation
  int *bar_err;
  unsigned nblocks;
};

// About a second of polling (2^22 waits of ~256 ns) before a barrier gives
// up, flags the error and lets its block go on: the launch then ends (its
// result void, reported by lbm_amr2d_sync as LBM_ETIMEDOUT) instead of
// holding the GPU. A cooperative launch has every block resident, so a
// healthy barrier releases within microseconds.
constexpr unsigned long long kBarrierSpins = 1ull << 22;

__device__ __forceinline__ void grid_barrier(unsigned *bar, int *err, unsigned nblocks) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == nblocks - 1) {
      atomicExch(bar, 0u);  // re-armed before the release
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned long long spins = 0;
      while (*gen == g) {
        if (++spins > kBarrierSpins) {
          atomicExch(err, 1);
          break;
        }
        __nanosleep(256);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kPoolThreads)
    amr_macro_fused(const __grid_constant__ AmrParams p, const __grid_constant__ StepParams rp,
                    const __grid_constant__ MacroArgs m) {
  __shared__ double sm[kForceSlots * (kPoolThreads / 32)];
  const int n = p.counts[1];
  const int FB = p.FB, FB2 = FB * FB, nch = (FB2 + kPoolThreads - 1) / kPoolThreads;
  const int nroot = (int)((p.N0 + kPoolThreads - 1) / kPoolThreads);
  // 0: force partials (time t, pool), ring fill (from the root at t), root step
  for (int w = blockIdx.x; w < n + n * nch + nroot; w += gridDim.x) {
    if (w < n) {
      const int s = p.activeList[w];
      const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
      ForceAcc acc;
      force_tile_acc(p, m.f1a, s, bx, by, acc);
      double v[kForceSlots];
#pragma unroll
      for (int k = 0; k < 6; ++k) v[k] = acc.v[k];
      v[6] = acc.bad;
      v[7] = 0.0;
      block_sum<kForceSlots, kPoolThreads>(v, sm);
      if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < kForceSlots; ++k) p.partials[(int64_t)w * kForceSlots + k] = v[k];
      __syncthreads();
    } else if (w < n + n * nch) {
      const int k = (w - n) / nch, c = ((w - n) % nch) * kPoolThreads + threadIdx.x;
      if (c < FB2) {
        const int s = p.activeList[k];
        const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
        const int fx = c % FB, fy = c / FB;
        const bool inX = fx >= p.G && fx < p.G + p.RB2, inY = fy >= p.G && fy < p.G + p.RB2;
        if (!(inX && inY)) fill_ring_cell(p, m.f0in, m.f1a, s, bx, by, fx, fy);
      }
    } else {
      const int c = (w - n - n * nch) * kPoolThreads + threadIdx.x;
      if (c < p.N0) {
        CellForce cf;
        cell2<float>(m.f0in, m.f0out, m.mac, rp, c % p.W, c / p.W, false, cf);
      }
    }
  }
  grid_barrier(m.bar, m.bar_err, m.nblocks);
  // 1: the force of this macro-step, and substep a -> b
  if (blockIdx.x == 0) {
    if (n == 0) {
      if (threadIdx.x < 4) p.force_out[threadIdx.x] = 0.0;
    } else if (threadIdx.x < 32) {
      sum_partials_warp<kForceSlots>(p.partials, n, p.force_out);
    }
  }
  for (int w = blockIdx.x; w < n * nch; w += gridDim.x) {
    const int k = w / nch, c = (w % nch) * kPoolThreads + threadIdx.x;
    if (c >= FB2) continue;
    const int s = p.activeList[k];
    const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
    substep_cell(p, m.f1a, m.f1b, m.vel1, s, bx, by, c % FB, c / FB);
  }
  grid_barrier(m.bar, m.bar_err, m.nblocks);
  // 2: substep b -> a
  for (int w = blockIdx.x; w < n * nch; w += gridDim.x) {
    const int k = w / nch, c = (w % nch) * kPoolThreads + threadIdx.x;
    if (c >= FB2) continue;
    const int s = p.activeList[k];
    const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
    substep_cell(p, m.f1b, m.f1a, m.vel1, s, bx, by, c % FB, c / FB);
  }
  grid_barrier(m.bar, m.bar_err, m.nblocks);
  // 3: restriction of the pool into the root at t + 1
  const int RR = p.RB * p.RB, nrr = (RR + kPoolThreads - 1) / kPoolThreads;
  for (int w = blockIdx.x; w < n * nrr; w += gridDim.x) {
    const int k = w / nrr, c = (w % nrr) * kPoolThreads + threadIdx.x;
    if (c >= RR) continue;
    const int s = p.activeList[k];
    const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
    average_cell(p, m.f1a, m.f0out, s, bx, by, c);
  }
}

// Blocks of the fused macro-step's cooperative launch on the current device
// (every one resident), or 0 where it cannot run: the explode interface, or
// a device without cooperative launches.
int fused_blocks(const AmrParams &p) {
  int dev = 0, sms = 0, coop = 0, per_sm = 0;
  if (p.explode || cudaGetDevice(&dev) != cudaSuccess) return 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  const bool ok = coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, amr_macro_fused, kPoolThreads, 0) ==
                              cudaSuccess;
  cudaGetLastError();
  return ok ? per_sm * sms : 0;
}

// ---- explode / coalesce interface ------------------------------------------------

__device__ __forceinline__ int wrap2(int v, int n) { return ((v % n) + n) % n; }

__device__ __forceinline__ bool covered2(const AmrParams &p, int x, int y) {
  return p.blockSlot[(wrap2(y, p.H) / p.RB) * p.NBX + wrap2(x, p.W) / p.RB] >= 0;
}

__device__ __forceinline__ int64_t rcell(const AmrParams &p, int x, int y) {
  return (int64_t)wrap2(y, p.H) * p.W + wrap2(x, p.W);
}

// amr_explode.wgsl: every ring cell whose L0 cell V is unrefined takes V's
// time-t populations for the directions whose L0 target is covered (plus
// the linear term orthogonal to e_i), V's population where this child's own
// one-step destination lies in the tile (in-orphan), else 0.
__global__ void __launch_bounds__(kChunk)
    amr_explode(const float *__restrict__ f0, float *__restrict__ f1, const __grid_constant__ AmrParams p) {
  const int n = p.counts[1];
  const int NFX = 2 * p.W, NFY = 2 * p.H;
  const int FB2 = p.FB * p.FB, nch = (FB2 + kChunk - 1) / kChunk;
  for (int w = blockIdx.x; w < n * nch; w += gridDim.x) {
    const int k = w / nch, c0 = (w % nch) * kChunk, c1 = min(c0 + kChunk, FB2);
    const int s = p.activeList[k];
    const int bid = p.slotToBlock[s], bx = bid % p.NBX, by = bid / p.NBX;
    const int G = p.G, RB2 = p.RB2, FB = p.FB;
    for (int c = c0 + threadIdx.x; c < c1; c += kChunk) {
      const int fx = c % FB, fy = c / FB;
      if (fx >= G && fx < G + RB2 && fy >= G && fy < G + RB2) continue;
      const int gx = wrap2(bx * RB2 + fx - G, NFX), gy = wrap2(by * RB2 + fy - G, NFY);
      const int vx = gx / 2, vy = gy / 2;
      if (covered2(p, vx, vy)) continue;
      const int64_t vc = rcell(p, vx, vy);
      bool okx = false, oky = false;
      if (p.linear) {
        okx = !covered2(p, vx - 1, vy) && !covered2(p, vx + 1, vy);
        oky = !covered2(p, vx, vy - 1) && !covered2(p, vx, vy + 1);
      }
      const float dx = ((float)(gx - 2 * vx) - 0.5f) * 0.5f, dy = ((float)(gy - 2 * vy) - 0.5f) * 0.5f;
      const int64_t cell = pcell(p, s, fx, fy);
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        const int ex = L9::ex(i), ey = L9::ey(i);
        const float fv = __ldg(f0 + i * p.N0 + vc);
        float o;
        if (covered2(p, vx + ex, vy + ey)) {
          o = fv;
          if (p.linear && (okx || oky)) {
            float gxv = okx ? 0.5f * (__ldg(f0 + i * p.N0 + rcell(p, vx + 1, vy)) - __ldg(f0 + i * p.N0 + rcell(p, vx - 1, vy)))
                            : 0.f;
            float gyv = oky ? 0.5f * (__ldg(f0 + i * p.N0 + rcell(p, vx, vy + 1)) - __ldg(f0 + i * p.N0 + rcell(p, vx, vy - 1)))
                            : 0.f;
            const float ef = (gxv * (float)ex + gyv * (float)ey) / (float)(ex * ex + ey * ey);
            gxv -= (float)ex * ef;
            gyv -= (float)ey * ef;
            o += dx * gxv + dy * gyv;
          }
        } else {
          const int dgx = wrap2(gx + ex, NFX), dgy = wrap2(gy + ey, NFY);
          const bool into = covered2(p, dgx / 2, dgy / 2) && dgx / RB2 == bx && dgy / RB2 == by;
          o = into ? fv : 0.f;
        }
        f1[i * p.N1 + cell] = o;
      }
    }
  }
}

// amr_coalesce.wgsl, one thread per L0 cell (each writes only its own cell
// of the time-t buffer): a covered cell takes, for every direction whose
// target is unrefined, the mean of the four fine cells of that target that
// the L0 step will pull; an unrefined cell at the seam gets its out-orphans
// (half-step exits of the tiles) less the in-orphans explode injected.
__global__ void __launch_bounds__(256)
    amr_coalesce(const float *__restrict__ f1, float *__restrict__ f0, const __grid_constant__ AmrParams p) {
  const int64_t c = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (c >= p.N0) return;
  const int cx = (int)(c % p.W), cy = (int)(c / p.W);
  const int NFX = 2 * p.W, NFY = 2 * p.H;
  const int G = p.G, RB2 = p.RB2;
  if (covered2(p, cx, cy)) {
    const int cbx = cx / p.RB, cby = cy / p.RB;
    const int cs = p.blockSlot[cby * p.NBX + cbx];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const int tx = cx + L9::ex(i), ty = cy + L9::ey(i);
      if (covered2(p, tx, ty)) continue;
      float sum = 0.f;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int px = tx * 2 + (k & 1), py = ty * 2 + (k >> 1);
        sum += __ldg(f1 + i * p.N1 + pcell(p, cs, px - cbx * RB2 + G, py - cby * RB2 + G));
      }
      f0[i * p.N0 + c] = sum * 0.25f;
    }
    return;
  }
  bool nearc = false;
#pragma unroll
  for (int i = 1; i < 9; ++i) nearc = nearc || covered2(p, cx + L9::ex(i), cy + L9::ey(i));
  if (!nearc) return;
#pragma unroll
  for (int i = 1; i < 9; ++i) {
    const int ex = L9::ex(i), ey = L9::ey(i);
    if (covered2(p, cx + ex, cy + ey)) continue;
    float sum = 0.f, nin = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int ox = k & 1, oy = k >> 1;
      const int pux = (cx + ex) * 2 + ox, puy = (cy + ey) * 2 + oy;
      const int qx = wrap2(pux - ex, NFX), qy = wrap2(puy - ey, NFY);
      const int qbx = qx / RB2, qby = qy / RB2;
      const int qs = p.blockSlot[qby * p.NBX + qbx];
      if (qs >= 0) sum += __ldg(f1 + i * p.N1 + pcell(p, qs, qx - qbx * RB2 + G + ex, qy - qby * RB2 + G + ey));
      const int chx = wrap2(cx * 2 + ox + ex, NFX), chy = wrap2(cy * 2 + oy + ey, NFY);
      if (covered2(p, chx / 2, chy / 2)) nin += 1.f;
    }
    const float own = f0[i * p.N0 + c];
    const float net = sum - nin * own;
    if (net != 0.f) f0[i * p.N0 + c] = own + net * 0.25f;
  }
}

}  // namespace
}  // namespace lbm

// ---- session ---------------------------------------------------------------------

using namespace lbm;

struct lbm_amr2d {
  lbm_amr2d_config cfg{};
  AmrParams p{};
  StepParams root{};
  float *f0[2] = {nullptr, nullptr};
  float4 *mac = nullptr;
  float *f1[2] = {nullptr, nullptr};
  float2 *vel1 = nullptr;
  int cur = 0;
  int64_t step = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double *host = nullptr;
  int *host_counts = nullptr;
  int grid_slots = 0;
  // the fused macro-step: resident blocks of one cooperative launch (0: off)
  // and its grid barrier's state and timeout flag
  int fused_grid = 0;
  unsigned *bar = nullptr;
  int *bar_err = nullptr;
  std::string err;
};

namespace {

thread_local std::string g_amr_error;

int afail(lbm_amr2d *a, int code, const std::string &m) {
  if (a) a->err = m; else g_amr_error = m;
  return code;
}

#define ACK(a, call)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return afail(a, e_ == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA,        \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

void release_amr(lbm_amr2d *a) {
  if (!a) return;
  if (a->stream) cudaStreamSynchronize(a->stream);
  for (auto &g : a->graph)
    if (g) cudaGraphExecDestroy(g);
  cudaFree(a->f0[0]); cudaFree(a->f0[1]); cudaFree(a->mac);
  cudaFree(a->f1[0]); cudaFree(a->f1[1]); cudaFree(a->vel1);
  AmrParams &p = a->p;
  cudaFree(p.blockSlot); cudaFree(p.slotToBlock); cudaFree(p.parentSlot); cudaFree(p.freeList);
  cudaFree(p.counts); cudaFree(p.activeList); cudaFree(p.want); cudaFree(p.newly); cudaFree(p.crit);
  cudaFree(p.partials); cudaFree(p.counter); cudaFree(p.force_out);
  cudaFree(a->bar); cudaFree(a->bar_err);
  if (a->host) cudaFreeHost(a->host);
  if (a->host_counts) cudaFreeHost(a->host_counts);
  if (a->own) cudaStreamDestroy(a->own);
}

int validate_amr(const lbm_amr2d_config *c, std::string &why) {
  if (!c) { why = "config is NULL"; return LBM_EINVAL; }
  if (c->levels != 2) { why = "levels must be 2 (root + one pool level)"; return LBM_EINVAL; }
  if (c->rb < 2 || c->rb > 32) { why = "rb must be in [2, 32]"; return LBM_EINVAL; }
  if (c->nx <= 0 || c->ny <= 0 || c->nx % (2 * c->rb) || c->ny % (2 * c->rb)) {
    why = "nx and ny must be positive multiples of 2*rb (one root block is 2*rb cells)";
    return LBM_EINVAL;
  }
  if (c->max_slots <= 0 || c->max_slots % 4) { why = "max_slots must be a positive multiple of 4 (quad allocation)"; return LBM_EINVAL; }
  if (!(c->tau > 0.5f)) { why = "tau must be > 0.5"; return LBM_EINVAL; }
  if (lbm_tau_chain_singularity(c->tau, c->levels, 0.01) >= 0) {
    why = "a level's tau is within 0.01 of 1, where the post-collision coarse<->fine transfer is 0/0 "
          "(amr2d.mjs:189 tauChainSingularity)";
    return LBM_EINVAL;
  }
  if (c->body.shape != LBM_SHAPE_ELLIPSE || !(c->body.a > 0.f) || !(c->body.b > 0.f)) {
    why = "the body must be an ellipse (a, b > 0)";
    return LBM_EINVAL;
  }
  if (c->refine_every < 1) { why = "refine_every must be >= 1"; return LBM_EINVAL; }
  return LBM_OK;
}

int macro_launches(lbm_amr2d *a, cudaStream_t st, int from) {
  AmrParams &p = a->p;
  const int g = a->grid_slots;
  if (p.explode) {
    amr_force<<<g, kPoolThreads, 0, st>>>(a->f1[0], p);
    // amr2d-gpu.mjs:1096-1124 S_AdvanceExplode: the L0 step runs LAST
    amr_explode<<<g, kChunk, 0, st>>>(a->f0[from], a->f1[0], p);
    amr_substep<<<g, kChunk, 0, st>>>(a->f1[0], a->f1[1], a->vel1, p);
    amr_substep<<<g, kChunk, 0, st>>>(a->f1[1], a->f1[0], a->vel1, p);
    amr_coalesce<<<(int)((p.N0 + 255) / 256), 256, 0, st>>>(a->f1[0], a->f0[from], p);
    StepParams rp = a->root;
    rp.write_mac = 1;
    cudaError_t e = launch_step(9, 0, a->f0[from], a->f0[1 - from], (float *)a->mac, rp, st);
    if (e) return afail(a, LBM_ECUDA, std::string("root step: ") + cudaGetErrorString(e));
    amr_average<<<g, 64, 0, st>>>(a->f1[0], a->f0[1 - from], p);
    ACK(a, cudaGetLastError());
    return LBM_OK;
  }
  if (a->fused_grid > 0) {
    StepParams rp = a->root;
    rp.write_mac = 1;
    const MacroArgs m{a->f0[from], a->f0[1 - from], (float *)a->mac, a->f1[0], a->f1[1], a->vel1, a->bar,
                      a->bar_err, (unsigned)a->fused_grid};
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(a->fused_grid);
    lc.blockDim = dim3(kPoolThreads);
    lc.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    ACK(a, cudaLaunchKernelEx(&lc, amr_macro_fused, p, rp, m));
    return LBM_OK;
  }
  amr_force<<<g, kPoolThreads, 0, st>>>(a->f1[0], p);
  amr_fill<<<g, kChunk, 0, st>>>(a->f0[from], a->f1[0], 0, p);
  StepParams rp = a->root;
  rp.write_mac = 1;
  cudaError_t e = launch_step(9, 0, a->f0[from], a->f0[1 - from], (float *)a->mac, rp, st);
  if (e) return afail(a, LBM_ECUDA, std::string("root step: ") + cudaGetErrorString(e));
  amr_substep<<<g, kChunk, 0, st>>>(a->f1[0], a->f1[1], a->vel1, p);
  amr_substep<<<g, kChunk, 0, st>>>(a->f1[1], a->f1[0], a->vel1, p);
  amr_average<<<g, 64, 0, st>>>(a->f1[0], a->f0[1 - from], p);
  ACK(a, cudaGetLastError());
  return LBM_OK;
}

int refine_round(lbm_amr2d *a) {
  AmrParams &p = a->p;
  cudaStream_t st = a->stream;
  ACK(a, cudaMemsetAsync(p.newly, 0, p.S * sizeof(unsigned), st));
  amr_criterion<<<p.NBX * p.NBY, 64, 0, st>>>(a->mac, p);
  ACK(a, cudaMemsetAsync(p.want, 0, (size_t)p.NBX * p.NBY * sizeof(unsigned), st));
  amr_decide<<<(p.PNX * p.PNY + 127) / 128, 128, 0, st>>>(p);
  amr_coarsen_refine<<<1, kManageThreads, 0, st>>>(p);
  amr_fill<<<a->grid_slots, kChunk, 0, st>>>(a->f0[a->cur], a->f1[0], 1, p);
  ACK(a, cudaGetLastError());
  return LBM_OK;
}

int build_graph(lbm_amr2d *a, int from) {
  cudaStream_t cs;
  ACK(a, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  int rc = LBM_OK;
  if (e == cudaSuccess) rc = macro_launches(a, cs, from);
  cudaError_t e2 = cudaStreamEndCapture(cs, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess && rc == LBM_OK) e = cudaGraphInstantiate(&a->graph[from], g, 0);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  if ((rc || e != cudaSuccess) && a->fused_grid > 0) {
    // a cooperative kernel node this driver will not capture: the six launches
    cudaGetLastError();
    a->fused_grid = 0;
    return build_graph(a, from);
  }
  if (rc) return rc;
  if (e != cudaSuccess) return afail(a, LBM_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_amr2d_config_default(lbm_amr2d_config *c, int nx, int ny) {
  if (!c) return LBM_EINVAL;
  std::memset(c, 0, sizeof(*c));
  c->nx = nx; c->ny = ny;
  c->levels = 2;
  c->rb = 8;
  c->tau = 0.6f;
  c->max_slots = 4 * ((nx / 16) * (ny / 16));
  c->solid_eq = 1;
  c->k_eps = 1.5f;
  c->sponge_w = 4.0f;
  c->body.shape = LBM_SHAPE_ELLIPSE;
  c->body.qw = 1.f;
  c->body.a = c->body.b = 1.f;
  c->refine_every = 16;
  c->refine_thresh = -8.0f;
  c->refine_margin = 8.0f;
  c->refine_lookahead = 16.0f;
  c->auto_refine = 1;
  c->iface = 0;
  c->explode_linear = 1;
  return LBM_OK;
}

int lbm_amr2d_create(const lbm_amr2d_config *cfg, lbm_amr2d **out) {
  if (!out) return afail(nullptr, LBM_EINVAL, "out is NULL");
  *out = nullptr;
  std::string why;
  if (validate_amr(cfg, why)) return afail(nullptr, LBM_EINVAL, why);
  lbm_amr2d *a = new lbm_amr2d();
  a->cfg = *cfg;
  AmrParams &p = a->p;
  const lbm_amr2d_config &c = *cfg;
  p.W = c.nx; p.H = c.ny; p.RB = c.rb; p.G = 2; p.RB2 = 2 * c.rb; p.FB = p.RB2 + 2 * p.G;
  p.NBX = c.nx / c.rb; p.NBY = c.ny / c.rb; p.PNX = c.nx / p.RB2; p.PNY = c.ny / p.RB2; p.S = c.max_slots;
  p.N0 = (int64_t)c.nx * c.ny; p.N1 = (int64_t)p.S * p.FB * p.FB;
  p.tau_c = c.tau;
  p.tau_f = 2.0f * c.tau - 0.5f;
  p.omega_f = 1.0f / p.tau_f;
  p.eps_f = c.k_eps * 0.5f;
  p.sponge_w = c.sponge_w; p.sux = c.sponge_u[0]; p.suy = c.sponge_u[1];
  p.fx = c.force[0]; p.fy = c.force[1];
  p.margin = c.refine_margin; p.lookahead = c.refine_lookahead;
  p.resc_c2f = 0.5f * (p.tau_f - 1.0f) / (p.tau_c - 1.0f);
  p.resc_f2c = 2.0f * (p.tau_c - 1.0f) / (p.tau_f - 1.0f);
  p.vort_on = c.refine_thresh <= 1.0f;
  p.thr = std::exp2((double)c.refine_thresh);
  p.bb = c.use_bounceback; p.solid_eq = c.solid_eq;
  p.explode = c.iface == 1 ? 1 : 0;
  p.linear = c.explode_linear ? 1 : 0;
  p.body = c.body;
  for (int i = 0; i < 9; ++i) {
    const int ex = Lattice<9>::ex(i), ey = Lattice<9>::ey(i);
    const float eu = (float)ex * p.sux + (float)ey * p.suy;
    p.ftarget[i] = Lattice<9>::w(i) * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * (p.sux * p.sux + p.suy * p.suy));
  }
  // The root level is a dense D2Q9 domain stepped by the dense kernel.
  lbm_config rc;
  lbm_config_default(&rc, 9, c.nx, c.ny, 1);
  rc.tau = c.tau; rc.force[0] = c.force[0]; rc.force[1] = c.force[1];
  rc.has_body = 1; rc.use_bounceback = c.use_bounceback; rc.solid_eq = c.solid_eq; rc.chi_eps = c.k_eps;
  rc.sponge_w = c.sponge_w; rc.sponge_u[0] = c.sponge_u[0]; rc.sponge_u[1] = c.sponge_u[1];
  rc.body = c.body;
  fill_step_params(rc, p.N0, 0, a->root);
  a->root.force_on = 0;  // the body force is measured on the finest level
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  a->grid_slots = std::min(p.S, 8 * sms);
  auto bail = [&](cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    release_amr(a);
    delete a;
    return afail(nullptr, e == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA, m);
  };
  cudaError_t e;
#define AM(ptr, bytes) if ((e = cudaMalloc(&(ptr), (bytes)))) return bail(e, "cudaMalloc " #ptr)
  if ((e = cudaStreamCreateWithFlags(&a->own, cudaStreamNonBlocking))) return bail(e, "stream");
  a->stream = a->own;
  AM(a->f0[0], 9 * p.N0 * 4); AM(a->f0[1], 9 * p.N0 * 4); AM(a->mac, p.N0 * 16);
  AM(a->f1[0], 9 * p.N1 * 4); AM(a->f1[1], 9 * p.N1 * 4); AM(a->vel1, p.N1 * 8);
  AM(p.blockSlot, p.NBX * p.NBY * 4); AM(p.slotToBlock, p.S * 4); AM(p.parentSlot, p.S * 4);
  AM(p.freeList, (p.S / 4) * 4); AM(p.counts, 2 * 4); AM(p.activeList, p.S * 4);
  AM(p.want, p.NBX * p.NBY * 4); AM(p.newly, p.S * 4); AM(p.crit, p.NBX * p.NBY * 4);
  AM(p.partials, (size_t)p.S * kForceSlots * 8); AM(p.counter, 4); AM(p.force_out, kForceSlots * 8);
  AM(a->bar, 2 * sizeof(unsigned)); AM(a->bar_err, sizeof(int));
#undef AM
  if ((e = cudaMallocHost(&a->host, 16 * sizeof(double)))) return bail(e, "cudaMallocHost");
  if ((e = cudaMallocHost(&a->host_counts, 4 * sizeof(int)))) return bail(e, "cudaMallocHost");
  std::vector<int> neg(std::max<int64_t>(p.NBX * p.NBY, p.S), -1), fl(p.S / 4);
  for (int i = 0; i < p.S / 4; ++i) fl[i] = i;  // writePoolInitialState: free list 0..n-1
  int counts[2] = {p.S / 4, 0};
  cudaMemcpy(p.blockSlot, neg.data(), p.NBX * p.NBY * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(p.slotToBlock, neg.data(), p.S * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(p.freeList, fl.data(), (p.S / 4) * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(p.counts, counts, 8, cudaMemcpyHostToDevice);
  cudaMemset(p.parentSlot, 0, p.S * 4);
  cudaMemset(p.activeList, 0xff, p.S * 4);
  cudaMemset(p.want, 0, p.NBX * p.NBY * 4);
  cudaMemset(p.newly, 0, p.S * 4);
  cudaMemset(p.crit, 0, p.NBX * p.NBY * 4);
  cudaMemset(p.counter, 0, 4);
  cudaMemset(p.force_out, 0, kForceSlots * 8);
  cudaMemset(a->f1[0], 0, 9 * p.N1 * 4);
  cudaMemset(a->f1[1], 0, 9 * p.N1 * 4);
  cudaMemset(a->mac, 0, p.N0 * 16);
  cudaMemset(a->bar, 0, 2 * sizeof(unsigned));
  cudaMemset(a->bar_err, 0, sizeof(int));
  a->fused_grid = fused_blocks(p);
  if ((e = cudaDeviceSynchronize())) return bail(e, "initialise");
  *out = a;
  return LBM_OK;
}

void lbm_amr2d_destroy(lbm_amr2d *a) {
  release_amr(a);
  delete a;
}

const char *lbm_amr2d_last_error(const lbm_amr2d *a) { return a ? a->err.c_str() : g_amr_error.c_str(); }

int lbm_amr2d_set_stream(lbm_amr2d *a, void *stream) {
  if (!a) return LBM_EINVAL;
  ACK(a, cudaStreamSynchronize(a->stream));
  a->stream = stream ? (cudaStream_t)stream : a->own;
  return LBM_OK;
}

int lbm_amr2d_write_root(lbm_amr2d *a, const float *f, const float *vel) {
  if (!a || !f || !vel) return a ? afail(a, LBM_EINVAL, "NULL argument") : LBM_EINVAL;
  const AmrParams &p = a->p;
  ACK(a, cudaMemcpyAsync(a->f0[a->cur], f, 9 * p.N0 * 4, cudaMemcpyHostToDevice, a->stream));
  std::vector<float4> m(p.N0);
  for (int64_t k = 0; k < p.N0; ++k) m[k] = make_float4(1.f, vel[2 * k], vel[2 * k + 1], 0.f);
  ACK(a, cudaMemcpyAsync(a->mac, m.data(), p.N0 * 16, cudaMemcpyHostToDevice, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  return LBM_OK;
}

int lbm_amr2d_read_root(lbm_amr2d *a, float *f, float *vel) {
  if (!a) return LBM_EINVAL;
  const AmrParams &p = a->p;
  if (f) ACK(a, cudaMemcpyAsync(f, a->f0[a->cur], 9 * p.N0 * 4, cudaMemcpyDeviceToHost, a->stream));
  std::vector<float4> m;
  if (vel) {
    m.resize(p.N0);
    ACK(a, cudaMemcpyAsync(m.data(), a->mac, p.N0 * 16, cudaMemcpyDeviceToHost, a->stream));
  }
  ACK(a, cudaStreamSynchronize(a->stream));
  if (vel)
    for (int64_t k = 0; k < p.N0; ++k) { vel[2 * k] = m[k].y; vel[2 * k + 1] = m[k].z; }
  return LBM_OK;
}

int lbm_amr2d_read_pool(lbm_amr2d *a, float *f, float *vel) {
  if (!a) return LBM_EINVAL;
  const AmrParams &p = a->p;
  if (f) ACK(a, cudaMemcpyAsync(f, a->f1[0], 9 * p.N1 * 4, cudaMemcpyDeviceToHost, a->stream));
  if (vel) ACK(a, cudaMemcpyAsync(vel, a->vel1, p.N1 * 8, cudaMemcpyDeviceToHost, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  return LBM_OK;
}

int lbm_amr2d_step(lbm_amr2d *a, int n) {
  if (!a) return LBM_EINVAL;
  if (n < 0) return afail(a, LBM_EINVAL, "step count must be >= 0");
  for (int k = 0; k < n; ++k) {
    if (a->cfg.auto_refine && a->step % a->cfg.refine_every == 0) {
      int rc = refine_round(a);
      if (rc) return rc;
    }
    ++a->step;
    if (!a->graph[a->cur]) {
      int rc = build_graph(a, a->cur);
      if (rc) return rc;
    }
    ACK(a, cudaGraphLaunch(a->graph[a->cur], a->stream));
    a->cur = 1 - a->cur;
  }
  return LBM_OK;
}

int lbm_amr2d_refine_round(lbm_amr2d *a) {
  if (!a) return LBM_EINVAL;
  return refine_round(a);
}

int lbm_amr2d_set_auto_refine(lbm_amr2d *a, int on) {
  if (!a) return LBM_EINVAL;
  a->cfg.auto_refine = on ? 1 : 0;
  return LBM_OK;
}

int lbm_amr2d_set_fused(lbm_amr2d *a, int on) {
  if (!a) return LBM_EINVAL;
  ACK(a, cudaStreamSynchronize(a->stream));
  for (auto &g : a->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  a->fused_grid = on ? fused_blocks(a->p) : 0;
  return LBM_OK;
}

int lbm_amr2d_fused(const lbm_amr2d *a) { return a ? (a->fused_grid > 0 ? 1 : 0) : 0; }

int lbm_amr2d_forces(lbm_amr2d *a, double out[4]) {
  if (!a || !out) return a ? afail(a, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  ACK(a, cudaMemcpyAsync(a->host, a->p.force_out, kForceSlots * 8, cudaMemcpyDeviceToHost, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  out[0] = a->host[0]; out[1] = a->host[1]; out[2] = a->host[5]; out[3] = a->host[6];
  return LBM_OK;
}

int lbm_amr2d_read_topology(lbm_amr2d *a, int32_t *block_slot, int32_t *slot_to_block, int32_t *free_list,
                            int32_t counts[2], int32_t *active_list, float *criterion, uint32_t *want) {
  if (!a) return LBM_EINVAL;
  const AmrParams &p = a->p;
  cudaStream_t st = a->stream;
  const size_t nb = (size_t)p.NBX * p.NBY;
  if (block_slot) ACK(a, cudaMemcpyAsync(block_slot, p.blockSlot, nb * 4, cudaMemcpyDeviceToHost, st));
  if (slot_to_block) ACK(a, cudaMemcpyAsync(slot_to_block, p.slotToBlock, p.S * 4, cudaMemcpyDeviceToHost, st));
  if (free_list) ACK(a, cudaMemcpyAsync(free_list, p.freeList, (p.S / 4) * 4, cudaMemcpyDeviceToHost, st));
  if (counts) ACK(a, cudaMemcpyAsync(counts, p.counts, 8, cudaMemcpyDeviceToHost, st));
  if (active_list) ACK(a, cudaMemcpyAsync(active_list, p.activeList, p.S * 4, cudaMemcpyDeviceToHost, st));
  if (criterion) ACK(a, cudaMemcpyAsync(criterion, p.crit, nb * 4, cudaMemcpyDeviceToHost, st));
  if (want) ACK(a, cudaMemcpyAsync(want, p.want, nb * 4, cudaMemcpyDeviceToHost, st));
  ACK(a, cudaStreamSynchronize(st));
  return LBM_OK;
}

int64_t lbm_amr2d_cell_updates(const lbm_amr2d *a) {
  if (!a) return 0;
  lbm_amr2d *m = const_cast<lbm_amr2d *>(a);
  if (cudaMemcpyAsync(m->host_counts, a->p.counts, 8, cudaMemcpyDeviceToHost, a->stream) != cudaSuccess) return -1;
  if (cudaStreamSynchronize(a->stream) != cudaSuccess) return -1;
  const int64_t active = m->host_counts[1];
  return a->p.N0 + active * (int64_t)a->p.RB2 * a->p.RB2 * 2;
}

int lbm_amr2d_sync(lbm_amr2d *a) {
  if (!a) return LBM_EINVAL;
  ACK(a, cudaStreamSynchronize(a->stream));
  if (a->fused_grid > 0) {
    int flag = 0;
    ACK(a, cudaMemcpy(&flag, a->bar_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
      cudaMemset(a->bar_err, 0, sizeof(int));
      return afail(a, LBM_ETIMEDOUT, "a grid barrier of the fused macro-step timed out; its results are void");
    }
  }
  return LBM_OK;
}

int lbm_amr2d_write_pool(lbm_amr2d *a, const float *f, const float *vel) {
  if (!a || !f || !vel) return a ? afail(a, LBM_EINVAL, "NULL argument") : LBM_EINVAL;
  const AmrParams &p = a->p;
  ACK(a, cudaMemcpyAsync(a->f1[0], f, 9 * p.N1 * 4, cudaMemcpyHostToDevice, a->stream));
  ACK(a, cudaMemcpyAsync(a->vel1, vel, p.N1 * 8, cudaMemcpyHostToDevice, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  return LBM_OK;
}

int lbm_amr2d_read_parent_slots(lbm_amr2d *a, int32_t *parent_slot) {
  if (!a || !parent_slot) return a ? afail(a, LBM_EINVAL, "NULL argument") : LBM_EINVAL;
  ACK(a, cudaMemcpyAsync(parent_slot, a->p.parentSlot, a->p.S * 4, cudaMemcpyDeviceToHost, a->stream));
  ACK(a, cudaStreamSynchronize(a->stream));
  return LBM_OK;
}

int lbm_amr2d_write_topology(lbm_amr2d *a, const int32_t *block_slot, const int32_t *slot_to_block,
                             const int32_t *parent_slot, const int32_t *free_list, int32_t free_count) {
  if (!a || !block_slot || !slot_to_block || !parent_slot || !free_list)
    return a ? afail(a, LBM_EINVAL, "NULL argument") : LBM_EINVAL;
  const AmrParams &p = a->p;
  const int nb = p.NBX * p.NBY, nq = p.S / 4;
  if (free_count < 0 || free_count > nq) return afail(a, LBM_EINVAL, "free_count outside [0, max_slots/4]");
  for (int b = 0; b < nb; ++b) {
    const int s = block_slot[b];
    if (s < -1 || s >= p.S || (s >= 0 && slot_to_block[s] != b))
      return afail(a, LBM_EINVAL, "block_slot and slot_to_block are not inverse maps");
  }
  std::vector<int> quad_used(nq, 0), quad_free(nq, 0), active;
  for (int s = 0; s < p.S; ++s) {
    const int b = slot_to_block[s];
    if (b < -1 || b >= nb || (b >= 0 && block_slot[b] != s))
      return afail(a, LBM_EINVAL, "block_slot and slot_to_block are not inverse maps");
    if (b >= 0) {
      quad_used[s / 4] += 1;
      active.push_back(s);
    }
  }
  for (int q = 0; q < nq; ++q)
    if (quad_used[q] != 0 && quad_used[q] != 4) return afail(a, LBM_EINVAL, "a quad is partly in use");
  for (int k = 0; k < free_count; ++k) {
    const int q = free_list[k];
    if (q < 0 || q >= nq || quad_used[q] || quad_free[q]++)
      return afail(a, LBM_EINVAL, "the free list names a quad in use, twice, or out of range");
  }
  const int counts[2] = {free_count, (int)active.size()};
  active.resize(p.S, -1);
  cudaStream_t st = a->stream;
  ACK(a, cudaMemcpyAsync(p.blockSlot, block_slot, nb * 4, cudaMemcpyHostToDevice, st));
  ACK(a, cudaMemcpyAsync(p.slotToBlock, slot_to_block, p.S * 4, cudaMemcpyHostToDevice, st));
  ACK(a, cudaMemcpyAsync(p.parentSlot, parent_slot, p.S * 4, cudaMemcpyHostToDevice, st));
  ACK(a, cudaMemcpyAsync(p.freeList, free_list, nq * 4, cudaMemcpyHostToDevice, st));
  ACK(a, cudaMemcpyAsync(p.counts, counts, 8, cudaMemcpyHostToDevice, st));
  ACK(a, cudaMemcpyAsync(p.activeList, active.data(), p.S * 4, cudaMemcpyHostToDevice, st));
  ACK(a, cudaStreamSynchronize(st));
  return LBM_OK;
}

int64_t lbm_amr2d_get_step(const lbm_amr2d *a) { return a ? a->step : -1; }

int lbm_amr2d_set_step(lbm_amr2d *a, int64_t step) {
  if (!a || step < 0) return a ? afail(a, LBM_EINVAL, "step must be >= 0") : LBM_EINVAL;
  a->step = step;
  return LBM_OK;
}

int lbm_amr2d_set_body(lbm_amr2d *a, const lbm_body *body) {
  if (!a || !body) return a ? afail(a, LBM_EINVAL, "body is NULL") : LBM_EINVAL;
  if (body->shape != LBM_SHAPE_ELLIPSE || !(body->a > 0.f) || !(body->b > 0.f))
    return afail(a, LBM_EINVAL, "the body must be an ellipse (a, b > 0)");
  ACK(a, cudaStreamSynchronize(a->stream));
  a->cfg.body = *body;
  a->p.body = *body;
  a->root.body = *body;
  for (auto &g : a->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return LBM_OK;
}

}  // extern "C"
