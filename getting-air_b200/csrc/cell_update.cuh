// Per-cell LBM update shared by the dense, batched and served kernels, plus
// the storage codecs and the deterministic FP64 block reduction.
//
// A "domain" is a box of cells stored in an arena of Q planes with plane
// stride p.n; its cells start at arena index p.base and run
// (z*NY + y)*NX + x. The dense solver is one domain at base 0; the batched
// and served forms place many domains in one arena. Whatever the launch
// shape, every cell goes through cell3()/cell2() below, so the arithmetic of
// all forms is the same instruction stream.
//
// Reference arithmetic:
//   cell3   common_d3_step.wgsl:224-400 (step) + common_d3_force.wgsl:171-283
//   cell2   lbm_step.wgsl:137-270 (step) + lbm_force.wgsl main
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "dense.cuh"
#include "geometry.cuh"
#include "lattice.cuh"

namespace lbm {

// 1 / c_s^2. The moving-wall term 2 w_i rho_w (e_i . u_w) / c_s^2 multiplies
// by it: a division there is an IEEE-rounded divide with a slow-path branch
// per link, which in the 3D AMR substep (most tile cells near the body) cost
// a third of the kernel's instructions.
constexpr float kInvCS2 = 3.0f;

// ---- storage codecs --------------------------------------------------------
// FP32 planes hold f itself; the 16-bit planes hold (f - off_i) * scale (see
// Pack), rounded to nearest even. Arithmetic is f32 throughout.
#ifndef LBM_STREAMING_STORES
#define LBM_STREAMING_STORES 0
#endif
template <typename S> struct Codec;
template <> struct Codec<float> {
  static __device__ __forceinline__ float ld(const float *p, int, const Pack &) { return __ldg(p); }
  static __device__ __forceinline__ void st(float *p, float v, int, const Pack &) {
    if (LBM_STREAMING_STORES) __stcs(p, v); else *p = v;
  }
};
template <> struct Codec<__half> {
  static __device__ __forceinline__ float ld(const __half *p, int i, const Pack &k) {
    return fmaf(__half2float(__ldg(p)), k.inv, k.off[i]);
  }
  static __device__ __forceinline__ void st(__half *p, float v, int i, const Pack &k) {
    *p = __float2half_rn(fmaf(v, k.scale, k.noff[i]));
  }
};
template <> struct Codec<__nv_bfloat16> {
  static __device__ __forceinline__ float ld(const __nv_bfloat16 *p, int i, const Pack &k) {
    return fmaf(__bfloat162float(__ldg(p)), k.inv, k.off[i]);
  }
  static __device__ __forceinline__ void st(__nv_bfloat16 *p, float v, int i, const Pack &k) {
    *p = __float2bfloat16_rn(fmaf(v, k.scale, k.noff[i]));
  }
};

// ---- deterministic block reduction + last-block finish -------------------

template <int NV, int THREADS>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sm) {
  constexpr int NW = THREADS / 32;
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sm[k * NW + warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = lane < NW ? sm[k * NW + lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      v[k] = t;
    }
  }
}

// The fixed-order sum of nparts partials by one warp (lane = threadIdx.x):
// lane l adds partials l, l + 32, ... in order, then a shuffle tree; lane 0
// writes out. Every caller that sums the same partials this way gets the
// same bits.
template <int NV>
__device__ __forceinline__ void sum_partials_warp(const double *partials, int nparts, double *out) {
  const int lane = threadIdx.x & 31;
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (int j = lane; j < nparts; j += 32)
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[(int64_t)j * NV + k]);
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = acc[k];
}

// Writes this block's partial (thread 0 holds it), and if this block is the
// last of `nparts` to do so, sums all partials in a fixed order into `out`
// and re-arms the ticket counter for the next step. Only warp 0 takes part:
// the other warps leave as soon as their share is in `sm`, so they do not
// hold the SM while thread 0 waits on its fence and ticket. Returns true in
// warp 0 of the last block.
template <int NV, int THREADS>
__device__ bool finish_sum(const double (&v)[NV], double *partials, unsigned int *counter,
                           int nparts, int part, double *out, double *) {
  if (threadIdx.x >= 32) return false;
  const int lane = threadIdx.x;
  unsigned int last = 0u;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(int64_t)part * NV + k] = v[k];
    __threadfence();
    const unsigned int ticket = atomicAdd(counter, 1u);
    last = ticket == (unsigned int)(nparts - 1) ? 1u : 0u;
  }
  if (!__shfl_sync(0xffffffffu, last, 0)) return false;
  __threadfence();
  sum_partials_warp<NV>(partials, nparts, out);
  if (lane == 0) *counter = 0u;
  return true;
}

__device__ __forceinline__ float sponge_weight(float d, float sw) {
  if (sw <= 0.0f) return 0.0f;
  float w = fminf(fmaxf(1.0f - d / sw, 0.0f), 1.0f);
  return w * w * (3.0f - 2.0f * w);
}

__device__ __forceinline__ double finite_or_zero(float v, double &bad) {
  if (isfinite(v)) return (double)v;
  bad += 1.0;
  return 0.0;
}

// Force/torque contribution of one cell to the body (f32, as the reference
// forms it per cell).
struct CellForce {
  float fx = 0.f, fy = 0.f, fz = 0.f, tx = 0.f, ty = 0.f, tz = 0.f;
};

// A thread's FP64 running sum of cell contributions; a non-finite cell
// component is counted and contributes 0 (the reference's safeFixed).
struct ForceAcc {
  double v[6] = {0, 0, 0, 0, 0, 0};
  double bad = 0.0;
  __device__ __forceinline__ void add(const CellForce &c) {
    v[0] += finite_or_zero(c.fx, bad);
    v[1] += finite_or_zero(c.fy, bad);
    v[2] += finite_or_zero(c.fz, bad);
    v[3] += finite_or_zero(c.tx, bad);
    v[4] += finite_or_zero(c.ty, bad);
    v[5] += finite_or_zero(c.tz, bad);
  }
};

// The block's FP64 partial of the force, written by thread 0 to
// partials[part]; the caller's stream sums the partials after the launch.
// Most blocks of a force region hold no cell with a contribution (the
// region is the body's box; only its shell touches the body): when every
// thread's sums are +0 the block writes its zero partial directly instead
// of running the FP64 tree, whose result would be the same +0s.
template <int THREADS>
__device__ __forceinline__ void publish_force(const ForceAcc &a, double *partials, int part) {
  const bool mine = a.v[0] != 0.0 || a.v[1] != 0.0 || a.v[2] != 0.0 || a.v[3] != 0.0 || a.v[4] != 0.0 ||
                    a.v[5] != 0.0 || a.bad != 0.0;
  if (!__syncthreads_or(mine)) {
    if (threadIdx.x < kForceSlots) partials[(int64_t)part * kForceSlots + threadIdx.x] = 0.0;
    return;
  }
  __shared__ double sm[kForceSlots * (THREADS / 32)];
  double v[kForceSlots];
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = a.v[k];
  v[6] = a.bad;
  v[7] = 0.0;
  block_sum<kForceSlots, THREADS>(v, sm);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < kForceSlots; ++k) partials[(int64_t)part * kForceSlots + k] = v[k];
}

// The sum of a launch's force partials, spread over the first blocks of a
// later launch so that no block waits on more than one round of loads:
// block b adds the partials of group b (kSumGroup consecutive ones, one per
// thread, then the block tree) into groups[b]; the last group to finish
// (a ticket behind one fence per group, not per partial) sums the groups in
// order into out. The order depends only on nparts, so every launch that
// sums the same partials with THREADS = kSumGroup gets the same bits.
template <int THREADS>
__device__ __forceinline__ bool sum_partials_grouped(const double *partials, int nparts, double *groups,
                                                     unsigned int *counter, double *out, int b) {
  static_assert(THREADS == kSumGroup, "one partial per thread");
  __shared__ double sm[kForceSlots * (THREADS / 32)];
  double acc[kForceSlots];
  const int j = b * kSumGroup + (int)threadIdx.x;
#pragma unroll
  for (int k = 0; k < kForceSlots; ++k) acc[k] = j < nparts ? partials[(int64_t)j * kForceSlots + k] : 0.0;
  block_sum<kForceSlots, THREADS>(acc, sm);
  return finish_sum<kForceSlots, THREADS>(acc, groups, counter, sum_groups(nparts), b, out, sm);
}

// Returns true in the block that summed the partials (the last to finish).
template <int THREADS>
__device__ __forceinline__ bool reduce_force(const ForceAcc &a, double *partials, unsigned int *counter,
                                             int nparts, int part, double *out) {
  __shared__ double sm[kForceSlots * (THREADS / 32)];
  double v[kForceSlots];
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = a.v[k];
  v[6] = a.bad;
  v[7] = 0.0;
  block_sum<kForceSlots, THREADS>(v, sm);
  return finish_sum<kForceSlots, THREADS>(v, partials, counter, nparts, part, out, sm);
}

// The BGK collision with Guo forcing and the sponge blend, written over
// opposite pairs (e, -e). With a = (1-s) omega rho, b = (1-s)(1 - omega/2)
// (s the sponge weight) and per direction eu = e.u, eF = e.F:
//   (1-s)[omega feq + S](+-e) = w (A +- B),
//     A = c0 + eu (4.5 a eu + 9 b eF),   c0 = a (1 - 1.5 u.u) - 3 b u.F
//     B = 3 a eu + 3 b eF
//   f_out(+-e) = (1-s)(1-omega) f(+-e) + s f_far(+-e) + w (A +- B).
// The products of w with a, b and c0 are formed once per weight class, so
// a pair costs about a dozen FP32 instructions. Outside the sponge (s = 0)
// this is the plain BGK + Guo update. The reference's per-direction form
// (common_d3_step.wgsl:331-357) and mix() blend (common_sponge.wgsl:7-11),
// reassociated.
// Where a cell's post-collision populations go: MemSink stores them (the
// step); NullSink drops them (a force-only pass, whose collision the
// compiler then removes as dead code).
template <typename S> struct MemSink {
  S *fo;
  int64_t n;
  int cell;
  const Pack &pk;
  __device__ __forceinline__ void put(int i, float v) { Codec<S>::st(fo + (int64_t)i * n + cell, v, i, pk); }
};
struct NullSink {
  __device__ __forceinline__ void put(int, float) {}
};

// TRT (dw = omega_- - omega != 0): the odd part of each pair relaxes at
// omega_- instead, in the reference's delta form (plans/TRT.md sec 8.0(1)):
//   f_i += -dw (f_i^- - feq_i^-) - dw/2 S_i^-,
//   f_i^- = (f_i - f_j)/2, feq_i^- = 3 w rho e.u, S_i^- = 3 w e.F,
// the odd forcing prefactor becoming (1 - omega_-/2); the sponge blend
// scales it by (1 - s) like the rest of the collided value, and f_j takes
// the negative. TRT = false is the BGK loop alone (dw ignored); the kernels
// pick the instantiation from dw != 0 per launch, so the BGK code keeps its
// register allocation.
template <class L, int Q, class Sink, bool TRT = false>
__device__ __forceinline__ void collide_store(const float (&f)[Q], float rho, float ux, float uy, float uz, float Fx,
                                              float Fy, float Fz, float omg, float spw, const float *ftarget,
                                              Sink &sink, float dw = 0.f) {
  const float usq = ux * ux + uy * uy + uz * uz;
  const float uF = ux * Fx + uy * Fy + uz * Fz;
  const float ks = 1.0f - spw;
  const float a = (omg * ks) * rho;
  const float b = (1.0f - 0.5f * omg) * ks;
  const float keep = (1.0f - omg) * ks;
  const float c0 = fmaf(a, fmaf(-1.5f, usq, 1.0f), -3.0f * b * uF);
  sink.put(0, fmaf(keep, f[0], fmaf(spw, ftarget[0], L::w(0) * c0)));
  if (!TRT) {
#pragma unroll
    for (int i = 1; i < Q; ++i) {
      const int j = L::opp(i);
      if (j < i) continue;
      const float ex = (float)L::ex(i), ey = (float)L::ey(i), ez = (float)L::ez(i);
      const float w = L::w(i);
      const float eu = ex * ux + ey * uy + ez * uz;
      const float eF = ex * Fx + ey * Fy + ez * Fz;
      const float t = fmaf((9.0f * w) * b, eF, ((4.5f * w) * a) * eu);
      const float A = fmaf(eu, t, w * c0);
      const float B = fmaf((3.0f * w) * a, eu, ((3.0f * w) * b) * eF);
      sink.put(i, fmaf(keep, f[i], fmaf(spw, ftarget[i], A + B)));
      sink.put(j, fmaf(keep, f[j], fmaf(spw, ftarget[j], A - B)));
    }
  } else {
    const float kd = -ks * dw;
    const float rho3 = 3.0f * rho;
#pragma unroll
    for (int i = 1; i < Q; ++i) {
      const int j = L::opp(i);
      if (j < i) continue;
      const float ex = (float)L::ex(i), ey = (float)L::ey(i), ez = (float)L::ez(i);
      const float w = L::w(i);
      const float eu = ex * ux + ey * uy + ez * uz;
      const float eF = ex * Fx + ey * Fy + ez * Fz;
      const float t = fmaf((9.0f * w) * b, eF, ((4.5f * w) * a) * eu);
      const float A = fmaf(eu, t, w * c0);
      const float B = fmaf((3.0f * w) * a, eu, ((3.0f * w) * b) * eF);
      const float D = kd * fmaf(0.5f, f[i] - f[j], w * fmaf(1.5f, eF, -rho3 * eu));
      sink.put(i, fmaf(keep, f[i], fmaf(spw, ftarget[i], A + B)) + D);
      sink.put(j, fmaf(keep, f[j], fmaf(spw, ftarget[j], A - B)) - D);
    }
  }
}

// rho and rho u* from the gathered populations, summed over opposite pairs.
template <class L, int Q>
__device__ __forceinline__ void moments(const float (&f)[Q], float &rho, float &mx, float &my, float &mz) {
  rho = f[0];
  mx = my = mz = 0.f;
#pragma unroll
  for (int i = 1; i < Q; ++i) {
    const int j = L::opp(i);
    if (j < i) continue;
    const float s = f[i] + f[j], d = f[i] - f[j];
    rho += s;
    if (L::ex(i) == 1) mx += d; else if (L::ex(i) == -1) mx -= d;
    if (L::ey(i) == 1) my += d; else if (L::ey(i) == -1) my -= d;
    if (L::ez(i) == 1) mz += d; else if (L::ez(i) == -1) mz -= d;
  }
}

__device__ __forceinline__ float sponge_weight_inv(float d, float inv_sw) {
  float w = fminf(fmaxf(1.0f - d * inv_sw, 0.0f), 1.0f);
  return w * w * (3.0f - 2.0f * w);
}

// ---- row-major walks without divisions --------------------------------------
// A thread of a multi-domain launch visits cells c0, c0 + step, c0 + 2 step,
// ... of one domain. Its first cell takes the divisions; every later one
// adds the step's own decomposition (dx, dy, dz) with one carry per axis
// (x + dx < 2 nx and y + dy + 1 < 2 ny, so a single subtraction suffices).
struct CellWalk {
  int x, y, z;
  int dx, dy, dz;
  int nx, ny;
  __device__ __forceinline__ CellWalk(int c0, int step, int nx_, int ny_) : nx(nx_), ny(ny_) {
    const int r = c0 / nx;
    x = c0 - r * nx;
    y = r % ny;
    z = r / ny;
    const int rs = step / nx;
    dx = step - rs * nx;
    dy = rs % ny;
    dz = rs / ny;
  }
  __device__ __forceinline__ void advance() {
    x += dx;
    y += dy;
    z += dz;
    if (x >= nx) { x -= nx; ++y; }
    if (y >= ny) { y -= ny; ++z; }
  }
};

// ---- 3D cell update ---------------------------------------------------------
// Pull-stream (periodic sources, then bounce-back patches: body first with
// Ladd's correction at local rho_w, then walls), moments, Guo forcing with
// the chi penalty, BGK collide, sponge blend, SOLID_EQ. When `force` is set
// (the caller's block can see the body) the cell's force/torque contribution
// is returned in cf.

// Everything after the pull gather, for one cell: bounce-back patches,
// moments, forcing, collision into `sink`, mac, force. `fi` is the domain's
// base in the input arena (own-cell loads of the bounce-back patches).
template <int Q, typename S, class Sink, bool TRT = false>
__device__ __forceinline__ void cell3_core(const S *__restrict__ fi, float (&f)[Q], float *__restrict__ mac,
                                           const StepParams &p, int x, int y, int z, bool force, CellForce &cf,
                                           Sink &sink) {
  using L = Lattice<Q>;
  // z indexes the stored planes; the physics (body, walls, sponge, reach
  // box) sees the domain's own z, which for a slab is offset by p.zoff in a
  // domain p.nzg planes deep (both the identity for a whole domain)
  const int nx = p.nx, ny = p.ny, nz = p.nzg;
  const int64_t n = p.n;
  const int cell = (z * ny + y) * nx + x;
  z += p.zoff;
  const V3 pos = {(float)x, (float)y, (float)z};
  float phi = 1e30f;
  V3 us = {0.f, 0.f, 0.f};
  bool see = p.has_body;
  if (see && p.nbox_on) {
    int dx = x - p.nbox[0], dy = y - p.nbox[2], dz = z - p.nbox[4];
    dx += dx < 0 ? nx : 0;
    dy += dy < 0 ? ny : 0;
    dz += dz < 0 ? nz : 0;
    see = dx <= p.nbox[1] - p.nbox[0] && dy <= p.nbox[3] - p.nbox[2] && dz <= p.nbox[5] - p.nbox[4];
  }
  if (see) {
    phi = phi3(pos, p.body, p.win);
    us = body_velocity3(pos, p.body, p.win);
  }
  const bool bbody = p.has_body && p.bb;
  const bool at_wall = (p.wall_x && (x == 0 || x == nx - 1)) || (p.wall_y && (y == 0 || y == ny - 1)) ||
                       (p.wall_z && (z == 0 || z == nz - 1));
  // A link reaches a solid source only from within |e| <= sqrt(3) of the
  // surface, and a signed distance is 1-Lipschitz.
  const bool near = bbody && phi < 2.5f;
  float fbx = 0.f, fby = 0.f, fbz = 0.f;

  // 1b. Bounce-back links. Every link is classified first (SDF and wall
  // tests, no memory access), then the cell's own populations that the
  // patches read are loaded together: a near cell waits for one memory
  // latency instead of one per solid link. (The rest direction never
  // patches: its source is the cell itself.)
  if (near || at_wall) {
    unsigned solid = 0u, wall = 0u;
#pragma unroll
    for (int i = 1; i < Q; ++i) {
      const int ex = L::ex(i), ey = L::ey(i), ez = L::ez(i);
      if (near && phi3({pos.x - (float)ex, pos.y - (float)ey, pos.z - (float)ez}, p.body, p.win) < 0.f) {
        solid |= 1u << i;
      } else if (at_wall) {
        const int sx = x - ex, sy = y - ey, sz = z - ez;
        const bool out = (p.wall_x && (sx < 0 || sx >= nx)) || (p.wall_y && (sy < 0 || sy >= ny)) ||
                         (p.wall_z && (sz < 0 || sz >= nz));
        if (out) wall |= 1u << i;
      }
    }
    if (solid | wall) {
      const bool all = bbody && p.rho_w_local && phi < 2.f;  // rho_w sums every population
      float own[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i)
        own[i] = (all || (((solid | wall) >> L::opp(i)) & 1u)) ? Codec<S>::ld(fi + (int64_t)i * n + cell, i, p.pk)
                                                                 : 0.f;
      float rhoW = 1.f;
      if (all) {
        float s = 0.f;
#pragma unroll
        for (int i = 0; i < Q; ++i) s += own[i];
        rhoW = s;
      }
#pragma unroll
      for (int i = 1; i < Q; ++i) {
        const int ex = L::ex(i), ey = L::ey(i), ez = L::ez(i);
        const float fopp = own[L::opp(i)];
        if ((solid >> i) & 1u) {
          const float corr =
              2.f * L::w(i) * rhoW * ((float)ex * us.x + (float)ey * us.y + (float)ez * us.z) * kInvCS2;
          f[i] = fopp + corr;
          if (phi >= 0.f) {
            const float m = 2.f * fopp + corr;
            fbx += -(float)ex * m;
            fby += -(float)ey * m;
            fbz += -(float)ez * m;
          }
        } else if ((wall >> i) & 1u) {
          f[i] = fopp;
        }
      }
    }
  }

  // 2. Moments.
  float rho, mx, my, mz;
  moments<L, Q>(f, rho, mx, my, mz);
  const float rhoDen = fmaxf(rho, 1e-6f);
  const float inv = 1.0f / rhoDen;
  const float uxs = mx * inv, uys = my * inv, uzs = mz * inv;

  // 3. Solid coupling and Guo forcing: u = u* + F / (2 rho).
  const float chi = (p.has_body && !p.bb) ? chi_from_phi(phi, p.chi_eps) : 0.f;
  const float rc = rho * chi;
  const float Fx = rc * (us.x - uxs) + p.fx;
  const float Fy = rc * (us.y - uys) + p.fy;
  const float Fz = rc * (us.z - uzs) + p.fz;
  const float hinv = 0.5f * inv;
  const float ux = fmaf(Fx, hinv, uxs);
  const float uy = fmaf(Fy, hinv, uys);
  const float uz = fmaf(Fz, hinv, uzs);

  float spw = 0.f;
  if (p.sponge_w > 0.f) {
    // distances in window coordinates: under a moving window the band
    // travels with the body (the identity without one)
    V3 wp = pos;
    if (p.win.on) {
      wp.x = win_coord1(pos.x, win_offset1(p.body.cx, p.win.anchor[0], p.win.n[0]), p.win.n[0]);
      wp.y = win_coord1(pos.y, win_offset1(p.body.cy, p.win.anchor[1], p.win.n[1]), p.win.n[1]);
      wp.z = win_coord1(pos.z, win_offset1(p.body.cz, p.win.anchor[2], p.win.n[2]), p.win.n[2]);
    }
    const float dx = p.sax ? fminf(wp.x, (float)(nx - 1) - wp.x) : 1e30f;
    const float dy = p.say ? fminf(wp.y, (float)(ny - 1) - wp.y) : 1e30f;
    const float dz = p.saz ? fminf(wp.z, (float)(nz - 1) - wp.z) : 1e30f;
    spw = sponge_weight_inv(fminf(dx, fminf(dy, dz)), p.sponge_inv);
  }

  // 4. Collide + sponge blend, 5. solid interior held at feq(1, u_body).
  const bool in_solid = p.solid_eq && bbody && phi < 0.f;
  if (!in_solid) {
    collide_store<L, Q, Sink, TRT>(f, rho, ux, uy, uz, Fx, Fy, Fz, p.omega, spw, p.ftarget, sink, p.trt_dw);
  } else {
    const float ussq = us.x * us.x + us.y * us.y + us.z * us.z;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const float w = L::w(i);
      const float eu = (float)L::ex(i) * us.x + (float)L::ey(i) * us.y + (float)L::ez(i) * us.z;
      sink.put(i, w * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * ussq));
    }
  }
  if (p.write_mac) {
    float4 m = in_solid ? make_float4(1.f, us.x, us.y, us.z) : make_float4(rho, ux, uy, uz);
    reinterpret_cast<float4 *>(mac + 4 * p.base)[cell] = m;
  }

  // Force on the body from this cell (bounce-back links were summed above).
  if (force) {
    if (bbody) {
      if (p.swept && fabsf(phi) < p.swept_band) {
        const bool solid_now = phi < 0.f;
        const bool solid_next = phi3_ahead(pos, p.body, 1.f, p.win) < 0.f;
        if (solid_now != solid_next) {
          float cx = 0.f, cy = 0.f, cz = 0.f;
#pragma unroll
          for (int i = 0; i < Q; ++i) {
            const float v = Codec<S>::ld(fi + (int64_t)i * n + cell, i, p.pk);
            cx += v * (float)L::ex(i);
            cy += v * (float)L::ey(i);
            cz += v * (float)L::ez(i);
          }
          if (!solid_now) { fbx += cx; fby += cy; fbz += cz; }
          else { fbx += -cx; fby += -cy; fbz += -cz; }
        }
      }
    } else if (p.has_body) {
      const float c2 = chi_from_phi(phi, p.chi_eps);
      if (c2 >= 1e-6f) {
        const float rc2 = rho * c2;
        fbx = -(rc2 * (us.x - uxs));
        fby = -(rc2 * (us.y - uys));
        fbz = -(rc2 * (us.z - uzs));
      }
    }
    const V3 r = body_delta(pos, p.body, p.win);
    const float rx = r.x, ry = r.y, rz = r.z;
    cf.fx = fbx; cf.fy = fby; cf.fz = fbz;
    cf.tx = ry * fbz - rz * fby;
    cf.ty = rz * fbx - rx * fbz;
    cf.tz = rx * fby - ry * fbx;
  }
}


// Pull gather of one cell from the periodic sources.
template <int Q, typename S>
__device__ __forceinline__ void gather3(const S *__restrict__ fi, const StepParams &p, int x, int y, int z,
                                        float (&f)[Q]) {
  using L = Lattice<Q>;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int64_t n = p.n;
  const int nxny = nx * ny;
  const int cell = z * nxny + y * nx + x;
  // Offset of the pull source for e = +1 / -1 on each axis, periodic.
  const int xo_p = x == 0 ? nx - 1 : -1, xo_m = x == nx - 1 ? 1 - nx : 1;
  const int yo_p = y == 0 ? (ny - 1) * nx : -nx, yo_m = y == ny - 1 ? (1 - ny) * nx : nx;
  const int zo_p = z == 0 ? (nz - 1) * nxny : -nxny, zo_m = z == nz - 1 ? (1 - nz) * nxny : nxny;
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const int ex = L::ex(i), ey = L::ey(i), ez = L::ez(i);
    const int off = (ex == 1 ? xo_p : (ex == -1 ? xo_m : 0)) + (ey == 1 ? yo_p : (ey == -1 ? yo_m : 0)) +
                    (ez == 1 ? zo_p : (ez == -1 ? zo_m : 0));
    f[i] = Codec<S>::ld(fi + (int64_t)i * n + (cell + off), i, p.pk);
  }
}

// TRT: the collision is the two-relaxation-time one; callers pass
// p.trt_dw != 0 (see collide_store).
template <int Q, typename S, bool TRT = false>
__device__ __forceinline__ void cell3(const S *__restrict__ fin, S *__restrict__ fout,
                                      float *__restrict__ mac, const StepParams &p, int x, int y,
                                      int z, bool force, CellForce &cf) {
  const S *fi = fin + p.base;
  float f[Q];
  gather3<Q, S>(fi, p, x, y, z, f);
  MemSink<S> sink{fout + p.base, p.n, (z * p.ny + y) * p.nx + x, p.pk};
  cell3_core<Q, S, MemSink<S>, TRT>(fi, f, mac, p, x, y, z, force, cf, sink);
}

// cell3 with the collision picked from the launch's parameters (a
// warp-uniform branch), for kernels that do not instantiate per collision.
template <int Q, typename S>
__device__ __forceinline__ void cell3_any(const S *__restrict__ fin, S *__restrict__ fout,
                                          float *__restrict__ mac, const StepParams &p, int x, int y,
                                          int z, bool force, CellForce &cf) {
  if (p.trt_dw != 0.f) cell3<Q, S, true>(fin, fout, mac, p, x, y, z, force, cf);
  else cell3<Q, S, false>(fin, fout, mac, p, x, y, z, force, cf);
}

// A cell that only fluid can reach: no body link within reach (or no body),
// no wall on any of its links, no moving window, and not in the force
// reduction. For such a cell cell3() finds phi = 1e30, u_s = 0 and chi = 0,
// so its Guo force is the body force alone (rho chi (u_s - u*) = +-0, and
// +-0 + F = F) and nothing is patched; this is that path with the dead
// tests taken out, to the bit.
template <int Q, typename S, bool TRT = false>
__device__ __forceinline__ void cell3_fluid(const S *__restrict__ fin, S *__restrict__ fout,
                                            float *__restrict__ mac, const StepParams &p, int x, int y, int z) {
  using L = Lattice<Q>;
  const S *fi = fin + p.base;
  float f[Q];
  gather3<Q, S>(fi, p, x, y, z, f);
  float rho, mx, my, mz;
  moments<L, Q>(f, rho, mx, my, mz);
  const float inv = 1.0f / fmaxf(rho, 1e-6f);
  const float uxs = mx * inv, uys = my * inv, uzs = mz * inv;
  const float hinv = 0.5f * inv;
  const float ux = fmaf(p.fx, hinv, uxs);
  const float uy = fmaf(p.fy, hinv, uys);
  const float uz = fmaf(p.fz, hinv, uzs);
  float spw = 0.f;
  if (p.sponge_w > 0.f) {
    const float dx = p.sax ? fminf((float)x, (float)(p.nx - 1) - (float)x) : 1e30f;
    const float dy = p.say ? fminf((float)y, (float)(p.ny - 1) - (float)y) : 1e30f;
    const float zg = (float)(z + p.zoff);
    const float dz = p.saz ? fminf(zg, (float)(p.nzg - 1) - zg) : 1e30f;
    spw = sponge_weight_inv(fminf(dx, fminf(dy, dz)), p.sponge_inv);
  }
  const int cell = (z * p.ny + y) * p.nx + x;
  MemSink<S> sink{fout + p.base, p.n, cell, p.pk};
  collide_store<L, Q, MemSink<S>, TRT>(f, rho, ux, uy, uz, p.fx, p.fy, p.fz, p.omega, spw, p.ftarget, sink,
                                       p.trt_dw);
  if (p.write_mac) reinterpret_cast<float4 *>(mac + 4 * p.base)[cell] = make_float4(rho, ux, uy, uz);
}

// Force contribution of one cell without the collision (a free body's
// force pass).
template <int Q, typename S>
__device__ __forceinline__ void cell3_force(const S *__restrict__ fin, const StepParams &p, int x, int y, int z,
                                            CellForce &cf) {
  const S *fi = fin + p.base;
  float f[Q];
  gather3<Q, S>(fi, p, x, y, z, f);
  NullSink sink;
  cell3_core<Q, S>(fi, f, nullptr, p, x, y, z, true, cf, sink);
}

// ---- 2D cell update (D2Q9) ---------------------------------------------------

// Pull gather of one D2Q9 cell from its periodic sources.
template <typename S>
__device__ __forceinline__ void gather2(const S *__restrict__ fi, const StepParams &p, int x, int y, float (&f)[9]) {
  using L = Lattice<9>;
  const int W = p.nx, H = p.ny;
  const int64_t n = p.n;
  const int cell = y * W + x;
  const int xo_p = x == 0 ? W - 1 : -1, xo_m = x == W - 1 ? 1 - W : 1;
  const int yo_p = y == 0 ? (H - 1) * W : -W, yo_m = y == H - 1 ? (1 - H) * W : W;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int ex = L::ex(i), ey = L::ey(i);
    const int off = (ex == 1 ? xo_p : (ex == -1 ? xo_m : 0)) + (ey == 1 ? yo_p : (ey == -1 ? yo_m : 0));
    f[i] = Codec<S>::ld(fi + (int64_t)i * n + (cell + off), i, p.pk);
  }
}

template <typename S>
__device__ __forceinline__ void cell2_core(const S *__restrict__ fin, float (&f)[9], S *__restrict__ fout,
                                           float *__restrict__ mac, const StepParams &p, int x, int y, bool force,
                                           CellForce &cf);

template <typename S>
__device__ __forceinline__ void cell2(const S *__restrict__ fin, S *__restrict__ fout,
                                      float *__restrict__ mac, const StepParams &p, int x, int y,
                                      bool force, CellForce &cf) {
  float f[9];
  gather2<S>(fin + p.base, p, x, y, f);
  cell2_core<S>(fin, f, fout, mac, p, x, y, force, cf);
}

// Everything after the gather for one D2Q9 cell: bounce-back and wall
// patches, moments, forcing, collision, mac, force.
template <typename S>
__device__ __forceinline__ void cell2_core(const S *__restrict__ fin, float (&f)[9], S *__restrict__ fout,
                                           float *__restrict__ mac, const StepParams &p, int x, int y, bool force,
                                           CellForce &cf) {
  using L = Lattice<9>;
  const int W = p.nx, H = p.ny;
  const int64_t n = p.n;
  const S *fi = fin + p.base;
  S *fo_ = fout + p.base;
  const int cell = y * W + x;
  const float fW = (float)W, fH = (float)H;
  const float px = (float)x, py = (float)y;
  float rx = 0.f, ry = 0.f, usx = 0.f, usy = 0.f, phi = 1e30f;
  if (p.has_body) {
    rx = wrap_delta(px - p.body.cx, fW);
    ry = wrap_delta(py - p.body.cy, fH);
    usx = p.body.vx - p.body.wz * ry;
    usy = p.body.vy + p.body.wz * rx;
    phi = phi2(px, py, p.body, fW, fH);
  }
  const bool bbody = p.has_body && p.bb;
  const bool near = bbody && phi < 2.5f;
  const bool at_wall = p.wall_y && (y == 0 || y == H - 1);
  float fbx = 0.f, fby = 0.f;
  if (near || at_wall) {
    const int xm = x == 0 ? W - 1 : x - 1, xp = x == W - 1 ? 0 : x + 1;
    const int ym = y == 0 ? H - 1 : y - 1, yp = y == H - 1 ? 0 : y + 1;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const int ex = L::ex(i), ey = L::ey(i), o = L::opp(i);
      bool solid = false;
      if (near) {
        const int sx = ex == 1 ? xm : (ex == -1 ? xp : x);
        const int sy = ey == 1 ? ym : (ey == -1 ? yp : y);
        solid = phi2((float)sx, (float)sy, p.body, fW, fH) < 0.f;
      }
      if (solid) {
        const float fopp = Codec<S>::ld(fi + (int64_t)o * n + cell, o, p.pk);
        const float corr = 2.f * L::w(i) * ((float)ex * usx + (float)ey * usy) * kInvCS2;
        f[i] = fopp + corr;
        if (phi >= 0.f) {
          const float m = 2.f * fopp + corr;
          fbx += -(float)ex * m;
          fby += -(float)ey * m;
        }
      } else if (at_wall) {
        const int ysrc = y - ey;
        if (ysrc < 0 || ysrc >= H) {
          const float wu = ysrc < 0 ? p.wall_u0 : p.wall_u1;
          const float corr = 2.f * L::w(i) * (float)ex * wu * kInvCS2;
          f[i] = Codec<S>::ld(fi + (int64_t)o * n + cell, o, p.pk) + corr;
        }
      }
    }
  }
  float rho, mxs, mys, mzs;
  moments<L, 9>(f, rho, mxs, mys, mzs);
  const float rhoDen = fmaxf(rho, 1e-6f);
  const float inv = 1.0f / rhoDen;
  const float uxs = mxs * inv, uys = mys * inv;
  const float chi = (p.has_body && !p.bb) ? chi_from_phi(phi, p.chi_eps) : 0.f;
  const float Fx = rho * chi * (usx - uxs) + p.fx;
  const float Fy = rho * chi * (usy - uys) + p.fy;
  const float hinv = 0.5f * inv;
  const float ux = fmaf(Fx, hinv, uxs);
  const float uy = fmaf(Fy, hinv, uys);

  float spw = 0.f;
  if (p.sponge_w > 0.f) {
    const float dx = fminf(px, (float)(W - 1 - x));
    const float dy = fminf(py, (float)(H - 1 - y));
    spw = sponge_weight_inv(fminf(dx, dy), p.sponge_inv);
  }
  const bool in_solid = p.solid_eq && bbody && phi < 0.f;
  if (!in_solid) {
    MemSink<S> sink{fo_, n, cell, p.pk};
    collide_store<L, 9>(f, rho, ux, uy, 0.f, Fx, Fy, 0.f, p.omega, spw, p.ftarget, sink);
  } else {
    const float ussq = usx * usx + usy * usy;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const float w = L::w(i);
      const float eu = (float)L::ex(i) * usx + (float)L::ey(i) * usy;
      Codec<S>::st(fo_ + (int64_t)i * n + cell, w * 1.0f * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * ussq), i, p.pk);
    }
  }
  if (p.write_mac) reinterpret_cast<float4 *>(mac + 4 * p.base)[cell] = make_float4(rho, ux, uy, 0.f);

  if (force) {
    if (!bbody && p.has_body) {
      const float c2 = chi_from_phi(phi, p.chi_eps);
      if (c2 >= 1e-6f) {
        fbx = -(rho * c2 * (usx - uxs));
        fby = -(rho * c2 * (usy - uys));
      }
    }
    cf.fx = fbx;
    cf.fy = fby;
    cf.tz = rx * fby - ry * fbx;
  }
}

}  // namespace lbm
