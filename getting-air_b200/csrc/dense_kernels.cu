// Dense-grid kernels for sm_100a: the fused pull-stream / BGK / Guo-forcing
// step with its body-force reduction, equilibrium seeding, storage
// conversion and the FP64 conserved-totals reduction.
//
// Reference arithmetic:
//   3D step    common_d3_step.wgsl:224-400
//   3D force   common_d3_force.wgsl:171-283 (momentum exchange with local
//              rho_w and the swept-cell term, or the chi penalty)
//   2D step    lbm_step.wgsl:137-270
//   2D force   lbm_force.wgsl (main)
//   initEq     common_d3_step.wgsl:206-222
//   totals     amr2d-gpu.mjs:698-736 readConservedTotals
//
// Layout in HBM: f is Q planes, plane-major, `f[i * n + cell]` with
// cell = (z*NY + y)*NX + x -- the reference's layout, which is also the one
// that gives every warp a coalesced 128-byte row per plane. One thread owns
// one cell: it issues the Q pull loads up front (periodic sources), patches
// the few bounce-back links afterwards, collides in registers and writes
// the Q planes of its own cell. The mac field is written only when the
// host asks for it (the last step of a batch), not every step.
//
// The body force is summed INSIDE the step: the reference runs a separate
// full-grid force pass before each step over the same pre-streaming f_in,
// and every quantity it needs (f_opp at the cell, the streamed rho and u*)
// is already in this kernel's registers. Only the launch blocks whose cells
// can touch the body reduce; each writes one FP64 partial and the last
// block to finish sums the partials in a fixed order, so the result is
// deterministic and no second launch is needed.

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "dense.cuh"
#include "geometry.cuh"
#include "lattice.cuh"

namespace lbm {

namespace {

constexpr float kCS2 = 1.0f / 3.0f;

// ---- storage codecs --------------------------------------------------------
// The 16-bit forms hold f_i - w_i (the f-pack mode-2 offset,
// common_fpack.wgsl:91-121), rounded to nearest even; arithmetic stays f32.
template <typename S> struct Codec;
template <> struct Codec<float> {
  static __device__ __forceinline__ float ld(const float *p, float) { return __ldg(p); }
  static __device__ __forceinline__ void st(float *p, float v, float) { *p = v; }
};
template <> struct Codec<__half> {
  static __device__ __forceinline__ float ld(const __half *p, float w) {
    return __half2float(__ldg(p)) + w;
  }
  static __device__ __forceinline__ void st(__half *p, float v, float w) {
    *p = __float2half_rn(v - w);
  }
};
template <> struct Codec<__nv_bfloat16> {
  static __device__ __forceinline__ float ld(const __nv_bfloat16 *p, float w) {
    return __bfloat162float(__ldg(p)) + w;
  }
  static __device__ __forceinline__ void st(__nv_bfloat16 *p, float v, float w) {
    *p = __float2bfloat16_rn(v - w);
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

// Writes this block's partial (thread 0 holds it), and if this block is the
// last of `nparts` to do so, sums all partials in index order into `out`.
template <int NV, int THREADS>
__device__ void finish_sum(const double (&v)[NV], double *partials, unsigned int *counter,
                           int nparts, int part, double *out, double *sm) {
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[(int64_t)part * NV + k] = v[k];
    __threadfence();
    unsigned int ticket = atomicAdd(counter, 1u);
    s_last = (ticket == (unsigned int)(nparts - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (int j = threadIdx.x; j < nparts; j += THREADS)
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&partials[(int64_t)j * NV + k]);
  block_sum<NV, THREADS>(acc, sm);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = acc[k];
    *counter = 0u;
  }
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

// ---- 3D fused step ---------------------------------------------------------

template <int Q, typename S>
__global__ void __launch_bounds__(kStepThreads)
    d3_step(const S *__restrict__ fin, S *__restrict__ fout, float *__restrict__ mac,
            const StepParams p) {
  using L = Lattice<Q>;
  const int x = blockIdx.x * kStepThreads + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int64_t n = p.n;
  float fbx = 0.f, fby = 0.f, fbz = 0.f, tbx = 0.f, tby = 0.f, tbz = 0.f;

  if (x < nx) {
    const int cell = (z * ny + y) * nx + x;
    const int xm = x == 0 ? nx - 1 : x - 1, xp = x == nx - 1 ? 0 : x + 1;
    const int ym = y == 0 ? ny - 1 : y - 1, yp = y == ny - 1 ? 0 : y + 1;
    const int zm = z == 0 ? nz - 1 : z - 1, zp = z == nz - 1 ? 0 : z + 1;

    // 1. Pull-stream from the periodic sources.
    float f[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const int ex = L::ex(i), ey = L::ey(i), ez = L::ez(i);
      const int sx = ex == 1 ? xm : (ex == -1 ? xp : x);
      const int sy = ey == 1 ? ym : (ey == -1 ? yp : y);
      const int sz = ez == 1 ? zm : (ez == -1 ? zp : z);
      f[i] = Codec<S>::ld(fin + (int64_t)i * n + ((sz * ny + sy) * nx + sx), L::w(i));
    }

    const V3 pos = {(float)x, (float)y, (float)z};
    float phi = 1e30f;
    V3 us = {0.f, 0.f, 0.f};
    if (p.has_body) {
      phi = phi3(pos, p.body);
      us = body_velocity3(pos, p.body);
    }
    const bool bbody = p.has_body && p.bb;
    const bool at_wall = (p.wall_x && (x == 0 || x == nx - 1)) ||
                         (p.wall_y && (y == 0 || y == ny - 1)) ||
                         (p.wall_z && (z == 0 || z == nz - 1));
    // A link can only reach a solid source from within |e| <= sqrt(3) of the
    // surface, and a signed distance is 1-Lipschitz.
    const bool near = bbody && phi < 2.5f;

    // 1b. Bounce-back links: body (Ladd, with local rho_w) first, then walls.
    if (near || at_wall) {
      float rhoW = 1.f;
      if (bbody && p.rho_w_local && phi < 2.f) {
        float s = 0.f;
#pragma unroll
        for (int i = 0; i < Q; ++i) s += Codec<S>::ld(fin + (int64_t)i * n + cell, L::w(i));
        rhoW = s;
      }
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const int ex = L::ex(i), ey = L::ey(i), ez = L::ez(i);
        const int o = L::opp(i);
        bool solid = false;
        if (near) solid = phi3({pos.x - (float)ex, pos.y - (float)ey, pos.z - (float)ez}, p.body) < 0.f;
        if (solid) {
          const float fo = Codec<S>::ld(fin + (int64_t)o * n + cell, L::w(o));
          const float corr = 2.f * L::w(i) * rhoW *
                             ((float)ex * us.x + (float)ey * us.y + (float)ez * us.z) / kCS2;
          f[i] = fo + corr;
          if (phi >= 0.f) {
            const float m = 2.f * fo + corr;
            fbx += -(float)ex * m;
            fby += -(float)ey * m;
            fbz += -(float)ez * m;
          }
        } else if (at_wall) {
          const int sx = x - ex, sy = y - ey, sz = z - ez;
          const bool out = (p.wall_x && (sx < 0 || sx >= nx)) ||
                           (p.wall_y && (sy < 0 || sy >= ny)) ||
                           (p.wall_z && (sz < 0 || sz >= nz));
          if (out) f[i] = Codec<S>::ld(fin + (int64_t)o * n + cell, L::w(o));
        }
      }
    }

    // 2. Moments.
    float rho = 0.f, mx = 0.f, my = 0.f, mz = 0.f;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      rho += f[i];
      mx += f[i] * (float)L::ex(i);
      my += f[i] * (float)L::ey(i);
      mz += f[i] * (float)L::ez(i);
    }
    const float rhoDen = fmaxf(rho, 1e-6f);
    const float uxs = mx / rhoDen, uys = my / rhoDen, uzs = mz / rhoDen;

    // 3. Solid coupling and Guo forcing.
    const float chi = (p.has_body && !p.bb) ? chi_from_phi(phi, p.chi_eps) : 0.f;
    const float rc = rho * chi;
    const float Fx = rc * (us.x - uxs) + p.fx;
    const float Fy = rc * (us.y - uys) + p.fy;
    const float Fz = rc * (us.z - uzs) + p.fz;
    const float ux = uxs + Fx / (2.0f * rhoDen);
    const float uy = uys + Fy / (2.0f * rhoDen);
    const float uz = uzs + Fz / (2.0f * rhoDen);
    const float usq = ux * ux + uy * uy + uz * uz;

    float spw = 0.f;
    if (p.sponge_w > 0.f) {
      const float dx = p.sax ? fminf(pos.x, (float)(nx - 1 - x)) : 1e30f;
      const float dy = p.say ? fminf(pos.y, (float)(ny - 1 - y)) : 1e30f;
      const float dz = p.saz ? fminf(pos.z, (float)(nz - 1 - z)) : 1e30f;
      spw = sponge_weight(fminf(dx, fminf(dy, dz)), p.sponge_w);
    }

    // 4. Collide (+ sponge blend), 5. solid interior held at feq(1, u_body).
    const float omg = p.omega;
    const float sfac = 1.0f - 0.5f * omg;
    const bool in_solid = p.solid_eq && bbody && phi < 0.f;
    const float ussq = us.x * us.x + us.y * us.y + us.z * us.z;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const float exf = (float)L::ex(i), eyf = (float)L::ey(i), ezf = (float)L::ez(i);
      const float w = L::w(i);
      float out;
      if (in_solid) {
        const float eu = exf * us.x + eyf * us.y + ezf * us.z;
        out = w * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * ussq);
      } else {
        const float eu = exf * ux + eyf * uy + ezf * uz;
        const float feq = w * rho * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * usq);
        const float t2 = eu * 9.0f;
        const float Si = sfac * w *
                         (((exf - ux) * 3.0f + t2 * exf) * Fx + ((eyf - uy) * 3.0f + t2 * eyf) * Fy +
                          ((ezf - uz) * 3.0f + t2 * ezf) * Fz);
        const float fc = f[i] - omg * (f[i] - feq) + Si;
        out = spw > 0.f ? fc * (1.0f - spw) + p.ftarget[i] * spw : fc;
      }
      Codec<S>::st(fout + (int64_t)i * n + cell, out, w);
    }
    if (p.write_mac) {
      float4 m = in_solid ? make_float4(1.f, us.x, us.y, us.z) : make_float4(rho, ux, uy, uz);
      reinterpret_cast<float4 *>(mac)[cell] = m;
    }

    // Force on the body from this cell (the parts not already summed above).
    if (p.force_on) {
      if (bbody) {
        if (p.swept && fabsf(phi) < p.swept_band) {
          const bool solid_now = phi < 0.f;
          const bool solid_next = phi3_ahead(pos, p.body, 1.f) < 0.f;
          if (solid_now != solid_next) {
            float cx = 0.f, cy = 0.f, cz = 0.f;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
              const float v = Codec<S>::ld(fin + (int64_t)i * n + cell, L::w(i));
              cx += v * (float)L::ex(i);
              cy += v * (float)L::ey(i);
              cz += v * (float)L::ez(i);
            }
            if (!solid_now) { fbx += cx; fby += cy; fbz += cz; }
            else { fbx += -cx; fby += -cy; fbz += -cz; }
          }
        }
      } else if (p.has_body && chi_from_phi(phi, p.chi_eps) >= 1e-6f) {
        const float c2 = chi_from_phi(phi, p.chi_eps);
        const float rc2 = rho * c2;
        fbx = -(rc2 * (us.x - uxs));
        fby = -(rc2 * (us.y - uys));
        fbz = -(rc2 * (us.z - uzs));
      }
      const float rx = pos.x - p.body.cx, ry = pos.y - p.body.cy, rz = pos.z - p.body.cz;
      tbx = ry * fbz - rz * fby;
      tby = rz * fbx - rx * fbz;
      tbz = rx * fby - ry * fbx;
    }
  }

  if (p.force_on) {
    const int bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z;
    if (bx >= p.rbx0 && bx < p.rbx1 && by >= p.rby0 && by < p.rby1 && bz >= p.rbz0 &&
        bz < p.rbz1) {
      __shared__ double sm[kForceSlots * (kStepThreads / 32)];
      double bad = 0.0;
      double v[kForceSlots];
      v[0] = finite_or_zero(fbx, bad);
      v[1] = finite_or_zero(fby, bad);
      v[2] = finite_or_zero(fbz, bad);
      v[3] = finite_or_zero(tbx, bad);
      v[4] = finite_or_zero(tby, bad);
      v[5] = finite_or_zero(tbz, bad);
      v[6] = bad;
      v[7] = 0.0;
      block_sum<kForceSlots, kStepThreads>(v, sm);
      const int rx = p.rbx1 - p.rbx0, ry = p.rby1 - p.rby0, rz = p.rbz1 - p.rbz0;
      const int part = ((bz - p.rbz0) * ry + (by - p.rby0)) * rx + (bx - p.rbx0);
      finish_sum<kForceSlots, kStepThreads>(v, p.partials, p.counter, rx * ry * rz, part,
                                            p.force_out, sm);
    }
  }
}

// ---- 2D fused step (D2Q9) ---------------------------------------------------

template <typename S>
__global__ void __launch_bounds__(kStepThreads)
    d2_step(const S *__restrict__ fin, S *__restrict__ fout, float *__restrict__ mac,
            const StepParams p) {
  using L = Lattice<9>;
  const int x = blockIdx.x * kStepThreads + threadIdx.x;
  const int y = blockIdx.y;
  const int W = p.nx, H = p.ny;
  const int64_t n = p.n;
  float fbx = 0.f, fby = 0.f, tbz = 0.f;

  if (x < W) {
    const int cell = y * W + x;
    const int xm = x == 0 ? W - 1 : x - 1, xp = x == W - 1 ? 0 : x + 1;
    const int ym = y == 0 ? H - 1 : y - 1, yp = y == H - 1 ? 0 : y + 1;
    float f[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const int ex = L::ex(i), ey = L::ey(i);
      const int sx = ex == 1 ? xm : (ex == -1 ? xp : x);
      const int sy = ey == 1 ? ym : (ey == -1 ? yp : y);
      f[i] = Codec<S>::ld(fin + (int64_t)i * n + (sy * W + sx), L::w(i));
    }
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
    if (near || at_wall) {
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
          const float fo = Codec<S>::ld(fin + (int64_t)o * n + cell, L::w(o));
          const float corr = 2.f * L::w(i) * ((float)ex * usx + (float)ey * usy) / kCS2;
          f[i] = fo + corr;
          if (phi >= 0.f) {
            const float m = 2.f * fo + corr;
            fbx += -(float)ex * m;
            fby += -(float)ey * m;
          }
        } else if (at_wall) {
          const int ysrc = y - ey;
          if (ysrc < 0 || ysrc >= H) {
            const float wu = ysrc < 0 ? p.wall_u0 : p.wall_u1;
            const float corr = 2.f * L::w(i) * (float)ex * wu / kCS2;
            f[i] = Codec<S>::ld(fin + (int64_t)o * n + cell, L::w(o)) + corr;
          }
        }
      }
    }
    float rho = 0.f, uxs = 0.f, uys = 0.f;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      rho += f[i];
      uxs += f[i] * (float)L::ex(i);
      uys += f[i] * (float)L::ey(i);
    }
    const float rhoDen = fmaxf(rho, 1e-6f);
    uxs /= rhoDen;
    uys /= rhoDen;
    const float chi = (p.has_body && !p.bb) ? chi_from_phi(phi, p.chi_eps) : 0.f;
    const float Fx = rho * chi * (usx - uxs) + p.fx;
    const float Fy = rho * chi * (usy - uys) + p.fy;
    const float ux = uxs + Fx / (2.0f * rhoDen);
    const float uy = uys + Fy / (2.0f * rhoDen);
    const float usq = ux * ux + uy * uy;

    float spw = 0.f;
    if (p.sponge_w > 0.f) {
      const float dx = fminf(px, (float)(W - 1 - x));
      const float dy = fminf(py, (float)(H - 1 - y));
      spw = sponge_weight(fminf(dx, dy), p.sponge_w);
    }
    const float omg = p.omega;
    const float sfac = 1.0f - 0.5f * omg;
    const bool in_solid = p.solid_eq && bbody && phi < 0.f;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const float exf = (float)L::ex(i), eyf = (float)L::ey(i);
      const float w = L::w(i);
      float out;
      if (in_solid) {
        const float eu = exf * usx + eyf * usy;
        out = w * 1.0f * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * (usx * usx + usy * usy));
      } else {
        const float eu = exf * ux + eyf * uy;
        const float feq = w * rho * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * usq);
        const float term2 = (exf * ux + eyf * uy) * 9.0f;
        const float Si = sfac * w *
                         (((exf - ux) * 3.0f + term2 * exf) * Fx + ((eyf - uy) * 3.0f + term2 * eyf) * Fy);
        const float fc = f[i] - omg * (f[i] - feq) + Si;
        out = spw > 0.f ? fc * (1.0f - spw) + p.ftarget[i] * spw : fc;
      }
      Codec<S>::st(fout + (int64_t)i * n + cell, out, w);
    }
    if (p.write_mac) reinterpret_cast<float4 *>(mac)[cell] = make_float4(rho, ux, uy, 0.f);

    if (p.force_on) {
      if (!bbody && p.has_body) {
        const float c2 = chi_from_phi(phi, p.chi_eps);
        if (c2 >= 1e-6f) {
          fbx = -(rho * c2 * (usx - uxs));
          fby = -(rho * c2 * (usy - uys));
        }
        tbz = rx * fby - ry * fbx;
      } else if (phi >= 0.f) {
        tbz = rx * fby - ry * fbx;
      }
    }
  }

  if (p.force_on) {
    const int bx = blockIdx.x, by = blockIdx.y;
    if (bx >= p.rbx0 && bx < p.rbx1 && by >= p.rby0 && by < p.rby1) {
      __shared__ double sm[kForceSlots * (kStepThreads / 32)];
      double bad = 0.0;
      double v[kForceSlots];
      v[0] = finite_or_zero(fbx, bad);
      v[1] = finite_or_zero(fby, bad);
      v[2] = 0.0;
      v[3] = 0.0;
      v[4] = 0.0;
      v[5] = finite_or_zero(tbz, bad);
      v[6] = bad;
      v[7] = 0.0;
      block_sum<kForceSlots, kStepThreads>(v, sm);
      const int rx = p.rbx1 - p.rbx0, ry = p.rby1 - p.rby0;
      const int part = (by - p.rby0) * rx + (bx - p.rbx0);
      finish_sum<kForceSlots, kStepThreads>(v, p.partials, p.counter, rx * ry, part,
                                            p.force_out, sm);
    }
  }
}

// ---- seeding and storage conversion ----------------------------------------

template <int Q, typename S>
__global__ void init_eq(const float4 *__restrict__ mac, S *__restrict__ f, int64_t n) {
  using L = Lattice<Q>;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const float4 m = mac[c];
    const float rho = m.x, ux = m.y, uy = m.z, uz = Q == 9 ? 0.f : m.w;
    const float usq = Q == 9 ? (ux * ux + uy * uy) : (ux * ux + uy * uy + uz * uz);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const float eu = (float)L::ex(i) * ux + (float)L::ey(i) * uy + (float)L::ez(i) * uz;
      const float v = L::w(i) * rho * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * usq);
      Codec<S>::st(f + (int64_t)i * n + c, v, L::w(i));
    }
  }
}

template <int Q, typename S>
__global__ void pack_planes(const float *__restrict__ src, S *__restrict__ dst, int64_t n) {
  using L = Lattice<Q>;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int i = 0; i < Q; ++i) Codec<S>::st(dst + (int64_t)i * n + c, src[(int64_t)i * n + c], L::w(i));
}

template <int Q, typename S>
__global__ void unpack_planes(const S *__restrict__ src, float *__restrict__ dst, int64_t n) {
  using L = Lattice<Q>;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int i = 0; i < Q; ++i) dst[(int64_t)i * n + c] = Codec<S>::ld(src + (int64_t)i * n + c, L::w(i));
}

// ---- conserved totals ------------------------------------------------------
// Per cell the reference sums the f32 populations in f64 (JS numbers):
// rho, rho u, then mass += rho - 1. Same here, with FP64 partial sums per
// block and a fixed-order final sum.

constexpr int kTotalsBlocks = 148 * 4;

template <int Q, typename S>
__global__ void __launch_bounds__(kReduceThreads)
    totals_kernel(const S *__restrict__ f, int64_t n, double *partials, unsigned int *counter,
                  double *out) {
  using L = Lattice<Q>;
  double mass = 0.0, px = 0.0, py = 0.0, pz = 0.0, bad = 0.0;
  double rmin = 1e300, rmax = -1e300, u2max = 0.0;
  for (int64_t c = blockIdx.x * (int64_t)kReduceThreads + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * kReduceThreads) {
    double rho = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const double v = (double)Codec<S>::ld(f + (int64_t)i * n + c, L::w(i));
      rho += v;
      mx += v * L::ex(i);
      my += v * L::ey(i);
      mz += v * L::ez(i);
    }
    if (!isfinite(rho + mx + my + mz)) {
      bad += 1.0;
      continue;
    }
    mass += rho - 1.0;
    px += mx;
    py += my;
    pz += mz;
    rmin = fmin(rmin, rho);
    rmax = fmax(rmax, rho);
    u2max = fmax(u2max, (mx * mx + my * my + mz * mz) / (rho * rho));
  }
  // Sums via the shared block_sum; min/max folded through negation tricks
  // would lose determinism guarantees for ties, so they are reduced apart.
  __shared__ double sm[kTotalsSlots * (kReduceThreads / 32)];
  double v[5] = {mass, px, py, pz, bad};
  block_sum<5, kReduceThreads>(v, sm);
  double mm[3] = {rmin, -rmax, -u2max};
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mm[k] = fmin(mm[k], __shfl_down_sync(0xffffffffu, mm[k], o));
  __shared__ double smm[3 * (kReduceThreads / 32)];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 3; ++k) smm[k * (kReduceThreads / 32) + warp] = mm[k];
  __syncthreads();
  if (warp == 0) {
    for (int k = 0; k < 3; ++k) {
      double t = lane < kReduceThreads / 32 ? smm[k * (kReduceThreads / 32) + lane] : 1e300;
      for (int o = 16; o > 0; o >>= 1) t = fmin(t, __shfl_down_sync(0xffffffffu, t, o));
      mm[k] = t;
    }
  }
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    double *pp = partials + (int64_t)blockIdx.x * kTotalsSlots;
    pp[0] = v[0]; pp[1] = v[1]; pp[2] = v[2]; pp[3] = v[3];
    pp[4] = mm[0]; pp[5] = mm[1]; pp[6] = mm[2]; pp[7] = v[4];
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s7 = 0, m4 = 1e300, m5 = 1e300, m6 = 1e300;
    for (unsigned int j = 0; j < gridDim.x; ++j) {
      const double *pp = partials + (int64_t)j * kTotalsSlots;
      s0 += __ldcg(pp + 0); s1 += __ldcg(pp + 1); s2 += __ldcg(pp + 2); s3 += __ldcg(pp + 3);
      m4 = fmin(m4, __ldcg(pp + 4)); m5 = fmin(m5, __ldcg(pp + 5)); m6 = fmin(m6, __ldcg(pp + 6));
      s7 += __ldcg(pp + 7);
    }
    out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
    out[4] = m4; out[5] = -m5; out[6] = sqrt(-m6 < 0 ? 0.0 : -m6); out[7] = s7;
    *counter = 0u;
  }
}

template <typename F>
cudaError_t dispatch(int q, int storage, F &&fn) {
  switch (q * 4 + storage) {
    case 9 * 4 + 0: fn.template operator()<9, float>(); break;
    case 9 * 4 + 1: fn.template operator()<9, __half>(); break;
    case 9 * 4 + 2: fn.template operator()<9, __nv_bfloat16>(); break;
    case 19 * 4 + 0: fn.template operator()<19, float>(); break;
    case 19 * 4 + 1: fn.template operator()<19, __half>(); break;
    case 19 * 4 + 2: fn.template operator()<19, __nv_bfloat16>(); break;
    case 27 * 4 + 0: fn.template operator()<27, float>(); break;
    case 27 * 4 + 1: fn.template operator()<27, __half>(); break;
    case 27 * 4 + 2: fn.template operator()<27, __nv_bfloat16>(); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  return (int)(b < 148 * 8 ? (b < 1 ? 1 : b) : 148 * 8);
}

}  // namespace

cudaError_t launch_step(int q, int storage, const void *f_in, void *f_out, float *mac,
                        const StepParams &p, cudaStream_t st) {
  dim3 grid((p.nx + kStepThreads - 1) / kStepThreads, p.ny, q == 9 ? 1 : p.nz);
  return dispatch(q, storage, [&]<int Q, typename S>() {
    if constexpr (Q == 9)
      d2_step<S><<<grid, kStepThreads, 0, st>>>((const S *)f_in, (S *)f_out, mac, p);
    else
      d3_step<Q, S><<<grid, kStepThreads, 0, st>>>((const S *)f_in, (S *)f_out, mac, p);
  });
}

cudaError_t launch_init_eq(int q, int storage, const float *mac_in, void *f_out, int64_t n,
                           cudaStream_t st) {
  return dispatch(q, storage, [&]<int Q, typename S>() {
    init_eq<Q, S><<<grid_for(n, 256), 256, 0, st>>>((const float4 *)mac_in, (S *)f_out, n);
  });
}

cudaError_t launch_pack(int q, int storage, const float *f32, void *f_store, int64_t n,
                        cudaStream_t st) {
  return dispatch(q, storage, [&]<int Q, typename S>() {
    pack_planes<Q, S><<<grid_for(n, 256), 256, 0, st>>>(f32, (S *)f_store, n);
  });
}

cudaError_t launch_unpack(int q, int storage, const void *f_store, float *f32, int64_t n,
                          cudaStream_t st) {
  return dispatch(q, storage, [&]<int Q, typename S>() {
    unpack_planes<Q, S><<<grid_for(n, 256), 256, 0, st>>>((const S *)f_store, f32, n);
  });
}

int totals_blocks() { return kTotalsBlocks; }

cudaError_t launch_totals(int q, int storage, const void *f, int64_t n, double *partials,
                          unsigned int *counter, double *out, cudaStream_t st) {
  return dispatch(q, storage, [&]<int Q, typename S>() {
    totals_kernel<Q, S><<<kTotalsBlocks, kReduceThreads, 0, st>>>((const S *)f, n, partials,
                                                                  counter, out);
  });
}

}  // namespace lbm
