// Signed-distance geometry and rigid-body kinematics on the device, f32.
//
// 3D: common_d3_geometry.wgsl:60-253 (quaternion helpers qMul/qRotInv with
// [w,x,y,z] layout, sdSphere, sdRoundBox, sdSpheroid with 3 Newton steps on
// the meridional ellipse, get_phi3, get_phi3Ahead, bodyVelocity3,
// chiFromPhiEps3). bodyDelta3 takes the nearest periodic image on the
// axes of a moving window (common_d3_window.wgsl winWrapDelta) and is
// exactly p - c without one.
// 2D: common_geometry.wgsl:84-160 (get_phi: exact circle, far-field
// algebraic early-out at SDF_FAR = 64, otherwise 3 Newton steps) with the
// periodic nearest-image wrap `d -= N * round(d / N)`.
//
// Every expression keeps the reference's operation order so the solid mask
// (which link bounces back) is the same cell set as the reference's.
#pragma once

#include <cuda_runtime.h>
#include "../../include/lbm.h"
#include "body.cuh"

namespace lbm {

struct V3 { float x, y, z; };
struct Q4 { float w, x, y, z; };

// winWrap1: d - n round(d / n), round to nearest even as WGSL's round, each
// operation rounded on its own; the identity at n = 0.
__device__ __forceinline__ float win_wrap1(float d, float n) {
  return n > 0.f ? __fsub_rn(d, __fmul_rn(n, rintf(__fdiv_rn(d, n)))) : d;
}

// winOffset: whole cells the window has travelled, floor(c) - anchor.
__device__ __forceinline__ float win_offset1(float c, float anchor, float n) {
  return n > 0.f ? __fsub_rn(floorf(c), anchor) : 0.f;
}

// winCoord1: a buffer position as a window coordinate in [0, n).
__device__ __forceinline__ float win_coord1(float p, float off, float n) {
  if (!(n > 0.f)) return p;
  const float w = __fsub_rn(p, off);
  return __fsub_rn(w, __fmul_rn(n, floorf(__fdiv_rn(w, n))));
}

__device__ __forceinline__ Q4 q_mul(Q4 p, Q4 q) {
  return {p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z,
          p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y,
          p.w * q.y - p.x * q.z + p.y * q.w + p.z * q.x,
          p.w * q.z + p.x * q.y - p.y * q.x + p.z * q.w};
}

// WORLD -> BODY: conj(q) * (0, v) * q.
__device__ __forceinline__ V3 q_rot_inv(Q4 q, V3 v) {
  Q4 c = {q.w, -q.x, -q.y, -q.z};
  Q4 r = q_mul(q_mul(c, {0.f, v.x, v.y, v.z}), q);
  return {r.x, r.y, r.z};
}

// Explicitly rounded (no contraction) so every call site, inlined or not,
// produces the same bits -- which link bounces back must not depend on how
// the compiler fused a sum of squares.
__device__ __forceinline__ float len3(V3 v) {
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)), __fmul_rn(v.z, v.z)));
}

__device__ __forceinline__ float sd_round_box(V3 p, V3 h, float r) {
  V3 q = {fabsf(p.x) - (h.x - r), fabsf(p.y) - (h.y - r), fabsf(p.z) - (h.z - r)};
  V3 m = {fmaxf(q.x, 0.f), fmaxf(q.y, 0.f), fmaxf(q.z, 0.f)};
  return len3(m) + fminf(fmaxf(q.x, fmaxf(q.y, q.z)), 0.f) - r;
}

__device__ __forceinline__ float sd_spheroid(V3 p, float a, float c) {
  float r0 = sqrtf(p.x * p.x + p.y * p.y);
  if (fabsf(a - c) <= 1e-6f * fmaxf(a, c)) return sqrtf(r0 * r0 + p.z * p.z) - a;
  float x = fabsf(r0), y = fabsf(p.z);
  float rr = sqrtf((x * x) / (a * a) + (y * y) / (c * c));
  bool inside = rr < 1.0f;
  float t = atan2f(y * a, x * c);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float ct = cosf(t), st = sinf(t);
    float ex = x - a * ct, ey = y - c * st;
    float F = ex * (-a * st) + ey * (c * ct);
    float Fp = -(a * a * st * st + c * c * ct * ct) + ex * (-a * ct) + ey * (-c * st);
    t = t - F / (fabsf(Fp) < 1e-9f ? -1e-9f : Fp);
    t = fminf(fmaxf(t, 0.f), 1.5707963f);
  }
  float dx = x - a * cosf(t), dy = y - c * sinf(t);
  float d = sqrtf(dx * dx + dy * dy);
  return inside ? -d : d;
}

__device__ __forceinline__ float sdf_local3(V3 lp, const lbm_body &b) {
  if (b.shape == LBM_SHAPE_SPHERE) return len3(lp) - b.a;
  if (b.shape == LBM_SHAPE_SPHEROID) return sd_spheroid(lp, b.a, b.c);
  return sd_round_box(lp, {b.a, b.b, b.c}, b.r);
}

// bodyDelta3: p relative to the body centre, nearest image on windowed axes.
__device__ __forceinline__ V3 body_delta(V3 p, const lbm_body &b, const Win &w) {
  V3 d = {p.x - b.cx, p.y - b.cy, p.z - b.cz};
  if (w.on) {
    d.x = win_wrap1(d.x, w.n[0]);
    d.y = win_wrap1(d.y, w.n[1]);
    d.z = win_wrap1(d.z, w.n[2]);
  }
  return d;
}

__device__ __forceinline__ float phi3_inline(V3 p, const lbm_body &b, const Win &w) {
  return sdf_local3(q_rot_inv({b.qw, b.qx, b.qy, b.qz}, body_delta(p, b, w)), b);
}

// Out of line: called per bounce-back link candidate, which only the thin
// shell of cells next to the body evaluates; inlining it at 19-27 sites
// bloats the step kernel past the instruction cache.
static __device__ __noinline__ float phi3_call(float x, float y, float z, const lbm_body *b, const Win *w) {
  return phi3_inline({x, y, z}, *b, *w);
}

// A sphere's distance does not depend on its orientation, so the per-cell
// evaluation skips the rotation (bit-identical to the rotated form for the
// identity quaternion, the only orientation a pinned sphere has).
__device__ __forceinline__ float phi3(V3 p, const lbm_body &b, const Win &w) {
  if (b.shape == LBM_SHAPE_SPHERE && !w.on) return len3({p.x - b.cx, p.y - b.cy, p.z - b.cz}) - b.a;
  return phi3_call(p.x, p.y, p.z, &b, &w);
}

// exp map of an angular velocity over dt, common_d3_geometry.wgsl:86-91.
__device__ __forceinline__ Q4 exp_map(V3 w, float dt) {
  float m = len3(w);
  if (m <= 1e-12f) return {1.f, 0.f, 0.f, 0.f};
  float half = 0.5f * m * dt;
  float s = sinf(half);
  return {cosf(half), s * w.x / m, s * w.y / m, s * w.z / m};
}

// The same body one step ahead at its current velocities,
// common_d3_geometry.wgsl:199-203.
__device__ __forceinline__ float phi3_ahead(V3 p, const lbm_body &b, float dt, const Win &w) {
  V3 c = {b.cx + b.vx * dt, b.cy + b.vy * dt, b.cz + b.vz * dt};
  Q4 q = q_mul(exp_map({b.wx, b.wy, b.wz}, dt), {b.qw, b.qx, b.qy, b.qz});
  V3 d = {p.x - c.x, p.y - c.y, p.z - c.z};
  if (w.on) {
    d.x = win_wrap1(d.x, w.n[0]);
    d.y = win_wrap1(d.y, w.n[1]);
    d.z = win_wrap1(d.z, w.n[2]);
  }
  return sdf_local3(q_rot_inv(q, d), b);
}

__device__ __forceinline__ V3 body_velocity3(V3 p, const lbm_body &b, const Win &w) {
  const V3 r = body_delta(p, b, w);
  // v + w x r
  return {b.vx + (b.wy * r.z - b.wz * r.y), b.vy + (b.wz * r.x - b.wx * r.z),
          b.vz + (b.wx * r.y - b.wy * r.x)};
}

__device__ __forceinline__ float chi_from_phi(float phi, float eps) {
  return 0.5f * (1.0f - tanhf(fminf(fmaxf(phi / eps, -20.0f), 20.0f)));
}

// ---- 2D card geometry ----------------------------------------------------

// WGSL round() ties to even; rintf does the same in the default mode.
__device__ __forceinline__ float wrap_delta(float d, float n) { return d - n * rintf(d / n); }

__device__ __forceinline__ float phi2_inline(float px, float py, const lbm_body &b, float W, float H) {
  float ca = cosf(b.theta), sa = sinf(b.theta);
  float dx = px - b.cx, dy = py - b.cy;
  dx = wrap_delta(dx, W);
  dy = wrap_delta(dy, H);
  float lx = dx * ca + dy * sa;
  float ly = -dx * sa + dy * ca;
  float a = b.a, bb = b.b;
  if (fabsf(a - bb) <= 1e-6f * fmaxf(a, bb))
    return __fsqrt_rn(__fadd_rn(__fmul_rn(lx, lx), __fmul_rn(ly, ly))) - a;
  float x = fabsf(lx), y = fabsf(ly);
  float r = sqrtf((x * x) / (a * a) + (y * y) / (bb * bb));
  float algebraic = (r - 1.0f) * bb;
  if (algebraic > 64.0f) return algebraic;
  bool inside = r < 1.0f;
  float t = atan2f(y * a, x * bb);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float ct = cosf(t), st = sinf(t);
    float ex = x - a * ct, ey = y - bb * st;
    float F = ex * (-a * st) + ey * (bb * ct);
    float Fp = -(a * a * st * st + bb * bb * ct * ct) + ex * (-a * ct) + ey * (-bb * st);
    t = t - F / (fabsf(Fp) < 1e-9f ? -1e-9f : Fp);
    t = fminf(fmaxf(t, 0.0f), 1.5707963f);
  }
  float ddx = x - a * cosf(t), ddy = y - bb * sinf(t);
  float d = sqrtf(ddx * ddx + ddy * ddy);
  return inside ? -d : d;
}

static __device__ __noinline__ float phi2_call(float px, float py, const lbm_body *b, float W, float H) {
  return phi2_inline(px, py, *b, W, H);
}

// An unrotated circle (every pinned cylinder) takes the closed form inline:
// cos(0) = 1 and sin(0) = 0 make the rotation exact, so this is the same
// value the general path returns.
__device__ __forceinline__ float phi2(float px, float py, const lbm_body &b, float W, float H) {
  if (b.theta == 0.0f && fabsf(b.a - b.b) <= 1e-6f * fmaxf(b.a, b.b)) {
    const float lx = wrap_delta(px - b.cx, W), ly = wrap_delta(py - b.cy, H);
    return __fsqrt_rn(__fadd_rn(__fmul_rn(lx, lx), __fmul_rn(ly, ly))) - b.a;
  }
  return phi2_call(px, py, &b, W, H);
}

}  // namespace lbm
