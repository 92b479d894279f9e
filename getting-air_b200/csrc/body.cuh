// The rigid body outside the lattice: which cells can feel it, and (for a
// free body) its 6-DOF integrator. Host and device share every function
// here, so the library's host twin of the integrator (lbm_body_advance) is
// the same code the device runs after each force pass.
//
// Integrator: d3-body.mjs stepFreeBody (:244-290), the host reference that
// shaders/d3_physics.wgsl mirrors:
//   v  += F/m + g            (dt = 1 lattice step; planar holds v_z = 0)
//   |v| clamped to v_max     (a magnitude clamp: the direction is kept)
//   L  += T                  (planar keeps only L_z)
//   x  += v, wrapped on the windowed axes; d += v (unwrapped)
//   w  = R I^-1 R^T L,  |w| clamped to o_max with L scaled alike
//   q_half = exp(w/2) q,  w_half = R_half I^-1 R_half^T L,  q = exp(w_half) q
// Angular momentum is the integrated state, so |L| is conserved exactly
// under zero torque, and the midpoint rotation keeps a major-axis spin
// stable. The reference integrates in f64 on the host and in f32 on the
// GPU; this integrator is FP64 on both.
//
// Volume and principal inertia: d3-body.mjs bodyVolume / principalInertia
// (:114-160); the rounded box uses the unrounded box, as the reference does.
#pragma once

#include <math.h>

#include "../../include/lbm.h"

#ifdef __CUDACC__
#define LBM_HD __host__ __device__ __forceinline__
#else
#define LBM_HD inline
#endif

namespace lbm {

// The moving window (common_d3_window.wgsl, d3-window.mjs): n is the domain
// size on a windowed axis and 0 elsewhere (WIN_N*), anchor the cell the body
// sits in within the window (WIN_A*). The fluid never moves: the body wraps
// through the periodic buffer and the sponge band follows it.
struct Win {
  float n[3];
  float anchor[3];
  int on;
};

// ---- reach of the body ---------------------------------------------------

// Radius of the smallest sphere about the centre containing the body
// (d3-body.mjs bodyCircumradius :136; the 2D ellipse takes its major axis).
LBM_HD float body_circumradius(const lbm_body &b) {
  switch (b.shape) {
    case LBM_SHAPE_SPHERE: return b.a;
    case LBM_SHAPE_SPHEROID: return fmaxf(b.a, b.c);
    case LBM_SHAPE_ELLIPSE: return fmaxf(b.a, b.b);
    default: return sqrtf(b.a * b.a + b.b * b.b + b.c * b.c);
  }
}

// Inclusive cell box [x0,x1]x[y0,y1]x[z0,z1] outside which no cell can add
// to the body force: a bounce-back link is at most sqrt(3) long, the
// swept-cell term reaches one step of surface motion, and the penalty's chi
// is below 1e-6 beyond ~6.9 band widths. `swept`/`band` are the swept-cell
// switch and the |phi| band it applies in. Returns false when no cell of
// the domain is within reach. On a windowed axis (win[a] set) the box is
// not clipped: it may start below 0 or end past the last cell, to be read
// modulo the axis, and it covers the whole axis once it is that long.
LBM_HD bool body_cell_box(const lbm_body &b, int q, int nx, int ny, int nz, int bounceback, int swept_force,
                          float chi_eps, int box[6], int *swept, float *band, const int *win = nullptr) {
  const float rc = body_circumradius(b);
  const float speed = sqrtf(b.vx * b.vx + b.vy * b.vy + b.vz * b.vz) +
                      sqrtf(b.wx * b.wx + b.wy * b.wy + b.wz * b.wz) * rc;
  *swept = (q != 9 && bounceback && swept_force && speed > 0.f) ? 1 : 0;
  *band = 2.0f + speed;
  const float margin = bounceback ? (3.0f + speed) : (8.0f * chi_eps + 2.0f);
  const float reach = rc + margin;
  const bool wrap2d = (q == 9);  // the 2D SDF takes the nearest periodic image
  const float centre[3] = {b.cx, b.cy, b.cz};
  const int len[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    if (a == 2 && q == 9) { box[4] = box[5] = 0; break; }
    int lo = (int)floorf(centre[a] - reach), hi = (int)ceilf(centre[a] + reach);
    if (win && win[a]) {
      if (hi - lo + 1 >= len[a]) { lo = 0; hi = len[a] - 1; }
      box[2 * a] = lo;
      box[2 * a + 1] = hi;
      continue;
    }
    if (wrap2d && (lo < 0 || hi > len[a] - 1)) { lo = 0; hi = len[a] - 1; }
    box[2 * a] = lo < 0 ? 0 : lo;
    box[2 * a + 1] = hi > len[a] - 1 ? len[a] - 1 : hi;
  }
  return box[0] <= box[1] && box[2] <= box[3] && box[4] <= box[5];
}

// ---- FP64 quaternion algebra ([w, x, y, z], body -> world) --------------

struct DQuat {
  double w, x, y, z;
};

LBM_HD DQuat dq_mul(const DQuat &p, const DQuat &q) {
  return {p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z, p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y,
          p.w * q.y - p.x * q.z + p.y * q.w + p.z * q.x, p.w * q.z + p.x * q.y - p.y * q.x + p.z * q.w};
}

LBM_HD DQuat dq_conj(const DQuat &q) { return {q.w, -q.x, -q.y, -q.z}; }

LBM_HD double dnorm3(const double v[3]) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

// Unit quaternion; a degenerate one becomes the identity rather than NaN.
LBM_HD DQuat dq_normalize(const DQuat &q) {
  const double n = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  if (!(n > 1e-12)) return {1.0, 0.0, 0.0, 0.0};
  return {q.w / n, q.x / n, q.y / n, q.z / n};
}

// v_world = q v q*  /  v_body = q* v q.
LBM_HD void dq_rotate(const DQuat &q, const double v[3], double out[3]) {
  const DQuat r = dq_mul(dq_mul(q, {0.0, v[0], v[1], v[2]}), dq_conj(q));
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
LBM_HD void dq_rotate_inv(const DQuat &q, const double v[3], double out[3]) {
  const DQuat r = dq_mul(dq_mul(dq_conj(q), {0.0, v[0], v[1], v[2]}), q);
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

// Rotation by |w| dt about w (identity for a vanishing rate).
LBM_HD DQuat dq_expmap(const double w[3], double dt) {
  const double m = dnorm3(w);
  if (!(m > 1e-12)) return {1.0, 0.0, 0.0, 0.0};
  const double half = 0.5 * (m * dt);
  const double s = sin(half) / m;
  return {cos(half), w[0] * s, w[1] * s, w[2] * s};
}

// omega = R I_body^-1 R^T L (rotate into the body frame, divide, rotate back).
LBM_HD void omega_from_L(const DQuat &q, const double ibody[3], const double L[3], double w[3]) {
  double lb[3];
  dq_rotate_inv(q, L, lb);
  lb[0] /= ibody[0]; lb[1] /= ibody[1]; lb[2] /= ibody[2];
  dq_rotate(q, lb, w);
}

// ---- the body ---------------------------------------------------------------

LBM_HD double body_volume(const lbm_body &b) {
  const double pi = 3.14159265358979323846;
  switch (b.shape) {
    case LBM_SHAPE_SPHERE: return (4.0 / 3.0) * pi * (double)b.a * b.a * b.a;
    case LBM_SHAPE_SPHEROID: return (4.0 / 3.0) * pi * (double)b.a * b.a * b.c;
    default: return 8.0 * (double)b.a * b.b * b.c;
  }
}

LBM_HD void body_inertia(const lbm_body &b, double m, double I[3]) {
  const double a = b.a, bb = b.b, c = b.c;
  switch (b.shape) {
    case LBM_SHAPE_SPHERE: I[0] = I[1] = I[2] = 0.4 * m * a * a; break;
    case LBM_SHAPE_SPHEROID:
      I[0] = I[1] = m * (a * a + c * c) / 5.0;
      I[2] = 2.0 * m * a * a / 5.0;
      break;
    default:
      I[0] = m * (bb * bb + c * c) / 3.0;
      I[1] = m * (a * a + c * c) / 3.0;
      I[2] = m * (a * a + bb * bb) / 3.0;
  }
}

LBM_HD DQuat state_quat(const lbm_body_state &s) { return {s.q[0], s.q[1], s.q[2], s.q[3]}; }

// makeBodyState: mass from density x volume, L = R I_body R^T omega.
LBM_HD void body_state_make(const lbm_body &b, double density, lbm_body_state &s) {
  s.x[0] = b.cx; s.x[1] = b.cy; s.x[2] = b.cz;
  s.q[0] = b.qw; s.q[1] = b.qx; s.q[2] = b.qy; s.q[3] = b.qz;
  s.v[0] = b.vx; s.v[1] = b.vy; s.v[2] = b.vz;
  s.omega[0] = b.wx; s.omega[1] = b.wy; s.omega[2] = b.wz;
  s.mass = density * body_volume(b);
  body_inertia(b, s.mass, s.ibody);
  double wb[3];
  const DQuat q = state_quat(s);
  dq_rotate_inv(q, s.omega, wb);
  wb[0] *= s.ibody[0]; wb[1] *= s.ibody[1]; wb[2] *= s.ibody[2];
  dq_rotate(q, wb, s.L);
  for (int k = 0; k < 3; ++k) { s.d[k] = 0.0; s.force[k] = 0.0; s.torque[k] = 0.0; }
  s.steps = 0;
}

LBM_HD double wrap_position(double c, double n) { return n > 0.0 ? c - n * floor(c / n) : c; }

// One step (dt = 1) of stepFreeBody under `force`/`torque`. The load is
// recorded first; a pinned body stops there, and `no_fluid_force` zeroes
// the fluid load before it is applied.
LBM_HD void body_step(lbm_body_state &s, const double force[3], const double torque[3], const lbm_body_opts &o) {
  for (int k = 0; k < 3; ++k) { s.force[k] = force[k]; s.torque[k] = torque[k]; }
  s.steps += 1;
  if (o.pinned) return;
  const double use = o.no_fluid_force ? 0.0 : 1.0;
  const double m = s.mass;
  double v[3] = {s.v[0] + (use * force[0] / m + o.gravity[0]), s.v[1] + (use * force[1] / m + o.gravity[1]),
                 o.planar ? 0.0 : s.v[2] + (use * force[2] / m + o.gravity[2])};
  const double vmag = dnorm3(v);
  if (o.v_max > 0.0 && vmag > o.v_max) {
    const double k = o.v_max / vmag;
    v[0] *= k; v[1] *= k; v[2] *= k;
  }
  double L[3];
  if (o.planar) {
    L[0] = 0.0; L[1] = 0.0; L[2] = s.L[2] + use * torque[2];
  } else {
    for (int k = 0; k < 3; ++k) L[k] = s.L[k] + use * torque[k];
  }
  for (int k = 0; k < 3; ++k) {
    s.x[k] = wrap_position(s.x[k] + v[k], o.wrap[k]);
    s.d[k] += v[k];
  }
  const DQuat q0 = state_quat(s);
  double w[3];
  omega_from_L(q0, s.ibody, L, w);
  if (o.planar) { w[0] = 0.0; w[1] = 0.0; }
  const double wmag = dnorm3(w);
  if (o.o_max > 0.0 && wmag > o.o_max) {
    const double k = o.o_max / wmag;
    for (int j = 0; j < 3; ++j) { w[j] *= k; L[j] *= k; }
  }
  const DQuat qh = dq_normalize(dq_mul(dq_expmap(w, 0.5), q0));
  double wh[3];
  omega_from_L(qh, s.ibody, L, wh);
  if (o.planar) { wh[0] = 0.0; wh[1] = 0.0; }
  const DQuat qn = dq_normalize(dq_mul(dq_expmap(wh, 1.0), q0));
  for (int k = 0; k < 3; ++k) { s.v[k] = v[k]; s.L[k] = L[k]; s.omega[k] = wh[k]; }
  s.q[0] = qn.w; s.q[1] = qn.x; s.q[2] = qn.y; s.q[3] = qn.z;
}

// The f32 pose the lattice kernels read, from the FP64 state (shape and
// size kept from `shape`).
LBM_HD lbm_body body_pose(const lbm_body &shape, const lbm_body_state &s) {
  lbm_body b = shape;
  b.cx = (float)s.x[0]; b.cy = (float)s.x[1]; b.cz = (float)s.x[2];
  b.qw = (float)s.q[0]; b.qx = (float)s.q[1]; b.qy = (float)s.q[2]; b.qz = (float)s.q[3];
  b.vx = (float)s.v[0]; b.vy = (float)s.v[1]; b.vz = (float)s.v[2];
  b.wx = (float)s.omega[0]; b.wy = (float)s.omega[1]; b.wz = (float)s.omega[2];
  return b;
}

// ---- free-body coupling on the device --------------------------------------
// Per step: a force pass over the cells near the body (pose P_t, f_t) whose
// last block integrates the body (P_t -> P_t+1), then the lattice step with
// P_t+1 -- the reference's order (main-3d.js encodeSteps: force, physics,
// step). The pose is double-buffered by step parity so that no block of a
// force pass can see the pose its own last block writes.

struct BodyPose {
  lbm_body body;
  int region[6];     // launch blocks that can feel the body: per axis the
                     // first (in the grid) and first + count, read modulo it
  int swept;
  float swept_band;
};

struct BodyDyn {
  lbm_body_state st;
  lbm_body_opts opt;
  lbm_body shape;
  int q, nx, ny, nz, bounceback, swept_force;
  int win[3];        // moving-window axes (the box is not clipped on them)
  float chi_eps;
  int cap[3];        // force-pass grid: the largest box, in launch blocks
  int overflow;      // steps whose box exceeded cap (clipped)
};

}  // namespace lbm
