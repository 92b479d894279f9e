// ORACLE -- test infrastructure only. FP64 restatement of the reference's
// 6-DOF rigid body, d3-body.mjs (the host reference that
// shaders/d3_physics.wgsl mirrors):
//   qMul / qConj / qNormalize / qFromAxisAngle   d3-body.mjs:172-199
//   qRotate / qRotateInv (two quaternion products) :202-210
//   expMap / omegaFromL                            :219-229
//   stepFreeBody                                   :244-290
//   makeBodyState                                  :292-300
//   bodyVolume / principalInertia                  :114-160
//   wrapPosition                                   d3-window.mjs:148-151
// plus the WGSL kernel's additions (pinned record-only, NO_FLUID_FORCE).
// Vectors are std::array, written step by step as the JS does.
#pragma once

#include <array>
#include <cmath>

#include "../include/lbm.h"

namespace oracle {

using Vec3 = std::array<double, 3>;
using Quat = std::array<double, 4>;  // w, x, y, z

inline Quat q_mul(const Quat &p, const Quat &q) {
  return {p[0] * q[0] - p[1] * q[1] - p[2] * q[2] - p[3] * q[3],
          p[0] * q[1] + p[1] * q[0] + p[2] * q[3] - p[3] * q[2],
          p[0] * q[2] - p[1] * q[3] + p[2] * q[0] + p[3] * q[1],
          p[0] * q[3] + p[1] * q[2] - p[2] * q[1] + p[3] * q[0]};
}
inline Quat q_conj(const Quat &q) { return {q[0], -q[1], -q[2], -q[3]}; }
inline double hyp3(double a, double b, double c) { return std::sqrt(a * a + b * b + c * c); }
inline Quat q_normalize(const Quat &q) {
  const double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(n > 1e-12)) return {1, 0, 0, 0};
  return {q[0] / n, q[1] / n, q[2] / n, q[3] / n};
}
inline Quat q_axis_angle(const Vec3 &axis, double angle) {
  double n = hyp3(axis[0], axis[1], axis[2]);
  if (n == 0) n = 1;
  const double s = std::sin(angle / 2) / n;
  return {std::cos(angle / 2), axis[0] * s, axis[1] * s, axis[2] * s};
}
inline Vec3 q_rotate(const Quat &q, const Vec3 &v) {
  const Quat r = q_mul(q_mul(q, {0, v[0], v[1], v[2]}), q_conj(q));
  return {r[1], r[2], r[3]};
}
inline Vec3 q_rotate_inv(const Quat &q, const Vec3 &v) {
  const Quat r = q_mul(q_mul(q_conj(q), {0, v[0], v[1], v[2]}), q);
  return {r[1], r[2], r[3]};
}
inline Quat exp_map(const Vec3 &w, double dt) {
  const double m = hyp3(w[0], w[1], w[2]);
  return m > 1e-12 ? q_axis_angle(w, m * dt) : Quat{1, 0, 0, 0};
}
inline Vec3 omega_from_L(const Quat &q, const Vec3 &ib, const Vec3 &L) {
  const Vec3 lb = q_rotate_inv(q, L);
  return q_rotate(q, {lb[0] / ib[0], lb[1] / ib[1], lb[2] / ib[2]});
}

inline double volume(const lbm_body &b) {
  const double pi = 3.14159265358979323846;
  if (b.shape == LBM_SHAPE_SPHERE) return 4.0 / 3.0 * pi * std::pow((double)b.a, 3);
  if (b.shape == LBM_SHAPE_SPHEROID) return 4.0 / 3.0 * pi * (double)b.a * b.a * b.c;
  return 8.0 * (double)b.a * b.b * b.c;
}
inline Vec3 inertia(const lbm_body &b, double m) {
  const double a = b.a, bb = b.b, c = b.c;
  if (b.shape == LBM_SHAPE_SPHERE) { const double i = 0.4 * m * a * a; return {i, i, i}; }
  if (b.shape == LBM_SHAPE_SPHEROID) { const double ix = m * (a * a + c * c) / 5; return {ix, ix, 2 * m * a * a / 5}; }
  return {m * (bb * bb + c * c) / 3, m * (a * a + c * c) / 3, m * (a * a + bb * bb) / 3};
}

struct RigidBody {
  Vec3 x, v, L, omega, d, force, torque, ib;
  Quat q;
  double mass;
  long steps;
};

inline RigidBody make_body_state(const lbm_body &b, double density) {
  RigidBody s{};
  s.x = {b.cx, b.cy, b.cz};
  s.q = {b.qw, b.qx, b.qy, b.qz};
  s.v = {b.vx, b.vy, b.vz};
  s.omega = {b.wx, b.wy, b.wz};
  s.mass = density * volume(b);
  s.ib = inertia(b, s.mass);
  const Vec3 lb = q_rotate_inv(s.q, s.omega);
  s.L = q_rotate(s.q, {lb[0] * s.ib[0], lb[1] * s.ib[1], lb[2] * s.ib[2]});
  return s;
}

inline double wrap_pos(double c, double n) { return n > 0 ? c - n * std::floor(c / n) : c; }

inline void step_free_body(RigidBody &s, const Vec3 &F, const Vec3 &T, const lbm_body_opts &o) {
  s.force = F;
  s.torque = T;
  s.steps += 1;
  if (o.pinned) return;
  const Vec3 force = o.no_fluid_force ? Vec3{0, 0, 0} : F;
  const Vec3 torque = o.no_fluid_force ? Vec3{0, 0, 0} : T;
  const double m = s.mass;
  Vec3 v = {s.v[0] + (force[0] / m + o.gravity[0]), s.v[1] + (force[1] / m + o.gravity[1]),
            o.planar ? 0.0 : s.v[2] + (force[2] / m + o.gravity[2])};
  const double vmag = hyp3(v[0], v[1], v[2]);
  const double vmax = o.v_max > 0 ? o.v_max : INFINITY, omax = o.o_max > 0 ? o.o_max : INFINITY;
  if (vmag > vmax) for (double &c : v) c *= vmax / vmag;
  Vec3 L = o.planar ? Vec3{0, 0, s.L[2] + torque[2]}
                    : Vec3{s.L[0] + torque[0], s.L[1] + torque[1], s.L[2] + torque[2]};
  Vec3 x;
  for (int k = 0; k < 3; ++k) x[k] = wrap_pos(s.x[k] + v[k], o.wrap[k]);
  Vec3 dd = {s.d[0] + v[0], s.d[1] + v[1], s.d[2] + v[2]};
  Vec3 w = omega_from_L(s.q, s.ib, L);
  if (o.planar) w = {0, 0, w[2]};
  const double wmag = hyp3(w[0], w[1], w[2]);
  if (wmag > omax) {
    const double k = omax / wmag;
    for (int j = 0; j < 3; ++j) { w[j] *= k; L[j] *= k; }
  }
  const Quat qh = q_normalize(q_mul(exp_map(w, 0.5), s.q));
  Vec3 wh = omega_from_L(qh, s.ib, L);
  if (o.planar) wh = {0, 0, wh[2]};
  s.q = q_normalize(q_mul(exp_map(wh, 1.0), s.q));
  s.x = x;
  s.v = v;
  s.L = L;
  s.d = dd;
  s.omega = wh;
}

inline void to_state(const RigidBody &r, lbm_body_state &s) {
  for (int k = 0; k < 3; ++k) {
    s.x[k] = r.x[k]; s.v[k] = r.v[k]; s.L[k] = r.L[k]; s.omega[k] = r.omega[k]; s.d[k] = r.d[k];
    s.force[k] = r.force[k]; s.torque[k] = r.torque[k]; s.ibody[k] = r.ib[k];
  }
  for (int k = 0; k < 4; ++k) s.q[k] = r.q[k];
  s.mass = r.mass;
  s.steps = r.steps;
}

inline RigidBody from_state(const lbm_body_state &s) {
  RigidBody r{};
  for (int k = 0; k < 3; ++k) {
    r.x[k] = s.x[k]; r.v[k] = s.v[k]; r.L[k] = s.L[k]; r.omega[k] = s.omega[k]; r.d[k] = s.d[k];
    r.force[k] = s.force[k]; r.torque[k] = s.torque[k]; r.ib[k] = s.ibody[k];
  }
  for (int k = 0; k < 4; ++k) r.q[k] = s.q[k];
  r.mass = s.mass;
  r.steps = (long)s.steps;
  return r;
}

// The f32 pose the lattice reads (BodyState3D is f32 in the reference).
inline lbm_body pose_of(const lbm_body &shape, const RigidBody &r) {
  lbm_body b = shape;
  b.cx = (float)r.x[0]; b.cy = (float)r.x[1]; b.cz = (float)r.x[2];
  b.qw = (float)r.q[0]; b.qx = (float)r.q[1]; b.qy = (float)r.q[2]; b.qz = (float)r.q[3];
  b.vx = (float)r.v[0]; b.vy = (float)r.v[1]; b.vz = (float)r.v[2];
  b.wx = (float)r.omega[0]; b.wy = (float)r.omega[1]; b.wz = (float)r.omega[2];
  return b;
}

}  // namespace oracle
