// ORACLE -- test infrastructure only. CPU restatement of the reference's
// dense lattice-Boltzmann arithmetic, used by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
// It is never linked into or called by the product library.
//
// Two precisions from one template:
//   R = double  the FP64 oracle the GPU path is scored against (the
//               reference's "JS FP64" semantics: f32 table constants, f64
//               arithmetic);
//   R = float   the reference's own f32 operation order, built with
//               -ffp-contract=off so every operation rounds once, for
//               tight short-horizon comparisons.
//
// Followed line by line (reference paths):
//   lattice-2d.mjs:106-162        D2Q9 set, weights, OPP (derived here)
//   lattice-3d.mjs:50-210         D3Q19/27 derived ordering, ulp-tweaked weights
//   lbm_step.wgsl:137-270         2D fused step
//   lbm_force.wgsl                2D force (separate pass on f_in, as the reference)
//   common_geometry.wgsl:84-160   2D ellipse SDF
//   common_d3_step.wgsl:206-400   3D initEq + fused step
//   common_d3_force.wgsl:171-283  3D force (momentum exchange / swept / penalty)
//   common_d3_geometry.wgsl       3D SDFs, quaternions, body velocity
//   common_d3_sponge.wgsl, common_sponge.wgsl, common_walls.wgsl
//   amr2d-gpu.mjs:698-736         conserved totals
// Forces are summed in double in a fixed order (one partial per grid row,
// rows summed in index order), independent of the thread count.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/lbm.h"

#include "body.h"
#include "common.h"
#include "dense3.h"

namespace {
using namespace oracle;

// ---- 2D --------------------------------------------------------------------

template <class R>
void force2(const lbm_config &c, const std::vector<R> &fin, double out[8]) {
  const Tables &T = tables(9);
  const int W = c.nx, H = c.ny;
  const int64_t N = (int64_t)W * H;
  const lbm_body &b = c.body;
  const R CS2 = R(1) / R(3), fW = R(W), fH = R(H);
  std::vector<double> rows((size_t)H * 4, 0.0);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y) {
    double acc[4] = {0, 0, 0, 0};
    for (int x = 0; x < W; ++x) {
      const int64_t cell = (int64_t)y * W + x;
      R px = R(x), py = R(y);
      R phi = phi2(px, py, b, fW, fH);
      R chi = chi_of(phi, R(c.chi_eps));
      R rx = wrapd(px - R(b.cx), fW), ry = wrapd(py - R(b.cy), fH);
      R usx = R(b.vx) - R(b.wz) * ry, usy = R(b.vy) + R(b.wz) * rx;
      R fx = 0, fy = 0, tz = 0;
      if (c.use_bounceback) {
        if (phi >= R(0)) {
          for (int i = 0; i < 9; ++i) {
            int nx_ = (x - T.ex[i] + W) % W, ny_ = (y - T.ey[i] + H) % H;
            if (phi2(R(nx_), R(ny_), b, fW, fH) < R(0)) {
              R fo = fin[T.opp[i] * N + cell];
              R corr = R(2) * R(T.w[i]) * (R(T.ex[i]) * usx + R(T.ey[i]) * usy) / CS2;
              fx += -R(T.ex[i]) * (R(2) * fo + corr);
              fy += -R(T.ey[i]) * (R(2) * fo + corr);
            }
          }
          tz = rx * fy - ry * fx;
        }
      } else if (chi >= R(1e-6)) {
        R rho = 0, uxs = 0, uys = 0;
        for (int i = 0; i < 9; ++i) {
          int sx = (x - T.ex[i] + W) % W, sy = (y - T.ey[i] + H) % H;
          R v = fin[i * N + (int64_t)sy * W + sx];
          rho += v; uxs += v * R(T.ex[i]); uys += v * R(T.ey[i]);
        }
        uxs /= std::fmax(rho, R(1e-6)); uys /= std::fmax(rho, R(1e-6));
        R Fx = rho * chi * (usx - uxs), Fy = rho * chi * (usy - uys);
        fx = -Fx; fy = -Fy;
        tz = rx * fy - ry * fx;
      }
      R v3[3] = {fx, fy, tz};
      for (int k = 0; k < 3; ++k) {
        if (std::isfinite((double)v3[k])) acc[k] += (double)v3[k];
        else acc[3] += 1.0;
      }
    }
    for (int k = 0; k < 4; ++k) rows[(size_t)y * 4 + k] = acc[k];
  }
  for (int k = 0; k < 8; ++k) out[k] = 0.0;
  for (int y = 0; y < H; ++y) {
    out[0] += rows[y * 4 + 0];
    out[1] += rows[y * 4 + 1];
    out[5] += rows[y * 4 + 2];
    out[6] += rows[y * 4 + 3];
  }
}

template <class R>
void run(const lbm_config &c, double *f, int nsteps, double *mac, double *forces) {
  const int64_t N = (int64_t)c.nx * c.ny * c.nz;
  const int64_t tot = N * c.q;
  std::vector<R> a(tot), b(tot);
  for (int64_t i = 0; i < tot; ++i) a[i] = R(f[i]);
  for (int s = 0; s < nsteps; ++s) {
    double fo[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (c.has_body) {
      if (c.q == 9) force2<R>(c, a, fo); else force3<R>(c, a, fo);
    }
    if (forces) std::memcpy(forces + 8 * s, fo, sizeof(fo));
    double *m = (s == nsteps - 1) ? mac : nullptr;
    if (c.q == 9) step2<R>(c, a, b, m); else step3<R>(c, a, b, m);
    a.swap(b);
  }
  for (int64_t i = 0; i < tot; ++i) f[i] = (double)a[i];
}

// The free-body loop in the reference's order (main-3d.js encodeSteps):
// force pass on f_t at pose P_t, the 6-DOF update to P_t+1, then the step
// on f_t with P_t+1.
template <class R>
void run_free(const lbm_config &c0, double *f, int nsteps, RigidBody &body, const lbm_body_opts &o, double *mac,
              double *forces, double *traj) {
  lbm_config c = c0;
  const int64_t N = (int64_t)c.nx * c.ny * c.nz;
  const int64_t tot = N * c.q;
  std::vector<R> a(tot), b(tot);
  for (int64_t i = 0; i < tot; ++i) a[i] = R(f[i]);
  for (int s = 0; s < nsteps; ++s) {
    c.body = pose_of(c0.body, body);
    double fo[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    force3<R>(c, a, fo);
    if (forces) std::memcpy(forces + 8 * s, fo, sizeof(fo));
    step_free_body(body, {fo[0], fo[1], fo[2]}, {fo[3], fo[4], fo[5]}, o);
    if (traj) {
      double *t = traj + 16 * s;
      for (int k = 0; k < 3; ++k) { t[k] = body.x[k]; t[3 + k] = body.v[k]; t[6 + k] = body.L[k]; t[9 + k] = body.omega[k]; }
      for (int k = 0; k < 4; ++k) t[12 + k] = body.q[k];
    }
    c.body = pose_of(c0.body, body);
    double *m = (s == nsteps - 1) ? mac : nullptr;
    step3<R>(c, a, b, m);
    a.swap(b);
  }
  for (int64_t i = 0; i < tot; ++i) f[i] = (double)a[i];
}

}  // namespace

extern "C" {

// makeBodyState for a 3D pose.
int oracle_body_make(const lbm_body *pose, double density, lbm_body_state *out) {
  if (!pose || !out) return -1;
  *out = lbm_body_state{};
  to_state(make_body_state(*pose, density), *out);
  return 0;
}

// `nsteps` of stepFreeBody under a constant load.
int oracle_body_step(lbm_body_state *s, const double force[3], const double torque[3], const lbm_body_opts *o,
                     int nsteps) {
  if (!s || !o) return -1;
  RigidBody r = from_state(*s);
  for (int k = 0; k < nsteps; ++k) step_free_body(r, {force[0], force[1], force[2]}, {torque[0], torque[1], torque[2]}, *o);
  to_state(r, *s);
  return 0;
}

// The coupled free-body run (3D): f in place, the body state in place,
// mac of the last step, per-step forces (8 each) and trajectory (16 each:
// x, v, L, omega, q after the update), any of the three NULL.
int oracle_run_free(const lbm_config *c, int fp32, double *f, int nsteps, lbm_body_state *state,
                    const lbm_body_opts *o, double *mac, double *forces, double *traj) {
  if (!c || !f || !state || !o || c->q == 9 || nsteps < 0) return -1;
  RigidBody r = from_state(*state);
  lbm_body_opts oo = *o;
  const int len[3] = {c->nx, c->ny, c->nz};
  for (int k = 0; k < 3; ++k)
    if (c->window[k]) oo.wrap[k] = len[k];  // a windowed axis wraps the body (winWrapPos)
  if (fp32) run_free<float>(*c, f, nsteps, r, oo, mac, forces, traj);
  else run_free<double>(*c, f, nsteps, r, oo, mac, forces, traj);
  to_state(r, *state);
  return 0;
}

// The moving window's scalar maps (d3-window.mjs wrapDelta, windowOffset,
// windowCoord, wrapPosition), FP64; n = 0 is an unwindowed axis.
double oracle_win_wrap_delta(double d, double n) { return win_wrap1<double>(d, n); }
double oracle_win_offset(double c, double anchor, double n) { return win_offset1<double>(c, anchor, n); }
double oracle_win_coord(double p, double off, double n) { return win_coord1<double>(p, off, n); }
double oracle_win_wrap_position(double c, double n) { return wrap_pos(c, n); }

// Derived lattice tables (weights as exact f32 values).
int oracle_tables(int q, int32_t *ex, int32_t *ey, int32_t *ez, float *w, int32_t *opp) {
  if (q != 9 && q != 19 && q != 27) return -1;
  const Tables &t = tables(q);
  for (int i = 0; i < q; ++i) {
    ex[i] = t.ex[i]; ey[i] = t.ey[i]; ez[i] = t.ez[i]; w[i] = t.w[i]; opp[i] = t.opp[i];
  }
  return 0;
}

// Equilibrium seeding (initEq): f_i = feq(rho, u) per cell, in R precision.
int oracle_init_eq(int q, int64_t n, int fp32, const double *mac, double *f) {
  const Tables &t = tables(q);
  for (int64_t c = 0; c < n; ++c) {
    const double *m = mac + 4 * c;
    for (int i = 0; i < q; ++i) {
      if (fp32) {
        float rho = (float)m[0], ux = (float)m[1], uy = (float)m[2], uz = q == 9 ? 0.f : (float)m[3];
        float eu = (float)t.ex[i] * ux + (float)t.ey[i] * uy + (float)t.ez[i] * uz;
        float usq = q == 9 ? ux * ux + uy * uy : ux * ux + uy * uy + uz * uz;
        f[i * n + c] = t.w[i] * rho * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * usq);
      } else {
        double rho = m[0], ux = m[1], uy = m[2], uz = q == 9 ? 0.0 : m[3];
        double eu = t.ex[i] * ux + t.ey[i] * uy + t.ez[i] * uz;
        double usq = ux * ux + uy * uy + uz * uz;
        f[i * n + c] = (double)t.w[i] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq);
      }
    }
  }
  return 0;
}

// Runs `nsteps` of force pass + fused step in place on f (Q*n doubles).
// mac (4*n) receives the last step's macroscopic field, forces (8*nsteps)
// the per-step force/torque sums; either may be NULL.
int oracle_run(const lbm_config *c, int fp32, double *f, int nsteps, double *mac, double *forces) {
  if (!c || !f || nsteps < 0) return -1;
  if (fp32) run<float>(*c, f, nsteps, mac, forces);
  else run<double>(*c, f, nsteps, mac, forces);
  return 0;
}

// Conserved totals in f64, readConservedTotals semantics (amr2d-gpu.mjs:698).
int oracle_totals(int q, int64_t n, const double *f, double out[8]) {
  const Tables &t = tables(q);
  double mass = 0, px = 0, py = 0, pz = 0, rmin = 1e300, rmax = -1e300, u2 = 0, bad = 0;
  for (int64_t c = 0; c < n; ++c) {
    double rho = 0, mx = 0, my = 0, mz = 0;
    for (int i = 0; i < q; ++i) {
      double v = f[i * n + c];
      rho += v; mx += v * t.ex[i]; my += v * t.ey[i]; mz += v * t.ez[i];
    }
    if (!std::isfinite(rho + mx + my + mz)) { bad += 1; continue; }
    mass += rho - 1.0; px += mx; py += my; pz += mz;
    rmin = std::fmin(rmin, rho); rmax = std::fmax(rmax, rho);
    u2 = std::fmax(u2, (mx * mx + my * my + mz * mz) / (rho * rho));
  }
  out[0] = mass; out[1] = px; out[2] = py; out[3] = pz;
  out[4] = rmin; out[5] = rmax; out[6] = std::sqrt(u2); out[7] = bad;
  return 0;
}

// binary16 encode by exact arithmetic on the value (not bit surgery): scale
// into the 11-bit significand grid, round half to even with nearbyint.
uint16_t oracle_f16_bits(float v) {
  if (std::isnan(v)) return 0x7e00;
  const uint16_t sign = std::signbit(v) ? 0x8000 : 0;
  double a = std::fabs((double)v);
  if (a == 0.0) return sign;
  if (std::isinf(a)) return sign | 0x7c00;
  int e;
  std::frexp(a, &e);           // a = m * 2^e, m in [0.5, 1)
  int E = e - 1;               // a in [2^E, 2^(E+1))
  if (E < -14) E = -14;        // subnormal grid
  const double q = std::ldexp(1.0, E - 10);
  double k = std::nearbyint(a / q);  // ties to even under the default mode
  if (k >= 2048.0) { k /= 2; E += 1; }
  if (E > 15) return sign | 0x7c00;
  if (k < 1024.0) return (uint16_t)(sign | (uint16_t)k);  // subnormal (E == -14)
  return (uint16_t)(sign | (uint16_t)((E + 15) << 10) | (uint16_t)((int)k - 1024));
}

}  // extern "C"
