// ORACLE -- test infrastructure only. Shared pieces of the CPU restatement:
// lattice tables derived the reference's way, geometry in R precision.
// Included by dense_oracle.cpp and amr2d_oracle.cpp.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/lbm.h"

namespace oracle {

struct Tables {
  int q = 0;
  int ex[27], ey[27], ez[27], opp[27];
  float w[27];
};

inline float f32ulp(float x) {
  int e = (int)std::floor(std::log2(std::fabs((double)x)));
  return (float)std::ldexp(1.0, e - 23);
}

// Derives the velocity set and weights the way lattice-3d.mjs /
// lattice-2d.mjs do (enumeration order, fraction -> f32 -> ulp tweak).
inline Tables derive(int q) {
  Tables t;
  t.q = q;
  if (q == 9) {
    const int E[9][2] = {{0, 0}, {1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
    const int num[3] = {4, 1, 1}, den[3] = {9, 9, 36};
    for (int i = 0; i < 9; ++i) {
      t.ex[i] = E[i][0]; t.ey[i] = E[i][1]; t.ez[i] = 0;
      const int sh = E[i][0] * E[i][0] + E[i][1] * E[i][1];
      t.w[i] = (float)((double)num[sh] / den[sh]);  // WEIGHT_ULP_TWEAK = [0,0,0]
    }
    for (int i = 0; i < 9; ++i)
      for (int j = 0; j < 9; ++j)
        if (t.ex[j] == -t.ex[i] && t.ey[j] == -t.ey[i]) t.opp[i] = j;
    return t;
  }
  const int order[3] = {1, -1, 0};
  int all[27][3], k = 0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c) { all[k][0] = order[a]; all[k][1] = order[b]; all[k][2] = order[c]; ++k; }
  const int max_shell = q == 19 ? 2 : 3;
  bool seen[27] = {};
  int n = 0;
  for (int shell = 0; shell <= max_shell; ++shell)
    for (int j = 0; j < 27; ++j) {
      const int *e = all[j];
      if (e[0] * e[0] + e[1] * e[1] + e[2] * e[2] != shell || seen[j]) continue;
      seen[j] = true;
      t.ex[n] = e[0]; t.ey[n] = e[1]; t.ez[n] = e[2]; ++n;
      if (shell) {
        for (int m = 0; m < 27; ++m)
          if (all[m][0] == -e[0] && all[m][1] == -e[1] && all[m][2] == -e[2]) seen[m] = true;
        t.ex[n] = -e[0]; t.ey[n] = -e[1]; t.ez[n] = -e[2]; ++n;
      }
    }
  const int num19[3] = {1, 1, 1}, den19[3] = {3, 18, 36}, tw19[3] = {1, -4, 2};
  const int num27[4] = {8, 2, 1, 1}, den27[4] = {27, 27, 54, 216}, tw27[4] = {-1, 1, -1, 0};
  for (int i = 0; i < q; ++i) {
    const int sh = t.ex[i] * t.ex[i] + t.ey[i] * t.ey[i] + t.ez[i] * t.ez[i];
    const int nu = q == 19 ? num19[sh] : num27[sh], de = q == 19 ? den19[sh] : den27[sh];
    const int tw = q == 19 ? tw19[sh] : tw27[sh];
    const float base = (float)((double)nu / de);
    t.w[i] = (float)((double)base + tw * (double)f32ulp(base));
  }
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < q; ++j)
      if (t.ex[j] == -t.ex[i] && t.ey[j] == -t.ey[i] && t.ez[j] == -t.ez[i]) t.opp[i] = j;
  return t;
}

inline const Tables &tables(int q) {
  static const Tables t9 = derive(9), t19 = derive(19), t27 = derive(27);
  return q == 9 ? t9 : (q == 19 ? t19 : t27);
}

// ---- geometry (R precision) ------------------------------------------------

template <class R> struct V3 { R x, y, z; };
template <class R> struct Q4 { R w, x, y, z; };

template <class R> Q4<R> qmul(Q4<R> p, Q4<R> q) {
  return {p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z,
          p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y,
          p.w * q.y - p.x * q.z + p.y * q.w + p.z * q.x,
          p.w * q.z + p.x * q.y - p.y * q.x + p.z * q.w};
}
template <class R> V3<R> qrotinv(Q4<R> q, V3<R> v) {
  Q4<R> c{q.w, -q.x, -q.y, -q.z};
  Q4<R> r = qmul(qmul(c, Q4<R>{R(0), v.x, v.y, v.z}), q);
  return {r.x, r.y, r.z};
}
template <class R> R len3(V3<R> v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

template <class R> R spheroid(V3<R> p, R a, R c) {
  R r0 = std::sqrt(p.x * p.x + p.y * p.y);
  if (std::fabs(a - c) <= R(1e-6) * std::fmax(a, c)) return std::sqrt(r0 * r0 + p.z * p.z) - a;
  R x = std::fabs(r0), y = std::fabs(p.z);
  R rr = std::sqrt((x * x) / (a * a) + (y * y) / (c * c));
  bool inside = rr < R(1);
  R t = std::atan2(y * a, x * c);
  for (int i = 0; i < 3; ++i) {
    R ct = std::cos(t), st = std::sin(t);
    R ex = x - a * ct, ey = y - c * st;
    R F = ex * (-a * st) + ey * (c * ct);
    R Fp = -(a * a * st * st + c * c * ct * ct) + ex * (-a * ct) + ey * (-c * st);
    t = t - F / (std::fabs(Fp) < R(1e-9) ? R(-1e-9) : Fp);
    t = std::fmin(std::fmax(t, R(0)), R(1.5707963));
  }
  R dx = x - a * std::cos(t), dy = y - c * std::sin(t);
  R d = std::sqrt(dx * dx + dy * dy);
  return inside ? -d : d;
}

template <class R> R sdf_local(V3<R> lp, const lbm_body &b) {
  if (b.shape == LBM_SHAPE_SPHERE) return len3(lp) - R(b.a);
  if (b.shape == LBM_SHAPE_SPHEROID) return spheroid<R>(lp, R(b.a), R(b.c));
  V3<R> q{std::fabs(lp.x) - (R(b.a) - R(b.r)), std::fabs(lp.y) - (R(b.b) - R(b.r)),
          std::fabs(lp.z) - (R(b.c) - R(b.r))};
  V3<R> m{std::fmax(q.x, R(0)), std::fmax(q.y, R(0)), std::fmax(q.z, R(0))};
  return len3(m) + std::fmin(std::fmax(q.x, std::fmax(q.y, q.z)), R(0)) - R(b.r);
}

template <class R> Q4<R> bquat(const lbm_body &b) { return {R(b.qw), R(b.qx), R(b.qy), R(b.qz)}; }

// The moving window (common_d3_window.wgsl, d3-window.mjs:90-150): n is the
// domain size on a windowed axis, 0 elsewhere; anchor the body's cell in the
// window. winWrap1 takes the nearest image (round half to even, as WGSL),
// winOffset the whole cells travelled, winCoord a buffer position in [0, n).
struct Win {
  double n[3] = {0, 0, 0};
  double anchor[3] = {0, 0, 0};
  bool on = false;
};

inline Win window_of(const lbm_config &c) {
  Win w;
  if (c.q == 9) return w;
  const int len[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; ++a)
    if (c.window[a]) {
      w.n[a] = len[a];
      w.anchor[a] = c.win_anchor[a];
      w.on = true;
    }
  return w;
}

template <class R> R win_wrap1(R d, double n) { return n > 0 ? d - R(n) * std::nearbyint(d / R(n)) : d; }
template <class R> R win_offset1(R c, double anchor, double n) { return n > 0 ? std::floor(c) - R(anchor) : R(0); }
template <class R> R win_coord1(R p, R off, double n) {
  if (!(n > 0)) return p;
  const R w = p - off;
  return w - R(n) * std::floor(w / R(n));
}

// bodyDelta3: p relative to the body centre, nearest image on windowed axes.
template <class R> V3<R> bdelta(V3<R> p, const lbm_body &b, const Win *w) {
  V3<R> d{p.x - R(b.cx), p.y - R(b.cy), p.z - R(b.cz)};
  if (w && w->on) {
    d.x = win_wrap1(d.x, w->n[0]);
    d.y = win_wrap1(d.y, w->n[1]);
    d.z = win_wrap1(d.z, w->n[2]);
  }
  return d;
}

// The sponge's view of a position: window coordinates (identity without one).
template <class R> V3<R> win_coord(V3<R> p, const lbm_body &b, const Win *w) {
  if (!w || !w->on) return p;
  return {win_coord1(p.x, win_offset1(R(b.cx), w->anchor[0], w->n[0]), w->n[0]),
          win_coord1(p.y, win_offset1(R(b.cy), w->anchor[1], w->n[1]), w->n[1]),
          win_coord1(p.z, win_offset1(R(b.cz), w->anchor[2], w->n[2]), w->n[2])};
}

template <class R> R phi3(V3<R> p, const lbm_body &b, const Win *w = nullptr) {
  return sdf_local<R>(qrotinv(bquat<R>(b), bdelta(p, b, w)), b);
}

template <class R> R phi3_ahead(V3<R> p, const lbm_body &b, R dt, const Win *win = nullptr) {
  V3<R> w{R(b.wx), R(b.wy), R(b.wz)};
  R m = len3(w);
  Q4<R> e{R(1), R(0), R(0), R(0)};
  if (!(m <= R(1e-12))) {
    R half = R(0.5) * m * dt;
    R s = std::sin(half);
    e = {std::cos(half), s * w.x / m, s * w.y / m, s * w.z / m};
  }
  V3<R> c{R(b.cx) + R(b.vx) * dt, R(b.cy) + R(b.vy) * dt, R(b.cz) + R(b.vz) * dt};
  Q4<R> q = qmul(e, bquat<R>(b));
  V3<R> d{p.x - c.x, p.y - c.y, p.z - c.z};
  if (win && win->on) {
    d.x = win_wrap1(d.x, win->n[0]);
    d.y = win_wrap1(d.y, win->n[1]);
    d.z = win_wrap1(d.z, win->n[2]);
  }
  return sdf_local<R>(qrotinv(q, d), b);
}

template <class R> V3<R> body_vel3(V3<R> p, const lbm_body &b, const Win *w = nullptr) {
  const V3<R> r = bdelta(p, b, w);
  return {R(b.vx) + (R(b.wy) * r.z - R(b.wz) * r.y), R(b.vy) + (R(b.wz) * r.x - R(b.wx) * r.z),
          R(b.vz) + (R(b.wx) * r.y - R(b.wy) * r.x)};
}

template <class R> R chi_of(R phi, R eps) {
  R a = phi / eps;
  a = std::fmin(std::fmax(a, R(-20)), R(20));
  return R(0.5) * (R(1) - std::tanh(a));
}

template <class R> R wrapd(R d, R n) { return d - n * std::nearbyint(d / n); }

template <class R> R phi2(R px, R py, const lbm_body &b, R W, R H) {
  R ca = std::cos(R(b.theta)), sa = std::sin(R(b.theta));
  R dx = wrapd(px - R(b.cx), W), dy = wrapd(py - R(b.cy), H);
  R lx = dx * ca + dy * sa, ly = -dx * sa + dy * ca;
  R a = R(b.a), bb = R(b.b);
  if (std::fabs(a - bb) <= R(1e-6) * std::fmax(a, bb)) return std::sqrt(lx * lx + ly * ly) - a;
  R x = std::fabs(lx), y = std::fabs(ly);
  R r = std::sqrt((x * x) / (a * a) + (y * y) / (bb * bb));
  R alg = (r - R(1)) * bb;
  if (alg > R(64)) return alg;
  bool inside = r < R(1);
  R t = std::atan2(y * a, x * bb);
  for (int i = 0; i < 3; ++i) {
    R ct = std::cos(t), st = std::sin(t);
    R ex = x - a * ct, ey = y - bb * st;
    R F = ex * (-a * st) + ey * (bb * ct);
    R Fp = -(a * a * st * st + bb * bb * ct * ct) + ex * (-a * ct) + ey * (-bb * st);
    t = t - F / (std::fabs(Fp) < R(1e-9) ? R(-1e-9) : Fp);
    t = std::fmin(std::fmax(t, R(0)), R(1.5707963));
  }
  R ddx = x - a * std::cos(t), ddy = y - bb * std::sin(t);
  R d = std::sqrt(ddx * ddx + ddy * ddy);
  return inside ? -d : d;
}

template <class R> R sponge(R d, R sw) {
  if (sw <= R(0)) return R(0);
  R w = std::fmin(std::fmax(R(1) - d / sw, R(0)), R(1));
  return w * w * (R(3) - R(2) * w);
}

// lbm_step.wgsl:137-270, one fused step of a dense D2Q9 grid; mac (4 per
// cell, may be NULL) receives rho, ux, uy, 0.
template <class R>
void step2(const lbm_config &c, const std::vector<R> &fin, std::vector<R> &fout, double *mac) {
  const Tables &T = tables(9);
  const int W = c.nx, H = c.ny;
  const int64_t N = (int64_t)W * H;
  const lbm_body &b = c.body;
  const R CS2 = R(1) / R(3), fW = R(W), fH = R(H);
  const R omg = R(1) / R(c.tau);
  const R SUX = R(c.sponge_u[0]), SUY = R(c.sponge_u[1]);
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const int64_t cell = (int64_t)y * W + x;
      R px = R(x), py = R(y);
      R rx = 0, ry = 0, usx = 0, usy = 0, phi = R(1e30f);
      if (c.has_body) {
        rx = wrapd(px - R(b.cx), fW); ry = wrapd(py - R(b.cy), fH);
        usx = R(b.vx) - R(b.wz) * ry; usy = R(b.vy) + R(b.wz) * rx;
        phi = phi2(px, py, b, fW, fH);
      }
      R f[9];
      for (int i = 0; i < 9; ++i) {
        int sx = (x + W - T.ex[i]) % W, sy = (y + H - T.ey[i]) % H;
        int ysrc = y - T.ey[i];
        if (c.use_bounceback && c.has_body && phi2(R(sx), R(sy), b, fW, fH) < R(0)) {
          R corr = R(2) * R(T.w[i]) * (R(T.ex[i]) * usx + R(T.ey[i]) * usy) / CS2;
          f[i] = fin[T.opp[i] * N + cell] + corr;
        } else if (c.wall[1] && (ysrc < 0 || ysrc >= H)) {
          R wu = ysrc < 0 ? R(c.wall_u[0]) : R(c.wall_u[1]);
          R corr = R(2) * R(T.w[i]) * R(T.ex[i]) * wu / CS2;
          f[i] = fin[T.opp[i] * N + cell] + corr;
        } else {
          f[i] = fin[i * N + (int64_t)sy * W + sx];
        }
      }
      R rho = 0, uxs = 0, uys = 0;
      for (int i = 0; i < 9; ++i) { rho += f[i]; uxs += f[i] * R(T.ex[i]); uys += f[i] * R(T.ey[i]); }
      R den = std::fmax(rho, R(1e-6));
      uxs /= den; uys /= den;
      R chi = (c.use_bounceback || !c.has_body) ? R(0) : chi_of(phi, R(c.chi_eps));
      R Fx = rho * chi * (usx - uxs) + R(c.force[0]);
      R Fy = rho * chi * (usy - uys) + R(c.force[1]);
      R ux = uxs + Fx / (R(2) * den), uy = uys + Fy / (R(2) * den);
      R usq = ux * ux + uy * uy;
      R dx = std::fmin(px, R(W - 1 - x)), dy = std::fmin(py, R(H - 1 - y));
      R sw = sponge(std::fmin(dx, dy), R(c.sponge_w));
      const bool solid = c.solid_eq && c.use_bounceback && c.has_body && phi < R(0);
      for (int i = 0; i < 9; ++i) {
        R exf = R(T.ex[i]), eyf = R(T.ey[i]), w = R(T.w[i]);
        R o;
        if (solid) {
          R eu = exf * usx + eyf * usy;
          o = w * R(1) * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * (usx * usx + usy * usy));
        } else {
          R eu = exf * ux + eyf * uy;
          R feq = w * rho * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * usq);
          R t2 = (exf * ux + eyf * uy) * R(9);
          R Si = (R(1) - R(0.5) * omg) * w *
                 (((exf - ux) * R(3) + t2 * exf) * Fx + ((eyf - uy) * R(3) + t2 * eyf) * Fy);
          R fc = f[i] - omg * (f[i] - feq) + Si;
          R euf = exf * SUX + eyf * SUY;
          R ft = w * (R(1) + R(3) * euf + R(4.5) * euf * euf - R(1.5) * (SUX * SUX + SUY * SUY));
          o = fc * (R(1) - sw) + ft * sw;
        }
        fout[i * N + cell] = o;
      }
      if (mac) {
        double *m = mac + 4 * cell;
        m[0] = (double)rho; m[1] = (double)ux; m[2] = (double)uy; m[3] = 0;
      }
    }
}

}  // namespace oracle
