// ORACLE -- test infrastructure only. The dense 3D force pass and fused
// step of the reference (common_d3_force.wgsl:171-283,
// common_d3_step.wgsl:206-400), shared by the dense and AMR restatements.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

#include "../include/lbm.h"

#include "common.h"

namespace oracle {

// ---- 3D --------------------------------------------------------------------

template <class R>
void force3(const lbm_config &c, const std::vector<R> &fin, double out[8]) {
  const Tables &T = tables(c.q);
  const int NX = c.nx, NY = c.ny, NZ = c.nz, Q = c.q;
  const int64_t N = (int64_t)NX * NY * NZ;
  const lbm_body &b = c.body;
  const Win win = window_of(c);
  const R CS2 = R(1) / R(3);
  std::vector<double> rows((size_t)NY * NZ * 7, 0.0);
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < NZ; ++z)
    for (int y = 0; y < NY; ++y) {
      double acc[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int x = 0; x < NX; ++x) {
        const int64_t cell = ((int64_t)z * NY + y) * NX + x;
        V3<R> p{R(x), R(y), R(z)};
        R phi = phi3(p, b, &win);
        V3<R> r = bdelta(p, b, &win);
        V3<R> us = body_vel3(p, b, &win);
        V3<R> fb{0, 0, 0}, tb{0, 0, 0};
        if (c.use_bounceback) {
          if (phi >= R(0)) {
            R rhoW = R(1);
            if (c.rho_w_local && phi < R(2)) {
              R s = 0;
              for (int i = 0; i < Q; ++i) s += fin[i * N + cell];
              rhoW = s;
            }
            for (int i = 0; i < Q; ++i) {
              V3<R> sp{p.x - R(T.ex[i]), p.y - R(T.ey[i]), p.z - R(T.ez[i])};
              if (phi3(sp, b, &win) < R(0)) {
                R fo = fin[T.opp[i] * N + cell];
                R corr = R(2) * R(T.w[i]) * rhoW *
                         (R(T.ex[i]) * us.x + R(T.ey[i]) * us.y + R(T.ez[i]) * us.z) / CS2;
                R m = R(2) * fo + corr;
                fb.x += -R(T.ex[i]) * m;
                fb.y += -R(T.ey[i]) * m;
                fb.z += -R(T.ez[i]) * m;
              }
            }
          }
          if (c.swept_force) {
            bool now = phi < R(0);
            if (now != (phi3_ahead(p, b, R(1), &win) < R(0))) {
              V3<R> mc{0, 0, 0};
              for (int i = 0; i < Q; ++i) {
                R v = fin[i * N + cell];
                mc.x += v * R(T.ex[i]); mc.y += v * R(T.ey[i]); mc.z += v * R(T.ez[i]);
              }
              if (!now) { fb.x += mc.x; fb.y += mc.y; fb.z += mc.z; }
              else { fb.x += -mc.x; fb.y += -mc.y; fb.z += -mc.z; }
            }
          }
          tb = {r.y * fb.z - r.z * fb.y, r.z * fb.x - r.x * fb.z, r.x * fb.y - r.y * fb.x};
        } else {
          R chi = chi_of(phi, R(c.chi_eps));
          if (chi >= R(1e-6)) {
            R rho = 0, mx = 0, my = 0, mz = 0;
            for (int i = 0; i < Q; ++i) {
              int sx = (x - T.ex[i] + NX) % NX, sy = (y - T.ey[i] + NY) % NY, sz = (z - T.ez[i] + NZ) % NZ;
              R v = fin[i * N + ((int64_t)sz * NY + sy) * NX + sx];
              rho += v; mx += v * R(T.ex[i]); my += v * R(T.ey[i]); mz += v * R(T.ez[i]);
            }
            R den = std::fmax(rho, R(1e-6));
            V3<R> ust{mx / den, my / den, mz / den};
            R rc = rho * chi;
            fb = {-(rc * (us.x - ust.x)), -(rc * (us.y - ust.y)), -(rc * (us.z - ust.z))};
            tb = {r.y * fb.z - r.z * fb.y, r.z * fb.x - r.x * fb.z, r.x * fb.y - r.y * fb.x};
          }
        }
        R v6[6] = {fb.x, fb.y, fb.z, tb.x, tb.y, tb.z};
        for (int k = 0; k < 6; ++k) {
          if (std::isfinite((double)v6[k])) acc[k] += (double)v6[k];
          else acc[6] += 1.0;
        }
      }
      for (int k = 0; k < 7; ++k) rows[((size_t)z * NY + y) * 7 + k] = acc[k];
    }
  for (int k = 0; k < 8; ++k) out[k] = 0.0;
  for (size_t j = 0; j < (size_t)NY * NZ; ++j)
    for (int k = 0; k < 7; ++k) out[k] += rows[j * 7 + k];
}

// Blocks the dense step does not solve (the coarse level under a refined
// region, common_d3_step.wgsl:110 coveredByFiner): block_slot[b] >= 0.
struct Cover {
  const int32_t *block_slot = nullptr;
  int rb = 1, nbx = 1, nby = 1;
  bool at(int x, int y, int z) const {
    return block_slot && block_slot[((z / rb) * nby + y / rb) * nbx + x / rb] >= 0;
  }
};

template <class R>
void step3(const lbm_config &c, const std::vector<R> &fin, std::vector<R> &fout, double *mac,
           const Cover &cover = Cover()) {
  const Tables &T = tables(c.q);
  const int NX = c.nx, NY = c.ny, NZ = c.nz, Q = c.q;
  const int64_t N = (int64_t)NX * NY * NZ;
  const lbm_body &b = c.body;
  const Win win = window_of(c);
  const R CS2 = R(1) / R(3);
  const R OMEGA = R(1) / R(c.tau);
  // TRT (plans/TRT.md sec 8.0(1)-(2)): OMEGA_M = 1 / tau_- with
  // tau_- = 1/2 + Lambda / (tau - 1/2) formed in double on the host, the
  // odd part of each direction relaxing at OMEGA_M in the delta form
  const double tau_m = 0.5 + (double)c.trt_lambda / ((double)c.tau - 0.5);
  const R DW = c.trt ? R(1.0 / tau_m) - OMEGA : R(0);
  const R FX = R(c.force[0]), FY = R(c.force[1]), FZ = R(c.force[2]);
  const R SUX = R(c.sponge_u[0]), SUY = R(c.sponge_u[1]), SUZ = R(c.sponge_u[2]);
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < NZ; ++z)
    for (int y = 0; y < NY; ++y)
      for (int x = 0; x < NX; ++x) {
        if (cover.at(x, y, z)) continue;
        const int64_t cell = ((int64_t)z * NY + y) * NX + x;
        V3<R> p{R(x), R(y), R(z)};
        R phi = c.has_body ? phi3(p, b, &win) : R(1e30f);
        V3<R> us = c.has_body ? body_vel3(p, b, &win) : V3<R>{0, 0, 0};
        const bool bb = c.has_body && c.use_bounceback;
        R rhoW = R(1);
        if (bb && c.rho_w_local && phi < R(2)) {
          R s = 0;
          for (int i = 0; i < Q; ++i) s += fin[i * N + cell];
          rhoW = s;
        }
        R f[27];
        for (int i = 0; i < Q; ++i) {
          int sxi = x - T.ex[i], syi = y - T.ey[i], szi = z - T.ez[i];
          if (bb && phi3(V3<R>{R(sxi), R(syi), R(szi)}, b, &win) < R(0)) {
            R corr = R(2) * R(T.w[i]) * rhoW *
                     (R(T.ex[i]) * us.x + R(T.ey[i]) * us.y + R(T.ez[i]) * us.z) / CS2;
            f[i] = fin[T.opp[i] * N + cell] + corr;
          } else if ((c.wall[0] && (sxi < 0 || sxi >= NX)) || (c.wall[1] && (syi < 0 || syi >= NY)) ||
                     (c.wall[2] && (szi < 0 || szi >= NZ))) {
            f[i] = fin[T.opp[i] * N + cell];
          } else {
            int sx = (sxi + NX) % NX, sy = (syi + NY) % NY, sz = (szi + NZ) % NZ;
            f[i] = fin[i * N + ((int64_t)sz * NY + sy) * NX + sx];
          }
        }
        R rho = 0, mx = 0, my = 0, mz = 0;
        for (int i = 0; i < Q; ++i) {
          rho += f[i];
          mx += f[i] * R(T.ex[i]); my += f[i] * R(T.ey[i]); mz += f[i] * R(T.ez[i]);
        }
        R den = std::fmax(rho, R(1e-6));
        R uxs = mx / den, uys = my / den, uzs = mz / den;
        R chi = (c.has_body && !c.use_bounceback) ? chi_of(phi, R(c.chi_eps)) : R(0);
        R Fx = rho * chi * (us.x - uxs) + FX;
        R Fy = rho * chi * (us.y - uys) + FY;
        R Fz = rho * chi * (us.z - uzs) + FZ;
        R ux = uxs + Fx / (R(2) * den), uy = uys + Fy / (R(2) * den), uz = uzs + Fz / (R(2) * den);
        R usq = ux * ux + uy * uy + uz * uz;
        R sw = R(0);
        if (c.sponge_w > 0) {
          const V3<R> wp = win_coord(p, b, &win);  // common_d3_step.wgsl:316
          R dx = c.sponge_axis[0] ? std::fmin(wp.x, R(NX - 1) - wp.x) : R(1e30f);
          R dy = c.sponge_axis[1] ? std::fmin(wp.y, R(NY - 1) - wp.y) : R(1e30f);
          R dz = c.sponge_axis[2] ? std::fmin(wp.z, R(NZ - 1) - wp.z) : R(1e30f);
          sw = sponge(std::fmin(dx, std::fmin(dy, dz)), R(c.sponge_w));
        }
        const bool solid = c.solid_eq && bb && phi < R(0);
        R ussq = us.x * us.x + us.y * us.y + us.z * us.z;
        R ufar = SUX * SUX + SUY * SUY + SUZ * SUZ;
        for (int i = 0; i < Q; ++i) {
          R exf = R(T.ex[i]), eyf = R(T.ey[i]), ezf = R(T.ez[i]), w = R(T.w[i]);
          R o;
          if (solid) {
            R eu = exf * us.x + eyf * us.y + ezf * us.z;
            o = w * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * ussq);
          } else {
            R eu = exf * ux + eyf * uy + ezf * uz;
            R feq = w * rho * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * usq);
            R t2 = eu * R(9);
            R dot = ((exf - ux) * R(3) + t2 * exf) * Fx + ((eyf - uy) * R(3) + t2 * eyf) * Fy +
                    ((ezf - uz) * R(3) + t2 * ezf) * Fz;
            R Si = (R(1) - R(0.5) * OMEGA) * w * dot;
            R fc = f[i] - OMEGA * (f[i] - feq) + Si;
            if (c.trt) {
              // f_minus = (f_i - f_opp)/2, feq_minus = 3 w rho e.u, S_minus = 3 w e.F
              const R fminus = R(0.5) * (f[i] - f[T.opp[i]]);
              const R feqminus = R(3) * w * rho * eu;
              const R sminus = R(3) * w * (exf * Fx + eyf * Fy + ezf * Fz);
              fc = fc - DW * (fminus - feqminus) - R(0.5) * DW * sminus;
            }
            R euf = exf * SUX + eyf * SUY + ezf * SUZ;
            R ft = w * (R(1) + R(3) * euf + R(4.5) * euf * euf - R(1.5) * ufar);
            o = fc * (R(1) - sw) + ft * sw;
          }
          fout[i * N + cell] = o;
        }
        if (mac) {
          double *m = mac + 4 * cell;
          if (solid) { m[0] = 1; m[1] = (double)us.x; m[2] = (double)us.y; m[3] = (double)us.z; }
          else { m[0] = (double)rho; m[1] = (double)ux; m[2] = (double)uy; m[3] = (double)uz; }
        }
      }
}

}  // namespace oracle
