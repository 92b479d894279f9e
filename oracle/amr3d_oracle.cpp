// ORACLE -- test infrastructure only. CPU restatement of the reference's 3D
// block-structured AMR at two levels (the dense L0 grid plus one pool level
// of RB^3-block tiles at half spacing), used by tests/ as the checker and
// never linked into the product library.
//
// Followed (reference paths):
//   d3-amr.mjs:38-110            GHOST, fineToCoarseUnit, makePool, refineWhere
//   d3-amr.mjs:112-165           nearBodyWant branch and bound (SQRT3_UP, depth 3)
//   main-3d.js:450-480           the box / slab / bar / all predicates
//   common_d3_pool.wgsl          tile addressing, wrapFine3, localInTile3,
//                                interpCoarseToFine3, dcRescaleC2F
//   common_d3_amr_interp.wgsl    tile seed (GHOST_ONLY = 0)
//   common_d3_moments.wgsl       pool moments after the seed
//   common_d3_amr_explode.wgsl   coarse -> ring (linear explosion, in-orphans)
//   common_d3_amr_step1.wgsl     pool substep, DIRECT_GHOST, COLLIDE_RING = 0
//   common_d3_amr_coalesce.wgsl  ring -> covered coarse cells, out/in orphans
//   common_d3_step.wgsl:110      coarse step skipping covered blocks
//   common_d3_force_pool.wgsl    pool force, dx^2 and dx^3 weights
//   main-3d.js:3219-3341         macro-step order: force, explode, two fine
//                                substeps, coalesce, coarse step; with
//                                ?interface=interp (:3343-3356) the coarse
//                                step first, the ring interpolated
//                                (GHOST_ONLY), substeps collide the ring,
//                                common_d3_amr_average.wgsl into the new L0
//   common_d3_manage.wgsl        dynamic refinement: decide (boxNearBody in
//                                f32 with the lead of the body's motion),
//                                drain (common_d3_amr_average.wgsl, DYING_ONLY),
//                                coarsen / refine over the free-slot stack,
//                                fill (interp, NEW_ONLY); slots granted in
//                                ascending block id (the reference's atomics
//                                leave the order to the scheduler)
// R = double is the FP64 checker; R = float keeps the reference's f32
// operation order (built with -ffp-contract=off).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/lbm.h"

#include "common.h"
#include "dense3.h"

namespace {
using namespace oracle;

constexpr int GH = 2;
constexpr double SQRT3_UP = 1.7320509;

struct Topo {
  int nx, ny, nz, rb, nbx, nby, nbz, nb;
  std::vector<int32_t> block_slot, slot_to_block;  // slot_to_block: capacity entries, -1 = free
  int slots = 0;                                   // capacity
  int initial = 0;
};

// nearBodyWant: one SDF evaluation brackets the minimum over a box of
// half-edge h as phi(c) - h*sqrt(3) <= min <= phi(c); undecided boxes split
// into octants down to depth 3, where failing to reject accepts.
bool near_box(const lbm_body &b, const double c[3], double h, int depth, double margin) {
  const double R = h * SQRT3_UP;
  const double phi = phi3<double>({c[0], c[1], c[2]}, b);
  if (phi - R > margin) return false;
  if (phi <= margin) return true;
  if (depth == 0) return true;
  const double hh = h / 2;
  for (int i = 0; i < 8; ++i) {
    const double cc[3] = {c[0] + ((i & 1) ? hh : -hh), c[1] + ((i & 2) ? hh : -hh), c[2] + ((i & 4) ? hh : -hh)};
    if (near_box(b, cc, hh, depth - 1, margin)) return true;
  }
  return false;
}

// Blocks wanted by the predicate, slots handed out in ascending block id.
void refine(Topo &t, int mode, const lbm_body &body, double margin, double frac, const int32_t *list) {
  t.block_slot.assign(t.nb, -1);
  t.slot_to_block.clear();
  const double dims[3] = {(double)t.nx, (double)t.ny, (double)t.nz};
  for (int id = 0; id < t.nb; ++id) {
    const int bx = id % t.nbx, by = (id / t.nbx) % t.nby, bz = id / (t.nbx * t.nby);
    const double lo[3] = {(double)bx * t.rb, (double)by * t.rb, (double)bz * t.rb};
    const double mid[3] = {lo[0] + t.rb / 2.0, lo[1] + t.rb / 2.0, lo[2] + t.rb / 2.0};
    bool want = false;
    switch (mode) {
      case LBM_REFINE_ALL: want = true; break;
      case LBM_REFINE_BOX: {
        want = true;
        for (int a = 0; a < 3; ++a)
          want = want && mid[a] >= dims[a] * (1 - frac) / 2 && mid[a] < dims[a] * (1 + frac) / 2;
        break;
      }
      case LBM_REFINE_BAR: {
        want = true;
        for (int a = 0; a < 2; ++a)
          want = want && mid[a] >= dims[a] * (1 - frac) / 2 && mid[a] < dims[a] * (1 + frac) / 2;
        break;
      }
      case LBM_REFINE_SLAB: want = mid[0] >= dims[0] * (1 - frac) / 2 && mid[0] < dims[0] * (1 + frac) / 2; break;
      case LBM_REFINE_BODY: want = near_box(body, mid, t.rb / 2.0, 3, margin); break;
      case LBM_REFINE_LIST: want = list[id] != 0; break;
    }
    if (!want) continue;
    t.block_slot[id] = (int32_t)t.slot_to_block.size();
    t.slot_to_block.push_back(id);
  }
  t.slots = (int)t.slot_to_block.size();
  t.initial = t.slots;
}

template <class R> R feq(const Tables &T, int i, R rho, R ux, R uy, R uz) {
  const R eu = R(T.ex[i]) * ux + R(T.ey[i]) * uy + R(T.ez[i]) * uz;
  const R usq = ux * ux + uy * uy + uz * uz;
  return R(T.w[i]) * rho * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * usq);
}

inline int wrapi(int v, int n) { return ((v % n) + n) % n; }

// qAt (common_d3_criterion.wgsl): Q = 1/2 (|Omega|^2 - |S|^2) at an L0 cell
// from centred differences of u over its six face neighbours, periodic, in
// f32 with every product and sum rounded on its own. mac is [rho, u] per cell.
inline float q_cell(const float *mac, int nx, int ny, int nz, int x, int y, int z) {
  auto u = [&](int xx, int yy, int zz, int i) {
    const int64_t c = ((int64_t)wrapi(zz, nz) * ny + wrapi(yy, ny)) * nx + wrapi(xx, nx);
    return mac[4 * c + 1 + i];
  };
  float J[3][3];  // J[j][i] = du_i / dx_j
  for (int i = 0; i < 3; ++i) {
    J[0][i] = (u(x + 1, y, z, i) - u(x - 1, y, z, i)) * 0.5f;
    J[1][i] = (u(x, y + 1, z, i) - u(x, y - 1, z, i)) * 0.5f;
    J[2][i] = (u(x, y, z + 1, i) - u(x, y, z - 1, i)) * 0.5f;
  }
  float s2 = 0.f, om2 = 0.f;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const float a = J[j][i], b = J[i][j];
      const float S = 0.5f * (a + b), O = 0.5f * (a - b);
      s2 += S * S;
      om2 += O * O;
    }
  return 0.5f * (om2 - s2);
}

template <class R> struct Amr3D {
  lbm_config c;
  int Q, FB, RB2, T3;
  int64_t N, P;  // coarse cells, pool cells (slots * FB^3)
  Topo t;
  const Tables *T;
  R tau_f;
  std::vector<R> fc[2], fp[2];
  std::vector<double> macc, macp;
  int cp = 0;
  int linear = 1;
  int interp = 0;  // ?interface=interp instead of explode/coalesce
  int reflux_on = 0;  // ?reflux=1 (interp only)
  std::vector<R> flux_acc;
  // dynamic refinement
  int dynamic = 0, manage_every = 16, manage_start = 0;
  double margin = 2.0;
  long step_count = 0;
  std::vector<int32_t> free_list;
  std::vector<uint8_t> slot_new, want;
  int free_count = 0, refused = 0, min_free = 0, decisions = 0;
  Win win;  // the moving window of the L0 configuration
  // the field criterion (common_d3_criterion.wgsl): off at q_abs = 0
  float q_abs = 0.f, q_hyst = 1.f, q_lead = 0.f;
  std::vector<float> block_q;

  int bid(int bx, int by, int bz) const { return (bz * t.nby + by) * t.nbx + bx; }
  bool covered(int x, int y, int z) const {
    return t.block_slot[bid(wrapi(x, t.nx) / t.rb, wrapi(y, t.ny) / t.rb, wrapi(z, t.nz) / t.rb)] >= 0;
  }
  int64_t ccell(int x, int y, int z) const {
    return ((int64_t)wrapi(z, t.nz) * t.ny + wrapi(y, t.ny)) * t.nx + wrapi(x, t.nx);
  }
  int64_t pcell(int s, int fx, int fy, int fz) const { return (int64_t)s * T3 + ((int64_t)fz * FB + fy) * FB + fx; }
  bool interior(int j) const { return j >= GH && j < GH + RB2; }
  static R f2c(int j, int origin) { return R(origin) - R(0.25) + R(0.5) * R(j - GH); }
  R omega_f() const { return R(1) / tau_f; }

  // ---- seed: initEq on the coarse grid, interpolated tiles, moments ------
  void seed(const double *mac) {
    for (int k = 0; k < 2; ++k) fc[k].assign((size_t)Q * N, R(0));
    for (int64_t cell = 0; cell < N; ++cell) {
      const double *m = mac + 4 * cell;
      for (int i = 0; i < Q; ++i) {
        const R v = feq<R>(*T, i, R((float)m[0]), R((float)m[1]), R((float)m[2]), R((float)m[3]));
        fc[0][i * N + cell] = v;
        fc[1][i * N + cell] = v;
      }
    }
    for (int k = 0; k < 2; ++k) fp[k].assign((size_t)Q * P, R(0));
    macp.assign((size_t)4 * P, 0.0);
    macc.assign((size_t)4 * N, 0.0);
    for (int64_t cell = 0; cell < N; ++cell)
      for (int k = 0; k < 4; ++k) macc[4 * cell + k] = (double)(float)mac[4 * cell + k];
    interp_fill(fc[0], fp[0], false);
    moments(fp[0]);
    cp = 0;
    step_count = 0;
  }

  // interpCoarseToFine3 over every cell of every tile (or its ring only).
  void interp_fill(const std::vector<R> &f0, std::vector<R> &dst, bool ring_only, bool only_new = false) {
    const R tc = R(c.tau), tf = R(2) * tc - R(0.5);
    const R rescale = R(0.5) * (tf - R(1)) / (tc - R(1));
    for (int s = 0; s < t.slots; ++s) {
      const int id = t.slot_to_block[s];
      if (id < 0 || (only_new && !slot_new[s])) continue;
      const int bx = id % t.nbx, by = (id / t.nbx) % t.nby, bz = id / (t.nbx * t.nby);
      for (int fz = 0; fz < FB; ++fz)
        for (int fy = 0; fy < FB; ++fy)
          for (int fx = 0; fx < FB; ++fx) {
            if (ring_only && interior(fx) && interior(fy) && interior(fz)) continue;
            const R p[3] = {f2c(fx, bx * t.rb), f2c(fy, by * t.rb), f2c(fz, bz * t.rb)};
            int c0[3];
            R tt[3];
            for (int a = 0; a < 3; ++a) {
              c0[a] = (int)std::floor(p[a]);
              tt[a] = p[a] - R(c0[a]);
            }
            R rho = 0, ux = 0, uy = 0, uz = 0, fneq[27] = {};
            for (int k = 0; k < 8; ++k) {
              const int di = k & 1, dj = (k >> 1) & 1, dk = (k >> 2) & 1;
              const R w = (di ? tt[0] : R(1) - tt[0]) * (dj ? tt[1] : R(1) - tt[1]) * (dk ? tt[2] : R(1) - tt[2]);
              const int64_t cc = ccell(c0[0] + di, c0[1] + dj, c0[2] + dk);
              R f[27], r = 0, mx = 0, my = 0, mz = 0;
              for (int i = 0; i < Q; ++i) {
                f[i] = f0[i * N + cc];
                r += f[i];
                mx += f[i] * R(T->ex[i]); my += f[i] * R(T->ey[i]); mz += f[i] * R(T->ez[i]);
              }
              const R den = std::fmax(r, R(1e-6));
              const R u[3] = {mx / den, my / den, mz / den};
              rho += w * r;
              ux += w * u[0]; uy += w * u[1]; uz += w * u[2];
              for (int i = 0; i < Q; ++i) fneq[i] += w * (f[i] - feq<R>(*T, i, r, u[0], u[1], u[2]));
            }
            const int64_t pc = pcell(s, fx, fy, fz);
            for (int i = 0; i < Q; ++i) dst[i * P + pc] = feq<R>(*T, i, rho, ux, uy, uz) + rescale * fneq[i];
          }
    }
  }

  void moments(const std::vector<R> &f) {
    for (int s = 0; s < t.slots; ++s)
      for (int k = 0; k < T3 && t.slot_to_block[s] >= 0; ++k) {
        const int64_t pc = (int64_t)s * T3 + k;
        R rho = 0, mx = 0, my = 0, mz = 0;
        for (int i = 0; i < Q; ++i) {
          const R v = f[i * P + pc];
          rho += v; mx += v * R(T->ex[i]); my += v * R(T->ey[i]); mz += v * R(T->ez[i]);
        }
        const R den = std::fmax(rho, R(1e-6));
        macp[4 * pc] = (double)rho;
        macp[4 * pc + 1] = (double)(mx / den);
        macp[4 * pc + 2] = (double)(my / den);
        macp[4 * pc + 3] = (double)(mz / den);
      }
  }

  // ---- explode: coarse (time t) -> ring ----------------------------------
  void explode(const std::vector<R> &fco, std::vector<R> &dst) {
    const int NF[3] = {2 * t.nx, 2 * t.ny, 2 * t.nz};
    for (int s = 0; s < t.slots; ++s) {
      const int id = t.slot_to_block[s];
      if (id < 0) continue;
      const int b[3] = {id % t.nbx, (id / t.nbx) % t.nby, id / (t.nbx * t.nby)};
      for (int fz = 0; fz < FB; ++fz)
        for (int fy = 0; fy < FB; ++fy)
          for (int fx = 0; fx < FB; ++fx) {
            if (interior(fx) && interior(fy) && interior(fz)) continue;
            const int fi[3] = {fx, fy, fz};
            int g[3], v[3];
            for (int a = 0; a < 3; ++a) {
              g[a] = wrapi(b[a] * RB2 + fi[a] - GH, NF[a]);
              v[a] = g[a] / 2;
            }
            if (covered(v[0], v[1], v[2])) continue;
            const int64_t vc = ccell(v[0], v[1], v[2]);
            bool ok[3];
            int64_t vm[3], vp[3];
            for (int a = 0; a < 3; ++a) {
              int m[3] = {v[0], v[1], v[2]}, q[3] = {v[0], v[1], v[2]};
              m[a] -= 1; q[a] += 1;
              ok[a] = !covered(m[0], m[1], m[2]) && !covered(q[0], q[1], q[2]);
              vm[a] = ccell(m[0], m[1], m[2]);
              vp[a] = ccell(q[0], q[1], q[2]);
            }
            R d[3];
            for (int a = 0; a < 3; ++a) d[a] = (R(g[a] - 2 * v[a]) - R(0.5)) * R(0.5);
            const int64_t pc = pcell(s, fx, fy, fz);
            for (int i = 0; i < Q; ++i) {
              const int e[3] = {T->ex[i], T->ey[i], T->ez[i]};
              if (!covered(v[0] + e[0], v[1] + e[1], v[2] + e[2])) {
                int dg[3];
                for (int a = 0; a < 3; ++a) dg[a] = wrapi(g[a] + e[a], NF[a]);
                const bool into = covered(dg[0] / 2, dg[1] / 2, dg[2] / 2) && dg[0] / RB2 == b[0] &&
                                  dg[1] / RB2 == b[1] && dg[2] / RB2 == b[2];
                dst[i * P + pc] = into ? fco[i * N + vc] : R(0);
                continue;
              }
              const R f = fco[i * N + vc];
              if (!linear) { dst[i * P + pc] = f; continue; }
              R G[3];
              for (int a = 0; a < 3; ++a)
                G[a] = ok[a] ? R(0.5) * (fco[i * N + vp[a]] - fco[i * N + vm[a]]) : R(0);
              const R ee = R(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
              const R gd = (G[0] * R(e[0]) + G[1] * R(e[1]) + G[2] * R(e[2])) / ee;
              for (int a = 0; a < 3; ++a) G[a] -= R(e[a]) * gd;
              dst[i * P + pc] = f + (d[0] * G[0] + d[1] * G[1] + d[2] * G[2]);
            }
          }
    }
  }

  // ---- one pool substep ----------------------------------------------------
  void substep(const std::vector<R> &fin, std::vector<R> &fout, bool collide_ring) {
    const lbm_body &bd = c.body;
    const bool hb = c.has_body, bb = c.has_body && c.use_bounceback;
    const R CS2 = R(1) / R(3), OM = omega_f();
    const R SUX = R(c.sponge_u[0]), SUY = R(c.sponge_u[1]), SUZ = R(c.sponge_u[2]);
    const R FXc = R(c.force[0]), FYc = R(c.force[1]), FZc = R(c.force[2]);
#pragma omp parallel for schedule(static)
    for (int s = 0; s < t.slots; ++s) {
      const int id = t.slot_to_block[s];
      if (id < 0) continue;
      const int b[3] = {id % t.nbx, (id / t.nbx) % t.nby, id / (t.nbx * t.nby)};
      const int nbn[3] = {t.nbx, t.nby, t.nbz};
      for (int fz = 0; fz < FB; ++fz)
        for (int fy = 0; fy < FB; ++fy)
          for (int fx = 0; fx < FB; ++fx) {
            const int fi[3] = {fx, fy, fz};
            int off[3], bn[3];
            for (int a = 0; a < 3; ++a) {
              off[a] = fi[a] <= GH ? -1 : (fi[a] + 1 >= GH + RB2 ? 1 : 0);
              bn[a] = wrapi(b[a] + off[a], nbn[a]);
            }
            auto slot_at = [&](int dx, int dy, int dz) {
              return t.block_slot[bid(dx ? bn[0] : b[0], dy ? bn[1] : b[1], dz ? bn[2] : b[2])];
            };
            const int64_t cell = pcell(s, fx, fy, fz);
            const V3<R> p{f2c(fx, b[0] * t.rb), f2c(fy, b[1] * t.rb), f2c(fz, b[2] * t.rb)};
            const R phi = hb ? phi3(p, bd, &win) : R(1e30f);
            const V3<R> us = hb ? body_vel3(p, bd, &win) : V3<R>{0, 0, 0};
            R rhoW = R(1);
            if (bb && c.rho_w_local && phi < R(2)) {
              R sum = 0;
              for (int i = 0; i < Q; ++i) sum += fin[i * P + cell];
              rhoW = sum;
            }
            R f[27];
            for (int i = 0; i < Q; ++i) {
              const int e[3] = {T->ex[i], T->ey[i], T->ez[i]};
              int sc[3] = {fx - e[0], fy - e[1], fz - e[2]};
              if (bb) {
                const V3<R> sp{f2c(sc[0], b[0] * t.rb), f2c(sc[1], b[1] * t.rb), f2c(sc[2], b[2] * t.rb)};
                if (phi3(sp, bd, &win) < R(0)) {
                  const R corr = R(2) * R(T->w[i]) * rhoW * (R(e[0]) * us.x + R(e[1]) * us.y + R(e[2]) * us.z) / CS2;
                  f[i] = fin[T->opp[i] * P + cell] + corr;
                  continue;
                }
              }
              int o[3];
              for (int a = 0; a < 3; ++a) o[a] = (sc[a] < GH || sc[a] >= GH + RB2) ? off[a] : 0;
              int ns = -1;
              if (o[0] || o[1] || o[2]) ns = slot_at(o[0], o[1], o[2]);
              int src = s;
              if (ns >= 0) {
                src = ns;
                for (int a = 0; a < 3; ++a) sc[a] -= o[a] * RB2;
              }
              for (int a = 0; a < 3; ++a) sc[a] = std::min(std::max(sc[a], 0), FB - 1);
              f[i] = fin[i * P + pcell(src, sc[0], sc[1], sc[2])];
            }
            R rho = 0, mx = 0, my = 0, mz = 0;
            for (int i = 0; i < Q; ++i) {
              rho += f[i]; mx += f[i] * R(T->ex[i]); my += f[i] * R(T->ey[i]); mz += f[i] * R(T->ez[i]);
            }
            const R den = std::fmax(rho, R(1e-6));
            const R uxs = mx / den, uys = my / den, uzs = mz / den;
            const R chi = (hb && !c.use_bounceback) ? chi_of(phi, R(c.chi_eps) * R(0.5)) : R(0);
            const R Fx = rho * chi * (us.x - uxs) + FXc, Fy = rho * chi * (us.y - uys) + FYc,
                    Fz = rho * chi * (us.z - uzs) + FZc;
            const R ux = uxs + Fx / (R(2) * den), uy = uys + Fy / (R(2) * den), uz = uzs + Fz / (R(2) * den);
            macp[4 * cell] = (double)rho;
            macp[4 * cell + 1] = (double)ux;
            macp[4 * cell + 2] = (double)uy;
            macp[4 * cell + 3] = (double)uz;
            const bool inter = interior(fx) && interior(fy) && interior(fz);
            if (!collide_ring && !inter) {
              for (int i = 0; i < Q; ++i) fout[i * P + cell] = f[i];
              continue;
            }
            R sw = R(0);
            if (c.sponge_w > 0) {
              const V3<R> wp = win_coord(p, bd, &win);  // common_d3_amr_step1.wgsl:362
              const R dx = c.sponge_axis[0] ? std::fmin(wp.x, R(t.nx - 1) - wp.x) : R(1e30f);
              const R dy = c.sponge_axis[1] ? std::fmin(wp.y, R(t.ny - 1) - wp.y) : R(1e30f);
              const R dz = c.sponge_axis[2] ? std::fmin(wp.z, R(t.nz - 1) - wp.z) : R(1e30f);
              sw = sponge(std::fmin(dx, std::fmin(dy, dz)), R(c.sponge_w));
            }
            const R usq = ux * ux + uy * uy + uz * uz, ufar = SUX * SUX + SUY * SUY + SUZ * SUZ;
            const bool solid = c.solid_eq && bb && phi < R(0);
            const R ussq = us.x * us.x + us.y * us.y + us.z * us.z;
            for (int i = 0; i < Q; ++i) {
              const R exf = R(T->ex[i]), eyf = R(T->ey[i]), ezf = R(T->ez[i]), w = R(T->w[i]);
              R out;
              if (solid) {
                const R eu = exf * us.x + eyf * us.y + ezf * us.z;
                out = w * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * ussq);
              } else {
                const R eu = exf * ux + eyf * uy + ezf * uz;
                const R fq = w * rho * (R(1) + R(3) * eu + R(4.5) * eu * eu - R(1.5) * usq);
                const R t9 = eu * R(9);
                const R dot = ((exf - ux) * R(3) + t9 * exf) * Fx + ((eyf - uy) * R(3) + t9 * eyf) * Fy +
                              ((ezf - uz) * R(3) + t9 * ezf) * Fz;
                const R Si = (R(1) - R(0.5) * OM) * w * dot;
                const R fcol = f[i] - OM * (f[i] - fq) + Si;
                const R euf = exf * SUX + eyf * SUY + ezf * SUZ;
                const R ft = w * (R(1) + R(3) * euf + R(4.5) * euf * euf - R(1.5) * ufar);
                out = fcol * (R(1) - sw) + ft * sw;
              }
              fout[i * P + cell] = out;
            }
            if (solid) {
              macp[4 * cell] = 1.0;
              macp[4 * cell + 1] = (double)us.x;
              macp[4 * cell + 2] = (double)us.y;
              macp[4 * cell + 3] = (double)us.z;
            }
          }
    }
  }

  // ---- coalesce: ring -> the time-t coarse buffer ------------------------
  int64_t local_in_tile(int g, int b, int nfine) const {
    int d = g - b * RB2;
    if (d < -nfine / 2) d += nfine;
    if (d > nfine / 2) d -= nfine;
    return d + GH;
  }

  // ---- flux / reflux (common_d3_amr_flux.wgsl, common_d3_amr_reflux.wgsl) --
  // An unrefined L0 cell whose block touches a refined block on the side
  // (face, edge or corner) the cell sits at.
  bool seam_cell(int x, int y, int z) const {
    const int c3[3] = {x, y, z};
    const int b[3] = {x / t.rb, y / t.rb, z / t.rb};
    if (t.block_slot[bid(b[0], b[1], b[2])] >= 0) return false;
    int off[3];
    for (int a = 0; a < 3; ++a) off[a] = c3[a] % t.rb == 0 ? -1 : ((c3[a] + 1) % t.rb == 0 ? 1 : 0);
    const int nb[3] = {t.nbx, t.nby, t.nbz};
    for (int k = 0; k < 8; ++k) {
      int q[3];
      for (int a = 0; a < 3; ++a) q[a] = wrapi(b[a] + ((k >> a) & 1) * off[a], nb[a]);
      if (t.block_slot[bid(q[0], q[1], q[2])] >= 0) return true;
    }
    return false;
  }

  int slot_of_fine(const int g[3]) const { return t.block_slot[bid(g[0] / RB2, g[1] / RB2, g[2] / RB2)]; }

  // The mass and momentum the fine level moved across the seam into each
  // seam cell during one substep, in L0 units (1/8 per fine cell).
  void flux(const std::vector<R> &fpo, std::vector<R> &acc, bool accumulate) {
    const int NF[3] = {2 * t.nx, 2 * t.ny, 2 * t.nz};
    for (int z = 0; z < t.nz; ++z)
      for (int y = 0; y < t.ny; ++y)
        for (int x = 0; x < t.nx; ++x) {
          if (!seam_cell(x, y, z)) continue;
          const int64_t cell = ccell(x, y, z);
          R dm = 0, dp[3] = {0, 0, 0};
          for (int oc = 0; oc < 8; ++oc) {
            const int pp[3] = {2 * x + (oc & 1), 2 * y + ((oc >> 1) & 1), 2 * z + ((oc >> 2) & 1)};
            for (int i = 0; i < Q; ++i) {
              const int e[3] = {T->ex[i], T->ey[i], T->ez[i]};
              int q[3], tt[3];
              for (int a = 0; a < 3; ++a) {
                q[a] = wrapi(pp[a] - e[a], NF[a]);
                tt[a] = wrapi(pp[a] + e[a], NF[a]);
              }
              const int so = slot_of_fine(q);
              if (so >= 0) {
                const R f = fpo[i * P + pcell(so, (int)local_in_tile(q[0], q[0] / RB2, NF[0]),
                                              (int)local_in_tile(q[1], q[1] / RB2, NF[1]),
                                              (int)local_in_tile(q[2], q[2] / RB2, NF[2]))];
                dm += f;
                for (int a = 0; a < 3; ++a) dp[a] += f * R(e[a]);
              }
              const int si = slot_of_fine(tt);
              if (si >= 0) {
                const R f = fpo[i * P + pcell(si, (int)local_in_tile(pp[0], tt[0] / RB2, NF[0]),
                                              (int)local_in_tile(pp[1], tt[1] / RB2, NF[1]),
                                              (int)local_in_tile(pp[2], tt[2] / RB2, NF[2]))];
                dm -= f;
                for (int a = 0; a < 3; ++a) dp[a] -= f * R(e[a]);
              }
            }
          }
          const R v[4] = {dm * R(0.125), dp[0] * R(0.125), dp[1] * R(0.125), dp[2] * R(0.125)};
          for (int k = 0; k < 4; ++k) acc[4 * cell + k] = accumulate ? acc[4 * cell + k] + v[k] : v[k];
        }
  }

  // The fine flux less the flux L0 computed across the same faces, added to
  // the new L0 populations as w_i (dm + 3 e_i . dp); cells within 2 of the
  // body are left alone.
  void reflux(const std::vector<R> &fin, std::vector<R> &fout, std::vector<R> &acc) {
    for (int z = 0; z < t.nz; ++z)
      for (int y = 0; y < t.ny; ++y)
        for (int x = 0; x < t.nx; ++x) {
          if (!seam_cell(x, y, z)) continue;
          if (c.has_body && phi3<R>({R(x), R(y), R(z)}, c.body, &win) < R(2)) continue;
          const int64_t cell = ccell(x, y, z);
          R dm = acc[4 * cell], dp[3] = {acc[4 * cell + 1], acc[4 * cell + 2], acc[4 * cell + 3]};
          for (int i = 0; i < Q; ++i) {
            const int e[3] = {T->ex[i], T->ey[i], T->ez[i]};
            if (covered(x - e[0], y - e[1], z - e[2])) {
              const R v = fin[i * N + ccell(x - e[0], y - e[1], z - e[2])];
              dm -= v;
              for (int a = 0; a < 3; ++a) dp[a] -= v * R(e[a]);
            }
            if (covered(x + e[0], y + e[1], z + e[2])) {
              const R v = fin[i * N + cell];
              dm += v;
              for (int a = 0; a < 3; ++a) dp[a] += v * R(e[a]);
            }
          }
          acc[4 * cell] = dm;
          for (int a = 0; a < 3; ++a) acc[4 * cell + 1 + a] = dp[a];
          R rho = 0, m[3] = {0, 0, 0};
          for (int i = 0; i < Q; ++i) {
            const R fo = fout[i * N + cell] +
                         R(T->w[i]) * (dm + R(3) * (R(T->ex[i]) * dp[0] + R(T->ey[i]) * dp[1] + R(T->ez[i]) * dp[2]));
            fout[i * N + cell] = fo;
            rho += fo;
            m[0] += fo * R(T->ex[i]); m[1] += fo * R(T->ey[i]); m[2] += fo * R(T->ez[i]);
          }
          const R den = std::fmax(rho, R(1e-6));
          macc[4 * cell] = (double)rho;
          macc[4 * cell + 1] = (double)(m[0] / den + R(c.force[0]) / (R(2) * den));
          macc[4 * cell + 2] = (double)(m[1] / den + R(c.force[1]) / (R(2) * den));
          macc[4 * cell + 3] = (double)(m[2] / den + R(c.force[2]) / (R(2) * den));
        }
  }

  void coalesce(const std::vector<R> &fpo, std::vector<R> &fco) {
    const int NF[3] = {2 * t.nx, 2 * t.ny, 2 * t.nz};
    std::vector<R> out = fco;  // each coarse cell writes only itself
    for (int z = 0; z < t.nz; ++z)
      for (int y = 0; y < t.ny; ++y)
        for (int x = 0; x < t.nx; ++x) {
          const int cc[3] = {x, y, z};
          const int64_t cell = ccell(x, y, z);
          const int b[3] = {x / t.rb, y / t.rb, z / t.rb};
          const int slot = t.block_slot[bid(b[0], b[1], b[2])];
          if (slot < 0) {
            bool nearc = false;
            for (int i = 1; i < Q; ++i) nearc = nearc || covered(x + T->ex[i], y + T->ey[i], z + T->ez[i]);
            if (!nearc) continue;
            for (int i = 1; i < Q; ++i) {
              const int e[3] = {T->ex[i], T->ey[i], T->ez[i]};
              const int tc[3] = {wrapi(x + e[0], t.nx), wrapi(y + e[1], t.ny), wrapi(z + e[2], t.nz)};
              if (covered(tc[0], tc[1], tc[2])) continue;
              R sacc = 0, nin = 0;
              for (int k = 0; k < 8; ++k) {
                const int o[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
                int pp[3], q[3], qb[3];
                for (int a = 0; a < 3; ++a) {
                  pp[a] = wrapi(tc[a] * 2 + o[a], NF[a]);
                  q[a] = wrapi(pp[a] - e[a], NF[a]);
                  qb[a] = q[a] / RB2;
                }
                const int qs = t.block_slot[bid(qb[0], qb[1], qb[2])];
                if (qs >= 0) {
                  sacc += fpo[i * P + pcell(qs, (int)local_in_tile(pp[0], qb[0], NF[0]),
                                             (int)local_in_tile(pp[1], qb[1], NF[1]),
                                             (int)local_in_tile(pp[2], qb[2], NF[2]))];
                }
                int ch[3];
                for (int a = 0; a < 3; ++a) ch[a] = wrapi(cc[a] * 2 + o[a] + e[a], NF[a]);
                if (covered(ch[0] / 2, ch[1] / 2, ch[2] / 2)) nin += R(1);
              }
              const R net = sacc - nin * fco[i * N + cell];
              if (net != R(0)) out[i * N + cell] = fco[i * N + cell] + net * R(0.125);
            }
            continue;
          }
          // covered: parent mac, then the populations the coarse grid pulls
          R rs = 0, ms[3] = {0, 0, 0};
          for (int k = 0; k < 8; ++k) {
            const int o[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
            const int64_t pc = pcell(slot, GH + 2 * (x - b[0] * t.rb) + o[0], GH + 2 * (y - b[1] * t.rb) + o[1],
                                     GH + 2 * (z - b[2] * t.rb) + o[2]);
            const R rho = R(macp[4 * pc]);
            rs += rho;
            for (int a = 0; a < 3; ++a) ms[a] += rho * R(macp[4 * pc + 1 + a]);
          }
          const R inv = R(1) / std::fmax(rs, R(1e-6));
          macc[4 * cell] = (double)(rs * R(0.125));
          for (int a = 0; a < 3; ++a) macc[4 * cell + 1 + a] = (double)(ms[a] * inv);
          for (int i = 0; i < Q; ++i) {
            const int e[3] = {T->ex[i], T->ey[i], T->ez[i]};
            const int tc[3] = {x + e[0], y + e[1], z + e[2]};
            if (covered(tc[0], tc[1], tc[2])) continue;
            R sacc = 0;
            for (int k = 0; k < 8; ++k) {
              const int o[3] = {k & 1, (k >> 1) & 1, (k >> 2) & 1};
              int l[3];
              for (int a = 0; a < 3; ++a) l[a] = (int)local_in_tile(tc[a] * 2 + o[a], b[a], NF[a]);
              sacc += fpo[i * P + pcell(slot, l[0], l[1], l[2])];
            }
            out[i * N + cell] = sacc * R(0.125);
          }
        }
    fco.swap(out);
  }

  // ---- pool force (common_d3_force_pool.wgsl) -----------------------------
  void force(const std::vector<R> &f, double out[8]) {
    for (int k = 0; k < 8; ++k) out[k] = 0;
    if (!c.has_body) return;
    const lbm_body &bd = c.body;
    const R CS2 = R(1) / R(3);
    for (int s = 0; s < t.slots; ++s) {
      const int id = t.slot_to_block[s];
      if (id < 0) continue;
      const int b[3] = {id % t.nbx, (id / t.nbx) % t.nby, id / (t.nbx * t.nby)};
      for (int fz = GH; fz < GH + RB2; ++fz)
        for (int fy = GH; fy < GH + RB2; ++fy)
          for (int fx = GH; fx < GH + RB2; ++fx) {
            const int64_t cell = pcell(s, fx, fy, fz);
            const V3<R> p{f2c(fx, b[0] * t.rb), f2c(fy, b[1] * t.rb), f2c(fz, b[2] * t.rb)};
            const R phi = phi3(p, bd, &win);
            const V3<R> r = bdelta(p, bd, &win);
            const V3<R> us = body_vel3(p, bd, &win);
            V3<R> fb{0, 0, 0}, fs{0, 0, 0};
            if (c.use_bounceback) {
              if (phi >= R(0)) {
                R rhoW = R(1);
                if (c.rho_w_local && phi < R(2)) {
                  R sum = 0;
                  for (int i = 0; i < Q; ++i) sum += f[i * P + cell];
                  rhoW = sum;
                }
                for (int i = 0; i < Q; ++i) {
                  const V3<R> sp{f2c(fx - T->ex[i], b[0] * t.rb), f2c(fy - T->ey[i], b[1] * t.rb),
                                 f2c(fz - T->ez[i], b[2] * t.rb)};
                  if (phi3(sp, bd, &win) < R(0)) {
                    const R fo = f[T->opp[i] * P + cell];
                    const R corr = R(2) * R(T->w[i]) * rhoW *
                                   (R(T->ex[i]) * us.x + R(T->ey[i]) * us.y + R(T->ez[i]) * us.z) / CS2;
                    const R m = R(2) * fo + corr;
                    fb.x += -R(T->ex[i]) * m; fb.y += -R(T->ey[i]) * m; fb.z += -R(T->ez[i]) * m;
                  }
                }
              }
              if (c.swept_force) {
                const bool now = phi < R(0);
                if (now != (phi3_ahead(p, bd, R(1), &win) < R(0))) {
                  V3<R> mc{0, 0, 0};
                  for (int i = 0; i < Q; ++i) {
                    const R v = f[i * P + cell];
                    mc.x += v * R(T->ex[i]); mc.y += v * R(T->ey[i]); mc.z += v * R(T->ez[i]);
                  }
                  if (!now) fs = mc; else fs = {-mc.x, -mc.y, -mc.z};
                }
              }
            } else {
              const R chi = chi_of(phi, R(c.chi_eps) * R(0.5));
              if (chi >= R(1e-6)) {
                R rho = 0, mx = 0, my = 0, mz = 0;
                for (int i = 0; i < Q; ++i) {
                  const int sx = std::min(std::max(fx - T->ex[i], 0), FB - 1);
                  const int sy = std::min(std::max(fy - T->ey[i], 0), FB - 1);
                  const int sz = std::min(std::max(fz - T->ez[i], 0), FB - 1);
                  const R v = f[i * P + pcell(s, sx, sy, sz)];
                  rho += v; mx += v * R(T->ex[i]); my += v * R(T->ey[i]); mz += v * R(T->ez[i]);
                }
                const R den = std::fmax(rho, R(1e-6));
                fb = {-(rho * chi * (us.x - mx / den)), -(rho * chi * (us.y - my / den)),
                      -(rho * chi * (us.z - mz / den))};
              }
            }
            const V3<R> ft{fb.x * R(0.25) + fs.x * R(0.125), fb.y * R(0.25) + fs.y * R(0.125),
                           fb.z * R(0.25) + fs.z * R(0.125)};
            const R v6[6] = {ft.x, ft.y, ft.z, r.y * ft.z - r.z * ft.y, r.z * ft.x - r.x * ft.z,
                             r.x * ft.y - r.y * ft.x};
            for (int k = 0; k < 6; ++k) {
              if (std::isfinite((double)v6[k])) out[k] += (double)v6[k];
              else out[6] += 1;
            }
          }
    }
  }

  // ---- dynamic refinement (common_d3_manage.wgsl), in f32 as the kernel --
  static bool box_near(const lbm_body &b, const Win *w, float cx, float cy, float cz, float h0, float reach) {
    const float S3 = 1.7320509f;
    const float R0 = h0 * S3;
    const float p0 = phi3<float>({cx, cy, cz}, b, w);
    if (p0 - R0 > reach) return false;
    if (p0 <= reach) return true;
    const float h1 = h0 * 0.5f, R1 = R0 * 0.5f;
    for (int i = 0; i < 8; ++i) {
      const float c1x = cx + ((i & 1) ? h1 : -h1), c1y = cy + ((i & 2) ? h1 : -h1), c1z = cz + ((i & 4) ? h1 : -h1);
      const float p1 = phi3<float>({c1x, c1y, c1z}, b, w);
      if (p1 - R1 > reach) continue;
      if (p1 <= reach) return true;
      const float h2 = h1 * 0.5f, R2 = R1 * 0.5f;
      for (int j = 0; j < 8; ++j) {
        const float c2x = c1x + ((j & 1) ? h2 : -h2), c2y = c1y + ((j & 2) ? h2 : -h2), c2z = c1z + ((j & 4) ? h2 : -h2);
        const float p2 = phi3<float>({c2x, c2y, c2z}, b, w);
        if (p2 - R2 > reach) continue;
        if (p2 <= reach) return true;
        const float h3 = h2 * 0.5f, R3 = R2 * 0.5f;
        for (int k = 0; k < 8; ++k) {
          const float c3x = c2x + ((k & 1) ? h3 : -h3), c3y = c2y + ((k & 2) ? h3 : -h3), c3z = c2z + ((k & 4) ? h3 : -h3);
          if (phi3<float>({c3x, c3y, c3z}, b, w) - R3 <= reach) return true;
        }
      }
    }
    return false;
  }

  // common_d3_amr_average.wgsl: each tile restricted into its L0 cells (feq
  // of the children's mean rho and mass-weighted u plus the F2C-rescaled
  // mean fneq) and their mac; with `want`, only the tiles it no longer wants.
  void restrict_tiles(std::vector<R> &fco, const uint8_t *wanted) {
    const R tc = R(c.tau), tf = R(2) * tc - R(0.5);
    const R f2c = R(2) * (tc - R(1)) / (tf - R(1));
    for (int s = 0; s < t.slots; ++s) {
      const int id = t.slot_to_block[s];
      if (id < 0 || (wanted && wanted[id])) continue;
      const int b3[3] = {id % t.nbx, (id / t.nbx) % t.nby, id / (t.nbx * t.nby)};
      for (int lz = 0; lz < t.rb; ++lz)
        for (int ly = 0; ly < t.rb; ++ly)
          for (int lx = 0; lx < t.rb; ++lx) {
            R rs = 0, ms[3] = {0, 0, 0}, fneq[27] = {};
            for (int k = 0; k < 8; ++k) {
              const int64_t pc = pcell(s, GH + 2 * lx + (k & 1), GH + 2 * ly + ((k >> 1) & 1), GH + 2 * lz + ((k >> 2) & 1));
              R f[27], r = 0, mx = 0, my = 0, mz = 0;
              for (int i = 0; i < Q; ++i) {
                f[i] = fp[0][i * P + pc];
                r += f[i]; mx += f[i] * R(T->ex[i]); my += f[i] * R(T->ey[i]); mz += f[i] * R(T->ez[i]);
              }
              const R den = std::fmax(r, R(1e-6));
              const R u[3] = {mx / den, my / den, mz / den};
              rs += r;
              for (int a = 0; a < 3; ++a) ms[a] += r * u[a];
              for (int i = 0; i < Q; ++i) fneq[i] += f[i] - feq<R>(*T, i, r, u[0], u[1], u[2]);
            }
            const R ra = rs * R(0.125), inv = R(1) / std::fmax(rs, R(1e-6));
            const R ua = ms[0] * inv, va = ms[1] * inv, wa = ms[2] * inv;
            const int64_t dst = ccell(b3[0] * t.rb + lx, b3[1] * t.rb + ly, b3[2] * t.rb + lz);
            for (int i = 0; i < Q; ++i) fco[i * N + dst] = feq<R>(*T, i, ra, ua, va, wa) + f2c * (fneq[i] * R(0.125));
            macc[4 * dst] = (double)ra;
            macc[4 * dst + 1] = (double)ua; macc[4 * dst + 2] = (double)va; macc[4 * dst + 3] = (double)wa;
          }
    }
  }

  // reduceQ: per block, the max of q_cell over its L0 box dilated by `lead`
  // (floor / ceil), read from the coarse mac as the kernel reads it, in f32.
  void reduce_q(float lead, std::vector<float> &out) const {
    out.assign(t.nb, 0.f);
    std::vector<float> mac4((size_t)4 * N);
    for (int64_t i = 0; i < 4 * N; ++i) mac4[i] = (float)macc[i];
    for (int id = 0; id < t.nb; ++id) {
      const int b[3] = {id % t.nbx, (id / t.nbx) % t.nby, id / (t.nbx * t.nby)};
      int i0[3], n[3];
      for (int a = 0; a < 3; ++a) {
        const float lo = (float)b[a] * (float)t.rb - lead;
        const float hi = lo + (float)t.rb + 2.f * lead;
        i0[a] = (int)std::floor(lo);
        n[a] = std::max((int)std::ceil(hi) - i0[a], 0);
      }
      float best = -1e30f;
      for (int kz = 0; kz < n[2]; ++kz)
        for (int ky = 0; ky < n[1]; ++ky)
          for (int kx = 0; kx < n[0]; ++kx)
            best = std::fmax(best, q_cell(mac4.data(), t.nx, t.ny, t.nz, i0[0] + kx, i0[1] + ky, i0[2] + kz));
      out[id] = best;
    }
  }

  void manage() {
    const lbm_body &b = c.body;
    float rc = b.shape == LBM_SHAPE_SPHERE ? b.a : (b.shape == LBM_SHAPE_SPHEROID ? std::fmax(b.a, b.c)
                                                  : std::sqrt(b.a * b.a + b.b * b.b + b.c * b.c));
    const float lead = (float)manage_every * (std::sqrt(b.vx * b.vx + b.vy * b.vy + b.vz * b.vz) +
                                              std::sqrt(b.wx * b.wx + b.wy * b.wy + b.wz * b.wz) * rc);
    const float reach = (float)margin + lead;
    want.assign(t.nb, 0);
    const float half = 0.5f * (float)t.rb;
    for (int id = 0; id < t.nb; ++id) {
      const int bx = id % t.nbx, by = (id / t.nbx) % t.nby, bz = id / (t.nbx * t.nby);
      want[id] = box_near(b, &win, (float)(bx * t.rb) + half, (float)(by * t.rb) + half, (float)(bz * t.rb) + half, half,
                          reach);
    }
    if (q_abs > 0) {
      // the union with the field ladder at one level (common_d3_manage.wgsl
      // decide, common_refine.wgsl desiredLevel / desiredLevelCoarsen):
      // 1/2 log2 max(Q, 1e-30) >= 1/2 log2 max(Q_abs, 1e-30), less q_hyst for
      // a block that holds a tile, compared as Q >= Q_abs 4^-q_hyst
      const double qr = std::max((double)q_abs, 1e-30);
      const float q_refine = (float)qr, q_hold = (float)(qr * std::exp2(-2.0 * (double)q_hyst));
      reduce_q(q_lead, block_q);
      for (int id = 0; id < t.nb; ++id)
        if (!want[id]) want[id] = std::fmax(block_q[id], 1e-30f) >= (t.block_slot[id] >= 0 ? q_hold : q_refine);
    }
    // drain the dying tiles into the time-t L0 buffer
    restrict_tiles(fc[cp], want.data());
    // coarsen then refine over the free-slot stack, ascending block id
    std::fill(slot_new.begin(), slot_new.end(), 0);
    for (int id = 0; id < t.nb; ++id) {
      const int s = t.block_slot[id];
      if (s < 0 || want[id]) continue;
      free_list[free_count++] = s;
      t.block_slot[id] = -1;
      t.slot_to_block[s] = -1;
    }
    for (int id = 0; id < t.nb; ++id) {
      if (t.block_slot[id] >= 0 || !want[id]) continue;
      if (free_count == 0) { ++refused; continue; }
      const int s = free_list[--free_count];
      t.block_slot[id] = s;
      t.slot_to_block[s] = id;
      slot_new[s] = 1;
    }
    min_free = std::min(min_free, free_count);
    ++decisions;
    interp_fill(fc[cp], fp[0], false, true);
  }

  // ---- one macro-step ------------------------------------------------------
  void macro_step(double *force_out, bool want_mac) {
    if (dynamic && step_count >= manage_start && (step_count - manage_start) % manage_every == 0) manage();
    ++step_count;
    if (force_out) force(fp[0], force_out);
    if (interp) {
      // ?interface=interp (main-3d.js:3343-3356): the L0 step first, the ring
      // interpolated from L0 at t, two substeps with the ring collided, the
      // tiles restricted into L0's new buffer
      l0_step(want_mac);
      interp_fill(fc[1 - cp], fp[0], true);
      if (reflux_on) flux(fp[0], flux_acc, false);
      substep(fp[0], fp[1], true);
      if (reflux_on) flux(fp[1], flux_acc, true);
      substep(fp[1], fp[0], true);
      restrict_tiles(fc[cp], nullptr);
      if (reflux_on) reflux(fc[1 - cp], fc[cp], flux_acc);
      return;
    }
    explode(fc[cp], fp[0]);
    substep(fp[0], fp[1], false);
    substep(fp[1], fp[0], false);
    coalesce(fp[0], fc[cp]);
    l0_step(want_mac);
  }

  // The L0 step from parity cp, covered blocks skipped; flips cp.
  void l0_step(bool want_mac) {
    Cover cov;
    cov.block_slot = t.block_slot.data();
    cov.rb = t.rb; cov.nbx = t.nbx; cov.nby = t.nby;
    std::vector<double> mbuf;
    double *m = nullptr;
    if (want_mac) {
      mbuf.assign((size_t)4 * N, 0.0);
      m = mbuf.data();
    }
    step3<R>(c, fc[cp], fc[1 - cp], m, cov);
    if (want_mac) {
      for (int z = 0; z < t.nz; ++z)
        for (int y = 0; y < t.ny; ++y)
          for (int x = 0; x < t.nx; ++x) {
            if (covered(x, y, z)) continue;
            const int64_t cell = ccell(x, y, z);
            for (int k = 0; k < 4; ++k) macc[4 * cell + k] = mbuf[4 * cell + k];
          }
    }
    cp = 1 - cp;
  }
};

template <class R>
Amr3D<R> *make(const lbm_config &c, int rb, int mode, double margin, double frac, const int32_t *list, int linear,
               int capacity, int dynamic, int manage_every, int manage_start, int interp) {
  auto *a = new Amr3D<R>();
  a->c = c;
  a->win = window_of(c);
  a->Q = c.q;
  a->T = &tables(c.q);
  a->t.nx = c.nx; a->t.ny = c.ny; a->t.nz = c.nz; a->t.rb = rb;
  a->t.nbx = c.nx / rb; a->t.nby = c.ny / rb; a->t.nbz = c.nz / rb;
  a->t.nb = a->t.nbx * a->t.nby * a->t.nbz;
  refine(a->t, mode, c.body, margin, frac, list);
  if (capacity > a->t.slots) {
    a->t.slot_to_block.resize(capacity, -1);
    a->t.slots = capacity;
  }
  a->dynamic = dynamic;
  a->interp = interp & 1;
  a->reflux_on = (interp >> 1) & 1;
  a->flux_acc.assign((size_t)4 * a->t.nx * a->t.ny * a->t.nz, R(0));
  a->manage_every = manage_every;
  a->manage_start = manage_start;
  a->margin = margin;
  a->free_count = a->t.slots - a->t.initial;
  a->min_free = a->free_count;
  a->free_list.assign(std::max(1, a->t.slots), 0);
  for (int i = 0; i < a->free_count; ++i) a->free_list[i] = a->t.initial + i;
  a->slot_new.assign(a->t.slots, 0);
  a->FB = 2 * rb + 2 * GH;
  a->RB2 = 2 * rb;
  a->T3 = a->FB * a->FB * a->FB;
  a->N = (int64_t)c.nx * c.ny * c.nz;
  a->P = (int64_t)a->t.slots * a->T3;
  a->tau_f = R(2) * R(c.tau) - R(0.5);
  a->linear = linear;
  return a;
}

struct Handle {
  int fp32;
  void *p;
};

}  // namespace

extern "C" {

// Builds the two-level hierarchy (topology only; oracle_amr3d_seed fills it).
void *oracle_amr3d_create(const lbm_config *c, int rb, int mode, double margin, double frac, const int32_t *list,
                          int linear, int fp32, int capacity, int dynamic, int manage_every, int manage_start,
                          int interp) {
  if (!c || c->q == 9 || rb < 1 || c->nx % rb || c->ny % rb || c->nz % rb) return nullptr;
  auto *h = new Handle{fp32, nullptr};
  if (fp32)
    h->p = make<float>(*c, rb, mode, margin, frac, list, linear, capacity, dynamic, manage_every, manage_start, interp);
  else
    h->p = make<double>(*c, rb, mode, margin, frac, list, linear, capacity, dynamic, manage_every, manage_start, interp);
  return h;
}

void oracle_amr3d_destroy(void *hp) {
  auto *h = (Handle *)hp;
  if (!h) return;
  if (h->fp32) delete (Amr3D<float> *)h->p; else delete (Amr3D<double> *)h->p;
  delete h;
}

#define WITH(h, ...)                                    \
  do {                                                  \
    if (((Handle *)(h))->fp32) {                        \
      auto *a = (Amr3D<float> *)((Handle *)(h))->p;     \
      __VA_ARGS__;                                      \
    } else {                                            \
      auto *a = (Amr3D<double> *)((Handle *)(h))->p;    \
      __VA_ARGS__;                                      \
    }                                                   \
  } while (0)

// {in use, refusals, lowest free count, decisions}
int oracle_amr3d_pool_stats(void *h, int32_t out[4]) {
  WITH(h, {
    out[0] = a->t.slots - a->free_count;
    out[1] = a->refused;
    out[2] = a->min_free;
    out[3] = a->decisions;
  });
  return 0;
}

// Replaces the body pose (a prescribed motion).
int oracle_amr3d_set_body(void *h, const lbm_body *b) {
  WITH(h, a->c.body = *b);
  return 0;
}

// Topology: block_slot (nb), slot_to_block (slots); returns the slot count.
int oracle_amr3d_topology(void *h, int32_t *block_slot, int32_t *slot_to_block) {
  int n = 0;
  WITH(h, {
    if (block_slot) std::memcpy(block_slot, a->t.block_slot.data(), a->t.nb * sizeof(int32_t));
    if (slot_to_block) std::memcpy(slot_to_block, a->t.slot_to_block.data(), a->t.slots * sizeof(int32_t));
    n = a->t.slots;
  });
  return n;
}

// The field criterion of the manager: Q_abs (0 = off), hysteresis in
// octaves of rotation rate, lead in L0 cells.
int oracle_amr3d_set_q(void *h, float q_abs, float q_hyst, float q_lead) {
  WITH(h, {
    a->q_abs = q_abs;
    a->q_hyst = q_hyst;
    a->q_lead = q_lead;
  });
  return 0;
}

// Per-block max Q of the current coarse mac with the box dilated by `lead`.
int oracle_amr3d_block_q(void *h, float lead, float *out) {
  WITH(h, {
    std::vector<float> q;
    a->reduce_q(lead, q);
    std::memcpy(out, q.data(), q.size() * sizeof(float));
  });
  return 0;
}

// Q at every cell of an nx*ny*nz field of [rho, ux, uy, uz] (f32, periodic).
int oracle_q_cells(int nx, int ny, int nz, const float *mac, float *q) {
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) q[((int64_t)z * ny + y) * nx + x] = q_cell(mac, nx, ny, nz, x, y, z);
  return 0;
}

// qOfGrad (d3-criterion.mjs) in FP64 on a 3x3 gradient J[i][j] = du_i/dx_j.
double oracle_q_of_grad(const double *J) {
  double om2 = 0, s2 = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double S = 0.5 * (J[3 * i + j] + J[3 * j + i]), O = 0.5 * (J[3 * i + j] - J[3 * j + i]);
      s2 += S * S;
      om2 += O * O;
    }
  return 0.5 * (om2 - s2);
}

int oracle_amr3d_seed(void *h, const double *mac) {
  WITH(h, a->seed(mac));
  return 0;
}

// `n` macro-steps; forces (8 per step) and the last step's coarse mac kept.
int oracle_amr3d_step(void *h, int n, double *forces) {
  WITH(h, {
    for (int k = 0; k < n; ++k) a->macro_step(forces ? forces + 8 * k : nullptr, true);
  });
  return 0;
}

// Coarse f of the current time level (Q*N), coarse mac (4*N, [rho,u] per
// cell), pool f (Q*P, slot-major planes) and pool mac (4*P); any may be NULL.
int oracle_amr3d_read(void *h, double *fc, double *macc, double *fp, double *macp) {
  WITH(h, {
    const int64_t QN = (int64_t)a->Q * a->N, QP = (int64_t)a->Q * a->P;
    if (fc) for (int64_t i = 0; i < QN; ++i) fc[i] = (double)a->fc[a->cp][i];
    if (macc) std::memcpy(macc, a->macc.data(), 4 * a->N * sizeof(double));
    if (fp) for (int64_t i = 0; i < QP; ++i) fp[i] = (double)a->fp[0][i];
    if (macp) std::memcpy(macp, a->macp.data(), 4 * a->P * sizeof(double));
  });
  return 0;
}

}  // extern "C"
