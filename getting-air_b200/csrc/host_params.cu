// Host-side parameter translation shared by every form of the solver.
#include <cmath>

#include "host_params.cuh"
#include "lattice.cuh"

namespace lbm {

namespace {
template <int Q> float weight(int i) { return Lattice<Q>::w(i); }
void dir_of(int q, int i, int &ex, int &ey, int &ez) {
  if (q == 9) { ex = Lattice<9>::ex(i); ey = Lattice<9>::ey(i); ez = 0; }
  else { ex = Lattice<27>::ex(i); ey = Lattice<27>::ey(i); ez = Lattice<27>::ez(i); }
}
}  // namespace

float lattice_weight(int q, int i) {
  return q == 9 ? weight<9>(i) : (q == 19 ? weight<19>(i) : weight<27>(i));
}

int validate_config(const lbm_config *c, std::string &why) {
  if (!c) { why = "config is NULL"; return LBM_EINVAL; }
  if (c->q != 9 && c->q != 19 && c->q != 27) { why = "q must be 9, 19 or 27"; return LBM_EINVAL; }
  if (c->nx < 3 || c->ny < 3 || c->nz < 1) { why = "grid must be at least 3 cells per axis"; return LBM_EINVAL; }
  if (c->q == 9 && c->nz != 1) { why = "D2Q9 requires nz == 1"; return LBM_EINVAL; }
  if (c->q != 9 && c->nz < 3) { why = "3D lattices need nz >= 3"; return LBM_EINVAL; }
  if (c->ny > 65535 || c->nz > 65535) { why = "ny and nz are limited to 65535"; return LBM_EINVAL; }
  const int64_t n = (int64_t)c->nx * c->ny * c->nz;
  if (n > 0x7fffffffLL) { why = "grid exceeds 2^31-1 cells"; return LBM_EINVAL; }
  if (!(c->tau > 0.5f) || !std::isfinite(c->tau)) { why = "tau must be finite and > 0.5"; return LBM_EINVAL; }
  if (c->storage < 0 || c->storage > 2) { why = "unknown storage"; return LBM_EINVAL; }
  if (c->trt != 0 && c->trt != 1) { why = "trt must be 0 or 1"; return LBM_EINVAL; }
  if (c->trt) {
    // plans/TRT.md sec 8.0(7): the 2D solver stays BGK
    if (c->q == 9) { why = "the TRT collision is 3D (the D2Q9 solver stays BGK)"; return LBM_EINVAL; }
    if (!(c->trt_lambda > 0.f) || !std::isfinite(c->trt_lambda)) {
      why = "trt_lambda must be finite and > 0";
      return LBM_EINVAL;
    }
  }
  if (c->has_body) {
    const int sh = c->body.shape;
    if (c->q == 9 && sh != LBM_SHAPE_ELLIPSE) { why = "D2Q9 bodies are ellipses"; return LBM_EINVAL; }
    if (c->q != 9 && (sh < 0 || sh > 2)) { why = "3D body shape must be sphere, spheroid or roundbox"; return LBM_EINVAL; }
    if (!(c->body.a > 0.f)) { why = "body size must be positive"; return LBM_EINVAL; }
    if (!c->use_bounceback && !(c->chi_eps > 0.f)) { why = "chi_eps must be positive"; return LBM_EINVAL; }
  }
  // the moving window's refusals (main-3d.js:316-348)
  const bool win = c->window[0] || c->window[1] || c->window[2];
  for (int a = 0; a < 3; ++a)
    if (c->window[a] != 0 && c->window[a] != 1) { why = "window flags must be 0 or 1"; return LBM_EINVAL; }
  if (win) {
    if (c->q == 9) { why = "the moving window is 3D (the D2Q9 body already takes the nearest image)"; return LBM_EINVAL; }
    if (!c->has_body) { why = "the moving window needs a body to follow"; return LBM_EINVAL; }
    for (int a = 0; a < 3; ++a)
      if (c->window[a] && c->wall[a]) {
        why = "the moving window needs a periodic axis for the body to cross: no wall on a windowed axis";
        return LBM_EINVAL;
      }
    if (!(c->sponge_w > 0.f)) {
      why = "the moving window needs a sponge: without one the wake wraps around the periodic buffer";
      return LBM_EINVAL;
    }
  }
  return LBM_OK;
}

Pack make_pack(const lbm_config &c) {
  Pack k{};
  const float ux = c.sponge_u[0], uy = c.sponge_u[1], uz = c.q == 9 ? 0.f : c.sponge_u[2];
  const float usq = c.q == 9 ? (ux * ux + uy * uy) : (ux * ux + uy * uy + uz * uz);
  for (int i = 0; i < c.q; ++i) {
    int ex, ey, ez;
    dir_of(c.q, i, ex, ey, ez);
    const float eu = (float)ex * ux + (float)ey * uy + (float)ez * uz;
    k.off[i] = lattice_weight(c.q, i) * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq);
  }
  k.scale = c.storage == LBM_STORE_FP16 ? kF16Scale : 1.0f;
  k.inv = 1.0f / k.scale;
  for (int i = 0; i < 27; ++i) k.noff[i] = -k.off[i] * k.scale;
  return k;
}

void fill_step_params(const lbm_config &c, int64_t n, int64_t base, StepParams &p) {
  p.nx = c.nx; p.ny = c.ny; p.nz = c.nz; p.n = n; p.base = base;
  p.zoff = 0; p.nzg = c.nz; p.zlo = 0;
  p.omega = 1.0f / c.tau;
  // TRT: omega_- from tau_- = 1/2 + Lambda / (tau - 1/2), both in double and
  // rounded once to f32 as the reference's OMEGA_M override is; the kernels
  // take the difference (the delta form, plans/TRT.md sec 8.0(1)).
  p.trt_dw = 0.f;
  if (c.trt) {
    const float omega_m = (float)(1.0 / lbm_trt_tau_minus((double)c.tau, (double)c.trt_lambda));
    p.trt_dw = omega_m - p.omega;
  }
  p.fx = c.force[0]; p.fy = c.force[1]; p.fz = c.q == 9 ? 0.f : c.force[2];
  p.wall_x = c.q == 9 ? 0 : c.wall[0];
  p.wall_y = c.wall[1];
  p.wall_z = c.q == 9 ? 0 : c.wall[2];
  p.wall_u0 = c.wall_u[0]; p.wall_u1 = c.wall_u[1];
  p.has_body = c.has_body; p.bb = c.use_bounceback; p.solid_eq = c.solid_eq;
  p.rho_w_local = c.rho_w_local;
  p.chi_eps = c.chi_eps;
  p.sponge_w = c.sponge_w;
  p.sponge_inv = c.sponge_w > 0.f ? 1.0f / c.sponge_w : 0.f;
  p.sax = c.sponge_axis[0]; p.say = c.sponge_axis[1]; p.saz = c.sponge_axis[2];
  const float ux = c.sponge_u[0], uy = c.sponge_u[1], uz = c.q == 9 ? 0.f : c.sponge_u[2];
  const float ufar = c.q == 9 ? (ux * ux + uy * uy) : (ux * ux + uy * uy + uz * uz);
  for (int i = 0; i < 27; ++i) p.ftarget[i] = 0.f;
  for (int i = 0; i < c.q; ++i) {
    int ex, ey, ez;
    dir_of(c.q, i, ex, ey, ez);
    const float eu = (float)ex * ux + (float)ey * uy + (float)ez * uz;
    p.ftarget[i] = lattice_weight(c.q, i) * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * ufar);
  }
  p.pk = make_pack(c);
  p.body = c.body;
  p.win = Win{};
  if (c.q != 9) {
    const int len[3] = {c.nx, c.ny, c.nz};
    for (int a = 0; a < 3; ++a)
      if (c.window[a]) {
        p.win.n[a] = (float)len[a];
        p.win.anchor[a] = (float)c.win_anchor[a];
        p.win.on = 1;
      }
  }
  p.nbox_on = 0;
  p.write_mac = 0;
  p.force_on = 0;
  p.swept = 0;
  p.swept_band = 0.f;
  p.groups = nullptr;
  p.defer_force = 0;
  p.prev_parts = 0;
  p.prev_partials = nullptr;
}

bool force_cell_box(const lbm_config &c, StepParams &p, int box[6]) {
  if (!c.has_body) return false;
  return body_cell_box(c.body, c.q, c.nx, c.ny, c.nz, c.use_bounceback, c.swept_force, c.chi_eps, box, &p.swept,
                       &p.swept_band, c.q != 9 ? c.window : nullptr);
}

bool set_body_regions(const lbm_config &c, StepParams &p, bool force) {
  int box[6];
  const bool any = force_cell_box(c, p, box);
  p.nbox_on = 0;
  if (c.q != 9 && c.has_body && c.use_bounceback) {
    const int len[3] = {c.nx, c.ny, c.nz};
    p.nbox_on = 1;
    for (int a = 0; a < 3; ++a) {
      if (!any) {  // no cell within reach: an empty box
        p.nbox[2 * a] = 0;
        p.nbox[2 * a + 1] = -1;
        continue;
      }
      int lo = box[2 * a] % len[a];
      if (lo < 0) lo += len[a];
      p.nbox[2 * a] = lo;
      p.nbox[2 * a + 1] = lo + (box[2 * a + 1] - box[2 * a]);
    }
  }
  p.force_on = (force && any) ? 1 : 0;
  if (!p.force_on) return false;
  int r[6];
  box_region(box, p.nx, p.ny, p.nz, nullptr, r);
  p.rbx0 = r[0]; p.rbx1 = r[1];
  p.rby0 = r[2]; p.rby1 = r[3];
  p.rbz0 = r[4]; p.rbz1 = r[5];
  return true;
}

}  // namespace lbm
