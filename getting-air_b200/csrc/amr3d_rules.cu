// Host rules of the 3D hierarchy: which blocks a configuration refines
// (d3-amr.mjs refineWhere / nearBodyWant and the box, bar, slab and all
// predicates of main-3d.js:450-480) and where a tile-local source index
// lives (resolveSource, d3-amr.mjs:178-200). FP64, as the reference's host
// code.
#include <cmath>
#include <cstring>

#include "../../include/lbm.h"
#include "amr3d.cuh"

namespace lbm {

namespace {

struct D3 {
  double x, y, z;
};

D3 rot_inv(const lbm_body &b, D3 v) {
  // conj(q) (0, v) q, [w, x, y, z]
  const double w = b.qw, x = -(double)b.qx, y = -(double)b.qy, z = -(double)b.qz;
  const double tw = -x * v.x - y * v.y - z * v.z;
  const double tx = w * v.x + y * v.z - z * v.y;
  const double ty = w * v.y - x * v.z + z * v.x;
  const double tz = w * v.z + x * v.y - y * v.x;
  const double qw = b.qw, qx = b.qx, qy = b.qy, qz = b.qz;
  return {tw * qx + tx * qw + ty * qz - tz * qy, tw * qy - tx * qz + ty * qw + tz * qx,
          tw * qz + tx * qy - ty * qx + tz * qw};
}

double sd_spheroid(D3 p, double a, double c) {
  const double r0 = std::hypot(p.x, p.y);
  if (std::fabs(a - c) <= 1e-6 * std::fmax(a, c)) return std::hypot(r0, p.z) - a;
  const double x = std::fabs(r0), y = std::fabs(p.z);
  const bool inside = std::sqrt(x * x / (a * a) + y * y / (c * c)) < 1;
  double t = std::atan2(y * a, x * c);
  for (int i = 0; i < 3; ++i) {
    const double ct = std::cos(t), st = std::sin(t);
    const double ex = x - a * ct, ey = y - c * st;
    const double F = ex * (-a * st) + ey * (c * ct);
    const double Fp = -(a * a * st * st + c * c * ct * ct) + ex * (-a * ct) + ey * (-c * st);
    t -= F / (std::fabs(Fp) < 1e-9 ? -1e-9 : Fp);
    t = std::fmin(std::fmax(t, 0.0), M_PI / 2);
  }
  const double d = std::hypot(x - a * std::cos(t), y - c * std::sin(t));
  return inside ? -d : d;
}

// d3-body.mjs sdfBody at a world point.
double sdf_world(const lbm_body &b, D3 w) {
  const D3 p = rot_inv(b, {w.x - b.cx, w.y - b.cy, w.z - b.cz});
  switch (b.shape) {
    case LBM_SHAPE_SPHERE: return std::sqrt(p.x * p.x + p.y * p.y + p.z * p.z) - b.a;
    case LBM_SHAPE_SPHEROID: return sd_spheroid(p, b.a, b.c);
    default: {
      const double qx = std::fabs(p.x) - (b.a - b.r), qy = std::fabs(p.y) - (b.b - b.r),
                   qz = std::fabs(p.z) - (b.c - b.r);
      const double out = std::sqrt(std::pow(std::fmax(qx, 0.0), 2) + std::pow(std::fmax(qy, 0.0), 2) +
                                   std::pow(std::fmax(qz, 0.0), 2));
      return out + std::fmin(std::fmax(qx, std::fmax(qy, qz)), 0.0) - b.r;
    }
  }
}

// nearBodyWant: phi(c) - h sqrt(3) <= min over the box <= phi(c); split the
// undecided boxes into octants, three levels deep, accepting at the bottom.
// sqrt(3) is rounded up, as the reference's SQRT3_UP.
bool near_box(const lbm_body &b, D3 c, double h, int depth, double margin) {
  const double R = h * 1.7320509;
  const double phi = sdf_world(b, c);
  if (phi - R > margin) return false;
  if (phi <= margin) return true;
  if (depth == 0) return true;
  const double hh = h / 2;
  for (int i = 0; i < 8; ++i) {
    const D3 cc = {c.x + ((i & 1) ? hh : -hh), c.y + ((i & 2) ? hh : -hh), c.z + ((i & 4) ? hh : -hh)};
    if (near_box(b, cc, hh, depth - 1, margin)) return true;
  }
  return false;
}

}  // namespace

int amr3_validate(const lbm_amr3d_config *c, std::string &why) {
  if (!c) { why = "config is NULL"; return LBM_EINVAL; }
  const lbm_config &r = c->root;
  if (r.q != 19 && r.q != 27) { why = "3D AMR runs D3Q19 or D3Q27"; return LBM_EINVAL; }
  if (r.storage != LBM_STORE_FP32) { why = "3D AMR stores FP32 populations"; return LBM_ENOTSUP; }
  if (c->levels != 2) { why = "levels must be 2 (one pool level)"; return LBM_ENOTSUP; }
  if (c->rb < 2 || c->rb > kMaxAmrRb) { why = "rb must be in [2, 8]"; return LBM_EINVAL; }
  if (r.nx % c->rb || r.ny % c->rb || r.nz % c->rb) { why = "every dimension must be a multiple of rb"; return LBM_EINVAL; }
  if (c->refine < LBM_REFINE_BODY || c->refine > LBM_REFINE_LIST) { why = "unknown refine mode"; return LBM_EINVAL; }
  if (c->iface != 0 && c->iface != 1) { why = "iface must be 0 (explode/coalesce) or 1 (interp)"; return LBM_EINVAL; }
  if (c->reflux) {
    if (c->iface != 1) { why = "reflux needs the interp interface: explode/coalesce is conservative by construction"; return LBM_EINVAL; }
    if (r.wall[0] || r.wall[1] || r.wall[2]) { why = "reflux is not valid with walls"; return LBM_EINVAL; }
    if (r.nx / c->rb < 3 || r.ny / c->rb < 3 || r.nz / c->rb < 3) { why = "reflux needs at least 3 blocks per axis"; return LBM_EINVAL; }
  }
  if (!std::isfinite(c->q_abs) || c->q_abs < 0 || !std::isfinite(c->q_hyst) || !std::isfinite(c->q_lead) ||
      c->q_lead < 0) {
    why = "q_abs and q_lead must be finite and >= 0, q_hyst finite";
    return LBM_EINVAL;
  }
  if (c->q_abs > 0 && !c->dynamic) {
    why = "the Q-criterion needs dynamic refinement: a set chosen once at start would refine a flow that has not "
          "developed yet";
    return LBM_EINVAL;
  }
  if (c->refine == LBM_REFINE_BODY && !r.has_body) { why = "refine = body needs a body"; return LBM_EINVAL; }
  if (std::fabs(r.tau - 1.0f) < 1e-3f) {
    why = "tau = 1 leaves no non-equilibrium part for the coarse/fine transfer to rescale";
    return LBM_EINVAL;
  }
  return LBM_OK;
}

void amr3_want(const lbm_amr3d_config &c, const uint8_t *list, std::vector<uint8_t> &want) {
  const lbm_config &r = c.root;
  const int rb = c.rb, nbx = r.nx / rb, nby = r.ny / rb, nbz = r.nz / rb;
  const double dims[3] = {(double)r.nx, (double)r.ny, (double)r.nz};
  const double f = c.boxfrac;
  want.assign((size_t)nbx * nby * nbz, 0);
  for (int id = 0; id < nbx * nby * nbz; ++id) {
    const int bx = id % nbx, by = (id / nbx) % nby, bz = id / (nbx * nby);
    const double mid[3] = {bx * rb + rb / 2.0, by * rb + rb / 2.0, bz * rb + rb / 2.0};
    auto in = [&](int a) { return mid[a] >= dims[a] * (1 - f) / 2 && mid[a] < dims[a] * (1 + f) / 2; };
    bool w = false;
    switch (c.refine) {
      case LBM_REFINE_ALL: w = true; break;
      case LBM_REFINE_BOX: w = in(0) && in(1) && in(2); break;
      case LBM_REFINE_BAR: w = in(0) && in(1); break;
      case LBM_REFINE_SLAB: w = in(0); break;
      case LBM_REFINE_BODY: w = near_box(r.body, {mid[0], mid[1], mid[2]}, rb / 2.0, 3, c.margin); break;
      case LBM_REFINE_LIST: w = list && list[id]; break;
    }
    want[id] = w ? 1 : 0;
  }
}

}  // namespace lbm

extern "C" {

int lbm_amr3d_refine_blocks(const lbm_amr3d_config *c, uint8_t *want) {
  std::string why;
  if (lbm::amr3_validate(c, why) || !want) return LBM_EINVAL;
  if (c->refine == LBM_REFINE_LIST) return LBM_EINVAL;
  std::vector<uint8_t> w;
  lbm::amr3_want(*c, nullptr, w);
  std::memcpy(want, w.data(), w.size());
  return LBM_OK;
}

int lbm_resolve_source(int rb, const int32_t nb[3], const int32_t *block_slot, const int32_t block[3],
                       const int32_t src[3], int32_t out[4]) {
  if (rb < 1 || !nb || !block_slot || !block || !src || !out) return LBM_EINVAL;
  const int RB2 = 2 * rb, G = lbm::kAmrGhost;
  int o[3], nbr[3];
  for (int a = 0; a < 3; ++a) {
    const int s = src[a];
    if (s < G) { nbr[a] = -1; o[a] = s + RB2; }
    else if (s >= G + RB2) { nbr[a] = 1; o[a] = s - RB2; }
    else { nbr[a] = 0; o[a] = s; }
  }
  out[1] = o[0]; out[2] = o[1]; out[3] = o[2];
  if (!nbr[0] && !nbr[1] && !nbr[2]) { out[0] = -1; return LBM_OK; }
  int b[3];
  for (int a = 0; a < 3; ++a) b[a] = ((block[a] + nbr[a]) % nb[a] + nb[a]) % nb[a];
  const int slot = block_slot[(b[2] * nb[1] + b[1]) * nb[0] + b[0]];
  out[0] = slot < 0 ? -2 : slot;
  return LBM_OK;
}

}  // extern "C"
