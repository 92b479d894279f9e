// Host entry points of the rigid-body integrator (the library's host twin
// of d3-body.mjs): the same functions the device runs after each force pass
// of a free body, compiled for the host.
#include <cmath>

#include "../../include/lbm.h"
#include "body.cuh"

extern "C" {

void lbm_body_opts_default(lbm_body_opts *o) {
  if (!o) return;
  *o = lbm_body_opts{};
  o->v_max = 0.2;
  o->o_max = 0.1;
}

int lbm_body_state_make(const lbm_body *pose, double density, lbm_body_state *out) {
  if (!pose || !out) return LBM_EINVAL;
  if (pose->shape < LBM_SHAPE_SPHERE || pose->shape > LBM_SHAPE_ROUNDBOX) return LBM_EINVAL;
  if (!(pose->a > 0.f) || !(density > 0.0) || !std::isfinite(density)) return LBM_EINVAL;
  if (pose->shape == LBM_SHAPE_SPHEROID && !(pose->c > 0.f)) return LBM_EINVAL;
  if (pose->shape == LBM_SHAPE_ROUNDBOX && !(pose->b > 0.f && pose->c > 0.f)) return LBM_EINVAL;
  *out = lbm_body_state{};
  lbm::body_state_make(*pose, density, *out);
  return LBM_OK;
}

int lbm_body_advance(lbm_body_state *s, const double force[3], const double torque[3], const lbm_body_opts *o,
                     int nsteps) {
  if (!s || !o || nsteps < 0) return LBM_EINVAL;
  if (!(s->mass > 0.0) || !(s->ibody[0] > 0.0) || !(s->ibody[1] > 0.0) || !(s->ibody[2] > 0.0)) return LBM_EINVAL;
  const double zero[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < nsteps; ++k) lbm::body_step(*s, force ? force : zero, torque ? torque : zero, *o);
  return LBM_OK;
}

}  // extern "C"
