// Host-side translation of an lbm_config into the kernels' StepParams, and
// the box of cells that can contribute to the body force. Shared by the
// dense session, the batch and the server, so every form steps a domain
// with the same constants.
#pragma once

#include <string>

#include "../../include/lbm.h"
#include "dense.cuh"

namespace lbm {

// Checks a configuration the way the reference throws (returns LBM_EINVAL
// and a message).
int validate_config(const lbm_config *c, std::string &why);

// Fills every physics field of `p` for a domain of `c` stored at arena
// index `base` in an arena of plane stride `n`. Reduction pointers and
// regions are left for the caller.
void fill_step_params(const lbm_config &c, int64_t n, int64_t base, StepParams &p);

// Cell box [x0,x1]x[y0,y1]x[z0,z1] (inclusive) outside which no cell can
// contribute to the body force; also sets p.swept / p.swept_band. Returns
// false when the body has no cell in the domain (force off).
bool force_cell_box(const lbm_config &c, StepParams &p, int box[6]);

// The body's regions of a dense step, from force_cell_box(): the reach box
// p.nbox of a 3D bounce-back body (cells outside it are beyond every link,
// so the step skips the SDF there; an empty box when the body has no cell
// in the domain), and with `force` the launch blocks that reduce the force
// (p.rb*). Returns p.force_on.
bool set_body_regions(const lbm_config &c, StepParams &p, bool force);

float lattice_weight(int q, int i);

// 16-bit storage encoding of a domain (far-field equilibrium offsets).
Pack make_pack(const lbm_config &c);

}  // namespace lbm
