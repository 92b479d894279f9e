// Device-side layout and host rules of the 3D two-level hierarchy.
//
// L0 is a dense grid (f planes of N cells, as the dense solver). The pool
// holds one tile per refined block: FB^3 cells, FB = 2 RB + 2 GHOST, slot-
// major, cell (fz*FB + fy)*FB + fx, planes of stride P = capacity * FB^3
// (d3-amr.mjs makePool / cellIndex). A tile-local index j maps to the L0
// position origin - 1/4 + (j - GHOST)/2 (fineToCoarseUnit).
#pragma once

#include <string>
#include <vector>

#include "../../include/lbm.h"
#include "dense.cuh"

namespace lbm {

constexpr int kAmrGhost = 2;
// words per tile cell in the substep's pull table: Q rounded up to a multiple of 4
constexpr int pull_words(int q) { return (q + 3) & ~3; }
constexpr int kTileThreads = 128;    // 1D pool kernels (force, drain, coalesce)
constexpr int kMaxAmrRb = 8;         // tiles up to FB = 20: FB x FB threads per CTA
constexpr int kTileMaxThreads = (2 * kMaxAmrRb + 4) * (2 * kMaxAmrRb + 4);

struct Amr3Params {
  int nx, ny, nz, rb, nbx, nby, nbz;
  int FB, RB2, T3;              // tile edge, interior edge, cells per tile
  int64_t N, P;                 // L0 cells; pool plane stride
  int slots;                    // tile kernels' grid: slots 0 .. slots-1 (unused ones exit)
  const int *block_slot;        // per block: its slot, or -1
  const int *slot_to_block;     // per slot: its block, or -1
  const int *iface;             // blocks the coalesce visits, ascending (static topology)
  int n_iface;                  // ... or, with iface == NULL, every block with iface_flag set
  const unsigned char *iface_flag;
  float omega_f;                // fine BGK rate, 1 / (2 tau - 1/2)
  float rescale_c2f;            // 0.5 (tau_f - 1) / (tau_c - 1)
  float chi_eps_f;              // the chi band on the fine level (CHI_EPS / 2)
  int linear;                   // linear explosion
  int collide_ring;             // interp interface: the ring collides (COLLIDE_RING = 1)
  int write_mac;
  double *partials;             // pool force: 8 doubles per force CTA
  unsigned int *counter;
  double *force_out;
  StepParams c;                 // L0 physics (body, forcing, sponge, far field)
  const uint32_t *links;        // bounce-back link code per pool cell (pinned body), or NULL
  const uint32_t *pulls;        // substep pull sources per (direction, tile cell list position)
};

int amr3_validate(const lbm_amr3d_config *c, std::string &why);
void amr3_want(const lbm_amr3d_config &c, const uint8_t *list, std::vector<uint8_t> &want);

}  // namespace lbm
