// Launch parameters and entry points of the dense-grid kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/lbm.h"
#include "body.cuh"

namespace lbm {

// How 16-bit storage encodes a population: s = (f - off[i]) * scale, stored
// rounded to nearest even; f = s * inv + off[i]. off[i] is the equilibrium of
// the domain's far field, feq_i(rho = 1, u = U_far) (f-pack mode 2 with the
// rest state replaced by the free stream: the stored value is the flow's
// deviation from it), and scale = 2^10 for FP16 keeps small deviations out
// of the subnormal range. Unused by FP32 storage.
// noff[i] = -off[i] * scale (exact: scale is a power of two), so that the
// encode is one fused multiply-add, fma(f, scale, noff[i]) = (f - off) *
// scale to the bit.
constexpr float kF16Scale = 1024.0f;  // 2^10, the FP16 storage scale
struct Pack {
  float off[27];
  float noff[27];
  float scale, inv;
};

// Per-step constants of the fused stream-collide kernels. Mirrors the
// override constants of common_d3_step.wgsl:125-213 / lbm_step.wgsl:36-135.
struct StepParams {
  int nx, ny, nz;       // stored extent (a slab's nz counts its two ghost planes)
  // A z-slab of a larger domain (lbm_create_slab): stored plane z is the
  // domain's plane z + zoff, the domain is nzg planes deep, and the step
  // covers the stored planes [zlo, nz - zlo) (zlo = 1: the ghost planes
  // below and above are filled by the halo exchange). A whole domain has
  // zoff = 0, nzg = nz, zlo = 0.
  int zoff, nzg, zlo;
  int64_t n;            // plane stride of the arena the domain lives in (cells)
  int64_t base;         // arena index of the domain's cell 0
  float omega;          // 1 / tau
  float trt_dw;         // omega_- - omega of the TRT collision; 0 = BGK
  float fx, fy, fz;     // uniform Guo body force
  int wall_x, wall_y, wall_z;
  float wall_u0, wall_u1;  // D2Q9 moving y-walls
  int has_body, bb, solid_eq, rho_w_local, swept;
  float swept_band;     // |phi| below which a cell can change hands in one step
  float chi_eps;
  float sponge_w, sponge_inv;  // band width and its reciprocal
  int sax, say, saz;
  float ftarget[27];    // sponge far-field equilibrium per direction (rho = 1)
  lbm_body body;
  Win win;              // moving window (3D); win.on = 0 without one
  // Bounce-back body only: the cell box (read modulo the grid) outside which
  // no cell is within a link of the body, so the SDF and the body velocity
  // need not be evaluated there (nbox_on = 0: evaluate everywhere).
  int nbox_on;
  int nbox[6];
  int write_mac;
  // Force reduction: the blocks of the launch grid that can see the body.
  int force_on;
  int rbx0, rbx1, rby0, rby1, rbz0, rbz1;
  double *partials;        // 8 doubles per region block
  unsigned int *counter;   // last-block ticket, returns to 0 after each step
  double *force_out;       // 8 doubles: fx fy fz tx ty tz nonfinite 0
  // Dense steps sum their partials after the launch (sum_partials_grouped,
  // with `counter` as its ticket and `groups` as its first-level sums): with
  // defer_force = 0 launch_step() follows the step with a launch that does
  // it; with defer_force = 1 it is left to the next launch on the stream,
  // whose first blocks sum the prev_parts partials at prev_partials.
  double *groups;
  int defer_force;
  int prev_parts;
  const double *prev_partials;
  Pack pk;                 // 16-bit storage encoding
  // Multi-domain launches: the domain's first tile, and the tile range
  // [ft0, ft1) (relative to tile0) whose cells can see the body.
  int tile0, ft0, ft1;
  // Free body (dense 3D only; all NULL otherwise): the pose this launch
  // reads (and for a force pass, the pose its last block writes) and the
  // integrator state.
  const BodyPose *pose_in;
  BodyPose *pose_out;
  BodyDyn *dyn;
};

// Launch shape of the dense step (threads per CTA along x, and the CTAs per
// SM the register budget is sized for). Compile-time so the tuning sweep can
// build variants; the defaults are the measured best.
#ifndef LBM_STEP_THREADS
#define LBM_STEP_THREADS 64
#endif
#ifndef LBM_STEP_MIN_BLOCKS
#define LBM_STEP_MIN_BLOCKS 16
#endif
constexpr int kStepThreads = LBM_STEP_THREADS;
constexpr int kStepMinBlocks = LBM_STEP_MIN_BLOCKS;

LBM_HD int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// The launch blocks of the dense step grid (kStepThreads cells along x, one
// row per block in y and z) that cover an inclusive cell box: per axis the
// first block, wrapped into the grid, and first + count, read modulo the
// grid -- the box of a windowed axis can cross the periodic seam. A box as
// long as the grid covers all of it; a count above cap[a] is clipped to it
// and reported (cap NULL: no limit).
LBM_HD bool box_region(const int box[6], int nx, int ny, int nz, const int *cap, int r[6]) {
  const int unit[3] = {kStepThreads, 1, 1};
  const int nb[3] = {(nx + kStepThreads - 1) / kStepThreads, ny, nz};
  bool clipped = false;
  for (int a = 0; a < 3; ++a) {
    const int b0 = floor_div(box[2 * a], unit[a]), b1 = floor_div(box[2 * a + 1], unit[a]);
    int first = b0 % nb[a], count = b1 - b0 + 1;
    if (first < 0) first += nb[a];
    if (count >= nb[a]) { first = 0; count = nb[a]; }
    if (cap && count > cap[a]) { count = cap[a]; clipped = true; }
    r[2 * a] = first;
    r[2 * a + 1] = first + count;
  }
  return clipped;
}
// Force partials summed per block by sum_partials_grouped (one per thread),
// and the number of such groups.
constexpr int kSumGroup = 64;
LBM_HD int sum_groups(int nparts) { return (nparts + kSumGroup - 1) / kSumGroup; }

// Number of force partials (launch blocks of the force region) of a dense step.
inline int force_parts(int q, const StepParams &p) {
  return (p.rbx1 - p.rbx0) * (p.rby1 - p.rby0) * (q == 9 ? 1 : p.rbz1 - p.rbz0);
}
constexpr int kReduceThreads = 256;
constexpr int kForceSlots = 8;
constexpr int kTotalsSlots = 8;

// storage: 0 fp32, 1 fp16 offset, 2 bf16 offset
cudaError_t launch_step(int q, int storage, const void *f_in, void *f_out, float *mac,
                        const StepParams &p, cudaStream_t st);
// Free-body force pass: the cells near the body (pose p.pose_in), FP64
// force/torque into p.force_out, then the body integrated into p.pose_out.
// `cap` is the launch grid (the largest box, in blocks).
cudaError_t launch_force_pass(int q, int storage, const void *f_in, const StepParams &p, const int cap[3],
                              cudaStream_t st);
cudaError_t launch_init_eq(int q, int storage, const float *mac_in, void *f_out, int64_t n, const Pack &pk,
                           cudaStream_t st);
// The equilibrium of one state (rho, ux, uy, uz) in every cell, with that
// state written to mac: the same bits as launch_init_eq of a uniform field.
cudaError_t launch_init_uniform(int q, int storage, const float rho_u[4], float *mac_out, void *f_out, int64_t n,
                                const Pack &pk, cudaStream_t st);
cudaError_t launch_pack(int q, int storage, const float *f32, void *f_store, int64_t n, const Pack &pk,
                        cudaStream_t st);
cudaError_t launch_unpack(int q, int storage, const void *f_store, float *f32, int64_t n, const Pack &pk,
                          cudaStream_t st);
// Totals over the current f, FP64; `partials` holds totals_partials() * 8
// doubles, `counter` one zeroed unsigned int.
int totals_blocks();
// n cells from f (a plane stride of `stride` cells, n when 0).
cudaError_t launch_totals(int q, int storage, const void *f, int64_t n, const Pack &pk, double *partials,
                          unsigned int *counter, double *out, cudaStream_t st, int64_t stride = 0);

// One launch of a batch step over tile positions k0 .. k1-1 of `order`
// (batch.cu); `fluid` selects the lean D2Q9 kernel.
cudaError_t launch_batch_step(int q, int storage, int threads, int ctas, cudaStream_t st, const void *fin,
                              void *fout, float *mac, const StepParams *doms, const int2 *tiles, const int *order,
                              int k0, int k1, int cells_per_tile, int write_mac, bool fluid);

}  // namespace lbm
