// Dense-grid kernels for sm_100a: the fused pull-stream / BGK / Guo-forcing
// step with its body-force reduction, equilibrium seeding, storage
// conversion and the FP64 conserved-totals reduction.
//
// Reference arithmetic:
//   3D step    common_d3_step.wgsl:224-400
//   3D force   common_d3_force.wgsl:171-283 (momentum exchange with local
//              rho_w and the swept-cell term, or the chi penalty)
//   2D step    lbm_step.wgsl:137-270
//   2D force   lbm_force.wgsl (main)
//   initEq     common_d3_step.wgsl:206-222
//   totals     amr2d-gpu.mjs:698-736 readConservedTotals
//
// Layout in HBM: f is Q planes, plane-major, `f[i * n + cell]` with
// cell = (z*NY + y)*NX + x -- the reference's layout, which is also the one
// that gives every warp a coalesced 128-byte row per plane. One thread owns
// one cell: it issues the Q pull loads up front (periodic sources), patches
// the few bounce-back links afterwards, collides in registers and writes
// the Q planes of its own cell. The mac field is written only when the
// host asks for it (the last step of a batch), not every step.
//
// The body force is summed INSIDE the step: the reference runs a separate
// full-grid force pass before each step over the same pre-streaming f_in,
// and every quantity it needs (f_opp at the cell, the streamed rho and u*)
// is already in this kernel's registers. Only the launch blocks whose cells
// can touch the body reduce; each writes one FP64 partial, and the partials
// are summed in a fixed order after the launch, so the result is
// deterministic: by the first blocks of the next step when steps follow one
// another, else by a small launch of the same blocks. The kernel boundary is
// what orders the partials before the sum. A last-block ticket inside the
// step needs a release fence per partial, and under the step's full write
// traffic each fence held its CTA for microseconds; one block summing all
// partials waits on dozens of rounds of loads; and a one-block launch after
// every step costs its launch gaps (measured at 256x128x128: +9 %, +10 %
// and +7 % of the step against no force at all, and +1 % for this form).

#include <type_traits>
#include <utility>

#include "cell_update.cuh"

namespace lbm {

namespace {

// ---- dense fused steps -------------------------------------------------------
// One thread per cell, kStepThreads (64) cells of a row per CTA, grid
// (NX/64, NY, NZ): the row and plane come straight from blockIdx, no
// division.

// The previous step's force, in this launch's first blocks (before their
// own cells, so that the group's fence has no stores of theirs to wait on).
__device__ __forceinline__ void sum_previous(const StepParams &p) {
  const int b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (p.prev_parts && b < sum_groups(p.prev_parts))
    sum_partials_grouped<kStepThreads>(p.prev_partials, p.prev_parts, p.groups, p.counter, p.force_out, b);
}

// Whether a cell of [lo, hi] lies in the interval [a, a + len] read modulo
// n (a in [0, n); len < 0 is empty): the reach-box test of cell3_core for a
// whole span of cells.
__device__ __forceinline__ bool span_hits(int lo, int hi, int a, int len, int n) {
  if (len >= n - 1) return true;
  const int b = a + len;
  return (lo <= b && hi >= a) || (lo + n <= b && hi + n >= a);
}

// What a launch block of the 3D step must evaluate, decided once per block
// (warp-uniform): kGeneral runs cell3 for every cell; kFluid runs
// cell3_fluid, for blocks that take no part in the force reduction, have no
// cell within reach of a bounce-back body (or no body), touch no wall and
// are not windowed. Penalty bodies reach every cell through chi and always
// take kGeneral. (A third kind without the sponge blend, for blocks beyond
// the sponge band, had fewer instructions per update but a slower step: a
// third hot copy of the update raised instruction-fetch and memory stalls.)
enum BlockKind { kGeneral = 0, kFluid = 1 };

__device__ __forceinline__ int block_kind(const StepParams &p, int lo, int hi, int y, int z, bool region) {
  if (region || p.win.on) return kGeneral;
  if (p.has_body) {
    if (!p.bb || !p.nbox_on) return kGeneral;
    if (span_hits(lo, hi, p.nbox[0], p.nbox[1] - p.nbox[0], p.nx) &&
        span_hits(y, y, p.nbox[2], p.nbox[3] - p.nbox[2], p.ny) &&
        span_hits(z, z, p.nbox[4], p.nbox[5] - p.nbox[4], p.nzg))
      return kGeneral;
  }
  if ((p.wall_x && (lo == 0 || hi == p.nx - 1)) || (p.wall_y && (y == 0 || y == p.ny - 1)) ||
      (p.wall_z && (z == 0 || z == p.nzg - 1)))
    return kGeneral;
  return kFluid;
}

template <int Q, typename S, bool TRT>
__device__ __forceinline__ void d3_step_block(const S *__restrict__ fin, S *__restrict__ fout,
                                              float *__restrict__ mac, const StepParams &p) {
  sum_previous(p);
  const int x = blockIdx.x * kStepThreads + threadIdx.x;
  // bz: the stored plane (a slab skips its ghost plane below); zg: the
  // domain's plane, which the force region and the block kind are in
  const int bx = blockIdx.x, by = blockIdx.y, bz = blockIdx.z + p.zlo;
  const int zg = bz + p.zoff;
  // the force region, read modulo the grid (it can cross a windowed seam;
  // a slab's region is its own share, with no seam)
  int dx = bx - p.rbx0, dy = by - p.rby0, dz = zg - p.rbz0;
  dx += dx < 0 ? (int)gridDim.x : 0;
  dy += dy < 0 ? (int)gridDim.y : 0;
  dz += (dz < 0 && p.zlo == 0) ? p.nzg : 0;
  const int rx = p.rbx1 - p.rbx0, ry = p.rby1 - p.rby0, rz = p.rbz1 - p.rbz0;
  const bool region = p.force_on && dx < rx && dy < ry && dz < rz;
  // The fluid path pays for 16-bit storage (issue-bound: 0.1106 against
  // 0.1167 ms per step on the 256x128x128 sphere) but not for FP32, whose
  // step is bound by memory latency and ran 0.1123 against 0.1110 ms with
  // it (D3Q27: 0.1589 against 0.1537 ms): FP32 takes the general path
  // everywhere.
  const int lo = bx * kStepThreads, hi = min(lo + kStepThreads, p.nx) - 1;
  const int kind = std::is_same<S, float>::value ? kGeneral : block_kind(p, lo, hi, by, zg, region);
  if (kind == kFluid) {
    if (x < p.nx) cell3_fluid<Q, S, TRT>(fin, fout, mac, p, x, by, bz);
    return;
  }
  CellForce cf;
  if (x < p.nx) cell3<Q, S, TRT>(fin, fout, mac, p, x, by, bz, region, cf);
  if (region) {
    ForceAcc acc;
    acc.add(cf);
    publish_force<kStepThreads>(acc, p.partials, (dz * ry + dy) * rx + dx);
  }
}

// A copy of the launch's parameters in shared memory with the body pose,
// swept-cell band and force region of this step taken from the device
// (free-body launches, where the pose is produced on the device).
__device__ __forceinline__ void stage_pose(const StepParams &p, StepParams &sp) {
  const unsigned *src = reinterpret_cast<const unsigned *>(&p);
  unsigned *dst = reinterpret_cast<unsigned *>(&sp);
  for (int k = threadIdx.x; k < (int)(sizeof(StepParams) / 4); k += blockDim.x) dst[k] = src[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    const BodyPose &bp = *p.pose_in;
    sp.body = bp.body;
    sp.nbox_on = 0;  // the pose moves on the device: evaluate the SDF everywhere
    sp.swept = bp.swept;
    sp.swept_band = bp.swept_band;
    sp.rbx0 = bp.region[0];
    sp.rbx1 = bp.region[1];
    sp.rby0 = bp.region[2];
    sp.rby1 = bp.region[3];
    sp.rbz0 = bp.region[4];
    sp.rbz1 = bp.region[5];
  }
  __syncthreads();
}

template <int Q, typename S, bool TRT>
__global__ void __launch_bounds__(kStepThreads, Q == 27 ? (kStepMinBlocks * 3) / 4 : kStepMinBlocks)
    d3_step(const S *__restrict__ fin, S *__restrict__ fout, float *__restrict__ mac,
            const __grid_constant__ StepParams p) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a no-op unless launched by launch_pdl
  d3_step_block<Q, S, TRT>(fin, fout, mac, p);
}

// The step of a free body: the pose comes from the device (written by the
// force pass just before); no force reduction.
template <int Q, typename S, bool TRT>
__global__ void __launch_bounds__(kStepThreads, Q == 27 ? (kStepMinBlocks * 3) / 4 : kStepMinBlocks)
    d3_step_free(const S *__restrict__ fin, S *__restrict__ fout, float *__restrict__ mac,
                 const __grid_constant__ StepParams p) {
  __shared__ StepParams sp;
  stage_pose(p, sp);
  d3_step_block<Q, S, TRT>(fin, fout, mac, sp);
}

// Integrates the free body under the force just summed and publishes the
// next pose with its force box (clipped to the launch capacity; a body
// outside the domain keeps one block so the integrator still runs).
__device__ __noinline__ void integrate_and_publish(BodyDyn *dyn, const double *force, BodyPose *next) {
  const double F[3] = {force[0], force[1], force[2]}, T[3] = {force[3], force[4], force[5]};
  body_step(dyn->st, F, T, dyn->opt);
  BodyPose np;
  np.body = body_pose(dyn->shape, dyn->st);
  int box[6];
  if (!body_cell_box(np.body, dyn->q, dyn->nx, dyn->ny, dyn->nz, dyn->bounceback, dyn->swept_force, dyn->chi_eps,
                     box, &np.swept, &np.swept_band, dyn->win)) {
    const float c[3] = {np.body.cx, np.body.cy, np.body.cz};
    const int len[3] = {dyn->nx, dyn->ny, dyn->nz};
    for (int a = 0; a < 3; ++a) {
      const int v = (int)fminf(fmaxf(c[a], 0.f), (float)(len[a] - 1));
      box[2 * a] = box[2 * a + 1] = v;
    }
  }
  if (box_region(box, dyn->nx, dyn->ny, dyn->nz, dyn->cap, np.region)) dyn->overflow += 1;
  *next = np;
}

// Free-body force pass over the blocks of the current force box (the
// launch grid is the largest box; blocks past this step's box leave at
// once and take no part in the reduction). The last block to finish sums
// the partials and integrates the body.
template <int Q, typename S>
__global__ void __launch_bounds__(kStepThreads)
    d3_force_pass(const S *__restrict__ fin, const __grid_constant__ StepParams p) {
  __shared__ StepParams sp;
  stage_pose(p, sp);
  const int rx = sp.rbx1 - sp.rbx0, ry = sp.rby1 - sp.rby0, rz = sp.rbz1 - sp.rbz0;
  if ((int)blockIdx.x >= rx || (int)blockIdx.y >= ry || (int)blockIdx.z >= rz) return;
  // blocks of the region, wrapped into the grid
  const int nbx = (sp.nx + kStepThreads - 1) / kStepThreads;
  int bx = sp.rbx0 + blockIdx.x, by = sp.rby0 + blockIdx.y, bz = sp.rbz0 + blockIdx.z;
  bx -= bx >= nbx ? nbx : 0;
  by -= by >= sp.ny ? sp.ny : 0;
  bz -= bz >= sp.nz ? sp.nz : 0;
  const int x = bx * kStepThreads + threadIdx.x;
  CellForce cf;
  if (x < sp.nx) cell3_force<Q, S>(fin, sp, x, by, bz, cf);
  const int part = ((int)blockIdx.z * ry + (int)blockIdx.y) * rx + (int)blockIdx.x;
  ForceAcc acc;
  acc.add(cf);
  const bool last = reduce_force<kStepThreads>(acc, sp.partials, sp.counter, rx * ry * rz, part, sp.force_out);
  if (last && threadIdx.x == 0) integrate_and_publish(sp.dyn, sp.force_out, sp.pose_out);
}

template <typename S>
__global__ void __launch_bounds__(kStepThreads)
    d2_step(const S *__restrict__ fin, S *__restrict__ fout, float *__restrict__ mac,
            const __grid_constant__ StepParams p) {
  sum_previous(p);
  const int x = blockIdx.x * kStepThreads + threadIdx.x;
  const int bx = blockIdx.x, by = blockIdx.y;
  const bool region = p.force_on && bx >= p.rbx0 && bx < p.rbx1 && by >= p.rby0 && by < p.rby1;
  CellForce cf;
  if (x < p.nx) cell2<S>(fin, fout, mac, p, x, by, region, cf);
  if (region) {
    const int rx = p.rbx1 - p.rbx0;
    ForceAcc acc;
    acc.add(cf);
    publish_force<kStepThreads>(acc, p.partials, (by - p.rby0) * rx + (bx - p.rbx0));
  }
}

// The force of a step that no following launch sums: the same blocks, with
// the same arithmetic, as the first blocks of a following step.
__global__ void __launch_bounds__(kStepThreads)
    force_finish(const double *__restrict__ partials, int nparts, double *__restrict__ groups,
                 unsigned int *__restrict__ counter, double *__restrict__ out) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  sum_partials_grouped<kStepThreads>(partials, nparts, groups, counter, out, blockIdx.x);
}

// ---- seeding and storage conversion ----------------------------------------

// f at equilibrium of the mac field; UNIFORM: of the one state `mu`, which
// is also written to every cell of mac (a uniform seed needs no host data).
template <int Q, typename S, bool UNIFORM = false>
__global__ void init_eq(const float4 *__restrict__ mac, S *__restrict__ f, int64_t n, const Pack pk,
                        float4 mu = {}, float4 *__restrict__ mac_out = nullptr) {
  using L = Lattice<Q>;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    const float4 m = UNIFORM ? mu : mac[c];
    if (UNIFORM) mac_out[c] = mu;
    const float rho = m.x, ux = m.y, uy = m.z, uz = Q == 9 ? 0.f : m.w;
    const float usq = Q == 9 ? (ux * ux + uy * uy) : (ux * ux + uy * uy + uz * uz);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const float eu = (float)L::ex(i) * ux + (float)L::ey(i) * uy + (float)L::ez(i) * uz;
      const float v = L::w(i) * rho * (1.f + 3.f * eu + 4.5f * eu * eu - 1.5f * usq);
      Codec<S>::st(f + (int64_t)i * n + c, v, i, pk);
    }
  }
}

template <int Q, typename S>
__global__ void pack_planes(const float *__restrict__ src, S *__restrict__ dst, int64_t n, const Pack pk) {
  using L = Lattice<Q>;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int i = 0; i < Q; ++i) Codec<S>::st(dst + (int64_t)i * n + c, src[(int64_t)i * n + c], i, pk);
}

template <int Q, typename S>
__global__ void unpack_planes(const S *__restrict__ src, float *__restrict__ dst, int64_t n, const Pack pk) {
  using L = Lattice<Q>;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int i = 0; i < Q; ++i) dst[(int64_t)i * n + c] = Codec<S>::ld(src + (int64_t)i * n + c, i, pk);
}

// ---- conserved totals ------------------------------------------------------
// Per cell the reference sums the f32 populations in f64 (JS numbers):
// rho, rho u, then mass += rho - 1. Same here, with FP64 partial sums per
// block and a fixed-order final sum.

constexpr int kTotalsBlocks = 148 * 4;

template <int Q, typename S>
__global__ void __launch_bounds__(kReduceThreads)
    totals_kernel(const S *__restrict__ f, int64_t n, int64_t stride, const Pack pk, double *partials,
                  unsigned int *counter, double *out) {
  using L = Lattice<Q>;
  double mass = 0.0, px = 0.0, py = 0.0, pz = 0.0, bad = 0.0;
  double rmin = 1e300, rmax = -1e300, u2max = 0.0;
  for (int64_t c = blockIdx.x * (int64_t)kReduceThreads + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * kReduceThreads) {
    double rho = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const double v = (double)Codec<S>::ld(f + (int64_t)i * stride + c, i, pk);
      rho += v;
      mx += v * L::ex(i);
      my += v * L::ey(i);
      mz += v * L::ez(i);
    }
    if (!isfinite(rho + mx + my + mz)) {
      bad += 1.0;
      continue;
    }
    mass += rho - 1.0;
    px += mx;
    py += my;
    pz += mz;
    rmin = fmin(rmin, rho);
    rmax = fmax(rmax, rho);
    u2max = fmax(u2max, (mx * mx + my * my + mz * mz) / (rho * rho));
  }
  // Sums via the shared block_sum; min/max folded through negation tricks
  // would lose determinism guarantees for ties, so they are reduced apart.
  __shared__ double sm[kTotalsSlots * (kReduceThreads / 32)];
  double v[5] = {mass, px, py, pz, bad};
  block_sum<5, kReduceThreads>(v, sm);
  double mm[3] = {rmin, -rmax, -u2max};
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mm[k] = fmin(mm[k], __shfl_down_sync(0xffffffffu, mm[k], o));
  __shared__ double smm[3 * (kReduceThreads / 32)];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 3; ++k) smm[k * (kReduceThreads / 32) + warp] = mm[k];
  __syncthreads();
  if (warp == 0) {
    for (int k = 0; k < 3; ++k) {
      double t = lane < kReduceThreads / 32 ? smm[k * (kReduceThreads / 32) + lane] : 1e300;
      for (int o = 16; o > 0; o >>= 1) t = fmin(t, __shfl_down_sync(0xffffffffu, t, o));
      mm[k] = t;
    }
  }
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    double *pp = partials + (int64_t)blockIdx.x * kTotalsSlots;
    pp[0] = v[0]; pp[1] = v[1]; pp[2] = v[2]; pp[3] = v[3];
    pp[4] = mm[0]; pp[5] = mm[1]; pp[6] = mm[2]; pp[7] = v[4];
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s7 = 0, m4 = 1e300, m5 = 1e300, m6 = 1e300;
    for (unsigned int j = 0; j < gridDim.x; ++j) {
      const double *pp = partials + (int64_t)j * kTotalsSlots;
      s0 += __ldcg(pp + 0); s1 += __ldcg(pp + 1); s2 += __ldcg(pp + 2); s3 += __ldcg(pp + 3);
      m4 = fmin(m4, __ldcg(pp + 4)); m5 = fmin(m5, __ldcg(pp + 5)); m6 = fmin(m6, __ldcg(pp + 6));
      s7 += __ldcg(pp + 7);
    }
    out[0] = s0; out[1] = s1; out[2] = s2; out[3] = s3;
    out[4] = m4; out[5] = -m5; out[6] = sqrt(-m6 < 0 ? 0.0 : -m6); out[7] = s7;
    *counter = 0u;
  }
}

// Expands the body once per (Q, storage) pair with Q and S bound.
#define LBM_DISPATCH(q, storage, ...)                                           \
  switch ((q) * 4 + (storage)) {                                                 \
    case 9 * 4 + 0: { constexpr int Q = 9; using S = float; __VA_ARGS__; } break;        \
    case 9 * 4 + 1: { constexpr int Q = 9; using S = __half; __VA_ARGS__; } break;       \
    case 9 * 4 + 2: { constexpr int Q = 9; using S = __nv_bfloat16; __VA_ARGS__; } break; \
    case 19 * 4 + 0: { constexpr int Q = 19; using S = float; __VA_ARGS__; } break;      \
    case 19 * 4 + 1: { constexpr int Q = 19; using S = __half; __VA_ARGS__; } break;     \
    case 19 * 4 + 2: { constexpr int Q = 19; using S = __nv_bfloat16; __VA_ARGS__; } break; \
    case 27 * 4 + 0: { constexpr int Q = 27; using S = float; __VA_ARGS__; } break;      \
    case 27 * 4 + 1: { constexpr int Q = 27; using S = __half; __VA_ARGS__; } break;     \
    case 27 * 4 + 2: { constexpr int Q = 27; using S = __nv_bfloat16; __VA_ARGS__; } break; \
    default: return cudaErrorInvalidValue;                                       \
  }                                                                              \
  return cudaGetLastError();

int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  return (int)(b < 148 * 8 ? (b < 1 ? 1 : b) : 148 * 8);
}

}  // namespace

namespace {
// A launch that may begin while the previous kernel on the stream drains
// (programmatic dependent launch): the step and force-sum kernels wait at
// their first instruction (griddepcontrol.wait) until that kernel has
// completed and its writes are visible, so the order is the stream's; what
// overlaps is the new grid's launch and scheduling with the old one's tail.
// Measured on B200 for one-step calls: 0.124 -> 0.120 ms per step, and with
// a force readback after each 0.129 -> 0.124 ms.
template <typename... K, typename... A>
void launch_pdl(dim3 g, dim3 b, cudaStream_t st, void (*k)(K...), A &&...args) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = g;
  lc.blockDim = b;
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  cudaLaunchKernelEx(&lc, k, std::forward<A>(args)...);
}
cudaError_t launch_step_kernel(int q, int storage, const void *f_in, void *f_out, float *mac, const StepParams &p,
                               cudaStream_t st) {
  dim3 grid((p.nx + kStepThreads - 1) / kStepThreads, p.ny, q == 9 ? 1 : p.nz - 2 * p.zlo);
  LBM_DISPATCH(q, storage, {
    if constexpr (Q == 9)
      d2_step<S><<<grid, kStepThreads, 0, st>>>((const S *)f_in, (S *)f_out, mac, p);
    else if (p.pose_in && p.trt_dw != 0.f)
      d3_step_free<Q, S, true><<<grid, kStepThreads, 0, st>>>((const S *)f_in, (S *)f_out, mac, p);
    else if (p.pose_in)
      d3_step_free<Q, S, false><<<grid, kStepThreads, 0, st>>>((const S *)f_in, (S *)f_out, mac, p);
    else if (p.trt_dw != 0.f)
      launch_pdl(grid, dim3(kStepThreads), st, d3_step<Q, S, true>, (const S *)f_in, (S *)f_out, mac, p);
    else
      launch_pdl(grid, dim3(kStepThreads), st, d3_step<Q, S, false>, (const S *)f_in, (S *)f_out, mac, p);
  });
}
}  // namespace

cudaError_t launch_step(int q, int storage, const void *f_in, void *f_out, float *mac,
                        const StepParams &p, cudaStream_t st) {
  // a free body's step takes no force (its force pass does)
  if (p.pose_in && p.force_on) return cudaErrorInvalidValue;
  if (p.force_on && (!p.partials || !p.groups || !p.counter || !p.force_out)) return cudaErrorInvalidValue;
  if (p.prev_parts && (!p.prev_partials || !p.groups || !p.counter || !p.force_out)) return cudaErrorInvalidValue;
  const cudaError_t e = launch_step_kernel(q, storage, f_in, f_out, mac, p, st);
  if (e != cudaSuccess || !p.force_on || p.defer_force) return e;
  const int parts = force_parts(q, p);
  launch_pdl(dim3(sum_groups(parts)), dim3(kStepThreads), st, force_finish, (const double *)p.partials, parts,
             p.groups, p.counter, p.force_out);
  return cudaGetLastError();
}

cudaError_t launch_force_pass(int q, int storage, const void *f_in, const StepParams &p, const int cap[3],
                              cudaStream_t st) {
  if (q == 9 || !p.pose_in || !p.pose_out || !p.dyn) return cudaErrorInvalidValue;
  dim3 grid(cap[0], cap[1], cap[2]);
  LBM_DISPATCH(q, storage, {
    if constexpr (Q != 9) d3_force_pass<Q, S><<<grid, kStepThreads, 0, st>>>((const S *)f_in, p);
  });
}

cudaError_t launch_init_eq(int q, int storage, const float *mac_in, void *f_out, int64_t n, const Pack &pk,
                           cudaStream_t st) {
  LBM_DISPATCH(q, storage, init_eq<Q, S><<<grid_for(n, 256), 256, 0, st>>>((const float4 *)mac_in, (S *)f_out, n, pk));
}

cudaError_t launch_init_uniform(int q, int storage, const float rho_u[4], float *mac_out, void *f_out, int64_t n,
                                const Pack &pk, cudaStream_t st) {
  const float4 mu = make_float4(rho_u[0], rho_u[1], rho_u[2], rho_u[3]);
  LBM_DISPATCH(q, storage, (init_eq<Q, S, true><<<grid_for(n, 256), 256, 0, st>>>(nullptr, (S *)f_out, n, pk, mu,
                                                                                 (float4 *)mac_out)));
}

cudaError_t launch_pack(int q, int storage, const float *f32, void *f_store, int64_t n, const Pack &pk,
                        cudaStream_t st) {
  LBM_DISPATCH(q, storage, pack_planes<Q, S><<<grid_for(n, 256), 256, 0, st>>>(f32, (S *)f_store, n, pk));
}

cudaError_t launch_unpack(int q, int storage, const void *f_store, float *f32, int64_t n, const Pack &pk,
                          cudaStream_t st) {
  LBM_DISPATCH(q, storage, unpack_planes<Q, S><<<grid_for(n, 256), 256, 0, st>>>((const S *)f_store, f32, n, pk));
}

int totals_blocks() { return kTotalsBlocks; }

cudaError_t launch_totals(int q, int storage, const void *f, int64_t n, const Pack &pk, double *partials,
                          unsigned int *counter, double *out, cudaStream_t st, int64_t stride) {
  if (stride <= 0) stride = n;
  LBM_DISPATCH(q, storage, (totals_kernel<Q, S><<<kTotalsBlocks, kReduceThreads, 0, st>>>((const S *)f, n, stride, pk, partials, counter, out)));
}

}  // namespace lbm
