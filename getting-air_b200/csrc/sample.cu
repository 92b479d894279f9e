// Headless views of the field, as compute kernels into a buffer.
//
// sampleTree (common_d3_tree_sample.wgsl): the value at a continuous L0
// point is the nearest cell of the finest level present there. A level-m
// cell has size 2^-m and centre (g + 1/2) 2^-m - 1/2, so the cell holding p
// is g = floor((p + 1/2) 2^m), owned by block g / (2 RB) -- one division,
// never a ring cell. Level 0 is the dense grid and is present everywhere.
//
// resample (common_d3_resample.wgsl): one sample per voxel centre
// origin + (v + 1/2) h - 1/2, stored as (ux, uy, uz, rho) in binary16 (the
// rgba16float texture) or f32, plus the level it came from.
//
// slice (common_d3_render_slice.wgsl fs_main, common_vortcolor.wgsl): one
// pixel per fragment of the full-screen quad, uv at pixel centres, the
// picture turned by quarter turns, speed / out-of-plane vorticity (centred
// differences taken from a level-consistent pair, dPlane) / normal velocity,
// the magnitude and signed tone-mapped ramps, RGBA8 rounded to nearest.
//
// Every coordinate expression is rounded operation by operation (no
// contraction), so the sample positions -- and with them which cell
// answers -- are the plain f32 arithmetic of the formulas.
#include <cmath>

#include <cuda_fp16.h>

#include "amr3d.cuh"
#include "sample.cuh"

namespace lbm {

namespace {

struct Sample {
  float4 v;   // [rho, ux, uy, uz]
  int level;
  float h;
  float3 c;   // centre of the answering cell, unwrapped
};

__device__ __forceinline__ int tree_wrap(int v, int n) {
  const int r = v % n;
  return r < 0 ? r + n : r;
}

__device__ Sample sample_dense(const TreeView &t, float3 p) {
  Sample o;
  const float gx = floorf(__fadd_rn(p.x, 0.5f)), gy = floorf(__fadd_rn(p.y, 0.5f)),
              gz = floorf(__fadd_rn(p.z, 0.5f));
  o.c = make_float3(gx, gy, gz);
  const int cx = tree_wrap((int)gx, t.nx), cy = tree_wrap((int)gy, t.ny), cz = tree_wrap((int)gz, t.nz);
  o.v = t.mac[((int64_t)cz * t.ny + cy) * t.nx + cx];
  o.level = 0;
  o.h = 1.f;
  return o;
}

// Level 1: the tile of the block owning p, if it has one.
__device__ bool sample_level1(const TreeView &t, float3 p, Sample &o) {
  const float gf[3] = {floorf(__fmul_rn(__fadd_rn(p.x, 0.5f), 2.f)), floorf(__fmul_rn(__fadd_rn(p.y, 0.5f), 2.f)),
                       floorf(__fmul_rn(__fadd_rn(p.z, 0.5f), 2.f))};
  const int dims[3] = {2 * t.nx, 2 * t.ny, 2 * t.nz};
  const int rb2 = 2 * t.rb;
  int g[3], b[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    g[a] = tree_wrap((int)gf[a], dims[a]);
    b[a] = g[a] / rb2;
  }
  const int nbx = t.nx / t.rb, nby = t.ny / t.rb;
  const int slot = t.block_slot[(b[2] * nby + b[1]) * nbx + b[0]];
  if (slot < 0) return false;
  const int G = kAmrGhost;
  const int64_t cell = (int64_t)slot * t.t3 +
                       ((int64_t)(g[2] - b[2] * rb2 + G) * t.fb + (g[1] - b[1] * rb2 + G)) * t.fb +
                       (g[0] - b[0] * rb2 + G);
  o.v = t.macp[cell];
  o.level = 1;
  o.h = 0.5f;
  o.c = make_float3(__fsub_rn(__fdiv_rn(__fadd_rn(gf[0], 0.5f), 2.f), 0.5f),
                    __fsub_rn(__fdiv_rn(__fadd_rn(gf[1], 0.5f), 2.f), 0.5f),
                    __fsub_rn(__fdiv_rn(__fadd_rn(gf[2], 0.5f), 2.f), 0.5f));
  return true;
}

// sampleTreeAtMost: the finest level present at p that is no finer than mmax.
__device__ Sample sample_tree(const TreeView &t, float3 p, int mmax) {
  if (min(mmax, t.levels) >= 1) {
    Sample o;
    if (sample_level1(t, p, o)) return o;
  }
  return sample_dense(t, p);
}

// ---- resample ----------------------------------------------------------------

struct VolParams {
  float ox, oy, oz, hx, hy, hz;
  int nx, ny, nz;
};

template <bool kHalf>
__global__ void resample_kernel(const TreeView t, const VolParams vp, void *__restrict__ out,
                                uint8_t *__restrict__ level) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= vp.nx || y >= vp.ny) return;
  const float3 p = make_float3(__fsub_rn(__fadd_rn(vp.ox, __fmul_rn(__fadd_rn((float)x, 0.5f), vp.hx)), 0.5f),
                               __fsub_rn(__fadd_rn(vp.oy, __fmul_rn(__fadd_rn((float)y, 0.5f), vp.hy)), 0.5f),
                               __fsub_rn(__fadd_rn(vp.oz, __fmul_rn(__fadd_rn((float)z, 0.5f), vp.hz)), 0.5f));
  const Sample s = sample_tree(t, p, t.levels);
  const int64_t idx = ((int64_t)z * vp.ny + y) * vp.nx + x;
  if (kHalf) {
    __half2 *o = reinterpret_cast<__half2 *>(out) + 2 * idx;
    o[0] = __floats2half2_rn(s.v.y, s.v.z);
    o[1] = __floats2half2_rn(s.v.w, s.v.x);
  } else {
    reinterpret_cast<float4 *>(out)[idx] = make_float4(s.v.y, s.v.z, s.v.w, s.v.x);
  }
  if (level) level[idx] = (uint8_t)s.level;
}

// ---- slice -------------------------------------------------------------------

struct SliceParams {
  int axis, slice, mode, rot;
  float u_scale, v_scale, vort_scale, vort_gamma;
  int W, H;
  float off[3];
};

struct PlaneSample {
  float uvw[3];
  float ab[3];
  int level;
};

__device__ __forceinline__ void rotate_uvw(int axis, float x, float y, float z, float out[3]) {
  if (axis == 0) { out[0] = y; out[1] = z; out[2] = x; }
  else if (axis == 1) { out[0] = z; out[1] = x; out[2] = y; }
  else { out[0] = x; out[1] = y; out[2] = z; }
}

__device__ __forceinline__ float3 plane_point(const SliceParams &sp, float a, float b) {
  const float sl = (float)sp.slice;
  float3 p;
  if (sp.axis == 0) p = make_float3(sl, a, b);
  else if (sp.axis == 1) p = make_float3(b, sl, a);
  else p = make_float3(a, b, sl);
  return make_float3(__fadd_rn(p.x, sp.off[0]), __fadd_rn(p.y, sp.off[1]), __fadd_rn(p.z, sp.off[2]));
}

__device__ PlaneSample sample_plane_at(const TreeView &t, const SliceParams &sp, float a, float b, int mmax) {
  const Sample s = sample_tree(t, plane_point(sp, a, b), mmax);
  PlaneSample o;
  rotate_uvw(sp.axis, s.v.y, s.v.z, s.v.w, o.uvw);
  rotate_uvw(sp.axis, s.c.x, s.c.y, s.c.z, o.ab);
  o.level = s.level;
  return o;
}

// dPlane: d(uvw[comp]) / d(in-plane axis `axis`) by a centred difference
// whose two arms come from one level, divided by the separation of the
// centres that answered.
__device__ float d_plane(const TreeView &t, const SliceParams &sp, float pa, float pb, int comp, int axis,
                         int mstart) {
  int m = mstart;
  float h = 1.f / (float)(1 << m);
  PlaneSample plus = sample_plane_at(t, sp, __fadd_rn(pa, axis == 0 ? h : 0.f), __fadd_rn(pb, axis == 1 ? h : 0.f), m);
  PlaneSample minus = sample_plane_at(t, sp, __fsub_rn(pa, axis == 0 ? h : 0.f), __fsub_rn(pb, axis == 1 ? h : 0.f), m);
  for (int it = 0; it < t.levels && plus.level != minus.level; ++it) {
    m = min(plus.level, minus.level);
    h = 1.f / (float)(1 << m);
    plus = sample_plane_at(t, sp, __fadd_rn(pa, axis == 0 ? h : 0.f), __fadd_rn(pb, axis == 1 ? h : 0.f), m);
    minus = sample_plane_at(t, sp, __fsub_rn(pa, axis == 0 ? h : 0.f), __fsub_rn(pb, axis == 1 ? h : 0.f), m);
  }
  const float dx = __fsub_rn(plus.ab[axis], minus.ab[axis]);
  if (fabsf(dx) < __fmul_rn(1e-6f, fmaxf(h, 1e-6f))) return 0.f;
  return __fdiv_rn(__fsub_rn(plus.uvw[comp], minus.uvw[comp]), dx);
}

__device__ __forceinline__ float mix1(float a, float b, float t) {
  return __fadd_rn(__fmul_rn(a, __fsub_rn(1.f, t)), __fmul_rn(b, t));
}

__device__ __forceinline__ float smooth(float e0, float e1, float x) {
  const float t = fminf(fmaxf(__fdiv_rn(__fsub_rn(x, e0), __fsub_rn(e1, e0)), 0.f), 1.f);
  return __fmul_rn(__fmul_rn(t, t), __fsub_rn(3.f, __fmul_rn(2.f, t)));
}

// magColor: dark blue -> cyan -> yellow for unsigned magnitudes.
__device__ void mag_color(float v, float rgb[3]) {
  const float c = fminf(fmaxf(v, 0.f), 1.f);
  const float lo0[3] = {0.05f, 0.05f, 0.12f}, lo1[3] = {0.1f, 0.65f, 0.75f}, hi[3] = {1.0f, 0.92f, 0.35f};
  const float s0 = smooth(0.f, 0.55f, c), s1 = smooth(0.55f, 1.f, c);
#pragma unroll
  for (int k = 0; k < 3; ++k) rgb[k] = mix1(mix1(lo0[k], lo1[k], s0), hi[k], s1);
}

// vorticityColor: Reinhard-compressed magnitude shaped by a gamma, blended
// from the near-black background toward warm red (positive) or cool blue.
__device__ void vort_color(float omega, float scale, float gamma, float rgb[3]) {
  const float a = __fmul_rn(fabsf(omega), scale);
  const float compressed = __fdiv_rn(a, __fadd_rn(1.f, a));
  const float mag = powf(compressed, gamma);
  const float val = omega >= 0.f ? mag : -mag;
  const float bg[3] = {0.05f, 0.05f, 0.1f}, pos[3] = {1.0f, 0.3f, 0.2f}, neg[3] = {0.2f, 0.5f, 1.0f};
#pragma unroll
  for (int k = 0; k < 3; ++k) rgb[k] = val > 0.f ? mix1(bg[k], pos[k], val) : mix1(bg[k], neg[k], -val);
}

__device__ __forceinline__ uint8_t unorm8(float x) { return (uint8_t)__float2uint_rn(__fmul_rn(__saturatef(x), 255.f)); }

__global__ void slice_kernel(const TreeView t, const SliceParams sp, uint8_t *__restrict__ rgba) {
  const int px = blockIdx.x * blockDim.x + threadIdx.x;
  const int py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= sp.W || py >= sp.H) return;
  const int nd[3] = {t.nx, t.ny, t.nz};
  const int da = nd[(sp.axis + 1) % 3], db = nd[(sp.axis + 2) % 3];
  const float dx = (float)da, dy = (float)db;
  // uv at the pixel centre; uv.y = 1 is the top row
  const float u = __fdiv_rn(__fadd_rn((float)px, 0.5f), (float)sp.W);
  const float v = __fsub_rn(1.f, __fdiv_rn(__fadd_rn((float)py, 0.5f), (float)sp.H));
  float pa, pb;
  if (sp.rot == 1) {
    pa = __fsub_rn(__fmul_rn(__fsub_rn(1.f, v), dx), 0.5f);
    pb = __fsub_rn(__fmul_rn(__fsub_rn(1.f, u), dy), 0.5f);
  } else if (sp.rot == 2) {
    pa = __fsub_rn(__fmul_rn(__fsub_rn(1.f, u), dx), 0.5f);
    pb = __fsub_rn(__fmul_rn(v, dy), 0.5f);
  } else if (sp.rot == 3) {
    pa = __fsub_rn(__fmul_rn(v, dx), 0.5f);
    pb = __fsub_rn(__fmul_rn(u, dy), 0.5f);
  } else {
    pa = __fsub_rn(__fmul_rn(u, dx), 0.5f);
    pb = __fsub_rn(__fmul_rn(__fsub_rn(1.f, v), dy), 0.5f);
  }
  const PlaneSample s = sample_plane_at(t, sp, pa, pb, t.levels);
  float rgb[3];
  if (sp.mode == 1) {
    const float omega = __fsub_rn(d_plane(t, sp, pa, pb, 1, 0, s.level), d_plane(t, sp, pa, pb, 0, 1, s.level));
    vort_color(__fdiv_rn(omega, fmaxf(sp.v_scale, 1e-12f)), sp.vort_scale, sp.vort_gamma, rgb);
  } else if (sp.mode == 2) {
    vort_color(__fdiv_rn(s.uvw[2], fmaxf(sp.u_scale, 1e-9f)), sp.vort_scale, sp.vort_gamma, rgb);
  } else {
    const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(s.uvw[0], s.uvw[0]), __fmul_rn(s.uvw[1], s.uvw[1])),
                                           __fmul_rn(s.uvw[2], s.uvw[2])));
    mag_color(__fdiv_rn(len, fmaxf(sp.u_scale, 1e-9f)), rgb);
  }
  uint8_t *o = rgba + 4 * ((int64_t)py * sp.W + px);
  o[0] = unorm8(rgb[0]);
  o[1] = unorm8(rgb[1]);
  o[2] = unorm8(rgb[2]);
  o[3] = 255;
}

}  // namespace

int validate_volume(const lbm_volume_spec *s, std::string &why) {
  if (!s) { why = "volume spec is NULL"; return LBM_EINVAL; }
  int64_t n = 1;
  for (int a = 0; a < 3; ++a) {
    if (s->shape[a] < 1) { why = "volume shape must be >= 1 per axis"; return LBM_EINVAL; }
    n *= s->shape[a];
    if (!std::isfinite(s->origin[a]) || std::fabs(s->origin[a]) > 1e7f) {
      why = "volume origin must be finite (|origin| <= 1e7)";
      return LBM_EINVAL;
    }
    if (!(s->h[a] > 0.f) || !(s->h[a] <= 1e6f)) { why = "voxel size must be in (0, 1e6]"; return LBM_EINVAL; }
  }
  if (s->shape[2] > 65535) { why = "volume shape z is limited to 65535"; return LBM_EINVAL; }
  if (n > ((int64_t)1 << 32)) { why = "volume exceeds 2^32 voxels"; return LBM_EINVAL; }
  if (s->fp16 != 0 && s->fp16 != 1) { why = "fp16 must be 0 or 1"; return LBM_EINVAL; }
  return LBM_OK;
}

int validate_slice(const lbm_slice_spec *s, int nx, int ny, int nz, std::string &why) {
  if (!s) { why = "slice spec is NULL"; return LBM_EINVAL; }
  if (s->axis < 0 || s->axis > 2) { why = "axis must be 0, 1 or 2"; return LBM_EINVAL; }
  if (s->mode < 0 || s->mode > 2) { why = "mode must be 0 (speed), 1 (vorticity) or 2 (normal velocity)"; return LBM_EINVAL; }
  if (s->rot < 0 || s->rot > 3) { why = "rot must be 0..3 quarter turns"; return LBM_EINVAL; }
  const int len[3] = {nx, ny, nz};
  if (s->slice < 0 || s->slice >= len[s->axis]) { why = "slice index outside the domain"; return LBM_EINVAL; }
  if (s->width < 1 || s->height < 1 || s->width > 16384 || s->height > 16384) {
    why = "image size must be 1..16384 pixels per side";
    return LBM_EINVAL;
  }
  if (!std::isfinite(s->u_scale) || !std::isfinite(s->v_scale) || !std::isfinite(s->vort_scale) ||
      s->vort_scale < 0.f || !(s->vort_gamma > 0.f) || !std::isfinite(s->vort_gamma)) {
    why = "scales must be finite (vort_scale >= 0, vort_gamma > 0)";
    return LBM_EINVAL;
  }
  return LBM_OK;
}

cudaError_t launch_resample(const TreeView &t, const lbm_volume_spec &s, void *out, uint8_t *level,
                            cudaStream_t st) {
  VolParams vp{s.origin[0], s.origin[1], s.origin[2], s.h[0], s.h[1], s.h[2], s.shape[0], s.shape[1], s.shape[2]};
  const dim3 blk(32, 8);
  const dim3 grid((vp.nx + 31) / 32, (vp.ny + 7) / 8, vp.nz);
  if (s.fp16) resample_kernel<true><<<grid, blk, 0, st>>>(t, vp, out, level);
  else resample_kernel<false><<<grid, blk, 0, st>>>(t, vp, out, level);
  return cudaGetLastError();
}

cudaError_t launch_slice(const TreeView &t, const lbm_slice_spec &s, ViewOffset off, uint8_t *rgba,
                         cudaStream_t st) {
  SliceParams sp{s.axis, s.slice, s.mode, s.rot, s.u_scale, s.v_scale, s.vort_scale, s.vort_gamma,
                 s.width, s.height, {off.v[0], off.v[1], off.v[2]}};
  const dim3 blk(16, 16);
  const dim3 grid((s.width + 15) / 16, (s.height + 15) / 16);
  slice_kernel<<<grid, blk, 0, st>>>(t, sp, rgba);
  return cudaGetLastError();
}

cudaError_t run_resample(const TreeView &t, const lbm_volume_spec &s, void *out, uint8_t *level, cudaStream_t st) {
  if (s.device) return launch_resample(t, s, out, level, st);
  const size_t nvox = (size_t)s.shape[0] * s.shape[1] * s.shape[2];
  const size_t bytes = nvox * (s.fp16 ? 8 : 16);
  void *d_out = nullptr;
  uint8_t *d_lvl = nullptr;
  cudaError_t e = cudaMallocAsync(&d_out, bytes, st);
  if (e == cudaSuccess && level) e = cudaMallocAsync((void **)&d_lvl, nvox, st);
  if (e == cudaSuccess) e = launch_resample(t, s, d_out, d_lvl, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && level) e = cudaMemcpyAsync(level, d_lvl, nvox, cudaMemcpyDeviceToHost, st);
  if (d_out) cudaFreeAsync(d_out, st);
  if (d_lvl) cudaFreeAsync(d_lvl, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  return e != cudaSuccess ? e : e2;
}

cudaError_t run_slice(const TreeView &t, const lbm_slice_spec &s, ViewOffset off, uint8_t *rgba, cudaStream_t st) {
  if (s.device) return launch_slice(t, s, off, rgba, st);
  const size_t bytes = (size_t)s.width * s.height * 4;
  uint8_t *d = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&d, bytes, st);
  if (e == cudaSuccess) e = launch_slice(t, s, off, d, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(rgba, d, bytes, cudaMemcpyDeviceToHost, st);
  if (d) cudaFreeAsync(d, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  return e != cudaSuccess ? e : e2;
}

}  // namespace lbm

extern "C" {

int lbm_volume_spec_default(lbm_volume_spec *v, int nx, int ny, int nz) {
  if (!v || nx < 1 || ny < 1 || nz < 1) return LBM_EINVAL;
  *v = lbm_volume_spec{};
  v->shape[0] = nx; v->shape[1] = ny; v->shape[2] = nz;
  v->h[0] = v->h[1] = v->h[2] = 1.f;
  return LBM_OK;
}

int lbm_slice_spec_default(lbm_slice_spec *v, int nx, int ny, int nz) {
  if (!v || nx < 1 || ny < 1 || nz < 1) return LBM_EINVAL;
  *v = lbm_slice_spec{};
  v->axis = 2;
  v->slice = nz / 2;
  v->u_scale = 0.05f;
  v->v_scale = 0.01f;
  v->vort_scale = 1.f;
  v->vort_gamma = 1.2f;
  v->width = nx;
  v->height = ny;
  return LBM_OK;
}

}  // extern "C"
