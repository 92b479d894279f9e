// Headless views of the field: the tree sampler (common_d3_tree_sample.wgsl),
// the voxel resample (common_d3_resample.wgsl) and the axis-aligned slice
// (common_d3_render_slice.wgsl + common_vortcolor.wgsl) as compute kernels
// into a buffer.
#pragma once

#include <string>

#include <cuda_runtime.h>

#include "../../include/lbm.h"

namespace lbm {

// What the sampler reads: the dense L0 [rho, ux, uy, uz] per cell and, with
// levels = 1, the level-1 pool's [rho, u] per tile cell and its block map.
struct TreeView {
  const float4 *mac;
  int nx, ny, nz;
  int levels;
  const float4 *macp;
  const int *block_slot;
  int rb, fb, t3;
};

// Continuous view offset of a moving window (winViewOffset): the body's
// centre less its anchor on windowed axes.
struct ViewOffset {
  float v[3];
};

int validate_volume(const lbm_volume_spec *s, std::string &why);
int validate_slice(const lbm_slice_spec *s, int nx, int ny, int nz, std::string &why);

// Launches into device buffers (out: 4 halves or 4 floats per voxel; level
// may be NULL).
cudaError_t launch_resample(const TreeView &t, const lbm_volume_spec &s, void *out, uint8_t *level,
                            cudaStream_t st);
cudaError_t launch_slice(const TreeView &t, const lbm_slice_spec &s, ViewOffset off, uint8_t *rgba,
                         cudaStream_t st);

// The host side of both entry points: device pointers are used as given;
// host pointers get a device staging buffer, a copy back and a sync.
cudaError_t run_resample(const TreeView &t, const lbm_volume_spec &s, void *out, uint8_t *level, cudaStream_t st);
cudaError_t run_slice(const TreeView &t, const lbm_slice_spec &s, ViewOffset off, uint8_t *rgba, cudaStream_t st);

}  // namespace lbm
