// Block-wide exclusive prefix sum for the deterministic managers: one value
// per thread of a CTA of up to 1024 threads (a multiple of 32), warp
// shuffles then one warp over the warp totals. Every thread of the CTA must
// call it; `sm` holds 64 ints of shared memory.
#pragma once

#include <cuda_runtime.h>

namespace lbm {

__device__ __forceinline__ int block_scan(int v, int *sm, int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    sm[32 + lane] = w;
  }
  __syncthreads();
  total = sm[32 + (blockDim.x >> 5) - 1];
  const int before = (warp ? sm[32 + warp - 1] : 0) + x - v;
  __syncthreads();
  return before;
}

}  // namespace lbm
