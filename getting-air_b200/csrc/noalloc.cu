// A dense step that allocates nothing: lbm_step_noalloc().
//
// Who needs it. Some callers cannot call cudaMalloc: a host that owns every
// byte of device memory through its own arena (an engine binding its own
// buffers through the FFI), a time-stepping loop that must not hit the
// implicit device-wide synchronisation of cudaMalloc/cudaFree while other
// streams are busy, or code that runs under a fixed memory budget decided
// up front. They already hold the populations; what the step additionally
// needs is scratch for the deterministic FP64 body-force reduction (one
// partial per launch block near the body, first-level group sums and a
// ticket counter, used by the sum launched after the step on the same
// stream). Here that scratch is a file-scope device array, so the entry
// point only launches.
//
// Limits and rules of use:
//  * the scratch holds kNoAllocMaxParts block partials (520 KiB with their
//    group sums and the ticket); a body whose force region needs more
//    launch blocks is refused with LBM_ENOSPC before anything is launched;
//  * every GPU that loads this library holds the array until the process
//    exits;
//  * a call outside stream capture looks up the array's device address
//    (cudaGetSymbolAddress) with the calling device current and keeps it
//    for that device; a call made while its stream is capturing uses the
//    kept address, so the first call on a device must come before any
//    capture. The lookup on every uncaptured call also means that a context
//    torn down by cudaDeviceReset is followed by a fresh address, not a
//    stale one; a graph captured before such a reset must not be replayed;
//  * all calls on a device share the one array, which keeps the last call's
//    contents. Each call clears the sum's ticket on its stream before the
//    step (the only scratch that must start at zero; partials and group
//    sums are written before they are read), so a sum that an earlier call
//    left unfinished cannot skew a later one. Two calls whose kernels
//    overlap on the GPU still race on the array: serialise them (one stream,
//    or events between streams);
//  * force_out, when given, is always written on the stream: the body's
//    force, or zeros when no cell of the domain can reach the body.
//
// The step itself is the dense kernel of dense_kernels.cu, unchanged.

#include <cstring>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/lbm.h"
#include "dense.cuh"
#include "host_params.cuh"

namespace {

constexpr int kNoAllocMaxParts = 8192;
// Partials (kForceSlots doubles per block), the group sums, then one slot
// whose first four bytes are the ticket (zero at load, and after every sum).
constexpr int kMaxGroups = (kNoAllocMaxParts + lbm::kSumGroup - 1) / lbm::kSumGroup;
constexpr int kScratchDoubles = (kNoAllocMaxParts + kMaxGroups) * lbm::kForceSlots + 32;

static __device__ __align__(256) double g_step_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double *g_scratch_addr[kMaxDevices] = {};
thread_local std::string g_noalloc_error;

int nfail(int code, const std::string &m) {
  g_noalloc_error = m;
  return code;
}

// Device address of the scratch array on the current device: looked up
// (and kept) when the stream is not capturing, the kept one otherwise.
int scratch_for_current_device(cudaStream_t st, double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return nfail(LBM_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return nfail(LBM_ENOTSUP, "device index beyond the scratch cache");
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cs);
  if (e != cudaSuccess) return nfail(LBM_ECUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_mutex);
  if (cs == cudaStreamCaptureStatusNone) {
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_step_scratch);
    if (e != cudaSuccess || !ptr)
      return nfail(LBM_ECUDA, std::string("cudaGetSymbolAddress(step scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = (double *)ptr;
  } else if (!g_scratch_addr[dev]) {
    return nfail(LBM_ESTATE, "the first lbm_step_noalloc call on a device must come before any stream capture");
  }
  *out = g_scratch_addr[dev];
  return LBM_OK;
}

}  // namespace

extern "C" {

const char *lbm_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

int lbm_step_noalloc(const lbm_config *cfg, const void *f_in, void *f_out, float *mac, double *force_out,
                     void *cuda_stream) {
  std::string why;
  if (lbm::validate_config(cfg, why)) return nfail(LBM_EINVAL, why);
  const int64_t n = (int64_t)cfg->nx * cfg->ny * cfg->nz;
  lbm::StepParams p{};
  lbm::fill_step_params(*cfg, n, 0, p);
  // the reach box and force region exactly as a session sets them
  if (lbm::set_body_regions(*cfg, p, force_out != nullptr)) {
    const int64_t parts = (int64_t)(p.rbx1 - p.rbx0) * (p.rby1 - p.rby0) * (p.rbz1 - p.rbz0);
    if (parts > kNoAllocMaxParts)
      return nfail(LBM_ENOSPC, "the body's force region spans " + std::to_string(parts) +
                                   " launch blocks; the fixed scratch holds " + std::to_string(kNoAllocMaxParts));
  }
  if (!f_in || !f_out || f_in == f_out) return nfail(LBM_EINVAL, "f_in and f_out must be distinct device buffers");
  cudaStream_t st = (cudaStream_t)cuda_stream;
  double *scratch = nullptr;
  int rc = scratch_for_current_device(st, &scratch);
  if (rc) return rc;
  p.partials = scratch;
  p.groups = scratch + kNoAllocMaxParts * lbm::kForceSlots;
  p.counter = reinterpret_cast<unsigned int *>(p.groups + kMaxGroups * lbm::kForceSlots);
  p.force_out = force_out;
  p.write_mac = mac ? 1 : 0;
  cudaError_t z = cudaSuccess;
  if (p.force_on)
    z = cudaMemsetAsync(p.counter, 0, sizeof(unsigned int), st);
  else if (force_out)
    z = cudaMemsetAsync(force_out, 0, lbm::kForceSlots * sizeof(double), st);
  if (z != cudaSuccess) return nfail(LBM_ECUDA, std::string("clear: ") + cudaGetErrorString(z));
  const cudaError_t e = lbm::launch_step(cfg->q, cfg->storage, f_in, f_out, mac, p, st);
  if (e != cudaSuccess) return nfail(LBM_ECUDA, std::string("step: ") + cudaGetErrorString(e));
  return LBM_OK;
}

}  // extern "C"
