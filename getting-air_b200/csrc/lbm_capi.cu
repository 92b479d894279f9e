// C ABI of the dense solver: session lifetime, state transfer, stepping and
// the FP64 reductions. Host side of the reference's page objects
// (main-3d.js encodeSteps / debugStepSync / readStats and
// main-cylinder.js's step loop), without WebGPU: a session owns two f
// buffers (ping-pong), the mac field and the reduction scratch, and launches
// on one CUDA stream.

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "../../include/lbm.h"
#include "dense.cuh"
#include "host_params.cuh"
#include "lattice.cuh"
#include "sample.cuh"

using namespace lbm;

struct lbm_session {
  lbm_config cfg{};
  int q = 0, storage = 0, elem = 4;
  int64_t n = 0;
  void *f[2] = {nullptr, nullptr};
  int cur = 0;
  float *mac = nullptr;
  double *force_partials = nullptr;
  double *force_groups = nullptr;  // first-level sums of the partials
  unsigned int *force_counter = nullptr;
  double *force_out = nullptr;
  int force_nparts = 0;
  double *tot_partials = nullptr;
  unsigned int *tot_counter = nullptr;
  double *tot_out = nullptr;
  double *host_out = nullptr;  // pinned, 16 doubles
  cudaStream_t own = nullptr, stream = nullptr;
  StepParams sp{};
  int64_t bytes = 0;
  std::string err;
  // Free body: two poses (by step parity) and the integrator state.
  bool free_body = false;
  int body_par = 0;
  int cap[3] = {0, 0, 0};
  BodyPose *pose = nullptr;
  BodyDyn *dyn = nullptr;
  // A z-slab of the domain cfg describes (lbm_create_slab): planes
  // [z0, z0 + nzl) stored as planes 1..nzl between two ghost planes, so n
  // counts nzl + 2 planes and `cells` the nzl the caller sees.
  bool slab = false;
  int z0 = 0, nzl = 0;
  int64_t nxy = 0, cells = 0;
};

namespace {

thread_local std::string g_create_error;

int fail(lbm_session *s, int code, const std::string &msg) {
  if (s) s->err = msg; else g_create_error = msg;
  return code;
}

int cuda_fail(lbm_session *s, cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return fail(s, e == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA, m);
}

#define CK(s, call)                                   \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(s, e_, #call); \
  } while (0)

template <int Q> void tables(int32_t *ex, int32_t *ey, int32_t *ez, float *w, int32_t *opp) {
  for (int i = 0; i < Q; ++i) {
    if (ex) ex[i] = Lattice<Q>::ex(i);
    if (ey) ey[i] = Lattice<Q>::ey(i);
    if (ez) ez[i] = Lattice<Q>::ez(i);
    if (w) w[i] = Lattice<Q>::w(i);
    if (opp) opp[i] = Lattice<Q>::opp(i);
  }
}

// Which launch blocks can receive a force contribution (the blocks covering
// the cell box of force_cell_box()) and the bounce-back reach box.
void set_force_region(lbm_session *s) { set_body_regions(s->cfg, s->sp, true); }

// Force scratch for `need` partials per step (grown, never shrunk; the
// stream is drained first since launches in flight may still read it).
int grow_force_scratch(lbm_session *s, int need) {
  if (need <= s->force_nparts) return LBM_OK;
  if (s->force_partials) {
    cudaStreamSynchronize(s->stream);
    cudaFree(s->force_partials);
    cudaFree(s->force_groups);
    s->bytes -= (int64_t)(2 * s->force_nparts + sum_groups(s->force_nparts)) * kForceSlots * 8;
  }
  s->force_partials = nullptr;
  s->force_groups = nullptr;
  s->force_nparts = 0;
  // two sets of partials: consecutive steps of one lbm_step() alternate
  CK(s, cudaMalloc(&s->force_partials, (size_t)2 * need * kForceSlots * sizeof(double)));
  CK(s, cudaMalloc(&s->force_groups, (size_t)sum_groups(need) * kForceSlots * sizeof(double)));
  s->force_nparts = need;
  s->bytes += (int64_t)(2 * need + sum_groups(need)) * kForceSlots * 8;
  s->sp.partials = s->force_partials;
  s->sp.groups = s->force_groups;
  return LBM_OK;
}

int ensure_force_scratch(lbm_session *s) {
  const StepParams &p = s->sp;
  if (!p.force_on) return LBM_OK;
  return grow_force_scratch(s, (p.rbx1 - p.rbx0) * (p.rby1 - p.rby0) * (p.rbz1 - p.rbz0));
}

void fill_params(lbm_session *s) {
  StepParams &p = s->sp;
  fill_step_params(s->cfg, s->n, 0, p);
  p.partials = s->force_partials;
  p.groups = s->force_groups;
  p.counter = s->force_counter;
  p.force_out = s->force_out;
  set_force_region(s);  // in the whole domain's planes
  if (!s->slab) return;
  // a slab: stored plane z is domain plane z + z0 - 1; its force region is
  // its own share of the domain's (slabs take no window, so no seam)
  p.nz = s->nzl + 2;
  p.zoff = s->z0 - 1;
  p.nzg = s->cfg.nz;
  p.zlo = 1;
  if (p.force_on) {
    p.rbz0 = std::max(p.rbz0, s->z0);
    p.rbz1 = std::min(p.rbz1, s->z0 + s->nzl);
    if (p.rbz0 >= p.rbz1) p.force_on = 0;
  }
}

// Copies between the caller's array of the session's cells (Q planes of
// `cells`, or 4 floats per cell with planes = 1, width 16) and a device
// array of the stored layout: a slab skips its ghost plane below and above.
cudaError_t copy_cells(lbm_session *s, void *dst, const void *src, size_t elem, int planes, cudaMemcpyKind kind) {
  if (!s->slab)
    return cudaMemcpyAsync(dst, src, elem * (size_t)planes * s->n, kind, s->stream);
  const size_t w = elem * (size_t)s->cells, skip = elem * (size_t)s->nxy, stored = elem * (size_t)s->n;
  if (kind == cudaMemcpyDeviceToHost)
    return cudaMemcpy2DAsync(dst, w, (const char *)src + skip, stored, w, planes, kind, s->stream);
  return cudaMemcpy2DAsync((char *)dst + skip, stored, src, w, w, planes, kind, s->stream);
}

void release(lbm_session *s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  cudaFree(s->f[0]);
  cudaFree(s->f[1]);
  cudaFree(s->mac);
  cudaFree(s->force_partials);
  cudaFree(s->force_groups);
  cudaFree(s->force_counter);
  cudaFree(s->force_out);
  cudaFree(s->tot_partials);
  cudaFree(s->tot_counter);
  cudaFree(s->tot_out);
  cudaFree(s->pose);
  cudaFree(s->dyn);
  if (s->host_out) cudaFreeHost(s->host_out);
  if (s->own) cudaStreamDestroy(s->own);
}

}  // namespace

extern "C" {

const char *lbm_version(void) { return "getting-air-b200 dense 0.1 (sm_100a)"; }
int lbm_abi_version(void) { return LBM_ABI_VERSION; }

int lbm_config_default(lbm_config *cfg, int q, int nx, int ny, int nz) {
  if (!cfg) return LBM_EINVAL;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->q = q;
  cfg->nx = nx; cfg->ny = ny; cfg->nz = nz;
  cfg->tau = 0.8f;  // OMEGA 1.25 (common_d3_step.wgsl:151)
  cfg->solid_eq = 1;
  cfg->rho_w_local = 1;
  cfg->swept_force = 1;
  cfg->chi_eps = 1.5f;
  cfg->sponge_w = q == 9 ? 4.0f : 0.0f;  // lbm_step.wgsl SPONGE_W = 4; 3D default 0
  cfg->sponge_axis[0] = cfg->sponge_axis[1] = cfg->sponge_axis[2] = 1;
  cfg->body.qw = 1.0f;
  cfg->body.shape = q == 9 ? LBM_SHAPE_ELLIPSE : LBM_SHAPE_SPHERE;
  cfg->storage = LBM_STORE_FP32;
  return LBM_OK;
}

namespace {
int create_session(const lbm_config *cfg, int z0, int nzl, bool slab, lbm_session **out) {
  if (!out) return fail(nullptr, LBM_EINVAL, "out is NULL");
  *out = nullptr;
  std::string why;
  int rc = validate_config(cfg, why);
  if (rc) return fail(nullptr, rc, why);
  if (slab) {
    if (cfg->q == 9) return fail(nullptr, LBM_EINVAL, "slabs split a 3D domain along z");
    if (cfg->window[0] || cfg->window[1] || cfg->window[2])
      return fail(nullptr, LBM_ENOTSUP, "a slab takes no moving window");
    if (nzl < 1 || z0 < 0 || z0 + nzl > cfg->nz)
      return fail(nullptr, LBM_EINVAL, "the slab [z0, z0 + nz_local) must lie in [0, nz)");
  }
  lbm_session *s = new lbm_session();
  s->cfg = *cfg;
  s->q = cfg->q;
  s->storage = cfg->storage;
  s->elem = cfg->storage == LBM_STORE_FP32 ? 4 : 2;
  s->slab = slab;
  s->z0 = slab ? z0 : 0;
  s->nzl = slab ? nzl : cfg->nz;
  s->nxy = (int64_t)cfg->nx * cfg->ny;
  s->cells = s->nxy * s->nzl;
  s->n = s->nxy * (slab ? nzl + 2 : cfg->nz);
  auto bail = [&](cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    release(s);
    delete s;
    return fail(nullptr, e == cudaErrorMemoryAllocation ? LBM_ENOMEM : LBM_ECUDA, m);
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking))) return bail(e, "stream");
  s->stream = s->own;
  const size_t fbytes = (size_t)s->q * s->n * s->elem;
  if ((e = cudaMalloc(&s->f[0], fbytes))) return bail(e, "cudaMalloc f[0]");
  if ((e = cudaMalloc(&s->f[1], fbytes))) return bail(e, "cudaMalloc f[1]");
  if ((e = cudaMalloc(&s->mac, (size_t)s->n * 16))) return bail(e, "cudaMalloc mac");
  if ((e = cudaMalloc(&s->force_counter, sizeof(unsigned int)))) return bail(e, "cudaMalloc counter");
  if ((e = cudaMalloc(&s->force_out, kForceSlots * sizeof(double)))) return bail(e, "cudaMalloc force");
  if ((e = cudaMalloc(&s->tot_partials, (size_t)totals_blocks() * kTotalsSlots * sizeof(double))))
    return bail(e, "cudaMalloc totals");
  if ((e = cudaMalloc(&s->tot_counter, sizeof(unsigned int)))) return bail(e, "cudaMalloc counter");
  if ((e = cudaMalloc(&s->tot_out, kTotalsSlots * sizeof(double)))) return bail(e, "cudaMalloc totals");
  if ((e = cudaMallocHost(&s->host_out, 16 * sizeof(double)))) return bail(e, "cudaMallocHost");
  cudaMemsetAsync(s->force_counter, 0, sizeof(unsigned int), s->stream);
  cudaMemsetAsync(s->tot_counter, 0, sizeof(unsigned int), s->stream);
  cudaMemsetAsync(s->force_out, 0, kForceSlots * sizeof(double), s->stream);
  cudaMemsetAsync(s->mac, 0, (size_t)s->n * 16, s->stream);
  cudaMemsetAsync(s->f[0], 0, fbytes, s->stream);
  s->bytes = 2 * (int64_t)fbytes + s->n * 16 + totals_blocks() * kTotalsSlots * 8 + 200;
  fill_params(s);
  if (ensure_force_scratch(s)) {
    std::string m = s->err;
    release(s);
    delete s;
    return fail(nullptr, LBM_ENOMEM, m);
  }
  s->sp.partials = s->force_partials;
  if ((e = cudaStreamSynchronize(s->stream))) return bail(e, "initialise");
  *out = s;
  return LBM_OK;
}
}  // namespace

int lbm_create(const lbm_config *cfg, lbm_session **out) { return create_session(cfg, 0, 0, false, out); }

int lbm_create_slab(const lbm_config *cfg, int z0, int nz_local, lbm_session **out) {
  return create_session(cfg, z0, nz_local, true, out);
}

int64_t lbm_slab_halo_bytes(const lbm_session *s) {
  if (!s || !s->slab) return 0;
  return s->nxy * (s->q == 19 ? 5 : 9) * s->elem;
}

namespace {
// The populations that cross a slab's z faces: ez = +1 leave through the top
// (the slab above pulls them from its ghost plane below), ez = -1 through
// the bottom; in ascending direction order on every slab.
int crossing(int q, int ez, int idx[9]) {
  int k = 0;
  for (int i = 0; i < q; ++i) {
    const int e = q == 19 ? Lattice<19>::ez(i) : Lattice<27>::ez(i);
    if (e == ez) idx[k++] = i;
  }
  return k;
}
}  // namespace

int lbm_slab_pack(lbm_session *s, void *send_lo, void *send_hi) {
  if (!s || !s->slab) return s ? fail(s, LBM_EINVAL, "not a slab session") : LBM_EINVAL;
  if (!send_lo || !send_hi) return fail(s, LBM_EINVAL, "send buffers are NULL");
  const size_t plane = (size_t)s->nxy * s->elem;
  const char *f = (const char *)s->f[s->cur];
  int idx[9];
  // the first stored plane's downward populations, the last one's upward
  int k = crossing(s->q, -1, idx);
  for (int j = 0; j < k; ++j)
    CK(s, cudaMemcpyAsync((char *)send_lo + j * plane, f + ((size_t)idx[j] * s->n + s->nxy) * s->elem, plane,
                          cudaMemcpyDeviceToDevice, s->stream));
  k = crossing(s->q, 1, idx);
  for (int j = 0; j < k; ++j)
    CK(s, cudaMemcpyAsync((char *)send_hi + j * plane,
                          f + ((size_t)idx[j] * s->n + (size_t)s->nzl * s->nxy) * s->elem, plane,
                          cudaMemcpyDeviceToDevice, s->stream));
  return LBM_OK;
}

int lbm_slab_unpack(lbm_session *s, const void *recv_lo, const void *recv_hi) {
  if (!s || !s->slab) return s ? fail(s, LBM_EINVAL, "not a slab session") : LBM_EINVAL;
  if (!recv_lo || !recv_hi) return fail(s, LBM_EINVAL, "receive buffers are NULL");
  const size_t plane = (size_t)s->nxy * s->elem;
  char *f = (char *)s->f[s->cur];
  int idx[9];
  // from the slab below: its upward populations, into the ghost plane below
  int k = crossing(s->q, 1, idx);
  for (int j = 0; j < k; ++j)
    CK(s, cudaMemcpyAsync(f + (size_t)idx[j] * s->n * s->elem, (const char *)recv_lo + j * plane, plane,
                          cudaMemcpyDeviceToDevice, s->stream));
  // from the slab above: its downward populations, into the ghost plane above
  k = crossing(s->q, -1, idx);
  for (int j = 0; j < k; ++j)
    CK(s, cudaMemcpyAsync(f + ((size_t)idx[j] * s->n + (size_t)(s->nzl + 1) * s->nxy) * s->elem,
                          (const char *)recv_hi + j * plane, plane, cudaMemcpyDeviceToDevice, s->stream));
  return LBM_OK;
}

void lbm_destroy(lbm_session *s) {
  release(s);
  delete s;
}

const char *lbm_last_error(const lbm_session *s) {
  return s ? s->err.c_str() : g_create_error.c_str();
}

int lbm_set_stream(lbm_session *s, void *stream) {
  if (!s) return LBM_EINVAL;
  CK(s, cudaStreamSynchronize(s->stream));
  s->stream = stream ? (cudaStream_t)stream : s->own;
  return LBM_OK;
}

int lbm_init_macro(lbm_session *s, const float *mac) {
  if (!s || !mac) return s ? fail(s, LBM_EINVAL, "mac is NULL") : LBM_EINVAL;
  // (a slab's ghost planes keep a zero mac: their populations are only read
  // after a halo exchange has written them)
  CK(s, copy_cells(s, s->mac, mac, 16, 1, cudaMemcpyHostToDevice));
  CK(s, launch_init_eq(s->q, s->storage, s->mac, s->f[s->cur], s->n, s->sp.pk, s->stream));
  CK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int lbm_write_f(lbm_session *s, const float *f) {
  if (!s || !f) return s ? fail(s, LBM_EINVAL, "f is NULL") : LBM_EINVAL;
  const size_t bytes = (size_t)s->q * s->n * 4;
  if (s->storage == LBM_STORE_FP32) {
    CK(s, copy_cells(s, s->f[s->cur], f, 4, s->q, cudaMemcpyHostToDevice));
  } else {
    float *tmp = nullptr;
    CK(s, cudaMallocAsync(&tmp, bytes, s->stream));
    cudaError_t e = copy_cells(s, tmp, f, 4, s->q, cudaMemcpyHostToDevice);
    if (!e) e = launch_pack(s->q, s->storage, tmp, s->f[s->cur], s->n, s->sp.pk, s->stream);
    cudaFreeAsync(tmp, s->stream);
    if (e) return cuda_fail(s, e, "pack f");
  }
  CK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int lbm_read_f(lbm_session *s, float *f) {
  if (!s || !f) return s ? fail(s, LBM_EINVAL, "f is NULL") : LBM_EINVAL;
  const size_t bytes = (size_t)s->q * s->n * 4;
  if (s->storage == LBM_STORE_FP32) {
    CK(s, copy_cells(s, f, s->f[s->cur], 4, s->q, cudaMemcpyDeviceToHost));
  } else {
    float *tmp = nullptr;
    CK(s, cudaMallocAsync(&tmp, bytes, s->stream));
    cudaError_t e = launch_unpack(s->q, s->storage, s->f[s->cur], tmp, s->n, s->sp.pk, s->stream);
    if (!e) e = copy_cells(s, f, tmp, 4, s->q, cudaMemcpyDeviceToHost);
    cudaFreeAsync(tmp, s->stream);
    if (e) return cuda_fail(s, e, "unpack f");
  }
  CK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int lbm_write_f_raw(lbm_session *s, const void *planes) {
  if (!s || !planes) return s ? fail(s, LBM_EINVAL, "planes is NULL") : LBM_EINVAL;
  CK(s, copy_cells(s, s->f[s->cur], planes, s->elem, s->q, cudaMemcpyHostToDevice));
  CK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int lbm_read_f_raw(lbm_session *s, void *planes) {
  if (!s || !planes) return s ? fail(s, LBM_EINVAL, "planes is NULL") : LBM_EINVAL;
  CK(s, copy_cells(s, planes, s->f[s->cur], s->elem, s->q, cudaMemcpyDeviceToHost));
  CK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int lbm_read_mac(lbm_session *s, float *mac) {
  if (!s || !mac) return s ? fail(s, LBM_EINVAL, "mac is NULL") : LBM_EINVAL;
  CK(s, copy_cells(s, mac, s->mac, 16, 1, cudaMemcpyDeviceToHost));
  CK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int lbm_step(lbm_session *s, int n) {
  if (!s) return LBM_EINVAL;
  if (n < 0) return fail(s, LBM_EINVAL, "step count must be >= 0");
  if (s->free_body) {
    for (int k = 0; k < n; ++k) {
      StepParams fp = s->sp;
      fp.pose_in = s->pose + s->body_par;
      fp.pose_out = s->pose + (1 - s->body_par);
      fp.dyn = s->dyn;
      fp.force_on = 1;
      fp.write_mac = 0;
      CK(s, launch_force_pass(s->q, s->storage, s->f[s->cur], fp, s->cap, s->stream));
      StepParams sp = s->sp;
      sp.pose_in = s->pose + (1 - s->body_par);
      sp.force_on = 0;
      sp.write_mac = (k == n - 1);
      CK(s, launch_step(s->q, s->storage, s->f[s->cur], s->f[1 - s->cur], s->mac, sp, s->stream));
      s->cur = 1 - s->cur;
      s->body_par = 1 - s->body_par;
    }
    return LBM_OK;
  }
  // Each step's force partials are summed by the next step's first block;
  // the last step's by the one-CTA sum launch_step() adds after it.
  const int64_t half = (int64_t)s->force_nparts * kForceSlots;
  const int parts = s->sp.force_on ? force_parts(s->q, s->sp) : 0;
  for (int k = 0; k < n; ++k) {
    StepParams &sp = s->sp;
    sp.write_mac = (k == n - 1);
    sp.partials = s->force_partials + (k & 1) * half;
    sp.defer_force = k < n - 1;
    sp.prev_parts = k > 0 ? parts : 0;
    sp.prev_partials = s->force_partials + ((k + 1) & 1) * half;
    CK(s, launch_step(s->q, s->storage, s->f[s->cur], s->f[1 - s->cur], s->mac, sp, s->stream));
    s->cur = 1 - s->cur;
  }
  s->sp.partials = s->force_partials;
  s->sp.defer_force = 0;
  s->sp.prev_parts = 0;
  return LBM_OK;
}

int lbm_set_body(lbm_session *s, const lbm_body *body) {
  if (!s || !body) return s ? fail(s, LBM_EINVAL, "body is NULL") : LBM_EINVAL;
  lbm_config c = s->cfg;
  c.body = *body;
  std::string why;
  if (validate_config(&c, why)) return fail(s, LBM_EINVAL, why);
  s->cfg = c;
  s->free_body = false;
  fill_params(s);
  int rc = ensure_force_scratch(s);
  if (rc) return rc;
  s->sp.partials = s->force_partials;
  return LBM_OK;
}

int lbm_set_free_body(lbm_session *s, const lbm_body_state *state, const lbm_body_opts *opts) {
  if (!s) return LBM_EINVAL;
  if (!state) {
    s->free_body = false;
    return LBM_OK;
  }
  const lbm_config &c = s->cfg;
  if (c.q == 9) return fail(s, LBM_ENOTSUP, "free bodies are 3D only");
  if (s->slab) return fail(s, LBM_ENOTSUP, "a free body moves across slabs: it runs in a whole domain");
  if (!c.has_body) return fail(s, LBM_EINVAL, "the session has no body");
  const lbm_body_state &st = *state;
  bool ok = st.mass > 0.0 && std::isfinite(st.mass);
  for (int k = 0; k < 3; ++k)
    ok = ok && st.ibody[k] > 0.0 && std::isfinite(st.ibody[k]) && std::isfinite(st.x[k]) &&
         std::isfinite(st.v[k]) && std::isfinite(st.L[k]);
  const double qn = st.q[0] * st.q[0] + st.q[1] * st.q[1] + st.q[2] * st.q[2] + st.q[3] * st.q[3];
  if (!ok || !(qn > 0.5 && qn < 2.0)) return fail(s, LBM_EINVAL, "body state must be finite, massive and unit-quaternion");
  lbm_body_opts o;
  if (opts) o = *opts; else lbm_body_opts_default(&o);
  {
    // a windowed axis wraps the body at the domain length (winWrapPos)
    const int len[3] = {c.nx, c.ny, c.nz};
    for (int k = 0; k < 3; ++k)
      if (c.window[k]) o.wrap[k] = len[k];
  }
  BodyDyn d{};
  d.st = st;
  d.opt = o;
  d.shape = c.body;
  d.q = c.q; d.nx = c.nx; d.ny = c.ny; d.nz = c.nz;
  d.bounceback = c.use_bounceback;
  d.swept_force = c.swept_force;
  d.chi_eps = c.chi_eps;
  for (int k = 0; k < 3; ++k) d.win[k] = c.window[k];
  // Largest force box the body can need: its reach at the clamped speeds
  // (the whole domain when a clamp is off).
  const double rc = body_circumradius(c.body);
  const double vmax = (o.v_max > 0.0 && std::isfinite(o.v_max)) ? o.v_max : INFINITY;
  const double omax = (o.o_max > 0.0 && std::isfinite(o.o_max)) ? o.o_max : INFINITY;
  const double speed = vmax + 1.5 * omax * rc + 0.5;
  const double margin = c.use_bounceback ? 3.0 + speed : 8.0 * c.chi_eps + 2.0;
  const double cells = 2.0 * std::ceil(rc + margin) + 3.0;
  const int nbx = (c.nx + kStepThreads - 1) / kStepThreads;
  d.cap[0] = std::isfinite(cells) ? (int)std::min<double>(nbx, std::ceil(cells / kStepThreads) + 1) : nbx;
  d.cap[1] = std::isfinite(cells) ? (int)std::min<double>(c.ny, cells) : c.ny;
  d.cap[2] = std::isfinite(cells) ? (int)std::min<double>(c.nz, cells) : c.nz;
  BodyPose p0{};
  p0.body = body_pose(c.body, st);
  int box[6];
  if (!body_cell_box(p0.body, c.q, c.nx, c.ny, c.nz, c.use_bounceback, c.swept_force, c.chi_eps, box, &p0.swept,
                     &p0.swept_band, c.window)) {
    const float ctr[3] = {p0.body.cx, p0.body.cy, p0.body.cz};
    const int len[3] = {c.nx, c.ny, c.nz};
    for (int a = 0; a < 3; ++a) {
      const int v = (int)std::fmin(std::fmax(ctr[a], 0.f), (float)(len[a] - 1));
      box[2 * a] = box[2 * a + 1] = v;
    }
  }
  box_region(box, c.nx, c.ny, c.nz, d.cap, p0.region);
  const int need = d.cap[0] * d.cap[1] * d.cap[2];
  if (int rc = grow_force_scratch(s, need)) return rc;
  if (!s->pose) {
    CK(s, cudaMalloc(&s->pose, 2 * sizeof(BodyPose)));
    CK(s, cudaMalloc(&s->dyn, sizeof(BodyDyn)));
    s->bytes += 2 * sizeof(BodyPose) + sizeof(BodyDyn);
  }
  CK(s, cudaMemcpyAsync(s->pose, &p0, sizeof(BodyPose), cudaMemcpyHostToDevice, s->stream));
  CK(s, cudaMemcpyAsync(s->dyn, &d, sizeof(BodyDyn), cudaMemcpyHostToDevice, s->stream));
  CK(s, cudaStreamSynchronize(s->stream));
  for (int k = 0; k < 3; ++k) s->cap[k] = d.cap[k];
  s->body_par = 0;
  s->free_body = true;
  return LBM_OK;
}

int lbm_resample(lbm_session *s, const lbm_volume_spec *spec, void *out, uint8_t *level) {
  if (!s) return LBM_EINVAL;
  std::string why;
  if (validate_volume(spec, why)) return fail(s, LBM_EINVAL, why);
  if (s->slab) return fail(s, LBM_ENOTSUP, "the headless views read a whole domain");
  if (!out) return fail(s, LBM_EINVAL, "out is NULL");
  if (s->q == 9) return fail(s, LBM_ENOTSUP, "the headless views are 3D");
  const lbm_config &c = s->cfg;
  const TreeView t{(const float4 *)s->mac, c.nx, c.ny, c.nz, 0, nullptr, nullptr, 1, 1, 1};
  CK(s, run_resample(t, *spec, out, level, s->stream));
  return LBM_OK;
}

int lbm_render_slice(lbm_session *s, const lbm_slice_spec *spec, uint8_t *rgba) {
  if (!s) return LBM_EINVAL;
  const lbm_config &c = s->cfg;
  std::string why;
  if (validate_slice(spec, c.nx, c.ny, c.nz, why)) return fail(s, LBM_EINVAL, why);
  if (!rgba) return fail(s, LBM_EINVAL, "rgba is NULL");
  if (s->slab) return fail(s, LBM_ENOTSUP, "the headless views read a whole domain");
  if (s->q == 9) return fail(s, LBM_ENOTSUP, "the headless views are 3D");
  // winViewOffset: the view pans with the body under a moving window
  ViewOffset off{{0.f, 0.f, 0.f}};
  if (c.window[0] || c.window[1] || c.window[2]) {
    float ctr[3] = {c.body.cx, c.body.cy, c.body.cz};
    if (s->free_body) {
      lbm_body_state st;
      CK(s, cudaMemcpyAsync(&st, &s->dyn->st, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
      CK(s, cudaStreamSynchronize(s->stream));
      for (int k = 0; k < 3; ++k) ctr[k] = (float)st.x[k];
    }
    for (int k = 0; k < 3; ++k)
      if (c.window[k]) off.v[k] = ctr[k] - (float)c.win_anchor[k];
  }
  const TreeView t{(const float4 *)s->mac, c.nx, c.ny, c.nz, 0, nullptr, nullptr, 1, 1, 1};
  CK(s, run_slice(t, *spec, off, rgba, s->stream));
  return LBM_OK;
}

int lbm_read_body_state(lbm_session *s, lbm_body_state *out) {
  if (!s || !out) return s ? fail(s, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  if (!s->free_body) return fail(s, LBM_EINVAL, "the body is not free (lbm_set_free_body)");
  CK(s, cudaMemcpyAsync(out, &s->dyn->st, sizeof(lbm_body_state), cudaMemcpyDeviceToHost, s->stream));
  CK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int lbm_forces(lbm_session *s, double out[6]) {
  if (!s || !out) return s ? fail(s, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  if (!s->sp.force_on && !s->free_body) {
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    return LBM_OK;
  }
  CK(s, cudaMemcpyAsync(s->host_out, s->force_out, 6 * sizeof(double), cudaMemcpyDeviceToHost,
                        s->stream));
  CK(s, cudaStreamSynchronize(s->stream));
  for (int k = 0; k < 6; ++k) out[k] = s->host_out[k];
  return LBM_OK;
}

namespace {
// Six doubles from device memory into pinned host memory the device can
// address: a one-warp kernel on the stream instead of a copy-engine
// transfer, whose start and finish between two kernels cost the stream
// several microseconds (measured on B200 in a loop of one-step calls, each
// followed by the force readback: 0.135 ms per step with the copy).
__global__ void copy_force_to_host(const double *__restrict__ src, double *dst) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (threadIdx.x < 6) dst[threadIdx.x] = src[threadIdx.x];
}
}  // namespace

int lbm_forces_async(lbm_session *s, double out[6]) {
  if (!s || !out) return s ? fail(s, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  if (!s->sp.force_on && !s->free_body) {
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    return LBM_OK;
  }
  // Pinned (page-locked) host memory has a device address under unified
  // addressing; anything else goes through the copy engine as before.
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, out) == cudaSuccess && at.type == cudaMemoryTypeHost && at.devicePointer) {
    {
      // launched like the step kernels (programmatic dependent launch); the
      // kernel waits for the previous one before it reads the force
      cudaLaunchConfig_t lc = {};
      lc.gridDim = dim3(1);
      lc.blockDim = dim3(32);
      lc.stream = s->stream;
      cudaLaunchAttribute la[1];
      la[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      la[0].val.programmaticStreamSerializationAllowed = 1;
      lc.attrs = la;
      lc.numAttrs = 1;
      cudaLaunchKernelEx(&lc, copy_force_to_host, (const double *)s->force_out, (double *)at.devicePointer);
    }
    CK(s, cudaGetLastError());
    return LBM_OK;
  }
  cudaGetLastError();  // a pageable pointer is no error here
  CK(s, cudaMemcpyAsync(out, s->force_out, 6 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  return LBM_OK;
}

int lbm_totals(lbm_session *s, double out[8]) {
  if (!s || !out) return s ? fail(s, LBM_EINVAL, "out is NULL") : LBM_EINVAL;
  // a slab's own planes: past the ghost plane below, n cells apart per population
  const char *f0 = (const char *)s->f[s->cur] + (s->slab ? s->nxy * s->elem : 0);
  CK(s, launch_totals(s->q, s->storage, f0, s->cells, s->sp.pk, s->tot_partials, s->tot_counter, s->tot_out,
                      s->stream, s->n));
  CK(s, cudaMemcpyAsync(s->host_out, s->tot_out, 8 * sizeof(double), cudaMemcpyDeviceToHost,
                        s->stream));
  CK(s, cudaStreamSynchronize(s->stream));
  for (int k = 0; k < 8; ++k) out[k] = s->host_out[k];
  return LBM_OK;
}

int lbm_sync(lbm_session *s) {
  if (!s) return LBM_EINVAL;
  CK(s, cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

int64_t lbm_device_bytes(const lbm_session *s) { return s ? s->bytes : 0; }

int lbm_lattice_tables(int q, int32_t *ex, int32_t *ey, int32_t *ez, float *w, int32_t *opp) {
  switch (q) {
    case 9: tables<9>(ex, ey, ez, w, opp); return LBM_OK;
    case 19: tables<19>(ex, ey, ez, w, opp); return LBM_OK;
    case 27: tables<27>(ex, ey, ez, w, opp); return LBM_OK;
    default: return LBM_EINVAL;
  }
}

// Round-to-nearest-even f32 -> binary16 through the f32 bit pattern, the
// semantics of f-pack.mjs:44-77 (which is what the GPU's pack2x16float does).
uint16_t lbm_f32_to_f16_bits(float v) {
  uint32_t x;
  std::memcpy(&x, &v, 4);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const int exp = (int)((x >> 23) & 0xffu);
  uint32_t man = x & 0x7fffffu;
  if (exp == 0xff) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u : 0u));
  const int e = exp - 112;
  if (e >= 0x1f) return (uint16_t)(sign | 0x7c00u);
  if (e <= 0) {
    if (e < -10) return (uint16_t)sign;
    man |= 0x800000u;
    const int shift = 14 - e;
    uint32_t h = man >> shift;
    const uint32_t rem = man & ((1u << shift) - 1u);
    const uint32_t half = 1u << (shift - 1);
    if (rem > half || (rem == half && (h & 1u))) h += 1;
    return (uint16_t)(sign | h);
  }
  uint32_t h = ((uint32_t)e << 10) | (man >> 13);
  const uint32_t rem = man & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1;
  return (uint16_t)(sign | h);
}

float lbm_f16_bits_to_f32(uint16_t h) {
  const float s = (h & 0x8000u) ? -1.0f : 1.0f;
  const int e = (h >> 10) & 0x1f;
  const int m = h & 0x3ff;
  if (e == 0) return s * (float)m * 5.9604644775390625e-8f;
  if (e == 31) return m ? NAN : s * INFINITY;
  return s * (1.0f + (float)m / 1024.0f) * std::ldexp(1.0f, e - 15);
}

}  // extern "C"
