/*
 * lbm.h -- C ABI of the B200 lattice-Boltzmann hot path.
 *
 * The reference (c7t/getting-air) drives its solver from JavaScript page
 * objects that own WebGPU buffers: `init` seeds f from a macroscopic field,
 * `step` encodes fused stream-collide dispatches, the force kernels feed
 * drag/lift, and host code sums conserved totals over a readback. This
 * header is the same behaviour as plain C entry points over an opaque
 * session that owns its device memory, so a Node N-API shim, a ctypes
 * stub or a C++ host can bind it without any torch or CUDA types.
 *
 * Conventions (mirroring the reference's error handling):
 *   - every call returns 0 (LBM_OK) or a negative lbm_status;
 *   - configuration errors the reference throws as `Error` (bad Q, bad
 *     tau, a non-dividing block size, ...) return LBM_EINVAL and leave a
 *     message for lbm_last_error();
 *   - device faults the reference counts rather than throws (non-finite
 *     force partials) are counted, see lbm_totals() out[7];
 *   - host buffers are caller-owned; device memory is library-owned;
 *   - one CUDA stream per session; a session is not thread-safe, distinct
 *     sessions are.
 *
 * Field wire format is the reference's: f as Q planes of f32, plane-major
 * (`f[i * ncells + cell]`, cell = (z*NY + y)*NX + x), whatever the on-device
 * storage (f-pack.mjs:6-17 keeps f32 plane-major on the wire for the same
 * reason). The macroscopic field is [rho, ux, uy, uz] per cell, interleaved
 * (common_d3_step.wgsl:57-61 `mac : array<vec4<f32>>`).
 */
#ifndef LBM_H
#define LBM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden visibility; everything declared here is
 * exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define LBM_ABI_VERSION 2

typedef enum {
  LBM_OK = 0,
  LBM_EINVAL = -1,    /* bad argument or configuration (reference: throws) */
  LBM_ENOMEM = -2,    /* device allocation failed */
  LBM_ECUDA = -3,     /* a CUDA call failed; message has the CUDA error */
  LBM_ETIMEDOUT = -4, /* a bounded device wait gave up */
  LBM_ENOTSUP = -5,   /* option not built into this library */
  LBM_ESTATE = -6,    /* call not valid in the session's current state */
  LBM_ENOSPC = -7     /* pool or budget exhausted (reference: refusal) */
} lbm_status;

/* On-device storage of f. The wire format is always f32 planes. */
typedef enum {
  LBM_STORE_FP32 = 0, /* plain f32 planes                                   */
  LBM_STORE_FP16 = 1, /* binary16 planes holding (f_i - feq_i(1, U_far)) * 2^10:
                         the deviation from the far-field (sponge) equilibrium,
                         f-pack mode 2 with the rest state replaced by the free
                         stream; w_i when there is no far-field velocity      */
  LBM_STORE_BF16 = 2  /* bfloat16 planes holding f_i - feq_i(1, U_far)         */
} lbm_storage;

/* Body shapes. 3D: common_d3_geometry.wgsl:40-42. D2Q9 uses ELLIPSE
 * (common_geometry.wgsl get_phi; a circle when a == b). */
typedef enum {
  LBM_SHAPE_SPHERE = 0,
  LBM_SHAPE_SPHEROID = 1,
  LBM_SHAPE_ROUNDBOX = 2,
  LBM_SHAPE_ELLIPSE = 3
} lbm_shape;

/* Rigid body pose and kinematics. The subset of BodyState3D
 * (common_d3_geometry.wgsl:25-58, d3-body.mjs:318 BODY_FIELDS) and CardState
 * (common_geometry.wgsl:8-35) that the step and force kernels read.
 * Quaternion order is [w, x, y, z] as in the reference. */
typedef struct {
  int32_t shape;
  float cx, cy, cz;       /* centre, lattice units (cell centres at integers) */
  float qw, qx, qy, qz;   /* 3D orientation, body -> world                    */
  float theta;            /* D2Q9 orientation angle                           */
  float vx, vy, vz;       /* linear velocity                                  */
  float wx, wy, wz;       /* angular velocity (D2Q9 uses wz as omega)         */
  float a, b, c, r;       /* semi-axes / half-extents; r = roundbox rounding  */
} lbm_body;

/* Dense-domain configuration: the override constants of
 * common_d3_step.wgsl:125-213 and lbm_step.wgsl:36-135, as a plain struct. */
typedef struct {
  int32_t q;              /* 9 (D2Q9), 19 (D3Q19) or 27 (D3Q27)              */
  int32_t nx, ny, nz;     /* nz must be 1 when q == 9                        */
  float tau;              /* BGK relaxation time; omega = 1/tau              */
  float force[3];         /* uniform Guo body-force density FORCE_X/Y/Z      */
  int32_t wall[3];        /* stationary no-slip walls normal to x, y, z      */
  float wall_u[2];        /* D2Q9: x-velocity of the y=0 / y=H-1 walls       */
  int32_t has_body;       /* HAS_BODY                                        */
  int32_t use_bounceback; /* USE_BOUNCEBACK: 1 = sharp Ladd, 0 = chi penalty */
  int32_t solid_eq;       /* SOLID_EQ                                        */
  int32_t rho_w_local;    /* RHO_W_LOCAL (3D)                                */
  int32_t swept_force;    /* SWEPT_FORCE (3D)                                */
  float chi_eps;          /* CHI_EPS / K_EPS band width, cells               */
  float sponge_w;         /* SPONGE_W; <= 0 disables the sponge              */
  int32_t sponge_axis[3]; /* SPONGE_AX/AY/AZ                                 */
  float sponge_u[3];      /* SPONGE_UX/UY/UZ far-field velocity              */
  lbm_body body;
  int32_t storage;        /* lbm_storage                                     */
  int32_t window[3];      /* moving window per axis (3D, common_d3_window.wgsl
                             WIN_N*): the body wraps through the periodic
                             buffer and the sponge band follows it; needs a
                             body, a sponge and no wall on the axis          */
  int32_t win_anchor[3];  /* WIN_AX/AY/AZ: the cell the body sits in within
                             the window, the floor of its initial centre    */
  int32_t trt;            /* two-relaxation-time collision (3D dense, batch,
                             server; plans/TRT.md sec 8.0): the odd part of
                             every direction pair relaxes at omega_- with
                             tau_- = 1/2 + trt_lambda / (tau - 1/2), the even
                             part at 1/tau as in BGK. 0 = BGK             */
  float trt_lambda;       /* the magic parameter Lambda (3/16 in the
                             reference's ?lambda= default); with trt = 1 it
                             must be > 0                                   */
} lbm_config;

typedef struct lbm_session lbm_session;

/* State of a free (integrated) 3D rigid body, FP64 -- d3-body.mjs
 * makeBodyState (:300-307) and the BodyState3D fields d3_physics.wgsl
 * advances. Quaternions are {w, x, y, z}, body -> world. */
typedef struct {
  double x[3];       /* centre, lattice units (wrapped on windowed axes)        */
  double q[4];       /* orientation                                             */
  double v[3];       /* linear velocity, cells per step                         */
  double L[3];       /* angular momentum, world frame (the integrated state)    */
  double omega[3];   /* angular velocity of the last step (its midpoint value)  */
  double d[3];       /* displacement since the state was made, unwrapped        */
  double force[3];   /* fluid force drained at the last step                    */
  double torque[3];  /* fluid torque drained at the last step                   */
  double mass;
  double ibody[3];   /* principal moments of inertia (body axes)                */
  int64_t steps;     /* steps integrated (pinned steps included)                */
} lbm_body_state;

/* Options of the integrator -- the override constants of d3_physics.wgsl
 * (GX/GY/GZ, NO_FLUID_FORCE, PLANAR), the v_max / o_max limiters of
 * BodyState3D and the moving window's wrap lengths (d3-window.mjs). */
typedef struct {
  double gravity[3];       /* uniform acceleration                             */
  double v_max, o_max;     /* magnitude clamps; <= 0 (or inf) = none           */
  double wrap[3];          /* per-axis wrap length of the position, 0 = none;
                              a session sets it to the domain length on the
                              axes of its moving window                     */
  int32_t planar;          /* no z translation, rotation about z only          */
  int32_t no_fluid_force;  /* integrate without the fluid load (it is still recorded) */
  int32_t pinned;          /* record the load, do not move                     */
  int32_t reserved;        /* zero                                             */
} lbm_body_opts;

/* Library version string and ABI version. */
const char *lbm_version(void);
int lbm_abi_version(void);

/* Fills `cfg` with the reference's defaults (common_d3_step.wgsl overrides:
 * OMEGA 1.25, CHI_EPS 1.5, SOLID_EQ 1, RHO_W_LOCAL 1, SWEPT_FORCE 1, sponge
 * axes on, no walls, no body, FP32 storage) for a q-lattice of the given
 * size. Pure host function. */
int lbm_config_default(lbm_config *cfg, int q, int nx, int ny, int nz);

/* Creates a dense session on the current CUDA device and allocates its
 * device state (two f buffers, the mac field, reduction scratch).
 * Replaces the page-side pipeline/buffer set-up of main-3d.js:980-1010 and
 * main-cylinder.js:400-430. Returns LBM_EINVAL for an invalid config. */
int lbm_create(const lbm_config *cfg, lbm_session **out);
void lbm_destroy(lbm_session *s);

/* Message for the last failed call on `s` (or, with s == NULL, the last
 * failed lbm_create on this thread). Never NULL. */
const char *lbm_last_error(const lbm_session *s);

/* Sets the CUDA stream (a cudaStream_t passed as void*) the session
 * launches on; NULL restores the session's own stream. */
int lbm_set_stream(lbm_session *s, void *cuda_stream);

/* Seeds f at equilibrium from a host macroscopic field, [rho,ux,uy,uz] per
 * cell -- common_d3_step.wgsl:206-222 initEq (and main-tgv.js:136 initF in
 * 2D). Also sets the session's mac field. Synchronous. */
int lbm_init_macro(lbm_session *s, const float *mac);

/* Writes / reads f in the f32 plane-major wire format (Q * ncells floats).
 * Packed storages convert on the device. Synchronous. */
int lbm_write_f(lbm_session *s, const float *f);
int lbm_read_f(lbm_session *s, float *f);

/* Writes / reads the populations exactly as stored: Q planes of ncells
 * elements of the session's storage type (4 bytes for FP32, 2 for the
 * 16-bit storages, which hold (f - off_i) * scale). An exact checkpoint of a
 * packed session, with no re-quantisation; for FP32 the same as
 * lbm_write_f / lbm_read_f. Synchronous. No reference counterpart (the
 * reference's snapshots carry f32 or f16 planes, f-pack.mjs:6-17). */
int lbm_write_f_raw(lbm_session *s, const void *planes);
int lbm_read_f_raw(lbm_session *s, void *planes);

/* Reads the macroscopic field of the last step (4 floats per cell). */
int lbm_read_mac(lbm_session *s, float *mac);

/* ---- headless views of the field (no graphics API) ----------------------
 * The reference resamples its hierarchy onto a 3D texture
 * (common_d3_resample.wgsl over common_d3_tree_sample.wgsl sampleTree:
 * nearest sample, finest level present wins) and draws axis-aligned slices
 * (common_d3_render_slice.wgsl fs_main with common_vortcolor.wgsl). Here
 * both are compute kernels writing into a buffer. */
typedef struct {
  float origin[3];    /* volOrigin: L0 cell units, cell centres at integers  */
  int32_t shape[3];   /* VOL_NX/NY/NZ voxels                                  */
  float h[3];         /* VOL_HX/HY/HZ: L0 cells per voxel                     */
  int32_t fp16;       /* 1: texels as IEEE binary16 (the rgba16float texture),
                         0: f32. Texel = (ux, uy, uz, rho), x fastest          */
  int32_t device;     /* 1: out / level are device pointers (no copy, no sync) */
} lbm_volume_spec;

typedef struct {
  int32_t axis;       /* slice normal: 0 x, 1 y, 2 z (in-plane axes cyclic)   */
  int32_t slice;      /* index along the normal, window coordinates           */
  int32_t mode;       /* 0 speed, 1 out-of-plane vorticity, 2 normal velocity */
  int32_t rot;        /* quarter turns of the picture, clockwise              */
  float u_scale;      /* velocity reference of modes 0 and 2                  */
  float v_scale;      /* vorticity reference of mode 1                        */
  float vort_scale;   /* common_vortcolor.wgsl VORT_SCALE (the 3D page: 1)    */
  float vort_gamma;   /* VORT_GAMMA (1.2)                                     */
  int32_t width, height;  /* pixels; RGBA8 rows top to bottom                 */
  int32_t device;     /* 1: rgba is a device pointer                          */
} lbm_slice_spec;

/* Defaults: full-domain L0 volume (origin 0, h 1, f32, host) / a z slice
 * through the middle, speed, 1:1 pixels, VORT_SCALE 1, VORT_GAMMA 1.2. */
int lbm_volume_spec_default(lbm_volume_spec *v, int nx, int ny, int nz);
int lbm_slice_spec_default(lbm_slice_spec *v, int nx, int ny, int nz);
/* The dense session's field (level 0 only) resampled / drawn; `level` (one
 * byte per voxel, may be NULL) receives the level each voxel came from. */
int lbm_resample(lbm_session *s, const lbm_volume_spec *spec, void *out, uint8_t *level);
int lbm_render_slice(lbm_session *s, const lbm_slice_spec *spec, uint8_t *rgba);

/* Advances n fused stream-collide steps (common_d3_step.wgsl:224 `step`,
 * lbm_step.wgsl:137 `main`), each fused with the body force/torque sum of
 * common_d3_force.wgsl / lbm_force.wgsl over the pre-streaming f. mac is
 * written on the last of the n steps only. Asynchronous on the session
 * stream. */
int lbm_step(lbm_session *s, int n);

/* Replaces the body pose/kinematics used by subsequent steps. */
int lbm_set_body(lbm_session *s, const lbm_body *body);

/* Makes the body free: from the next step on, every step is a force pass
 * over the cells near the body (FP64 sum), the 6-DOF update of `state` under
 * that load on the device, then the lattice step with the new pose -- the
 * reference's force -> physics -> step order (main-3d.js:3122-3145,
 * d3_physics.wgsl). The body's shape and size stay those of the session's
 * config. 3D sessions with a body only. NULL state leaves the body free with
 * its current device state replaced by nothing: it returns to the config's
 * prescribed pose (as lbm_set_body does). */
int lbm_set_free_body(lbm_session *s, const lbm_body_state *state, const lbm_body_opts *opts);

/* Reads the free body's state after the queued steps (synchronous). */
int lbm_read_body_state(lbm_session *s, lbm_body_state *out);

/* Force and torque on the body from the most recent step, FP64:
 * out = {fx, fy, fz, tx, ty, tz}. Synchronous (one 48-byte readback).
 * Replaces the i32 fixed-point atomics of common_d3_force.wgsl:265-282. */
int lbm_forces(lbm_session *s, double out[6]);

/* Queues a copy of the most recent step's {fx, fy, fz, tx, ty, tz} into
 * host memory `out` (pinned for a true asynchronous copy) on the session
 * stream and returns without waiting: a caller can record every step's force
 * while the device keeps stepping, then lbm_sync() once. The buffer must
 * stay valid until that sync. Pinned memory is written by a small kernel
 * on the stream (no copy-engine transfer between two steps); pageable
 * memory by cudaMemcpyAsync. */
int lbm_forces_async(lbm_session *s, double out[6]);

/* Conserved totals over the current f, FP64 on the device:
 * out = {sum(rho-1), sum(rho ux), sum(rho uy), sum(rho uz), rho_min, rho_max,
 *        max|u|, non-finite cell count}.
 * Replaces readConservedTotals (amr2d-gpu.mjs:698-736) and readStats
 * (main-3d.js:3610-3643). Synchronous. */
int lbm_totals(lbm_session *s, double out[8]);

/* Blocks until the session's queued work is done. */
int lbm_sync(lbm_session *s);

/* Bytes of device memory the session holds. */
int64_t lbm_device_bytes(const lbm_session *s);

/* ---- z-slabs: one domain split across GPUs ---------------------------------
 * No counterpart in the reference (one page steps one domain). A slab
 * session holds planes [z0, z0 + nz_local) of the 3D domain `cfg` describes
 * (one per GPU, one process per GPU): its physics -- body, walls, sponge,
 * force region -- is the whole domain's, at the domain's own coordinates,
 * and its cells are stored between a ghost plane below and one above. Every
 * step needs the populations that cross its z faces from the neighbouring
 * slabs (periodic in z: the last slab's upper neighbour is the first):
 *   lbm_slab_pack(s, send_lo, send_hi)   its first plane's ez = -1 and last
 *                                        plane's ez = +1 populations into
 *                                        caller device buffers of
 *                                        lbm_slab_halo_bytes(s) each;
 *   exchange: send_lo to the slab below (its recv_hi), send_hi to the slab
 *             above (its recv_lo) -- over NCCL or peer copies, by the caller;
 *   lbm_slab_unpack(s, recv_lo, recv_hi) into the ghost planes;
 *   lbm_step(s, 1).
 * A slab's f, mac and totals cover its own planes; its lbm_forces is its
 * share of the body force (the slabs' shares sum to the domain's). Slabs
 * take no moving window, free body or headless view. The result of a step
 * is the whole-domain step's, bit for bit, cell by cell. */
int lbm_create_slab(const lbm_config *cfg, int z0, int nz_local, lbm_session **out);
int64_t lbm_slab_halo_bytes(const lbm_session *s);
int lbm_slab_pack(lbm_session *s, void *send_lo, void *send_hi);
int lbm_slab_unpack(lbm_session *s, const void *recv_lo, const void *recv_hi);

/* ---- allocation-free stepping --------------------------------------------
 * No counterpart in the reference: added for callers that cannot call
 * cudaMalloc -- hosts that own all device memory through their own arena,
 * and loops that must not take the implicit device-wide synchronisation of
 * cudaMalloc/cudaFree. Advances one dense step of `cfg` from the caller's
 * device buffer f_in into the caller's f_out (Q planes in cfg->storage),
 * optionally writing mac (4 floats per cell, device) and the body's
 * force/torque (8 doubles, device: fx fy fz tx ty tz nonfinite 0), launched
 * on cuda_stream. Allocates nothing: the force reduction's scratch is a fixed
 * 520 KiB device array inside the library (8192 launch blocks of partials
 * plus their group sums and a ticket); a force region needing more returns
 * LBM_ENOSPC before anything is launched. force_out, when given, is always
 * written: zeros when no cell can reach the body. A call whose stream is not
 * capturing looks up the array's device address for the current device and
 * keeps it; a call during stream capture uses the kept one, so the first
 * call on a device must come before any capture (and a graph captured
 * before a cudaDeviceReset must not be replayed after it). All calls share
 * the array; each clears the ticket on its stream first, and calls whose
 * kernels overlap on the GPU race. Errors are reported by
 * lbm_noalloc_last_error(). */
int lbm_step_noalloc(const lbm_config *cfg, const void *f_in, void *f_out, float *mac, double *force_out,
                     void *cuda_stream);
const char *lbm_noalloc_last_error(void);

/* ---- batched form ----------------------------------------------------------
 * Many independent domains of uneven sizes (same q and storage) in one
 * arena, advanced by one persistent launch per step replayed from a CUDA
 * graph. Each domain is a full lbm_config and is stepped with exactly the
 * arithmetic of a dense session. The reference has no batched form (one page
 * per domain, main-3d.js encodeSteps); these calls are its N-page loop. */
typedef struct lbm_batch lbm_batch;

int lbm_batch_create(const lbm_config *domains, int ndomains, lbm_batch **out);
void lbm_batch_destroy(lbm_batch *b);
/* Last error of `b`, or with b == NULL of the last failed create. */
const char *lbm_batch_last_error(const lbm_batch *b);
int lbm_batch_set_stream(lbm_batch *b, void *cuda_stream);
int lbm_batch_domains(const lbm_batch *b);
int64_t lbm_batch_cells(const lbm_batch *b);
/* Per-domain state transfer, same formats as the dense calls. */
int lbm_batch_init_macro(lbm_batch *b, int domain, const float *mac);
int lbm_batch_write_f(lbm_batch *b, int domain, const float *f);
int lbm_batch_read_f(lbm_batch *b, int domain, float *f);
int lbm_batch_read_mac(lbm_batch *b, int domain, float *mac);
/* n steps of every domain; mac is written on the last one. */
int lbm_batch_step(lbm_batch *b, int n);
/* Tile shape of the persistent launch: threads per CTA (128 or 256), cells
 * per thread per tile, resident CTAs per SM. */
int lbm_batch_set_tiling(lbm_batch *b, int threads, int cells_per_thread, int ctas_per_sm);
int lbm_batch_get_tiling(const lbm_batch *b, int *threads, int *cells_per_thread, int *ctas_per_sm);
/* Times every candidate tiling on this batch (stepping into the spare
 * buffer, so the state is unchanged) and keeps the fastest. */
int lbm_batch_autotune(lbm_batch *b, int trials, float *best_ms);
/* Force/torque of every domain from the last step: 6 doubles per domain. */
int lbm_batch_forces(lbm_batch *b, double *out);
int lbm_batch_sync(lbm_batch *b);

/* ---- 2D block-structured AMR (D2Q9) --------------------------------------
 * Root level L0 is the dense W x H grid; level m >= 1 is a pool of tiles,
 * each one block of RB x RB cells of level m-1 refined 2:1 into
 * (2 RB + 2 G)^2 cells with a G = 2 ring (amr2d.mjs:220 makePool, FB = 20 at
 * RB = 8). Tiles are granted and released in quads (the four children of one
 * parent block, amr_manage_pool.wgsl grantQuad) from a deterministic free
 * list (the DET_SLOTS serial order, amr2d.mjs:1078 grantAssignment). One
 * macro-step follows main-cylinder-amr.js:1831 dispatchMacroStep with the
 * default `interp` interface (amr2d-gpu.mjs:1060 S_Advance): refine round
 * every refine_every steps, finest-level force, ring fill from the parent,
 * root step, two fine substeps at tau_f = 2 tau_c - 1/2, restriction back to
 * the root. */
typedef struct {
  int32_t nx, ny;            /* root grid; multiples of 2*rb                     */
  int32_t levels;            /* 2 (root + one pool level)                        */
  int32_t rb;                /* block size in parent cells (8)                   */
  float tau;                 /* root relaxation time                             */
  int32_t max_slots;         /* pool capacity in tiles, multiple of 4            */
  int32_t use_bounceback;    /* 0: chi penalty (default), 1: Ladd bounce-back    */
  int32_t solid_eq;
  float k_eps;               /* chi band in cells of each level (1.5)            */
  float sponge_w;            /* 4                                                */
  float sponge_u[2];         /* far-field velocity                               */
  float force[2];            /* uniform body force                               */
  lbm_body body;             /* LBM_SHAPE_ELLIPSE (circle when a == b)           */
  int32_t refine_every;      /* 16                                               */
  float refine_thresh;       /* -8: refine where log2 max|curl| >= this          */
  float refine_margin;       /* 8: refine blocks within this distance of body    */
  float refine_lookahead;    /* 16 macro-steps                                   */
  int32_t auto_refine;       /* 1                                                */
  int32_t iface;             /* 0: interp ring (the reference's 2D default),
                                1: explode/coalesce (amr_explode.wgsl,
                                amr_coalesce.wgsl; the ring advects only)       */
  int32_t explode_linear;    /* EXPLODE_LINEAR (1), explode only                 */
  int32_t reserved[6];
} lbm_amr2d_config;

typedef struct lbm_amr2d lbm_amr2d;

/* Defaults of main-cylinder-amr.js (REFINE_EVERY 16, REFINE_THRESH -8,
 * FORCE_REFINE_MARGIN 8, LOOKAHEAD 16, K_EPS 1.5, SPONGE_W 4, RB 8). */
int lbm_amr2d_config_default(lbm_amr2d_config *cfg, int nx, int ny);
int lbm_amr2d_create(const lbm_amr2d_config *cfg, lbm_amr2d **out);
void lbm_amr2d_destroy(lbm_amr2d *a);
const char *lbm_amr2d_last_error(const lbm_amr2d *a);
int lbm_amr2d_set_stream(lbm_amr2d *a, void *cuda_stream);
/* Root populations (9 planes of nx*ny) and root velocity (2 per cell, the
 * field the first refine round's criterion reads). */
int lbm_amr2d_write_root(lbm_amr2d *a, const float *f, const float *vel);
int lbm_amr2d_read_root(lbm_amr2d *a, float *f, float *vel);
/* Pool populations of level 1 (9 planes of max_slots * FB^2, FB = 2rb+4). */
int lbm_amr2d_read_pool(lbm_amr2d *a, float *f, float *vel);
/* n macro-steps. */
int lbm_amr2d_step(lbm_amr2d *a, int n);
/* One refine round now -- criterion over the root velocity of the last
 * macro-step, decide, coarsen, refine, fill the new tiles (amr2d-gpu.mjs
 * refineRound, the page's debug refine) -- and the switch of the rounds the
 * step runs every refine_every macro-steps (setAutoRefine). */
int lbm_amr2d_refine_round(lbm_amr2d *a);
int lbm_amr2d_set_auto_refine(lbm_amr2d *a, int on);
/* How the interp interface's macro-step runs: one cooperative launch whose
 * phases (force partials, ring fill and root step; substep; substep;
 * restriction) are separated by grid barriers (on, the default where the
 * device takes cooperative launches), or six launches (off). Both give the
 * same bits. lbm_amr2d_fused reports which is in use. A barrier that waits
 * longer than about a second gives up: lbm_amr2d_sync then returns
 * LBM_ETIMEDOUT. No counterpart in the reference (its macro-step is the six
 * dispatches). */
int lbm_amr2d_set_fused(lbm_amr2d *a, int on);
int lbm_amr2d_fused(const lbm_amr2d *a);
/* Drag/lift/torque of the last macro-step, FP64: {fx, fy, tz, nonfinite}. */
int lbm_amr2d_forces(lbm_amr2d *a, double out[4]);
/* Level-1 topology: block_slot[nbx*nby], slot_to_block[max_slots],
 * free_list[max_slots/4], counts = {free quads, active slots}, active list
 * (ascending slots), criterion[nbx*nby], want[nbx*nby]. Any may be NULL. */
int lbm_amr2d_read_topology(lbm_amr2d *a, int32_t *block_slot, int32_t *slot_to_block, int32_t *free_list,
                            int32_t counts[2], int32_t *active_list, float *criterion, uint32_t *want);
/* Lattice updates per macro-step at the current topology:
 * root cells + sum over levels of active * (2 rb)^2 * 2^m (amr2d.mjs:558). */
int64_t lbm_amr2d_cell_updates(const lbm_amr2d *a);
int lbm_amr2d_sync(lbm_amr2d *a);

/* State restore for checkpoints (the snapshot save/load of
 * main-cylinder-amr.js:1524-1705, whose version-7 layout the Python host
 * layer writes): the pool's time-t populations (9 planes of max_slots*FB^2)
 * and velocity ([ux,uy] per cell); the pool topology -- block_slot
 * (NBX*NBY), slot_to_block and parent_slot (max_slots), the quad free list
 * (max_slots/4 entries, the first free_count live) -- checked for
 * consistency (inverse maps, whole quads, no quad both free and in use) and
 * refused with LBM_EINVAL otherwise, the active list rebuilt from it; the
 * macro-step counter that schedules refine rounds; the body pose. */
int lbm_amr2d_write_pool(lbm_amr2d *a, const float *f, const float *vel);
int lbm_amr2d_read_parent_slots(lbm_amr2d *a, int32_t *parent_slot);
int lbm_amr2d_write_topology(lbm_amr2d *a, const int32_t *block_slot, const int32_t *slot_to_block,
                             const int32_t *parent_slot, const int32_t *free_list, int32_t free_count);
int64_t lbm_amr2d_get_step(const lbm_amr2d *a);
int lbm_amr2d_set_step(lbm_amr2d *a, int64_t step);
int lbm_amr2d_set_body(lbm_amr2d *a, const lbm_body *body);

/* ---- 3D block-structured AMR (D3Q19 / D3Q27, FP32) -----------------------
 * The dense L0 grid plus one pool level: blocks of RB^3 L0 cells, a refined
 * block owning a tile of FB^3 = (2 RB + 4)^3 cells at half spacing (interior
 * plus a two-cell ring). d3-amr.mjs (pool geometry, refineWhere,
 * nearBodyWant) and the kernels common_d3_amr_{explode,step1,coalesce,interp}
 * .wgsl, common_d3_force_pool.wgsl, common_d3_moments.wgsl; the macro-step
 * order of main-3d.js:3219-3341 (force, explode, two fine substeps, coalesce,
 * the coarse step skipping covered blocks). */

typedef enum {
  LBM_REFINE_BODY = 0,  /* blocks within `margin` of the body (nearBodyWant) */
  LBM_REFINE_BOX = 1,   /* centred cube, `boxfrac` of each axis            */
  LBM_REFINE_BAR = 2,   /* centred in x and y, all of z                    */
  LBM_REFINE_SLAB = 3,  /* centred band in x                               */
  LBM_REFINE_ALL = 4,
  LBM_REFINE_LIST = 5   /* the caller's per-block flags                    */
} lbm_refine;

typedef struct {
  lbm_config root;         /* L0 grid and physics; dims multiples of rb; FP32 */
  int32_t levels;          /* 2                                               */
  int32_t rb;              /* block edge, L0 cells (4)                        */
  int32_t refine;          /* lbm_refine                                      */
  float margin;            /* LBM_REFINE_BODY margin, L0 cells (2)            */
  float boxfrac;           /* box / bar / slab fraction (0.5)                 */
  int32_t explode_linear;  /* EXPLODE_LINEAR (1); 0 = uniform explosion       */
  int32_t dynamic;         /* re-decide the refined set on the device (0)     */
  int32_t manage_every;    /* macro-steps between decisions (16)              */
  int32_t manage_start;    /* first macro-step that decides (0)               */
  int32_t max_slots;       /* pool capacity; 0 = initial set (x slot_headroom when dynamic) */
  float slot_headroom;     /* 1.5                                             */
  int32_t iface;           /* 0: explode/coalesce (the reference's default);
                              1: interp -- the L0 step first, the ring
                              interpolated from L0, ring collided, tiles
                              restricted into L0 (main-3d.js:3343-3356)       */
  int32_t reflux;          /* interp only: the flux correction of
                              common_d3_amr_flux.wgsl / _reflux.wgsl
                              (?reflux=1); needs no walls and >= 3 blocks
                              per axis, as the reference requires             */
  float q_abs;             /* dynamic only: also refine blocks whose max
                              Q-criterion (common_d3_criterion.wgsl, from the
                              L0 velocity) reaches q_abs, lattice units --
                              the reference's qthresh x (U/D)^2; 0 = off      */
  float q_hyst;            /* a held block keeps its tile down to
                              q_abs * 4^-q_hyst (the reference's qhyst, 1)    */
  float q_lead;            /* cells the Q window is dilated by (qlead)        */
} lbm_amr3d_config;

typedef struct lbm_amr3d lbm_amr3d;

int lbm_amr3d_config_default(lbm_amr3d_config *c, int q, int nx, int ny, int nz);
/* `block_want` (one flag per block, id = (bz*NBY + by)*NBX + bx) is read for
 * LBM_REFINE_LIST only. Slots are handed out in ascending block id. */
int lbm_amr3d_create(const lbm_amr3d_config *c, const uint8_t *block_want, lbm_amr3d **out);
/* Device bytes the hierarchy of `c` holds (256-byte granules), computed
 * without touching the GPU; and the same hierarchy built inside a caller's
 * device block of at least that many bytes (256-byte aligned), which the
 * caller keeps and frees after lbm_amr3d_destroy (the server's arena). */
int lbm_amr3d_device_bytes(const lbm_amr3d_config *c, const uint8_t *block_want, int64_t *bytes);
int lbm_amr3d_create_in(const lbm_amr3d_config *c, const uint8_t *block_want, void *device_base, int64_t capacity,
                        lbm_amr3d **out);
void lbm_amr3d_destroy(lbm_amr3d *a);
const char *lbm_amr3d_last_error(const lbm_amr3d *a);
int lbm_amr3d_set_stream(lbm_amr3d *a, void *cuda_stream);
/* Seeds L0 at equilibrium from [rho,ux,uy,uz] per L0 cell (both buffers),
 * every tile by trilinear interpolation of it (DC rescale
 * 0.5 (tau_f - 1)/(tau_c - 1)), then the tiles' moments -- main-3d.js reset. */
int lbm_amr3d_init_macro(lbm_amr3d *a, const float *mac);
/* n macro-steps (one L0 step and two pool substeps each). With `dynamic`,
 * macro-steps manage_start + k * manage_every first re-decide the refined
 * set on the device (common_d3_manage.wgsl, in its order: decide, drain the
 * dying tiles into L0, free their slots, grant slots to new blocks, fill the
 * new tiles from L0), with slots granted in ascending block id. */
int lbm_amr3d_step(lbm_amr3d *a, int n);
/* Replaces the body pose (a prescribed motion); the next decision follows it. */
int lbm_amr3d_set_body(lbm_amr3d *a, const lbm_body *body);
/* One decision of the dynamic manager now, before the next macro-step
 * (the step runs them every manage_every macro-steps from manage_start). */
int lbm_amr3d_manage_now(lbm_amr3d *a);
/* The bounce-back link table (bounce-back bodies): one 32-bit code per pool
 * cell -- which pull sources lie inside the body, whether the cell is near
 * or inside it -- built when the hierarchy is seeded, after set_body and for
 * the tiles each decision grants, and read by the substeps and the pool
 * force instead of evaluating the body's distance at every cell and link
 * source. On by default; off evaluates them each step. The results are the
 * same bits either way. Returns LBM_OK (a hierarchy without a bounce-back
 * body has no table, and both calls leave it off). No counterpart in the
 * reference, which evaluates the distance in its step shader. */
int lbm_amr3d_set_links(lbm_amr3d *a, int on);
int lbm_amr3d_links(const lbm_amr3d *a);
/* {slots in use, refusals (pool exhausted), lowest free count seen, decisions}. */
int lbm_amr3d_pool_stats(lbm_amr3d *a, int32_t out[4]);
/* Per-block max Q-criterion of the L0 velocity of the last macro-step, over
 * each block's box dilated by `lead` L0 cells: nb floats into host memory.
 * Replaces the reference's criterion readback (common_d3_criterion.wgsl
 * reduceQ into blockQ, read by main-3d.js debugCriterion). */
int lbm_amr3d_block_q(lbm_amr3d *a, float lead, float *block_q);
/* The hierarchy's field of the last macro-step resampled onto a voxel box /
 * drawn as a slice, each point answered by the finest level present there
 * (common_d3_resample.wgsl, common_d3_render_slice.wgsl). */
int lbm_amr3d_resample(lbm_amr3d *a, const lbm_volume_spec *spec, void *out, uint8_t *level);
int lbm_amr3d_render_slice(lbm_amr3d *a, const lbm_slice_spec *spec, uint8_t *rgba);
/* Force and torque on the body at the last macro-step (pool force, FP64). */
int lbm_amr3d_forces(lbm_amr3d *a, double out[6]);
/* Over the L0 macroscopic field of the last step (covered cells carry the
 * tiles' projection): {sum(rho - 1), sum(rho ux), sum(rho uy), sum(rho uz)},
 * FP64 -- readInterfaceDiag (main-3d.js:4660). */
int lbm_amr3d_totals(lbm_amr3d *a, double out[4]);
/* L0 f (Q planes of NX*NY*NZ, current time level) and mac (4 per cell). */
int lbm_amr3d_read_coarse(lbm_amr3d *a, float *f, float *mac);
/* Pool f (Q planes of slots*FB^3, slot-major) and mac (4 per cell). */
int lbm_amr3d_read_pool(lbm_amr3d *a, float *f, float *mac);
/* block_slot (NBX*NBY*NBZ), slot_to_block (capacity; -1 = free slot);
 * counts = {capacity, FB, blocks}. Synchronous. */
int lbm_amr3d_topology(lbm_amr3d *a, int32_t *block_slot, int32_t *slot_to_block, int32_t counts[3]);
/* Cell updates of one macro-step at the current topology: the L0 cells
 * outside refined blocks plus two substeps of every refined interior cell. */
int64_t lbm_amr3d_cell_updates(lbm_amr3d *a);
int lbm_amr3d_sync(lbm_amr3d *a);

/* The block set a configuration refines (d3-amr.mjs refineWhere with the
 * predicate of `c->refine`); `want` has NBX*NBY*NBZ entries. */
int lbm_amr3d_refine_blocks(const lbm_amr3d_config *c, uint8_t *want);

/* d3-amr.mjs resolveSource: where a tile-local source index `src` of block
 * `block` lives. out = {slot, fx, fy, fz}; slot = -1 for the block's own
 * tile, -2 when no tile owns it (the ring is read). Returns 0. */
int lbm_resolve_source(int rb, const int32_t nb[3], const int32_t *block_slot, const int32_t block[3],
                       const int32_t src[3], int32_t out[4]);

/* ---- serving form -------------------------------------------------------------
 * A request loop over one device arena of `budget_bytes` allocated at
 * creation: submitted solves (a dense lbm_config + a step count) are admitted
 * first-fit in FIFO order as memory frees up, stay resident on the device,
 * and every poll advances all resident solves together (one persistent launch
 * per lattice per step) up to the soonest completion, then retires the
 * finished ones. A result is bit-identical to the same solve in a dense
 * session. No counterpart in the reference (one page, one domain). */
typedef struct lbm_server lbm_server;

typedef struct {
  int64_t id;          /* the caller's request id                          */
  int32_t status;      /* 0                                                 */
  int32_t steps;       /* steps run                                         */
  double forces[6];    /* body force/torque of the last step, FP64         */
  double submit_s;     /* server clock (seconds since create) at submit    */
  double admit_s;      /*   ... when admitted into device memory           */
  double done_s;       /*   ... when retired                                */
} lbm_result;

int lbm_server_create(int64_t budget_bytes, lbm_server **out);
void lbm_server_destroy(lbm_server *s);
const char *lbm_server_last_error(const lbm_server *s);
/* Queues a solve; `mac` (host, 4 floats per cell) seeds it, or NULL for the
 * uniform freestream at cfg->sponge_u. LBM_ENOSPC when it can never fit. */
int lbm_server_submit(lbm_server *s, int64_t id, const lbm_config *cfg, const float *mac, int steps);
/* Queues a 3D two-level AMR solve of `steps` macro-steps (refine = body,
 * box, bar, slab or all; static or dynamic), seeded like lbm_server_submit
 * on L0. Its hierarchy lives in the server's arena (lbm_amr3d_create_in) and
 * advances on its own stream beside the dense launches; lbm_server_read
 * returns its L0 f and mac, the result its pool force. */
int lbm_server_submit_amr3d(lbm_server *s, int64_t id, const lbm_amr3d_config *cfg, const float *mac, int steps);
/* Admission policy: 0 = FIFO (the default; a request waits while the one
 * ahead of it does not fit), 1 = the queued request with the least total
 * work (cells x steps) first. max_resident_cells > 0 caps the resident
 * requests' cells (a single request is always admitted when the device is
 * idle): enough to fill the GPU, so that short requests do not share it with
 * every long one. */
int lbm_server_set_policy(lbm_server *s, int policy, int64_t max_resident_cells);
/* Admits what fits, runs one tick of at most max_steps steps, and returns up
 * to max_done finished solves. Finished solves keep their device state until
 * lbm_server_release. */
int lbm_server_poll(lbm_server *s, int max_steps, lbm_result *done, int max_done, int *n_done);
/* Final f (FP32 storage only) and mac of a finished solve. */
int lbm_server_read(lbm_server *s, int64_t id, float *f, float *mac);
int lbm_server_release(lbm_server *s, int64_t id);
/* {queued, resident, finished-not-released, bytes in use, budget, lattice updates run}. */
int lbm_server_stats(lbm_server *s, int64_t out[6]);

/* ---- pure host functions (the reference's JS modules) ------------------- */

/* Integrator defaults (packBodyState: v_max 0.2, o_max 0.1; no gravity,
 * window, planar constraint or pinning). */
void lbm_body_opts_default(lbm_body_opts *o);

/* makeBodyState (d3-body.mjs:300): mass = density x volume, principal
 * inertia, L from the pose's angular velocity. 3D shapes only. */
int lbm_body_state_make(const lbm_body *pose, double density, lbm_body_state *out);

/* `nsteps` of stepFreeBody (d3-body.mjs:244-290) under a constant load, on
 * the host: the same code the device runs after each force pass. */
int lbm_body_advance(lbm_body_state *s, const double force[3], const double torque[3], const lbm_body_opts *o,
                     int nsteps);

/* Lattice tables, lattice-2d.mjs:106-162 and lattice-3d.mjs:50-210:
 * velocity set, f32 weights (exact bits), opposite index. Arrays hold q
 * entries; ez is all zero for q == 9. Any pointer may be NULL. */
int lbm_lattice_tables(int q, int32_t *ex, int32_t *ey, int32_t *ez,
                       float *w, int32_t *opp);

/* f32 -> IEEE binary16 bits with round-to-nearest-even, subnormals and
 * overflow to Inf, and its inverse (f-pack.mjs:44-88). */
uint16_t lbm_f32_to_f16_bits(float v);
float lbm_f16_bits_to_f32(uint16_t h);

/* AMR host rules of amr2d.mjs, as pure functions. */
/* tauAtLevel (card-params.mjs:188): tau_m = 2 tau_{m-1} - 1/2. */
double lbm_tau_at_level(double tau0, int m);
/* The TRT pair (plans/TRT.md sec 8.1, d3-trt.mjs tauMinusOf / lambdaOf on
 * the reference's TRT branch): tau_- = 1/2 + Lambda / (tau_+ - 1/2), and
 * Lambda = (tau_+ - 1/2)(tau_- - 1/2). */
double lbm_trt_tau_minus(double tau_plus, double lambda);
double lbm_trt_lambda(double tau_plus, double tau_minus);
/* Post-collision coarse->fine and fine->coarse non-equilibrium factors,
 * 0.5 (tf-1)/(tc-1) and 2 (tc-1)/(tf-1) (amr2d.mjs:136-141). */
double lbm_dc_rescale_c2f(double tau_coarse, double tau_fine);
double lbm_dc_rescale_f2c(double tau_coarse, double tau_fine);
/* First level within `band` of tau = 1 (the transfer's 0/0), or -1
 * (amr2d.mjs:189 tauChainSingularity). */
int lbm_tau_chain_singularity(double tau0, int levels, double band);
/* grantAssignment (amr2d.mjs:1078): candidates served in id order, each
 * popping free_list[--free_count]; granted_free_index[k] = -1 for refusals.
 * Returns the new free count. */
int lbm_grant_assignment(const int32_t *candidates, int n, int free_count, int32_t *granted_ids,
                         int32_t *granted_free_index, int32_t *n_granted);
/* releaseAssignment (amr2d.mjs:1094): releases pushed in id order at
 * free_count, free_count+1, ... Returns the new free count. */
int lbm_release_assignment(const int32_t *releases, int n, int free_count, int32_t *ids, int32_t *free_index);
/* activeSlotList (amr2d.mjs:578): ascending slots with slot_to_block >= 0. */
int lbm_active_slot_list(const int32_t *slot_to_block, int nslots, int32_t *out);
/* cascade21 (amr2d.mjs:988) on per-level block masks: want[m] is a
 * nbx(m)*nby(m) byte mask for m = 1..levels-1 (want[0] unused), nbx(m) =
 * nbx1 * 2^(m-1). Closes it in place deepest-first: quad completion at
 * m >= 2 and the parents of all 9 periodic neighbours. Returns the number of
 * blocks added. */
int lbm_cascade21(uint8_t **want, int levels, int nbx1, int nby1);
/* The same closure on the device (amr_cascade.wgsl:114-157 completeQuads and
 * balance, one deepest-first sweep of launches on cuda_stream): the masks
 * are copied in, closed and copied back; returns the number of blocks added,
 * or a negative status. Blocks until done. */
int lbm_cascade21_device(uint8_t **want, int levels, int nbx1, int nby1, void *cuda_stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* LBM_H */
