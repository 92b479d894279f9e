"""Host-side mirror of the reference's LBM module API over the C ABI.

The reference (c7t/getting-air) exposes its solver as JavaScript modules and
page session objects:

* lattice-2d.mjs / lattice-3d.mjs   -> :func:`lattice_tables`, :func:`feq`
* f-pack.mjs                         -> :func:`f32_to_f16_bits`, :func:`f16_bits_to_f32`
* d3-scenarios.mjs / main-tgv.js     -> :mod:`.scenarios`
* the page objects' init / step / forces / readStats
  (main-3d.js:3122 encodeSteps, :3610 readStats; amr2d-gpu.mjs:698
  readConservedTotals)            -> :class:`Solver`

Everything that computes runs in ``liblbm.so`` (hand-written sm_100a CUDA);
this module only marshals arguments. There is no CPU fallback: if the
library is missing, importing this package raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "liblbm.so"

# lbm_status
OK, EINVAL, ENOMEM, ECUDA, ETIMEDOUT, ENOTSUP, ESTATE, ENOSPC = 0, -1, -2, -3, -4, -5, -6, -7
STORAGE = {"fp32": 0, "fp16": 1, "bf16": 2}
SHAPE = {"sphere": 0, "spheroid": 1, "roundbox": 2, "ellipse": 3}


class LbmError(RuntimeError):
    """A C-ABI call returned a negative status (the reference throws `Error`)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"lbm status {code}: {msg}")
        self.code = code


class Body(C.Structure):
    _fields_ = [("shape", C.c_int32),
                ("cx", C.c_float), ("cy", C.c_float), ("cz", C.c_float),
                ("qw", C.c_float), ("qx", C.c_float), ("qy", C.c_float), ("qz", C.c_float),
                ("theta", C.c_float),
                ("vx", C.c_float), ("vy", C.c_float), ("vz", C.c_float),
                ("wx", C.c_float), ("wy", C.c_float), ("wz", C.c_float),
                ("a", C.c_float), ("b", C.c_float), ("c", C.c_float), ("r", C.c_float)]


class BodyState(C.Structure):
    """lbm_body_state: FP64 state of a free rigid body (d3-body.mjs makeBodyState)."""
    _fields_ = [("x", C.c_double * 3), ("q", C.c_double * 4), ("v", C.c_double * 3), ("L", C.c_double * 3),
                ("omega", C.c_double * 3), ("d", C.c_double * 3), ("force", C.c_double * 3),
                ("torque", C.c_double * 3), ("mass", C.c_double), ("ibody", C.c_double * 3),
                ("steps", C.c_int64)]

    def as_dict(self) -> dict:
        out = {k: np.array(getattr(self, k)[:]) for k in ("x", "q", "v", "L", "omega", "d", "force", "torque",
                                                          "ibody")}
        out["mass"] = float(self.mass)
        out["steps"] = int(self.steps)
        return out


class BodyOpts(C.Structure):
    """lbm_body_opts: the integrator's gravity, clamps, window wrap and switches."""
    _fields_ = [("gravity", C.c_double * 3), ("v_max", C.c_double), ("o_max", C.c_double),
                ("wrap", C.c_double * 3), ("planar", C.c_int32), ("no_fluid_force", C.c_int32),
                ("pinned", C.c_int32), ("reserved", C.c_int32)]


class Amr2DConfig(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("levels", C.c_int32), ("rb", C.c_int32),
                ("tau", C.c_float), ("max_slots", C.c_int32), ("use_bounceback", C.c_int32),
                ("solid_eq", C.c_int32), ("k_eps", C.c_float), ("sponge_w", C.c_float),
                ("sponge_u", C.c_float * 2), ("force", C.c_float * 2), ("body", Body),
                ("refine_every", C.c_int32), ("refine_thresh", C.c_float), ("refine_margin", C.c_float),
                ("refine_lookahead", C.c_float), ("auto_refine", C.c_int32), ("iface", C.c_int32),
                ("explode_linear", C.c_int32), ("reserved", C.c_int32 * 6)]


class Result(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int32), ("steps", C.c_int32), ("forces", C.c_double * 6),
                ("submit_s", C.c_double), ("admit_s", C.c_double), ("done_s", C.c_double)]


class Config(C.Structure):
    _fields_ = [("q", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("tau", C.c_float), ("force", C.c_float * 3), ("wall", C.c_int32 * 3),
                ("wall_u", C.c_float * 2), ("has_body", C.c_int32),
                ("use_bounceback", C.c_int32), ("solid_eq", C.c_int32),
                ("rho_w_local", C.c_int32), ("swept_force", C.c_int32),
                ("chi_eps", C.c_float), ("sponge_w", C.c_float),
                ("sponge_axis", C.c_int32 * 3), ("sponge_u", C.c_float * 3),
                ("body", Body), ("storage", C.c_int32), ("window", C.c_int32 * 3),
                ("win_anchor", C.c_int32 * 3), ("trt", C.c_int32), ("trt_lambda", C.c_float)]


class Amr3DConfig(C.Structure):
    _fields_ = [("root", Config), ("levels", C.c_int32), ("rb", C.c_int32), ("refine", C.c_int32),
                ("margin", C.c_float), ("boxfrac", C.c_float), ("explode_linear", C.c_int32),
                ("dynamic", C.c_int32), ("manage_every", C.c_int32), ("manage_start", C.c_int32),
                ("max_slots", C.c_int32), ("slot_headroom", C.c_float), ("iface", C.c_int32),
                ("reflux", C.c_int32), ("q_abs", C.c_float), ("q_hyst", C.c_float), ("q_lead", C.c_float)]


REFINE = {"body": 0, "box": 1, "bar": 2, "slab": 3, "all": 4, "list": 5}


class VolumeSpec(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("shape", C.c_int32 * 3), ("h", C.c_float * 3), ("fp16", C.c_int32),
                ("device", C.c_int32)]


class SliceSpec(C.Structure):
    _fields_ = [("axis", C.c_int32), ("slice", C.c_int32), ("mode", C.c_int32), ("rot", C.c_int32),
                ("u_scale", C.c_float), ("v_scale", C.c_float), ("vort_scale", C.c_float),
                ("vort_gamma", C.c_float), ("width", C.c_int32), ("height", C.c_int32), ("device", C.c_int32)]


SLICE_MODES = {"speed": 0, "vorticity": 1, "normal": 2}


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with getting-air_b200/build.py "
                          "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    P, I, D = C.c_void_p, C.c_int, C.POINTER(C.c_double)
    F = C.POINTER(C.c_float)
    sigs = {
        "lbm_version": ([], C.c_char_p),
        "lbm_abi_version": ([], I),
        "lbm_config_default": ([C.POINTER(Config), I, I, I, I], I),
        "lbm_create": ([C.POINTER(Config), C.POINTER(P)], I),
        "lbm_create_slab": ([C.POINTER(Config), I, I, C.POINTER(P)], I),
        "lbm_slab_halo_bytes": ([P], C.c_int64),
        "lbm_slab_pack": ([P, P, P], I),
        "lbm_slab_unpack": ([P, P, P], I),
        "lbm_destroy": ([P], None),
        "lbm_last_error": ([P], C.c_char_p),
        "lbm_set_stream": ([P, P], I),
        "lbm_init_macro": ([P, F], I),
        "lbm_write_f": ([P, F], I),
        "lbm_read_f": ([P, F], I),
        "lbm_write_f_raw": ([P, P], I),
        "lbm_read_f_raw": ([P, P], I),
        "lbm_read_mac": ([P, F], I),
        "lbm_volume_spec_default": ([C.POINTER(VolumeSpec), I, I, I], I),
        "lbm_slice_spec_default": ([C.POINTER(SliceSpec), I, I, I], I),
        "lbm_resample": ([P, C.POINTER(VolumeSpec), P, P], I),
        "lbm_render_slice": ([P, C.POINTER(SliceSpec), P], I),
        "lbm_amr3d_resample": ([P, C.POINTER(VolumeSpec), P, P], I),
        "lbm_amr3d_render_slice": ([P, C.POINTER(SliceSpec), P], I),
        "lbm_step": ([P, I], I),
        "lbm_set_body": ([P, C.POINTER(Body)], I),
        "lbm_forces": ([P, D], I),
        "lbm_totals": ([P, D], I),
        "lbm_forces_async": ([P, C.c_void_p], I),
        "lbm_sync": ([P], I),
        "lbm_device_bytes": ([P], C.c_int64),
        "lbm_batch_create": ([C.POINTER(Config), I, C.POINTER(P)], I),
        "lbm_batch_destroy": ([P], None),
        "lbm_batch_last_error": ([P], C.c_char_p),
        "lbm_batch_set_stream": ([P, P], I),
        "lbm_batch_domains": ([P], I),
        "lbm_batch_cells": ([P], C.c_int64),
        "lbm_batch_init_macro": ([P, I, F], I),
        "lbm_batch_write_f": ([P, I, F], I),
        "lbm_batch_read_f": ([P, I, F], I),
        "lbm_batch_read_mac": ([P, I, F], I),
        "lbm_batch_step": ([P, I], I),
        "lbm_batch_set_tiling": ([P, I, I, I], I),
        "lbm_batch_get_tiling": ([P, C.POINTER(I), C.POINTER(I), C.POINTER(I)], I),
        "lbm_batch_autotune": ([P, I, F], I),
        "lbm_batch_forces": ([P, D], I),
        "lbm_batch_sync": ([P], I),
        "lbm_amr2d_config_default": ([C.POINTER(Amr2DConfig), I, I], I),
        "lbm_amr2d_create": ([C.POINTER(Amr2DConfig), C.POINTER(P)], I),
        "lbm_amr2d_destroy": ([P], None),
        "lbm_amr2d_last_error": ([P], C.c_char_p),
        "lbm_amr2d_set_stream": ([P, P], I),
        "lbm_amr2d_write_root": ([P, F, F], I),
        "lbm_amr2d_read_root": ([P, F, F], I),
        "lbm_amr2d_read_pool": ([P, F, F], I),
        "lbm_amr2d_step": ([P, I], I),
        "lbm_amr2d_forces": ([P, D], I),
        "lbm_amr2d_read_topology": ([P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_int32), F, C.POINTER(C.c_uint32)], I),
        "lbm_amr2d_cell_updates": ([P], C.c_int64),
        "lbm_amr2d_sync": ([P], I),
        "lbm_amr2d_write_pool": ([P, F, F], I),
        "lbm_amr2d_read_parent_slots": ([P, C.POINTER(C.c_int32)], I),
        "lbm_amr2d_write_topology": ([P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32), C.c_int32], I),
        "lbm_amr2d_get_step": ([P], C.c_int64),
        "lbm_amr2d_set_step": ([P, C.c_int64], I),
        "lbm_amr2d_set_body": ([P, C.POINTER(Body)], I),
        "lbm_server_create": ([C.c_int64, C.POINTER(P)], I),
        "lbm_server_destroy": ([P], None),
        "lbm_server_last_error": ([P], C.c_char_p),
        "lbm_server_submit": ([P, C.c_int64, C.POINTER(Config), F, I], I),
        "lbm_server_poll": ([P, I, C.POINTER(Result), I, C.POINTER(I)], I),
        "lbm_server_read": ([P, C.c_int64, F, F], I),
        "lbm_server_release": ([P, C.c_int64], I),
        "lbm_server_stats": ([P, C.POINTER(C.c_int64)], I),
        "lbm_step_noalloc": ([C.POINTER(Config), P, P, P, P, P], I),
        "lbm_noalloc_last_error": ([], C.c_char_p),
        "lbm_tau_at_level": ([C.c_double, I], C.c_double),
        "lbm_trt_tau_minus": ([C.c_double, C.c_double], C.c_double),
        "lbm_trt_lambda": ([C.c_double, C.c_double], C.c_double),
        "lbm_dc_rescale_c2f": ([C.c_double, C.c_double], C.c_double),
        "lbm_dc_rescale_f2c": ([C.c_double, C.c_double], C.c_double),
        "lbm_tau_chain_singularity": ([C.c_double, I, C.c_double], I),
        "lbm_grant_assignment": ([C.POINTER(C.c_int32), I, I, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32)], I),
        "lbm_release_assignment": ([C.POINTER(C.c_int32), I, I, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], I),
        "lbm_active_slot_list": ([C.POINTER(C.c_int32), I, C.POINTER(C.c_int32)], I),
        "lbm_cascade21": ([C.POINTER(C.POINTER(C.c_uint8)), I, I, I], I),
        "lbm_cascade21_device": ([C.POINTER(C.POINTER(C.c_uint8)), I, I, I, P], I),
        "lbm_lattice_tables": ([I, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32), F, C.POINTER(C.c_int32)], I),
        "lbm_set_free_body": ([P, C.POINTER(BodyState), C.POINTER(BodyOpts)], I),
        "lbm_read_body_state": ([P, C.POINTER(BodyState)], I),
        "lbm_body_opts_default": ([C.POINTER(BodyOpts)], None),
        "lbm_body_state_make": ([C.POINTER(Body), C.c_double, C.POINTER(BodyState)], I),
        "lbm_body_advance": ([C.POINTER(BodyState), D, D, C.POINTER(BodyOpts), I], I),
        "lbm_amr3d_config_default": ([C.POINTER(Amr3DConfig), I, I, I, I], I),
        "lbm_amr3d_create": ([C.POINTER(Amr3DConfig), C.POINTER(C.c_uint8), C.POINTER(P)], I),
        "lbm_amr3d_destroy": ([P], None),
        "lbm_amr3d_last_error": ([P], C.c_char_p),
        "lbm_amr3d_set_stream": ([P, P], I),
        "lbm_amr3d_init_macro": ([P, F], I),
        "lbm_amr3d_step": ([P, I], I),
        "lbm_amr3d_forces": ([P, D], I),
        "lbm_amr3d_set_body": ([P, C.POINTER(Body)], I),
        "lbm_amr3d_pool_stats": ([P, C.POINTER(C.c_int32)], I),
        "lbm_amr3d_block_q": ([P, C.c_float, C.POINTER(C.c_float)], I),
        "lbm_amr3d_manage_now": ([P], I),
        "lbm_amr3d_set_links": ([P, I], I),
        "lbm_amr3d_links": ([P], I),
        "lbm_amr2d_refine_round": ([P], I),
        "lbm_amr2d_set_auto_refine": ([P, I], I),
        "lbm_amr2d_set_fused": ([P, I], I),
        "lbm_amr2d_fused": ([P], I),
        "lbm_amr3d_device_bytes": ([C.POINTER(Amr3DConfig), P, C.POINTER(C.c_int64)], I),
        "lbm_amr3d_create_in": ([C.POINTER(Amr3DConfig), P, P, C.c_int64, C.POINTER(P)], I),
        "lbm_server_submit_amr3d": ([P, C.c_int64, C.POINTER(Amr3DConfig), F, I], I),
        "lbm_server_set_policy": ([P, I, C.c_int64], I),
        "lbm_amr3d_totals": ([P, D], I),
        "lbm_amr3d_read_coarse": ([P, F, F], I),
        "lbm_amr3d_read_pool": ([P, F, F], I),
        "lbm_amr3d_topology": ([P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)], I),
        "lbm_amr3d_cell_updates": ([P], C.c_int64),
        "lbm_amr3d_sync": ([P], I),
        "lbm_amr3d_refine_blocks": ([C.POINTER(Amr3DConfig), C.POINTER(C.c_uint8)], I),
        "lbm_resolve_source": ([I, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32), C.POINTER(C.c_int32)], I),
        "lbm_f32_to_f16_bits": ([C.c_float], C.c_uint16),
        "lbm_f16_bits_to_f32": ([C.c_uint16], C.c_float),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


# ---- pure functions (lattice-2d.mjs, lattice-3d.mjs, f-pack.mjs) -----------

CS2 = 1.0 / 3.0


def lattice_tables(q: int) -> dict:
    """Velocity set, f32 weights and opposite index for D2Q9/D3Q19/D3Q27."""
    ex, ey, ez, opp = (np.zeros(q, np.int32) for _ in range(4))
    w = np.zeros(q, np.float32)
    rc = lib.lbm_lattice_tables(q, _ptr(ex, C.c_int32), _ptr(ey, C.c_int32), _ptr(ez, C.c_int32),
                                _ptr(w, C.c_float), _ptr(opp, C.c_int32))
    if rc:
        raise LbmError(rc, f"unsupported velocity set Q={q}")
    return {"ex": ex, "ey": ey, "ez": ez, "w": w, "opp": opp}


def feq(q: int, rho, ux, uy, uz, i: int):
    """BGK equilibrium, host side (lattice-3d.mjs:216 feq)."""
    t = lattice_tables(q)
    eu = t["ex"][i] * ux + t["ey"][i] * uy + t["ez"][i] * uz
    usq = ux * ux + uy * uy + uz * uz
    return float(t["w"][i]) * rho * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * usq)


def f32_to_f16_bits(v: float) -> int:
    return int(lib.lbm_f32_to_f16_bits(float(v)))


def f16_bits_to_f32(h: int) -> float:
    return float(lib.lbm_f16_bits_to_f32(int(h) & 0xFFFF))


# ---- the solver session ------------------------------------------------------

def default_config(q: int, dims) -> Config:
    nx, ny = int(dims[0]), int(dims[1])
    nz = int(dims[2]) if len(dims) > 2 else 1
    cfg = Config()
    rc = lib.lbm_config_default(C.byref(cfg), q, nx, ny, nz)
    if rc:
        raise LbmError(rc, "lbm_config_default")
    return cfg


def make_body(shape="sphere", centre=(0.0, 0.0, 0.0), a=1.0, b=None, c=None, r=0.0,
              quat=(1.0, 0.0, 0.0, 0.0), theta=0.0, v=(0.0, 0.0, 0.0), w=(0.0, 0.0, 0.0)) -> Body:
    bd = Body()
    bd.shape = SHAPE[shape] if isinstance(shape, str) else int(shape)
    bd.cx, bd.cy, bd.cz = (float(x) for x in (list(centre) + [0.0])[:3])
    bd.qw, bd.qx, bd.qy, bd.qz = (float(x) for x in quat)
    bd.theta = float(theta)
    bd.vx, bd.vy, bd.vz = (float(x) for x in v)
    bd.wx, bd.wy, bd.wz = (float(x) for x in w)
    bd.a = float(a)
    bd.b = float(a if b is None else b)
    bd.c = float(a if c is None else c)
    bd.r = float(r)
    return bd


class Solver:
    """One dense domain on the current GPU (the page session object).

    Mirrors the reference's page-level calls: ``init_macro`` (initEq),
    ``step`` (encodeSteps), ``forces`` (the drained force accumulators),
    ``totals`` (readConservedTotals / readStats), ``read_mac``, ``read_f``.
    """

    def __init__(self, cfg: Config, slab: tuple | None = None):
        """slab = (z0, nz_local): planes [z0, z0 + nz_local) of the domain
        (lbm_create_slab); its arrays then cover those planes only."""
        self.cfg = cfg
        self.q = cfg.q
        self.slab = slab
        nz = cfg.nz if slab is None else int(slab[1])
        self.dims = (cfg.nx, cfg.ny, nz)
        self.ncells = cfg.nx * cfg.ny * nz
        h = C.c_void_p()
        if slab is None:
            rc = lib.lbm_create(C.byref(cfg), C.byref(h))
        else:
            rc = lib.lbm_create_slab(C.byref(cfg), int(slab[0]), int(slab[1]), C.byref(h))
        if rc:
            raise LbmError(rc, lib.lbm_last_error(None).decode())
        self._h = h

    @classmethod
    def create(cls, q: int, dims, **kw) -> "Solver":
        return cls(config_from(q, dims, **kw))

    def _check(self, rc: int):
        if rc:
            raise LbmError(rc, lib.lbm_last_error(self._h).decode())

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self):
        if getattr(self, "_h", None):
            lib.lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_ptr: int | None):
        self._check(lib.lbm_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def init_macro(self, mac: np.ndarray):
        mac = np.ascontiguousarray(mac, dtype=np.float32).reshape(self.ncells, 4)
        self._check(lib.lbm_init_macro(self._h, _ptr(mac, C.c_float)))

    def write_f(self, f: np.ndarray):
        f = np.ascontiguousarray(f, dtype=np.float32).reshape(self.q, self.ncells)
        self._check(lib.lbm_write_f(self._h, _ptr(f, C.c_float)))

    def read_f(self) -> np.ndarray:
        out = np.empty((self.q, self.ncells), np.float32)
        self._check(lib.lbm_read_f(self._h, _ptr(out, C.c_float)))
        return out

    def _raw_dtype(self):
        return np.float32 if self.cfg.storage == STORAGE["fp32"] else np.uint16

    def write_f_raw(self, planes: np.ndarray):
        """Stored planes verbatim (uint16 bit patterns for the 16-bit storages)."""
        planes = np.ascontiguousarray(planes, dtype=self._raw_dtype()).reshape(self.q, self.ncells)
        self._check(lib.lbm_write_f_raw(self._h, planes.ctypes.data_as(C.c_void_p)))

    def read_f_raw(self) -> np.ndarray:
        out = np.empty((self.q, self.ncells), self._raw_dtype())
        self._check(lib.lbm_read_f_raw(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def read_mac(self, out: np.ndarray | None = None) -> np.ndarray:
        """The mac field (rho, ux, uy, uz per cell). `out`, if given, is a
        C-contiguous float32 array of ncells x 4 values to fill in place (a
        pinned one makes the copy a direct DMA)."""
        if out is None:
            out = np.empty((self.ncells, 4), np.float32)
        elif out.dtype != np.float32 or not out.flags.c_contiguous or out.size != self.ncells * 4:
            raise ValueError("out must be a C-contiguous float32 array of ncells x 4 values")
        self._check(lib.lbm_read_mac(self._h, _ptr(out, C.c_float)))
        return out

    def step(self, n: int = 1):
        self._check(lib.lbm_step(self._h, int(n)))

    # ---- slabs (lbm_create_slab) ----
    def halo_bytes(self) -> int:
        return int(lib.lbm_slab_halo_bytes(self._h))

    def pack(self, send_lo_ptr: int, send_hi_ptr: int):
        """The populations leaving through the bottom / top face into device buffers."""
        self._check(lib.lbm_slab_pack(self._h, C.c_void_p(send_lo_ptr), C.c_void_p(send_hi_ptr)))

    def unpack(self, recv_lo_ptr: int, recv_hi_ptr: int):
        """The neighbours' populations into the ghost planes below / above."""
        self._check(lib.lbm_slab_unpack(self._h, C.c_void_p(recv_lo_ptr), C.c_void_p(recv_hi_ptr)))

    def resample(self, **kw):
        """The field on a voxel box (volume_spec keywords; `level`, `out`)."""
        return _resample(lib.lbm_resample, self._h, self._check, self.dims, **kw)

    def render_slice(self, **kw) -> np.ndarray:
        """An axis-aligned slice picture, (height, width, 4) RGBA8."""
        return _render(lib.lbm_render_slice, self._h, self._check, self.dims, **kw)

    def set_body(self, body: Body):
        self._check(lib.lbm_set_body(self._h, C.byref(body)))

    def set_free_body(self, state: "BodyState | None", opts: "BodyOpts | None" = None):
        """Integrate the body on the device from now on (force pass, 6-DOF
        update, step); None returns it to the config's prescribed pose."""
        self._check(lib.lbm_set_free_body(self._h, C.byref(state) if state is not None else None,
                                          C.byref(opts) if opts is not None else None))

    def body_state(self) -> BodyState:
        out = BodyState()
        self._check(lib.lbm_read_body_state(self._h, C.byref(out)))
        return out

    def forces(self) -> np.ndarray:
        out = np.zeros(6, np.float64)
        self._check(lib.lbm_forces(self._h, _ptr(out, C.c_double)))
        return out

    def forces_async(self, out_ptr: int):
        """Queue the last step's force/torque (6 doubles) into host memory at
        out_ptr (pinned) without waiting; valid after sync()."""
        self._check(lib.lbm_forces_async(self._h, C.c_void_p(out_ptr)))

    def totals(self) -> dict:
        out = np.zeros(8, np.float64)
        self._check(lib.lbm_totals(self._h, _ptr(out, C.c_double)))
        keys = ("mass", "px", "py", "pz", "rho_min", "rho_max", "max_u", "nonfinite")
        return dict(zip(keys, out.tolist()))

    def sync(self):
        self._check(lib.lbm_sync(self._h))

    def device_bytes(self) -> int:
        return int(lib.lbm_device_bytes(self._h))


def body_opts(**kw) -> BodyOpts:
    """lbm_body_opts_default (v_max 0.2, o_max 0.1) with fields overridden;
    v_max / o_max of math.inf switch a clamp off."""
    o = BodyOpts()
    lib.lbm_body_opts_default(C.byref(o))
    for k, v in kw.items():
        if isinstance(getattr(o, k), C.Array):
            arr = getattr(o, k)
            for j, x in enumerate(v):
                arr[j] = x
        else:
            setattr(o, k, v)
    return o


def body_state(body: Body, density: float = 1.0) -> BodyState:
    """makeBodyState for a 3D body pose (make_body(...))."""
    out = BodyState()
    rc = lib.lbm_body_state_make(C.byref(body), float(density), C.byref(out))
    if rc:
        raise LbmError(rc, "invalid body for a body state")
    return out


def body_advance(state: BodyState, opts: BodyOpts, n: int = 1, force=(0.0, 0.0, 0.0),
                 torque=(0.0, 0.0, 0.0)) -> BodyState:
    """n host steps of stepFreeBody under a constant load (in place; returns state)."""
    f = np.ascontiguousarray(force, np.float64)
    t = np.ascontiguousarray(torque, np.float64)
    rc = lib.lbm_body_advance(C.byref(state), _ptr(f, C.c_double), _ptr(t, C.c_double), C.byref(opts), int(n))
    if rc:
        raise LbmError(rc, "invalid body state or options")
    return state


def volume_spec(dims, origin=(0.0, 0.0, 0.0), shape=None, h=(1.0, 1.0, 1.0), fp16=False) -> VolumeSpec:
    """A voxel box in L0 cell units (cell centres at integers): `shape`
    voxels of `h` L0 cells from `origin`; the whole L0 grid by default."""
    v = VolumeSpec()
    lib.lbm_volume_spec_default(C.byref(v), *dims)
    for k in range(3):
        v.origin[k] = float(origin[k])
        v.h[k] = float(h[k])
        if shape is not None:
            v.shape[k] = int(shape[k])
    v.fp16 = int(bool(fp16))
    return v


def slice_spec(dims, axis=2, slice=None, mode="speed", rot=0, width=None, height=None, u_scale=0.05,
               v_scale=0.01, vort_scale=1.0, vort_gamma=1.2) -> SliceSpec:
    """An axis-aligned slice picture (common_d3_render_slice.wgsl RParams);
    one pixel per L0 cell of the plane by default."""
    v = SliceSpec()
    lib.lbm_slice_spec_default(C.byref(v), *dims)
    v.axis = int(axis)
    v.slice = int(dims[axis] // 2 if slice is None else slice)
    v.mode = SLICE_MODES[mode] if isinstance(mode, str) else int(mode)
    v.rot = int(rot)
    pa, pb = dims[(axis + 1) % 3], dims[(axis + 2) % 3]
    if rot % 2:
        pa, pb = pb, pa
    v.width = int(pa if width is None else width)
    v.height = int(pb if height is None else height)
    v.u_scale, v.v_scale = float(u_scale), float(v_scale)
    v.vort_scale, v.vort_gamma = float(vort_scale), float(vort_gamma)
    return v


def _resample(fn, handle, check, dims, out=None, level=False, **kw):
    """Host arrays (nz, ny, nx, 4) float16/float32 and (nz, ny, nx) uint8, or
    into a device tensor `out` (its data pointer, no copy)."""
    spec = volume_spec(dims, **kw)
    shp = (spec.shape[2], spec.shape[1], spec.shape[0])
    if out is not None and hasattr(out, "data_ptr"):
        spec.device = 1
        lv = level if (level is not False and hasattr(level, "data_ptr")) else None
        check(fn(handle, C.byref(spec), C.c_void_p(out.data_ptr()),
                 C.c_void_p(lv.data_ptr() if lv is not None else 0)))
        return out, lv
    arr = np.empty(shp + (4,), np.float16 if spec.fp16 else np.float32)
    lv = np.empty(shp, np.uint8) if level else None
    check(fn(handle, C.byref(spec), arr.ctypes.data_as(C.c_void_p),
             lv.ctypes.data_as(C.c_void_p) if lv is not None else None))
    return arr, lv


def _render(fn, handle, check, dims, **kw):
    spec = slice_spec(dims, **kw)
    img = np.empty((spec.height, spec.width, 4), np.uint8)
    check(fn(handle, C.byref(spec), img.ctypes.data_as(C.c_void_p)))
    return img


def config_from(q: int, dims, **kw) -> Config:
    """An lbm_config for q/dims with fields overridden by keyword (the same
    keywords Solver.create takes)."""
    cfg = default_config(q, dims)
    for k, v in kw.items():
        if k == "storage" and isinstance(v, str):
            v = STORAGE[v]
        if k == "body" and isinstance(v, dict):
            v = make_body(**v)
        if k == "window" and (v is None or isinstance(v, str)):
            v = window_axes(v)
        if isinstance(getattr(cfg, k), C.Array):
            arr = getattr(cfg, k)
            for j, x in enumerate(v):
                arr[j] = x
        else:
            setattr(cfg, k, v)
    if any(cfg.window) and "win_anchor" not in kw:
        # the anchor is the body's initial cell, so the window's offset is 0
        # at step 0 (main-3d.js WIN_ANCHOR)
        for j, c in enumerate((cfg.body.cx, cfg.body.cy, cfg.body.cz)):
            cfg.win_anchor[j] = int(np.floor(c))
    return cfg


def window_axes(spec) -> tuple:
    """A window spec as per-axis flags (d3-window.mjs parseWindowAxes): '',
    '0', 'none' and None are off; '1', 'all', 'xyz' all three; otherwise
    the axes named. An unknown character is refused."""
    if spec is None:
        return (0, 0, 0)
    s = str(spec).strip().lower()
    if s in ("", "0", "none"):
        return (0, 0, 0)
    if s in ("1", "all", "xyz"):
        return (1, 1, 1)
    out = [0, 0, 0]
    for ch in s:
        i = "xyz".find(ch)
        if i < 0:
            raise ValueError(f"window={spec!r}: expected some of xyz, or 0/none/all")
        out[i] = 1
    return tuple(out)


class Batch:
    """Many independent domains advanced by one persistent launch per step.

    ``cfgs`` is a list of :class:`Config` (same q and storage). Per-domain
    calls take the domain index; ``forces()`` returns an (n, 6) array."""

    def __init__(self, cfgs):
        arr = (Config * len(cfgs))(*cfgs)
        self.cfgs = list(cfgs)
        self.q = cfgs[0].q
        self.ncells = [c.nx * c.ny * c.nz for c in cfgs]
        h = C.c_void_p()
        rc = lib.lbm_batch_create(arr, len(cfgs), C.byref(h))
        if rc:
            raise LbmError(rc, lib.lbm_batch_last_error(None).decode())
        self._h = h

    def _check(self, rc):
        if rc:
            raise LbmError(rc, lib.lbm_batch_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            lib.lbm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def cells(self) -> int:
        return int(lib.lbm_batch_cells(self._h))

    def set_stream(self, stream_ptr):
        self._check(lib.lbm_batch_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def init_macro(self, d: int, mac):
        mac = np.ascontiguousarray(mac, dtype=np.float32).reshape(self.ncells[d], 4)
        self._check(lib.lbm_batch_init_macro(self._h, d, _ptr(mac, C.c_float)))

    def write_f(self, d: int, f):
        f = np.ascontiguousarray(f, dtype=np.float32).reshape(self.q, self.ncells[d])
        self._check(lib.lbm_batch_write_f(self._h, d, _ptr(f, C.c_float)))

    def read_f(self, d: int) -> np.ndarray:
        out = np.empty((self.q, self.ncells[d]), np.float32)
        self._check(lib.lbm_batch_read_f(self._h, d, _ptr(out, C.c_float)))
        return out

    def read_mac(self, d: int) -> np.ndarray:
        out = np.empty((self.ncells[d], 4), np.float32)
        self._check(lib.lbm_batch_read_mac(self._h, d, _ptr(out, C.c_float)))
        return out

    def step(self, n: int = 1):
        self._check(lib.lbm_batch_step(self._h, int(n)))

    def set_tiling(self, threads: int, cells_per_thread: int, ctas_per_sm: int):
        self._check(lib.lbm_batch_set_tiling(self._h, threads, cells_per_thread, ctas_per_sm))

    def tiling(self):
        t, c, k = C.c_int(), C.c_int(), C.c_int()
        self._check(lib.lbm_batch_get_tiling(self._h, C.byref(t), C.byref(c), C.byref(k)))
        return t.value, c.value, k.value

    def autotune(self, trials: int = 3) -> float:
        ms = C.c_float()
        self._check(lib.lbm_batch_autotune(self._h, trials, C.byref(ms)))
        return ms.value

    def forces(self) -> np.ndarray:
        out = np.zeros((len(self.cfgs), 6), np.float64)
        self._check(lib.lbm_batch_forces(self._h, _ptr(out, C.c_double)))
        return out

    def sync(self):
        self._check(lib.lbm_batch_sync(self._h))


# ---- AMR host rules (amr2d.mjs) ------------------------------------------------

def tau_at_level(tau0: float, m: int) -> float:
    return float(lib.lbm_tau_at_level(tau0, m))


def trt_tau_minus(tau_plus: float, lam: float) -> float:
    """tau_- of the TRT collision for a given Lambda (plans/TRT.md sec 8.1 tauMinusOf)."""
    return float(lib.lbm_trt_tau_minus(tau_plus, lam))


def trt_lambda(tau_plus: float, tau_minus: float) -> float:
    """Lambda = (tau_+ - 1/2)(tau_- - 1/2) (plans/TRT.md sec 8.1 lambdaOf)."""
    return float(lib.lbm_trt_lambda(tau_plus, tau_minus))


def dc_rescale_c2f(tc: float, tf: float) -> float:
    return float(lib.lbm_dc_rescale_c2f(tc, tf))


def dc_rescale_f2c(tc: float, tf: float) -> float:
    return float(lib.lbm_dc_rescale_f2c(tc, tf))


def tau_chain_singularity(tau0: float, levels: int, band: float = 0.01):
    m = int(lib.lbm_tau_chain_singularity(tau0, levels, band))
    return None if m < 0 else m


def grant_assignment(candidates, free_count: int):
    """grantAssignment: ({granted: [(id, free_index)], refused: [ids], free_count})."""
    c = np.ascontiguousarray(candidates, np.int32)
    ids = np.zeros(max(len(c), 1), np.int32)
    idx = np.zeros(max(len(c), 1), np.int32)
    ng = C.c_int32()
    fc = lib.lbm_grant_assignment(_ptr(c, C.c_int32), len(c), free_count, _ptr(ids, C.c_int32),
                                  _ptr(idx, C.c_int32), C.byref(ng))
    granted = [(int(i), int(j)) for i, j in zip(ids[:len(c)], idx[:len(c)]) if j >= 0]
    refused = [int(i) for i, j in zip(ids[:len(c)], idx[:len(c)]) if j < 0]
    return {"granted": granted, "refused": refused, "free_count": int(fc)}


def release_assignment(releases, free_count: int):
    r = np.ascontiguousarray(releases, np.int32)
    ids = np.zeros(max(len(r), 1), np.int32)
    idx = np.zeros(max(len(r), 1), np.int32)
    fc = lib.lbm_release_assignment(_ptr(r, C.c_int32), len(r), free_count, _ptr(ids, C.c_int32),
                                    _ptr(idx, C.c_int32))
    return {"writes": [(int(i), int(j)) for i, j in zip(ids[:len(r)], idx[:len(r)])], "free_count": int(fc)}


def active_slot_list(slot_to_block):
    s = np.ascontiguousarray(slot_to_block, np.int32)
    out = np.zeros(max(len(s), 1), np.int32)
    n = lib.lbm_active_slot_list(_ptr(s, C.c_int32), len(s), _ptr(out, C.c_int32))
    return out[:n].tolist()


def cascade21(want_levels, levels: int, nbx1: int, nby1: int):
    """Closes per-level block masks in place (list indexed by level; entry 0
    unused). Returns (masks, number added)."""
    masks = [None] + [np.ascontiguousarray(want_levels[m], np.uint8).ravel().copy() for m in range(1, levels)]
    ptrs = (C.POINTER(C.c_uint8) * levels)()
    for m in range(1, levels):
        ptrs[m] = masks[m].ctypes.data_as(C.POINTER(C.c_uint8))
    n = lib.lbm_cascade21(ptrs, levels, nbx1, nby1)
    if n < 0:
        raise LbmError(n, "cascade21")
    return masks, int(n)


def cascade21_device(want_levels, levels: int, nbx1: int, nby1: int, stream_ptr: int | None = None):
    """cascade21 run by the device kernels (amr_cascade.wgsl's completeQuads
    and balance). Same arguments and result as cascade21."""
    masks = [None] + [np.ascontiguousarray(want_levels[m], np.uint8).ravel().copy() for m in range(1, levels)]
    ptrs = (C.POINTER(C.c_uint8) * levels)()
    for m in range(1, levels):
        ptrs[m] = masks[m].ctypes.data_as(C.POINTER(C.c_uint8))
    n = lib.lbm_cascade21_device(ptrs, levels, nbx1, nby1, C.c_void_p(stream_ptr or 0))
    if n < 0:
        raise LbmError(n, "cascade21_device")
    return masks, int(n)


def amr2d_config(nx: int, ny: int, **kw) -> Amr2DConfig:
    cfg = Amr2DConfig()
    lib.lbm_amr2d_config_default(C.byref(cfg), nx, ny)
    for k, v in kw.items():
        if k == "body" and isinstance(v, dict):
            v = make_body(**v)
        if isinstance(getattr(cfg, k), C.Array):
            arr = getattr(cfg, k)
            for j, x in enumerate(v):
                arr[j] = x
        else:
            setattr(cfg, k, v)
    return cfg


class Amr2D:
    """Two-level D2Q9 block-structured AMR session (root + one pool level)."""

    def __init__(self, cfg: Amr2DConfig):
        self.cfg = cfg
        self.W, self.H, self.rb = cfg.nx, cfg.ny, cfg.rb
        self.fb = 2 * cfg.rb + 4
        self.nbx, self.nby = cfg.nx // cfg.rb, cfg.ny // cfg.rb
        self.slots = cfg.max_slots
        h = C.c_void_p()
        rc = lib.lbm_amr2d_create(C.byref(cfg), C.byref(h))
        if rc:
            raise LbmError(rc, lib.lbm_amr2d_last_error(None).decode())
        self._h = h

    def _check(self, rc):
        if rc:
            raise LbmError(rc, lib.lbm_amr2d_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            lib.lbm_amr2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, ptr):
        self._check(lib.lbm_amr2d_set_stream(self._h, C.c_void_p(ptr or 0)))

    def write_root(self, f, vel):
        f = np.ascontiguousarray(f, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        self._check(lib.lbm_amr2d_write_root(self._h, _ptr(f, C.c_float), _ptr(vel, C.c_float)))

    def read_root(self):
        f = np.empty((9, self.W * self.H), np.float32)
        v = np.empty((self.W * self.H, 2), np.float32)
        self._check(lib.lbm_amr2d_read_root(self._h, _ptr(f, C.c_float), _ptr(v, C.c_float)))
        return f, v

    def read_pool(self):
        n = self.slots * self.fb * self.fb
        f = np.empty((9, n), np.float32)
        v = np.empty((n, 2), np.float32)
        self._check(lib.lbm_amr2d_read_pool(self._h, _ptr(f, C.c_float), _ptr(v, C.c_float)))
        return f, v

    def step(self, n: int = 1):
        self._check(lib.lbm_amr2d_step(self._h, int(n)))

    def refine_round(self):
        """One refine round now (criterion, decide, coarsen, refine, fill)."""
        self._check(lib.lbm_amr2d_refine_round(self._h))

    def set_auto_refine(self, on: bool):
        self._check(lib.lbm_amr2d_set_auto_refine(self._h, int(bool(on))))

    def set_fused(self, on: bool):
        """One cooperative launch per macro-step (on) or six launches (off)."""
        self._check(lib.lbm_amr2d_set_fused(self._h, int(bool(on))))

    @property
    def fused(self) -> bool:
        return bool(lib.lbm_amr2d_fused(self._h))

    def forces(self):
        out = np.zeros(4, np.float64)
        self._check(lib.lbm_amr2d_forces(self._h, _ptr(out, C.c_double)))
        return out

    def topology(self) -> dict:
        nb = self.nbx * self.nby
        bs, sb = np.zeros(nb, np.int32), np.zeros(self.slots, np.int32)
        fl, cnt = np.zeros(self.slots // 4, np.int32), np.zeros(2, np.int32)
        al, cr, wa = np.zeros(self.slots, np.int32), np.zeros(nb, np.float32), np.zeros(nb, np.uint32)
        self._check(lib.lbm_amr2d_read_topology(self._h, _ptr(bs, C.c_int32), _ptr(sb, C.c_int32),
                                                 _ptr(fl, C.c_int32), _ptr(cnt, C.c_int32), _ptr(al, C.c_int32),
                                                 _ptr(cr, C.c_float), _ptr(wa, C.c_uint32)))
        return {"block_slot": bs, "slot_to_block": sb, "free_list": fl, "free_count": int(cnt[0]),
                "active": al[:cnt[1]].copy(), "criterion": cr, "want": wa}

    def cell_updates(self) -> int:
        return int(lib.lbm_amr2d_cell_updates(self._h))

    def sync(self):
        self._check(lib.lbm_amr2d_sync(self._h))

    def write_pool(self, f, vel):
        f = np.ascontiguousarray(f, np.float32).reshape(9, -1)
        vel = np.ascontiguousarray(vel, np.float32).reshape(-1, 2)
        self._check(lib.lbm_amr2d_write_pool(self._h, _ptr(f, C.c_float), _ptr(vel, C.c_float)))

    def parent_slots(self) -> np.ndarray:
        out = np.zeros(self.slots, np.int32)
        self._check(lib.lbm_amr2d_read_parent_slots(self._h, _ptr(out, C.c_int32)))
        return out

    def write_topology(self, block_slot, slot_to_block, parent_slot, free_list, free_count: int):
        i32 = lambda a: np.ascontiguousarray(a, np.int32)
        bs, sb, ps, fl = i32(block_slot), i32(slot_to_block), i32(parent_slot), i32(free_list)
        self._check(lib.lbm_amr2d_write_topology(self._h, _ptr(bs, C.c_int32), _ptr(sb, C.c_int32),
                                                  _ptr(ps, C.c_int32), _ptr(fl, C.c_int32), int(free_count)))

    @property
    def macro_step(self) -> int:
        return int(lib.lbm_amr2d_get_step(self._h))

    @macro_step.setter
    def macro_step(self, step: int):
        self._check(lib.lbm_amr2d_set_step(self._h, int(step)))

    def set_body(self, body: Body):
        self._check(lib.lbm_amr2d_set_body(self._h, C.byref(body)))


def amr3d_config(q: int, dims, refine="body", rb: int = 4, margin: float = 2.0, boxfrac: float = 0.5,
                 explode_linear: int = 1, dynamic: int = 0, manage_every: int = 16, manage_start: int = 0,
                 max_slots: int = 0, slot_headroom: float = 1.5, iface: int = 0, reflux: int = 0,
                 q_abs: float = 0.0, q_hyst: float = 1.0, q_lead: float = 0.0, **root_kw) -> Amr3DConfig:
    """lbm_amr3d_config: the L0 grid/physics as config_from's keywords, plus the hierarchy."""
    c = Amr3DConfig()
    rc = lib.lbm_amr3d_config_default(C.byref(c), q, *dims)
    if rc:
        raise LbmError(rc, "bad dims")
    c.root = config_from(q, dims, **root_kw)
    c.rb = rb
    c.refine = REFINE[refine] if isinstance(refine, str) else int(refine)
    c.margin = margin
    c.boxfrac = boxfrac
    c.explode_linear = explode_linear
    c.dynamic = dynamic
    c.manage_every = manage_every
    c.manage_start = manage_start
    c.max_slots = max_slots
    c.slot_headroom = slot_headroom
    c.iface = iface
    c.reflux = reflux
    c.q_abs = q_abs
    c.q_hyst = q_hyst
    c.q_lead = q_lead
    return c


def amr3d_device_bytes(cfg: Amr3DConfig) -> int:
    """Device bytes the hierarchy holds (no GPU needed)."""
    out = C.c_int64()
    rc = lib.lbm_amr3d_device_bytes(C.byref(cfg), None, C.byref(out))
    if rc:
        raise LbmError(rc, lib.lbm_amr3d_last_error(None).decode())
    return int(out.value)


def amr3d_refine_blocks(cfg: Amr3DConfig) -> np.ndarray:
    nb = (cfg.root.nx // cfg.rb) * (cfg.root.ny // cfg.rb) * (cfg.root.nz // cfg.rb)
    out = np.zeros(nb, np.uint8)
    rc = lib.lbm_amr3d_refine_blocks(C.byref(cfg), _ptr(out, C.c_uint8))
    if rc:
        raise LbmError(rc, "lbm_amr3d_refine_blocks")
    return out


def resolve_source(rb: int, nb, block_slot, block, src):
    """d3-amr.mjs resolveSource: (slot, fx, fy, fz); slot -1 = own tile, -2 = no tile."""
    nb = np.ascontiguousarray(nb, np.int32)
    bs = np.ascontiguousarray(block_slot, np.int32)
    b = np.ascontiguousarray(block, np.int32)
    s = np.ascontiguousarray(src, np.int32)
    out = np.zeros(4, np.int32)
    i32 = lambda a: _ptr(a, C.c_int32)
    rc = lib.lbm_resolve_source(int(rb), i32(nb), i32(bs), i32(b), i32(s), i32(out))
    if rc:
        raise LbmError(rc, "lbm_resolve_source")
    return tuple(int(v) for v in out)


class Amr3D:
    """Two-level 3D AMR on the current GPU (the 3D page's AMR session)."""

    def __init__(self, cfg: Amr3DConfig, block_want=None):
        self.cfg = cfg
        self.q = cfg.root.q
        self.dims = (cfg.root.nx, cfg.root.ny, cfg.root.nz)
        self.ncells = int(np.prod(self.dims))
        h = C.c_void_p()
        w = None
        if block_want is not None:
            self._want = np.ascontiguousarray(block_want, np.uint8)
            w = _ptr(self._want, C.c_uint8)
        rc = lib.lbm_amr3d_create(C.byref(cfg), w, C.byref(h))
        if rc:
            raise LbmError(rc, lib.lbm_amr3d_last_error(None).decode())
        self._h = h
        self.nb = tuple(d // cfg.rb for d in self.dims)
        t = self.topology()
        self.slots, self.fb = t["slots"], t["fb"]

    def _check(self, rc: int):
        if rc:
            raise LbmError(rc, lib.lbm_amr3d_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            lib.lbm_amr3d_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_stream(self, stream_ptr: int | None):
        self._check(lib.lbm_amr3d_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def init_macro(self, mac: np.ndarray):
        mac = np.ascontiguousarray(mac, dtype=np.float32).reshape(self.ncells, 4)
        self._check(lib.lbm_amr3d_init_macro(self._h, _ptr(mac, C.c_float)))

    def step(self, n: int = 1):
        self._check(lib.lbm_amr3d_step(self._h, int(n)))

    def forces(self) -> np.ndarray:
        out = np.zeros(6)
        self._check(lib.lbm_amr3d_forces(self._h, _ptr(out, C.c_double)))
        return out

    def totals(self) -> np.ndarray:
        out = np.zeros(4)
        self._check(lib.lbm_amr3d_totals(self._h, _ptr(out, C.c_double)))
        return out

    def read_coarse(self):
        f = np.empty((self.q, self.ncells), np.float32)
        mac = np.empty((self.ncells, 4), np.float32)
        self._check(lib.lbm_amr3d_read_coarse(self._h, _ptr(f, C.c_float), _ptr(mac, C.c_float)))
        return f, mac

    def read_pool(self):
        n = self.slots * self.fb ** 3
        f = np.empty((self.q, n), np.float32)
        mac = np.empty((n, 4), np.float32)
        self._check(lib.lbm_amr3d_read_pool(self._h, _ptr(f, C.c_float), _ptr(mac, C.c_float)))
        return f, mac

    def topology(self) -> dict:
        nb = int(np.prod([d // self.cfg.rb for d in self.dims]))
        bs = np.zeros(nb, np.int32)
        sb = np.zeros(nb, np.int32)
        cnt = np.zeros(3, np.int32)
        self._check(lib.lbm_amr3d_topology(self._h, _ptr(bs, C.c_int32), _ptr(sb, C.c_int32), _ptr(cnt, C.c_int32)))
        return {"block_slot": bs, "slot_to_block": sb[:cnt[0]].copy(), "slots": int(cnt[0]), "fb": int(cnt[1])}

    def set_body(self, body: Body):
        self._check(lib.lbm_amr3d_set_body(self._h, C.byref(body)))

    def pool_stats(self) -> dict:
        out = np.zeros(4, np.int32)
        self._check(lib.lbm_amr3d_pool_stats(self._h, _ptr(out, C.c_int32)))
        return {"in_use": int(out[0]), "refusals": int(out[1]), "min_free": int(out[2]), "decisions": int(out[3])}

    def resample(self, **kw):
        """The hierarchy on a voxel box, finest level wins (volume_spec keywords)."""
        return _resample(lib.lbm_amr3d_resample, self._h, self._check, self.dims, **kw)

    def render_slice(self, **kw) -> np.ndarray:
        """An axis-aligned slice picture of the hierarchy, (height, width, 4)."""
        return _render(lib.lbm_amr3d_render_slice, self._h, self._check, self.dims, **kw)

    def manage_now(self):
        """One decision of the dynamic manager before the next macro-step."""
        self._check(lib.lbm_amr3d_manage_now(self._h))

    def set_links(self, on: bool):
        """The bounce-back link table on (the default) or off: the same bits
        either way, off evaluates the body's distance in every step."""
        self._check(lib.lbm_amr3d_set_links(self._h, 1 if on else 0))

    @property
    def links(self) -> bool:
        return bool(lib.lbm_amr3d_links(self._h))

    def block_q(self, lead: float = 0.0) -> np.ndarray:
        """Per-block max Q-criterion of the L0 velocity, box dilated by `lead`."""
        out = np.zeros(int(np.prod(self.nb)), np.float32)
        self._check(lib.lbm_amr3d_block_q(self._h, float(lead), _ptr(out, C.c_float)))
        return out

    def cell_updates(self) -> int:
        return int(lib.lbm_amr3d_cell_updates(self._h))

    def sync(self):
        self._check(lib.lbm_amr3d_sync(self._h))


def step_noalloc(cfg: Config, f_in_ptr: int, f_out_ptr: int, mac_ptr: int | None = None,
                 force_ptr: int | None = None, stream_ptr: int | None = None):
    """One dense step between caller-owned device buffers, with no device
    allocation inside the library (lbm_step_noalloc)."""
    rc = lib.lbm_step_noalloc(C.byref(cfg), C.c_void_p(f_in_ptr), C.c_void_p(f_out_ptr),
                              C.c_void_p(mac_ptr or 0), C.c_void_p(force_ptr or 0), C.c_void_p(stream_ptr or 0))
    if rc:
        raise LbmError(rc, lib.lbm_noalloc_last_error().decode())


class Server:
    """Continuous-batching request loop over one device arena (lbm_server)."""

    def __init__(self, budget_bytes: int):
        h = C.c_void_p()
        rc = lib.lbm_server_create(int(budget_bytes), C.byref(h))
        if rc:
            raise LbmError(rc, lib.lbm_server_last_error(None).decode())
        self._h = h
        self._results = (Result * 256)()

    def _check(self, rc):
        if rc:
            raise LbmError(rc, lib.lbm_server_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            lib.lbm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, rid: int, cfg: Config, steps: int, mac=None):
        ptr = None
        if mac is not None:
            mac = np.ascontiguousarray(mac, np.float32)
            ptr = _ptr(mac, C.c_float)
        self._check(lib.lbm_server_submit(self._h, int(rid), C.byref(cfg), ptr, int(steps)))

    def set_policy(self, policy: str = "fifo", max_resident_cells: int = 0):
        """Admission order ("fifo" or "sjf": least cells x steps first) and a
        cap on the resident requests' cells (0: the budget alone)."""
        p = {"fifo": 0, "sjf": 1}[policy]
        self._check(lib.lbm_server_set_policy(self._h, p, int(max_resident_cells)))

    def submit_amr3d(self, rid: int, cfg: Amr3DConfig, steps: int, mac=None):
        """Queues a 3D two-level AMR solve of `steps` macro-steps."""
        ptr = None
        if mac is not None:
            mac = np.ascontiguousarray(mac, np.float32)
            ptr = _ptr(mac, C.c_float)
        self._check(lib.lbm_server_submit_amr3d(self._h, int(rid), C.byref(cfg), ptr, int(steps)))

    def poll(self, max_steps: int = 64):
        n = C.c_int()
        self._check(lib.lbm_server_poll(self._h, int(max_steps), self._results, len(self._results), C.byref(n)))
        out = []
        for k in range(n.value):
            r = self._results[k]
            out.append({"id": r.id, "steps": r.steps, "forces": list(r.forces), "submit_s": r.submit_s,
                        "admit_s": r.admit_s, "done_s": r.done_s})
        return out

    def read(self, rid: int, cfg, f: bool = True):
        """Final f and mac of a finished solve (an AMR solve's L0 level)."""
        if isinstance(cfg, Amr3DConfig):
            cfg = cfg.root
        n = cfg.nx * cfg.ny * cfg.nz
        mac = np.empty((n, 4), np.float32)
        ff = np.empty((cfg.q, n), np.float32) if f else None
        self._check(lib.lbm_server_read(self._h, int(rid), _ptr(ff, C.c_float) if f else None, _ptr(mac, C.c_float)))
        return ff, mac

    def release(self, rid: int):
        self._check(lib.lbm_server_release(self._h, int(rid)))

    def stats(self) -> dict:
        out = np.zeros(6, np.int64)
        self._check(lib.lbm_server_stats(self._h, out.ctypes.data_as(C.POINTER(C.c_int64))))
        return dict(zip(("queued", "resident", "finished", "bytes_used", "budget", "lattice_updates"),
                        out.tolist()))
