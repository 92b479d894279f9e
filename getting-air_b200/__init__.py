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


class Config(C.Structure):
    _fields_ = [("q", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("tau", C.c_float), ("force", C.c_float * 3), ("wall", C.c_int32 * 3),
                ("wall_u", C.c_float * 2), ("has_body", C.c_int32),
                ("use_bounceback", C.c_int32), ("solid_eq", C.c_int32),
                ("rho_w_local", C.c_int32), ("swept_force", C.c_int32),
                ("chi_eps", C.c_float), ("sponge_w", C.c_float),
                ("sponge_axis", C.c_int32 * 3), ("sponge_u", C.c_float * 3),
                ("body", Body), ("storage", C.c_int32), ("reserved", C.c_int32 * 7)]


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
        "lbm_destroy": ([P], None),
        "lbm_last_error": ([P], C.c_char_p),
        "lbm_set_stream": ([P, P], I),
        "lbm_init_macro": ([P, F], I),
        "lbm_write_f": ([P, F], I),
        "lbm_read_f": ([P, F], I),
        "lbm_read_mac": ([P, F], I),
        "lbm_step": ([P, I], I),
        "lbm_set_body": ([P, C.POINTER(Body)], I),
        "lbm_forces": ([P, D], I),
        "lbm_totals": ([P, D], I),
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
        "lbm_lattice_tables": ([I, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                C.POINTER(C.c_int32), F, C.POINTER(C.c_int32)], I),
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

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.q = cfg.q
        self.dims = (cfg.nx, cfg.ny, cfg.nz)
        self.ncells = cfg.nx * cfg.ny * cfg.nz
        h = C.c_void_p()
        rc = lib.lbm_create(C.byref(cfg), C.byref(h))
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

    def read_mac(self) -> np.ndarray:
        out = np.empty((self.ncells, 4), np.float32)
        self._check(lib.lbm_read_mac(self._h, _ptr(out, C.c_float)))
        return out

    def step(self, n: int = 1):
        self._check(lib.lbm_step(self._h, int(n)))

    def set_body(self, body: Body):
        self._check(lib.lbm_set_body(self._h, C.byref(body)))

    def forces(self) -> np.ndarray:
        out = np.zeros(6, np.float64)
        self._check(lib.lbm_forces(self._h, _ptr(out, C.c_double)))
        return out

    def totals(self) -> dict:
        out = np.zeros(8, np.float64)
        self._check(lib.lbm_totals(self._h, _ptr(out, C.c_double)))
        keys = ("mass", "px", "py", "pz", "rho_min", "rho_max", "max_u", "nonfinite")
        return dict(zip(keys, out.tolist()))

    def sync(self):
        self._check(lib.lbm_sync(self._h))

    def device_bytes(self) -> int:
        return int(lib.lbm_device_bytes(self._h))


def config_from(q: int, dims, **kw) -> Config:
    """An lbm_config for q/dims with fields overridden by keyword (the same
    keywords Solver.create takes)."""
    cfg = default_config(q, dims)
    for k, v in kw.items():
        if k == "storage" and isinstance(v, str):
            v = STORAGE[v]
        if k == "body" and isinstance(v, dict):
            v = make_body(**v)
        if isinstance(getattr(cfg, k), C.Array):
            arr = getattr(cfg, k)
            for j, x in enumerate(v):
                arr[j] = x
        else:
            setattr(cfg, k, v)
    return cfg


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
