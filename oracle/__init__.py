"""ORACLE -- test infrastructure only.

ctypes wrapper over oracle/_build/liboracle.so, the CPU (FP64 / FP32
operation-order) restatement of the reference's shader arithmetic. Only the
tests, the smoke check and the benchmark's CPU-baseline leg import this, and
only as the checker: the product library never calls it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = _build.OUT
        if not path.exists():
            path = _build.build()
        L = C.CDLL(str(path))
        D, I, P = C.POINTER(C.c_double), C.c_int, C.c_void_p
        I32 = C.POINTER(C.c_int32)
        L.oracle_tables.argtypes = [I, I32, I32, I32, C.POINTER(C.c_float), I32]
        L.oracle_init_eq.argtypes = [I, C.c_int64, I, D, D]
        L.oracle_run.argtypes = [P, I, D, I, D, D]
        L.oracle_totals.argtypes = [I, C.c_int64, D, D]
        L.oracle_amr2d_create.argtypes = [P, I]
        L.oracle_amr2d_create.restype = P
        L.oracle_amr2d_destroy.argtypes = [P]
        L.oracle_amr2d_write_root.argtypes = [P, D, D]
        L.oracle_amr2d_step.argtypes = [P, I]
        L.oracle_amr2d_refine_from_vel.argtypes = [P, C.POINTER(C.c_float)]
        L.oracle_amr2d_set_topology.argtypes = [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                                C.POINTER(C.c_int32), C.c_int32]
        L.oracle_amr2d_read.argtypes = [P, D, D, D, D, C.POINTER(C.c_int32), C.POINTER(C.c_float), D]
        L.oracle_body_make.argtypes = [P, C.c_double, P]
        L.oracle_body_step.argtypes = [P, D, D, P, I]
        L.oracle_run_free.argtypes = [P, I, D, I, P, P, D, D, D]
        L.oracle_f16_bits.argtypes = [C.c_float]
        L.oracle_f16_bits.restype = C.c_uint16
        _LIB = L
    return _LIB


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def tables(q: int) -> dict:
    ex, ey, ez, opp = (np.zeros(q, np.int32) for _ in range(4))
    w = np.zeros(q, np.float32)
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    rc = lib().oracle_tables(q, p(ex), p(ey), p(ez), w.ctypes.data_as(C.POINTER(C.c_float)), p(opp))
    if rc:
        raise ValueError(q)
    return {"ex": ex, "ey": ey, "ez": ez, "w": w, "opp": opp}


def init_eq(q: int, mac: np.ndarray, fp32: bool = False) -> np.ndarray:
    mac = np.ascontiguousarray(mac, np.float64).reshape(-1, 4)
    n = mac.shape[0]
    f = np.zeros((q, n), np.float64)
    lib().oracle_init_eq(q, n, int(fp32), _d(mac), _d(f))
    return f


def run(cfg, f: np.ndarray, nsteps: int, fp32: bool = False):
    """Advances f (Q x n, float64) by nsteps; returns (f, mac, forces[nsteps, 8])."""
    f = np.array(f, np.float64, order="C", copy=True)
    n = f.shape[-1]
    mac = np.zeros((n, 4), np.float64)
    forces = np.zeros((max(nsteps, 1), 8), np.float64)
    rc = lib().oracle_run(C.cast(C.byref(cfg), C.c_void_p), int(fp32), _d(f), int(nsteps), _d(mac), _d(forces))
    if rc:
        raise ValueError("oracle_run failed")
    return f, mac, forces[:nsteps]


def totals(q: int, f: np.ndarray) -> np.ndarray:
    f = np.ascontiguousarray(f, np.float64)
    out = np.zeros(8, np.float64)
    lib().oracle_totals(q, f.shape[-1], _d(f), _d(out))
    return out


def f16_bits(v: float) -> int:
    return int(lib().oracle_f16_bits(float(v)))


class Amr2D:
    """The AMR macro-step restated on the CPU (FP64, or the f32 operation
    order with fp32=True). cfg is the product's Amr2DConfig structure."""

    def __init__(self, cfg, fp32: bool = False):
        self.cfg = cfg
        self.W, self.H, self.rb, self.S = cfg.nx, cfg.ny, cfg.rb, cfg.max_slots
        self.fb = 2 * cfg.rb + 4
        self.nb = (cfg.nx // cfg.rb) * (cfg.ny // cfg.rb)
        self._h = lib().oracle_amr2d_create(C.cast(C.byref(cfg), C.c_void_p), int(fp32))

    def close(self):
        if self._h:
            lib().oracle_amr2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def write_root(self, f, vel):
        f = np.ascontiguousarray(f, np.float64)
        vel = np.ascontiguousarray(vel, np.float64)
        lib().oracle_amr2d_write_root(self._h, _d(f), _d(vel))

    def step(self, n=1):
        lib().oracle_amr2d_step(self._h, int(n))

    def refine_from_vel(self, vel):
        v = np.ascontiguousarray(vel, np.float32)
        lib().oracle_amr2d_refine_from_vel(self._h, v.ctypes.data_as(C.POINTER(C.c_float)))

    def set_topology(self, block_slot, slot_to_block, free_list, free_count: int):
        i32 = lambda a: np.ascontiguousarray(a, np.int32)
        bs, sb, fl = i32(block_slot), i32(slot_to_block), i32(free_list)
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        lib().oracle_amr2d_set_topology(self._h, p(bs), p(sb), p(fl), int(free_count))

    def read(self) -> dict:
        n0, n1 = self.W * self.H, self.S * self.fb * self.fb
        f0, v0 = np.zeros((9, n0)), np.zeros((n0, 2))
        f1, v1 = np.zeros((9, n1)), np.zeros((n1, 2))
        topo = np.zeros(self.nb + self.S + self.S // 4 + 2 + self.S + self.nb, np.int32)
        crit = np.zeros(self.nb, np.float32)
        force = np.zeros(4)
        lib().oracle_amr2d_read(self._h, _d(f0), _d(v0), _d(f1), _d(v1),
                                topo.ctypes.data_as(C.POINTER(C.c_int32)),
                                crit.ctypes.data_as(C.POINTER(C.c_float)), _d(force))
        o = 0
        out = {"f0": f0, "vel0": v0, "f1": f1, "vel1": v1, "criterion": crit, "force": force}
        out["block_slot"] = topo[o:o + self.nb]; o += self.nb
        out["slot_to_block"] = topo[o:o + self.S]; o += self.S
        out["free_list"] = topo[o:o + self.S // 4]; o += self.S // 4
        out["free_count"] = int(topo[o]); n_act = int(topo[o + 1]); o += 2
        out["active"] = topo[o:o + n_act].copy(); o += self.S
        out["want"] = topo[o:o + self.nb].astype(np.uint32)
        return out


def body_make(body, density: float = 1.0):
    """makeBodyState (FP64) -> the product's BodyState structure type."""
    from getting_air_b200 import BodyState  # the ctypes layout only
    out = BodyState()
    if lib().oracle_body_make(C.addressof(body), float(density), C.addressof(out)):
        raise ValueError("bad body")
    return out


def body_step(state, opts, n: int = 1, force=(0.0, 0.0, 0.0), torque=(0.0, 0.0, 0.0)):
    """n steps of stepFreeBody under a constant load, in place."""
    f = np.ascontiguousarray(force, np.float64)
    t = np.ascontiguousarray(torque, np.float64)
    lib().oracle_body_step(C.addressof(state), _d(f), _d(t), C.addressof(opts), int(n))
    return state


def run_free(cfg, f0: np.ndarray, nsteps: int, state, opts, fp32: bool = False):
    """Coupled free-body run: returns (f, mac, forces[nsteps, 8], traj[nsteps, 16]);
    `state` is advanced in place. traj rows: x(3) v(3) L(3) omega(3) q(4)."""
    f = np.ascontiguousarray(f0, np.float64).copy()
    n = cfg.nx * cfg.ny * cfg.nz
    mac = np.zeros((n, 4))
    forces = np.zeros((nsteps, 8))
    traj = np.zeros((nsteps, 16))
    rc = lib().oracle_run_free(C.addressof(cfg), int(fp32), _d(f), int(nsteps), C.addressof(state),
                               C.addressof(opts), _d(mac), _d(forces), _d(traj))
    if rc:
        raise ValueError("oracle_run_free failed")
    return f, mac, forces, traj


def q_cells(mac) -> np.ndarray:
    """Q-criterion at every cell of a periodic (nz, ny, nx, 4) [rho, u] field,
    f32 (common_d3_criterion.wgsl qAt)."""
    m = np.ascontiguousarray(mac, np.float32)
    nz, ny, nx = m.shape[:3]
    out = np.zeros((nz, ny, nx), np.float32)
    L = lib()
    L.oracle_q_cells.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.oracle_q_cells(nx, ny, nz, m.ctypes.data_as(C.POINTER(C.c_float)), out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def q_of_grad(J) -> float:
    """Q = 1/2 (|Omega|^2 - |S|^2) of a 3x3 gradient J[i][j] = du_i/dx_j, FP64
    (d3-criterion.mjs qOfGrad)."""
    j = np.ascontiguousarray(J, np.float64).reshape(9)
    L = lib()
    L.oracle_q_of_grad.argtypes = [C.POINTER(C.c_double)]
    L.oracle_q_of_grad.restype = C.c_double
    return float(L.oracle_q_of_grad(_d(j)))


class Amr3D:
    """The 3D two-level AMR restatement (FP64, or the reference's f32 order)."""

    def __init__(self, cfg, block_want=None, fp32: bool = False, capacity: int = 0):
        self._h = None
        L = lib()
        L.oracle_amr3d_create.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                          C.POINTER(C.c_int32), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_int, C.c_int]
        L.oracle_amr3d_pool_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
        L.oracle_amr3d_set_body.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_amr3d_create.restype = C.c_void_p
        L.oracle_amr3d_destroy.argtypes = [C.c_void_p]
        L.oracle_amr3d_topology.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.oracle_amr3d_seed.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.oracle_amr3d_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        L.oracle_amr3d_read.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 4
        r = cfg.root
        self.q, self.dims, self.rb = r.q, (r.nx, r.ny, r.nz), cfg.rb
        self.nb = tuple(d // cfg.rb for d in self.dims)
        self.fb = 2 * cfg.rb + 4
        lst = None
        if block_want is not None:
            arr = np.ascontiguousarray(block_want, np.int32)
            self._list = arr
            lst = arr.ctypes.data_as(C.POINTER(C.c_int32))
        self._h = L.oracle_amr3d_create(C.addressof(r), cfg.rb, cfg.refine, cfg.margin, cfg.boxfrac, lst,
                                        cfg.explode_linear, int(fp32), int(capacity), int(cfg.dynamic),
                                        int(cfg.manage_every), int(cfg.manage_start),
                                        int(cfg.iface) | (int(cfg.reflux) << 1))
        if not self._h:
            raise ValueError("oracle_amr3d_create failed")
        L.oracle_amr3d_set_q.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float]
        L.oracle_amr3d_block_q.argtypes = [C.c_void_p, C.c_float, C.POINTER(C.c_float)]
        L.oracle_amr3d_set_q(self._h, float(cfg.q_abs), float(cfg.q_hyst), float(cfg.q_lead))
        nbl = int(np.prod(self.nb))
        self.block_slot = np.zeros(nbl, np.int32)
        s2b = np.zeros(nbl, np.int32)
        self.slots = L.oracle_amr3d_topology(self._h, self.block_slot.ctypes.data_as(C.POINTER(C.c_int32)),
                                             s2b.ctypes.data_as(C.POINTER(C.c_int32)))
        self.slot_to_block = s2b[:self.slots].copy()

    def pool_stats(self) -> dict:
        out = np.zeros(4, np.int32)
        lib().oracle_amr3d_pool_stats(self._h, out.ctypes.data_as(C.POINTER(C.c_int32)))
        return {"in_use": int(out[0]), "refusals": int(out[1]), "min_free": int(out[2]), "decisions": int(out[3])}

    def set_body(self, body):
        lib().oracle_amr3d_set_body(self._h, C.addressof(body))

    def topology(self):
        nbl = int(np.prod(self.nb))
        bs = np.zeros(nbl, np.int32)
        s2b = np.zeros(max(nbl, self.slots), np.int32)
        n = lib().oracle_amr3d_topology(self._h, bs.ctypes.data_as(C.POINTER(C.c_int32)),
                                        s2b.ctypes.data_as(C.POINTER(C.c_int32)))
        return bs, s2b[:n].copy()

    def block_q(self, lead: float = 0.0) -> np.ndarray:
        """Per-block max Q of the current coarse mac, box dilated by `lead`."""
        out = np.zeros(int(np.prod(self.nb)), np.float32)
        lib().oracle_amr3d_block_q(self._h, float(lead), out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def seed(self, mac):
        m = np.ascontiguousarray(mac, np.float64).reshape(-1, 4)
        lib().oracle_amr3d_seed(self._h, _d(m))

    def step(self, n: int) -> np.ndarray:
        forces = np.zeros((max(n, 1), 8))
        lib().oracle_amr3d_step(self._h, int(n), _d(forces))
        return forces[:n]

    def read(self):
        n = int(np.prod(self.dims))
        p = self.slots * self.fb ** 3
        fc, macc = np.zeros((self.q, n)), np.zeros((n, 4))
        fp, macp = np.zeros((self.q, p)), np.zeros((p, 4))
        lib().oracle_amr3d_read(self._h, _d(fc), _d(macc), _d(fp), _d(macp))
        return fc, macc, fp, macp

    def close(self):
        if self._h:
            lib().oracle_amr3d_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def _win_fn(name, nargs):
    f = getattr(lib(), name)
    f.argtypes = [C.c_double] * nargs
    f.restype = C.c_double
    return f


def win_wrap_delta(d: float, n: float) -> float:
    """Nearest periodic image of a delta on an axis of length n (0 = no window)."""
    return _win_fn("oracle_win_wrap_delta", 2)(d, n)


def win_offset(c: float, anchor: float, n: float) -> float:
    """Whole cells the window has travelled: floor(c) - anchor (0 = no window)."""
    return _win_fn("oracle_win_offset", 3)(c, anchor, n)


def win_coord(p: float, off: float, n: float) -> float:
    """A buffer position as a window coordinate in [0, n)."""
    return _win_fn("oracle_win_coord", 3)(p, off, n)


def win_wrap_position(c: float, n: float) -> float:
    """A body position wrapped into the buffer [0, n)."""
    return _win_fn("oracle_win_wrap_position", 2)(c, n)


def _tree_args(mac, dims, levels, macp, block_slot, rb, fb):
    nx, ny, nz = dims
    mac = np.ascontiguousarray(mac, np.float32).reshape(-1, 4)
    if levels:
        macp = np.ascontiguousarray(macp, np.float32).reshape(-1, 4)
        bs = np.ascontiguousarray(block_slot, np.int32)
    else:
        macp = np.zeros((1, 4), np.float32)
        bs = np.zeros(1, np.int32)
    keep = (mac, macp, bs)
    F, I32 = C.POINTER(C.c_float), C.POINTER(C.c_int32)
    return keep, [nx, ny, nz, mac.ctypes.data_as(F), int(levels), macp.ctypes.data_as(F), bs.ctypes.data_as(I32),
                  int(rb), int(fb)]


def tree_resample(mac, dims, origin, shape, h, levels=0, macp=None, block_slot=None, rb=1, fb=1):
    """The voxel box sampled from the hierarchy (finest level wins): (nvox, 4)
    f32 texels (ux, uy, uz, rho), x fastest, and the level per voxel."""
    keep, args = _tree_args(mac, dims, levels, macp, block_slot, rb, fb)
    nvox = int(np.prod(shape))
    out = np.zeros((nvox, 4), np.float32)
    lvl = np.zeros(nvox, np.uint8)
    o = np.ascontiguousarray(origin, np.float32)
    s = np.ascontiguousarray(shape, np.int32)
    hh = np.ascontiguousarray(h, np.float32)
    F = C.POINTER(C.c_float)
    lib().oracle_tree_resample(*args, o.ctypes.data_as(F), s.ctypes.data_as(C.POINTER(C.c_int32)),
                               hh.ctypes.data_as(F), out.ctypes.data_as(F), lvl.ctypes.data_as(C.POINTER(C.c_uint8)))
    del keep
    return out, lvl


def tree_slice(mac, dims, axis, slice, mode, rot, width, height, u_scale, v_scale, vort_scale=1.0, vort_gamma=1.2,
               off=(0.0, 0.0, 0.0), levels=0, macp=None, block_slot=None, rb=1, fb=1):
    """One slice picture (height, width, 4) uint8, rows top to bottom."""
    keep, args = _tree_args(mac, dims, levels, macp, block_slot, rb, fb)
    params = np.array([axis, slice, mode, rot, width, height], np.int32)
    scales = np.array([u_scale, v_scale, vort_scale, vort_gamma], np.float32)
    o = np.ascontiguousarray(off, np.float32)
    img = np.zeros((height, width, 4), np.uint8)
    F = C.POINTER(C.c_float)
    lib().oracle_tree_slice(*args, params.ctypes.data_as(C.POINTER(C.c_int32)), scales.ctypes.data_as(F),
                            o.ctypes.data_as(F), img.ctypes.data_as(C.POINTER(C.c_uint8)))
    del keep
    return img
