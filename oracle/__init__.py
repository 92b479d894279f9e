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
