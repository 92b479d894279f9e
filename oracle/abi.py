"""ORACLE -- test infrastructure only.

A ctypes mirror of the C ABI's `lbm_body` and `lbm_config` structures
(include/lbm.h), and the library's configuration defaults restated, so that
the oracle can be configured without loading the product library: the
benchmark's reference arm times the oracle alone and must map no product
code. `tests/test_oracle_abi.py` checks that the layout and the defaults
equal the product's field by field.
"""
from __future__ import annotations

import ctypes as C

SHAPE = {"sphere": 0, "spheroid": 1, "roundbox": 2, "ellipse": 3}
STORAGE = {"fp32": 0, "fp16": 1, "bf16": 2}


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
                ("body", Body), ("storage", C.c_int32), ("window", C.c_int32 * 3),
                ("win_anchor", C.c_int32 * 3), ("trt", C.c_int32), ("trt_lambda", C.c_float)]


def config_default(q: int, dims) -> Config:
    """lbm_config_default restated: tau 0.8 (OMEGA 1.25,
    common_d3_step.wgsl:151), SOLID_EQ, local rho_w, the swept-cell term,
    K_EPS 1.5, sponge width 4 in 2D (lbm_step.wgsl SPONGE_W) and 0 in 3D on
    every axis, an identity-oriented ellipse (2D) or sphere (3D), FP32."""
    cfg = Config()
    cfg.q = int(q)
    cfg.nx, cfg.ny = int(dims[0]), int(dims[1])
    cfg.nz = int(dims[2]) if len(dims) > 2 else 1
    cfg.tau = 0.8
    cfg.solid_eq = 1
    cfg.rho_w_local = 1
    cfg.swept_force = 1
    cfg.chi_eps = 1.5
    cfg.sponge_w = 4.0 if q == 9 else 0.0
    for j in range(3):
        cfg.sponge_axis[j] = 1
    cfg.body.qw = 1.0
    cfg.body.shape = SHAPE["ellipse"] if q == 9 else SHAPE["sphere"]
    cfg.storage = STORAGE["fp32"]
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


def config_from(q: int, dims, **kw) -> Config:
    """A Config with fields overridden by keyword, as the scenario builders
    give them (body as a dict, storage by name, arrays as sequences)."""
    cfg = config_default(q, dims)
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
