"""The oracle's mirror of lbm_config (oracle/abi.py), which lets the
benchmark's reference arm configure the oracle without loading the product
library, against the product's own structure and lbm_config_default."""
import ctypes as C

import numpy as np


def _layout(struct):
    return [(name, getattr(struct, name).offset, getattr(struct, name).size) for name, _ in struct._fields_]


def test_config_layout_matches_the_product(lbm):
    from oracle import abi
    assert C.sizeof(abi.Config) == C.sizeof(lbm.Config)
    assert C.sizeof(abi.Body) == C.sizeof(lbm.Body)
    assert _layout(abi.Config) == _layout(lbm.Config)
    assert _layout(abi.Body) == _layout(lbm.Body)


def test_config_defaults_match_the_product(lbm):
    from oracle import abi
    for q, dims in ((9, (64, 32)), (19, (32, 24, 16)), (27, (16, 16, 16))):
        mine = bytes(abi.config_default(q, dims))
        theirs = bytes(lbm.default_config(q, dims))
        assert mine == theirs, q


def test_config_from_matches_the_product(lbm):
    from oracle import abi
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=32, dims=(256, 128, 128), u0=0.05, tau=0.56, q=19, bounceback=True,
                  force=(1e-6, 0.0, 0.0), storage="fp32")
    a = bytes(abi.config_from(19, s["dims"], **s["kw"]))
    b = bytes(lbm.config_from(19, s["dims"], **s["kw"]))
    assert a == b
    assert np.frombuffer(a, np.uint8).any()
