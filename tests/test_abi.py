"""The C-ABI library loads and exports exactly what include/lbm.h declares,
and its host-side argument checks behave like the reference's throws. No
compute call is made here (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    syms = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        syms |= set(re.findall(r"\b(lbm\w*)\s*\(", text))
    return sorted(syms)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "lbm_create" in syms and "lbm_step" in syms and len(syms) >= 20


@pytest.mark.parametrize("sym", declared_symbols())
def test_library_exports_symbol(lbm, sym):
    assert hasattr(lbm.lib, sym), sym


def test_abi_version(lbm):
    assert lbm.lib.lbm_abi_version() == 2
    assert b"sm_100a" in lbm.lib.lbm_version()


def test_config_struct_size_matches_header(lbm):
    # lbm_config = 4 ints + tau + 3 floats + 3 ints + 2 floats + 5 ints + 2 floats
    # + 3 ints + 3 floats + lbm_body(19*4) + storage + window[3] + win_anchor[3] + trt + trt_lambda
    assert C.sizeof(lbm.Body) == 19 * 4
    assert C.sizeof(lbm.Config) == (4 + 1 + 3 + 3 + 2 + 5 + 2 + 3 + 3) * 4 + 19 * 4 + 9 * 4


@pytest.mark.parametrize("bad, msg", [
    (dict(q=7), "q must be"),
    (dict(q=9, nz=4), "nz == 1"),
    (dict(tau=0.5), "tau"),
    (dict(tau=float("nan")), "tau"),
    (dict(nx=2), "at least 3"),
    (dict(storage=5), "storage"),
    (dict(ny=70000), "65535"),
])
def test_invalid_config_is_rejected_before_any_device_work(lbm, bad, msg):
    q = bad.get("q", 19)
    dims = (16, 16, 1 if q == 9 and "nz" not in bad else 16)
    cfg = lbm.default_config(19 if q not in (9, 19, 27) else q, dims)
    for k, v in bad.items():
        setattr(cfg, k, v)
    with pytest.raises(lbm.LbmError) as ei:
        lbm.Solver(cfg)
    assert ei.value.code == lbm.EINVAL and msg in str(ei.value)


def test_body_shape_checked(lbm):
    cfg = lbm.default_config(9, (16, 16, 1))
    cfg.has_body = 1
    cfg.body = lbm.make_body("sphere", (8, 8, 0), a=2)
    with pytest.raises(lbm.LbmError, match="ellipse"):
        lbm.Solver(cfg)


def test_default_config_matches_reference_overrides(lbm):
    c = lbm.default_config(19, (8, 8, 8))
    assert abs(1 / c.tau - 1.25) < 1e-6           # OMEGA 1.25
    assert c.chi_eps == 1.5 and c.solid_eq == 1 and c.rho_w_local == 1 and c.swept_force == 1
    assert c.sponge_w == 0.0
    assert lbm.default_config(9, (8, 8, 1)).sponge_w == 4.0   # lbm_step.wgsl SPONGE_W


def test_batch_rejects_mixed_lattices_before_device_work(lbm):
    with pytest.raises(lbm.LbmError, match="share q"):
        lbm.Batch([lbm.config_from(19, (8, 8, 8)), lbm.config_from(27, (8, 8, 8))])
    with pytest.raises(lbm.LbmError, match="domain 1"):
        lbm.Batch([lbm.config_from(19, (8, 8, 8)), lbm.config_from(19, (8, 8, 8), tau=0.4)])
