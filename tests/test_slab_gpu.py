"""The z-slab form of the dense step on one GPU: R slab sessions stand in for
R ranks (their halos move by device copies in the ring order the ranks use;
no kernel waits on another), against one whole-domain session from the same
f32 state:

* f and mac of every slab equal the whole domain's planes bit for bit, after
  every step (body, sponge, walls on y and z, D3Q19 and D3Q27, FP32 and FP16);
* the slabs' force shares sum to the whole domain's force (FP64, another
  order of additions), and their totals to its totals.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ring_step(slabs, bufs):
    import torch
    for s, (lo, hi, _, _) in zip(slabs, bufs):
        s.pack(lo.data_ptr(), hi.data_ptr())
    for s in slabs:
        s.sync()
    R = len(slabs)
    for k, s in enumerate(slabs):
        below, above = bufs[(k - 1) % R], bufs[(k + 1) % R]
        # the slab below's upward buffer into my ghost plane below, the slab
        # above's downward buffer into my ghost plane above
        s.unpack(below[1].data_ptr(), above[0].data_ptr())
    for s in slabs:
        s.step(1)
    torch.cuda.synchronize()


@pytest.mark.parametrize("q,storage,R,walls", [
    (19, "fp32", 2, (0, 1, 0)), (19, "fp32", 3, (0, 0, 1)), (27, "fp32", 2, (0, 1, 1)), (19, "fp16", 3, (0, 1, 0))])
def test_slabs_equal_the_whole_domain(lbm, oracle, q, storage, R, walls):
    import torch
    from getting_air_b200 import scenarios as sc
    from getting_air_b200 import slab
    s = sc.sphere(n=8, dims=(40, 24, 26), u0=0.05, re=40, q=q, force=(2e-6, 0.0, 0.0), storage=storage)
    kw = dict(s["kw"], wall=walls)
    cfg = lbm.config_from(q, s["dims"], **kw)
    nx, ny, nz = s["dims"]
    nxy = nx * ny
    f0 = oracle.init_eq(q, s["mac"], fp32=True).astype(np.float32)
    whole = lbm.Solver(cfg)
    whole.write_f(f0)
    parts = slab.split(nz, R)
    slabs = [lbm.Solver(cfg, slab=p) for p in parts]
    for sl, (z0, k) in zip(slabs, parts):
        sl.write_f(np.ascontiguousarray(f0[:, z0 * nxy:(z0 + k) * nxy]))
    nb = slabs[0].halo_bytes()
    assert nb == nxy * (5 if q == 19 else 9) * (4 if storage == "fp32" else 2)
    bufs = [[torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(4)] for _ in slabs]
    for step in range(6):
        _ring_step(slabs, bufs)
        whole.step(1)
        wf, wm = whole.read_f_raw(), whole.read_mac()
        for sl, (z0, k) in zip(slabs, parts):
            assert np.array_equal(sl.read_f_raw(), wf[:, z0 * nxy:(z0 + k) * nxy]), (step, z0)
            assert np.array_equal(sl.read_mac(), wm[z0 * nxy:(z0 + k) * nxy]), (step, z0)
    F = sum(np.asarray(sl.forces()) for sl in slabs)
    Fw = np.asarray(whole.forces())
    assert abs(Fw[0]) > 0
    assert np.allclose(F, Fw, rtol=1e-11, atol=1e-13 * np.abs(Fw).max())
    tw = whole.totals()
    ts = [sl.totals() for sl in slabs]
    for key in ("mass", "px", "py", "pz"):
        assert abs(sum(t[key] for t in ts) - tw[key]) <= 1e-12 * max(1.0, abs(tw[key])) * cfg.nx * cfg.ny * cfg.nz
    assert min(t["rho_min"] for t in ts) == tw["rho_min"] and max(t["rho_max"] for t in ts) == tw["rho_max"]
    for sl in slabs:
        sl.close()
    whole.close()


def test_slab_refusals(lbm):
    cfg = lbm.config_from(19, (16, 16, 16))
    with pytest.raises(lbm.LbmError, match="must lie"):
        lbm.Solver(cfg, slab=(10, 8))
    with pytest.raises(lbm.LbmError, match="3D"):
        lbm.Solver(lbm.config_from(9, (16, 16)), slab=(0, 1))
