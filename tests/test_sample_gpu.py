"""The headless views on the GPU against the oracle, over the device's own
field (so the check isolates the sampler, resample and slice kernels):

* dense: the unit volume is the L0 mac bit for bit, in f32 and in binary16
  (round to nearest even, as the rgba16float texture stores it);
* 3D AMR: a half-spacing volume over the domain, finest level wins, bit for
  bit with the level map, and an offset, non-aligned box;
* slices of every mode and turn, dense and AMR (vorticity across the
  coarse/fine seam included): equal to the oracle's pictures except where
  powf's last bit moves a channel by one step;
* a moving window pans the slice with the body.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def seed(dims, s, amp=0.03):
    n = int(np.prod(dims))
    rng = np.random.default_rng(s)
    mac = np.zeros((n, 4), np.float32)
    mac[:, 0] = 1 + 0.01 * rng.standard_normal(n)
    mac[:, 1:] = amp * rng.standard_normal((n, 3))
    return mac


def close_images(a, b, frac=0.01):
    d = np.abs(a.astype(int) - b.astype(int))
    assert d.max() <= 1, d.max()
    assert (d > 0).mean() <= frac


def test_dense_unit_volume_is_the_mac(lbm, oracle):
    dims = (40, 24, 20)
    s = lbm.Solver.create(19, dims, tau=0.7)
    s.init_macro(seed(dims, 1))
    s.step(3)
    mac = s.read_mac()
    vol, lvl = s.resample(level=True)
    m = mac.reshape(dims[2], dims[1], dims[0], 4)
    assert np.array_equal(vol[..., :3], m[..., 1:]) and np.array_equal(vol[..., 3], m[..., 0])
    assert not lvl.any()
    v16, _ = s.resample(fp16=True)
    assert v16.dtype == np.float16
    assert np.array_equal(v16.view(np.uint16), vol.astype(np.float16).view(np.uint16))
    # into a device tensor, no host copy
    import torch
    t = torch.empty((dims[2], dims[1], dims[0], 4), dtype=torch.float32, device="cuda")
    s.resample(out=t)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), vol)
    s.close()


def amr_case(lbm):
    dims = (32, 24, 24)
    c = lbm.amr3d_config(19, dims, refine="body", tau=0.62, has_body=1, use_bounceback=1,
                         body=dict(shape="sphere", centre=(12.3, 11.8, 12.1), a=4.0))
    a = lbm.Amr3D(c)
    mac = seed(dims, 4, amp=0.02)
    mac[:, 1] += 0.04
    a.init_macro(mac)
    a.step(5)
    return a, dims


def tree_of(a):
    _, macc = a.read_coarse()
    _, macp = a.read_pool()
    topo = a.topology()
    return dict(levels=1, macp=macp, block_slot=topo["block_slot"], rb=a.cfg.rb, fb=a.fb), macc


def test_amr_volume_matches_oracle(lbm, oracle):
    a, dims = amr_case(lbm)
    tree, macc = tree_of(a)
    for origin, shape, h in (((-0.25, -0.25, -0.25), tuple(2 * d for d in dims), (0.5, 0.5, 0.5)),
                             ((5.1, 3.7, 8.05), (21, 17, 13), (0.37, 0.5, 0.61))):
        vol, lvl = a.resample(origin=origin, shape=shape, h=h, level=True)
        ov, ol = oracle.tree_resample(macc, dims, origin, shape, h, **tree)
        assert np.array_equal(vol.reshape(-1, 4), ov)
        assert np.array_equal(lvl.reshape(-1), ol)
        assert 0 < ol.mean() < 1  # both levels answer somewhere
        v16, _ = a.resample(origin=origin, shape=shape, h=h, fp16=True)
        assert np.array_equal(v16.reshape(-1, 4).view(np.uint16), ov.astype(np.float16).view(np.uint16))
    a.close()


@pytest.mark.parametrize("mode", ["speed", "vorticity", "normal"])
def test_amr_slices_match_oracle(lbm, oracle, mode):
    a, dims = amr_case(lbm)
    tree, macc = tree_of(a)
    m = lbm.SLICE_MODES[mode]
    for axis in (0, 1, 2):
        for rot in (0, 1, 2, 3):
            kw = dict(axis=axis, slice=12, mode=mode, rot=rot, u_scale=0.05, v_scale=0.01)
            spec = lbm.slice_spec(dims, **kw)
            # two pixels per L0 cell: the pool's resolution shows
            w, h = 2 * spec.width, 2 * spec.height
            img = a.render_slice(width=w, height=h, **kw)
            ref = oracle.tree_slice(macc, dims, axis, 12, m, rot, w, h, 0.05, 0.01, **tree)
            close_images(img, ref)
    a.close()


def test_dense_slice_and_window_pan(lbm, oracle):
    dims = (48, 24, 24)
    kw = dict(tau=0.6, has_body=1, use_bounceback=1, sponge_w=4.0, sponge_u=(0.0, 0.0, 0.0), window="x",
              win_anchor=(20, 11, 12), body=dict(shape="sphere", centre=(31.75, 11.5, 12.0), a=4.0))
    s = lbm.Solver.create(19, dims, **kw)
    s.init_macro(seed(dims, 6, amp=0.01))
    s.step(2)
    mac = s.read_mac()
    for mode in (0, 1, 2):
        img = s.render_slice(axis=2, slice=12, mode=mode, u_scale=0.02, v_scale=0.01)
        off = (31.75 - 20.0, 0.0, 0.0)
        ref = oracle.tree_slice(mac, dims, 2, 12, mode, 0, dims[0], dims[1], 0.02, 0.01, off=off)
        close_images(img, ref)
        unpanned = oracle.tree_slice(mac, dims, 2, 12, mode, 0, dims[0], dims[1], 0.02, 0.01)
        # the pan shifts the picture by the body's travel (12 whole cells at
        # one pixel per cell: 11.75 rounds to the cell 12 ahead)
        assert np.array_equal(ref, np.roll(unpanned, -12, axis=1))
    s.close()
