"""The moving window on the GPU (common_d3_window.wgsl, d3-window.mjs).

* translation invariance along the window axis, bit for bit: the body and the
  field shifted by k cells (the shifted body straddling the periodic seam)
  give the shifted populations, because the sponge band follows the body;
  without the window they do not;
* parity with the FP64 oracle with the body across the seam (the wrapped
  SDF, link velocity and torque arm, the force region read modulo the grid);
* a free body towed through the seam: position wrapped into the buffer,
  displacement unwrapped, trajectory and fields against the oracle;
* the 3D AMR manager and pool sponge under the window, against the oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def seed(dims, s, amp=0.01):
    n = int(np.prod(dims))
    rng = np.random.default_rng(s)
    mac = np.zeros((n, 4))
    mac[:, 0] = 1 + 1e-3 * rng.standard_normal(n)
    mac[:, 1:] = amp * rng.standard_normal((n, 3))
    return mac


DIMS = (64, 24, 24)


def wkw(cx, window="x", **kw):
    base = dict(tau=0.6, has_body=1, use_bounceback=1, sponge_w=5.0, sponge_u=(0.0, 0.0, 0.0),
                body=dict(shape="sphere", centre=(cx, 11.5, 12.0), a=4.5, v=(0.25, 0.0, 0.0)),
                window=window, win_anchor=(20, 11, 12))
    base.update(kw)
    return base


def run_dense(lbm, oracle, kw, f0, nsteps):
    s = lbm.Solver.create(19, DIMS, **kw)
    s.write_f(f0.astype(np.float32))
    s.step(nsteps)
    f, mac, F = s.read_f(), s.read_mac(), s.forces()
    s.close()
    return f, mac, F


@pytest.mark.parametrize("shape", ["sphere", "roundbox"])
def test_window_translation_invariance_bit_for_bit(lbm, oracle, shape):
    k = 41  # 20.25 + 41 = 61.25: the body straddles x = 64 -> 0
    mac = seed(DIMS, 7).reshape(DIMS[2], DIMS[1], DIMS[0], 4)
    out = {}
    for win in ("x", "0"):
        for shift in (0, k):
            kw = wkw(20.25 + shift, window=win)
            if shape == "roundbox":
                kw.update(use_bounceback=0, chi_eps=1.5,
                          body=dict(shape="roundbox", centre=(20.25 + shift, 11.5, 12.0), a=5.0, b=3.0, c=2.5,
                                    r=0.5, quat=(0.9238795, 0.0, 0.0, 0.3826834), v=(0.25, 0.0, 0.0),
                                    w=(0.0, 0.0, 0.0078125)))
            f0 = oracle.init_eq(19, np.roll(mac, shift, axis=2).reshape(-1, 4), fp32=True)
            f, _, F = run_dense(lbm, oracle, kw, f0, 6)
            out[win, shift] = (f.reshape(19, DIMS[2], DIMS[1], DIMS[0]), F)
    fa, Fa = out["x", 0]
    fb, Fb = out["x", k]
    assert np.array_equal(np.roll(fa, k, axis=3), fb)
    assert np.allclose(Fa, Fb, rtol=1e-9, atol=1e-12 * np.abs(Fa).max())
    assert np.abs(Fa[:3]).max() > 1e-4
    # the window starts as the unwindowed run (offset 0 at the anchor) ...
    assert np.array_equal(out["0", 0][0], fa)
    # ... and without it the sponge stays put, so the shifted run differs
    assert not np.array_equal(np.roll(out["0", 0][0], k, axis=3), out["0", k][0])


def test_window_across_the_seam_matches_oracle(lbm, oracle):
    kw = wkw(61.25)
    mac = seed(DIMS, 3)
    f0 = oracle.init_eq(19, mac, fp32=True)
    g_f, g_mac, g_F = run_dense(lbm, oracle, kw, f0, 10)
    s = lbm.Solver.create(19, DIMS, **kw)
    o_f, o_mac, o_F = oracle.run(s.cfg, f0, 10)
    s.close()
    assert rel_l2(g_mac[:, 1:4].astype(np.float64), o_mac[:, 1:4]) <= 1e-5
    assert rel_l2(g_mac[:, 0].astype(np.float64), o_mac[:, 0]) <= 1e-6
    scale = max(np.abs(o_F[-1, :6]).max(), 1e-3)
    assert np.abs(g_F - o_F[-1, :6]).max() <= 1e-4 * scale
    assert abs(o_F[-1, 0]) > 1e-3


def test_free_body_towed_through_the_seam(lbm, oracle):
    x0 = 55.25
    kw = wkw(x0)
    body = lbm.make_body(**kw.pop("body"))
    opts = lbm.body_opts(no_fluid_force=1, v_max=float("inf"), o_max=float("inf"))
    mac = seed(DIMS, 5, amp=0.005)
    f0 = oracle.init_eq(19, mac, fp32=True).astype(np.float32)
    s = lbm.Solver.create(19, DIMS, body=body, **kw)
    s.write_f(f0)
    st = lbm.body_state(body, 1.0)
    s.set_free_body(st, opts)
    nsteps = 48  # 12 cells at 0.25 per step: the centre crosses x = 64
    xs = []
    for _ in range(nsteps):
        s.step(1)
        xs.append(s.body_state().as_dict()["x"].copy())
    d = s.body_state().as_dict()
    g_mac, g_F = s.read_mac().astype(np.float64), s.forces()
    ost = oracle.body_make(body, 1.0)
    _, o_mac, o_F, o_traj = oracle.run_free(s.cfg, f0.astype(np.float64), nsteps, ost, opts)
    s.close()
    xs = np.array(xs)
    assert np.all((xs[:, 0] >= 0) & (xs[:, 0] < DIMS[0]))
    assert xs[-1, 0] == pytest.approx((x0 + 0.25 * nsteps) % DIMS[0], abs=1e-9)
    assert d["d"][0] == pytest.approx(0.25 * nsteps, abs=1e-9)
    assert np.abs(xs - o_traj[:, 0:3]).max() <= 1e-9
    assert rel_l2(g_mac[:, 1:4], o_mac[:, 1:4]) <= 2e-5
    fs = max(np.abs(o_F[-1, :6]).max(), 1e-3)
    assert np.abs(g_F - o_F[-1, :6]).max() <= 1e-3 * fs


def test_amr3d_window_towed_body_matches_oracle(lbm, oracle):
    """A sphere towed across the seam of a windowed 3D hierarchy: every
    decision of the manager (wrapped SDF) and the pool sponge in window
    coordinates, against the oracle."""
    dims = (40, 24, 24)
    body = dict(shape="sphere", centre=(33.25, 11.75, 12.25), a=3.0, v=(0.25, 0.0, 0.0))
    c = lbm.amr3d_config(19, dims, refine="body", margin=2.0, dynamic=1, manage_every=4, slot_headroom=2.0,
                         tau=0.62, has_body=1, use_bounceback=1, sponge_w=4.0, sponge_u=(0.03, 0.0, 0.0),
                         body=body, window="x")
    n = int(np.prod(dims))
    mac = np.zeros((n, 4), np.float32)
    mac[:, 0] = 1.0
    mac[:, 1] = 0.03
    a = lbm.Amr3D(c)
    o = oracle.Amr3D(c, capacity=a.slots)
    a.init_macro(mac)
    o.seed(mac.astype(np.float64))
    cx = body["centre"][0]
    for k in range(8):
        a.step(4)
        o.step(4)
        cx = (cx + 1.0) % dims[0]
        nb = lbm.make_body("sphere", (cx, 11.75, 12.25), a=3.0, v=(0.25, 0.0, 0.0))
        a.set_body(nb)
        o.set_body(nb)
        ta, to = a.topology(), o.topology()
        assert np.array_equal(ta["block_slot"], to[0]), k
        assert np.array_equal(ta["slot_to_block"], to[1]), k
    # the refined set followed the body across the seam
    bs = ta["block_slot"].reshape(dims[2] // 4, dims[1] // 4, dims[0] // 4)
    assert (bs[:, :, 0] >= 0).any() and (bs[:, :, -1] >= 0).any()
    assert a.pool_stats() == o.pool_stats()
    gfc, gmac = a.read_coarse()
    ofc, omac, ofp, _ = o.read()
    gfp, _ = a.read_pool()
    assert rel_l2(gfc.astype(np.float64), ofc) <= 5e-6
    used = np.repeat(to[1] >= 0, a.fb ** 3)
    assert rel_l2(gfp[:, used].astype(np.float64), ofp[:, used]) <= 5e-6
    a.close()
