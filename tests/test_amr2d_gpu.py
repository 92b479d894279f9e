"""GPU tests of the 2D AMR macro-step against the oracle.

* topology: every refine round's result (block->slot map, slot->block map,
  free list, free count, active list, want flags) is bit-identical to the
  oracle applying the same round to the device's own pre-round topology and
  root velocity; the criterion array is bit-identical too;
* fields and force: device vs FP64 oracle over whole macro-steps (refine
  rounds included) within U_TOL / F_TOL.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U_TOL = 1e-4
F_TOL = 1e-3


def make(lbm, W=256, H=128, r=10.0, bounceback=False, iface=0, **kw):
    from getting_air_b200 import scenarios as sc
    s = sc.cylinder_amr(W=W, H=H, r=r, centre=(64.0, 64.0), u0=0.08, re=100.0, bounceback=bounceback, **kw)
    cfg = lbm.amr2d_config(W, H, iface=iface, **s["kw"])
    return s, cfg


def topo_equal(t, o):
    assert np.array_equal(t["block_slot"], o["block_slot"])
    assert np.array_equal(t["slot_to_block"], o["slot_to_block"])
    assert t["free_count"] == o["free_count"]
    n = t["free_count"]
    # entries at or above free_count are stale in both (pushed and popped)
    assert np.array_equal(t["free_list"][:n], o["free_list"][:n])
    assert np.array_equal(t["active"], o["active"])
    assert np.array_equal(t["want"], o["want"])


@pytest.mark.parametrize("bounceback", [False, True])
def test_refine_rounds_are_bit_exact(lbm, oracle, bounceback):
    s, cfg = make(lbm, bounceback=bounceback)
    a = lbm.Amr2D(cfg)
    a.write_root(s["f"], s["vel"])
    o = oracle.Amr2D(cfg, fp32=True)
    # round 1 from the empty topology and the seed velocity
    a.step(1)
    o.refine_from_vel(s["vel"])
    t1, r1 = a.topology(), o.read()
    assert np.array_equal(t1["criterion"], r1["criterion"])
    topo_equal(t1, r1)
    assert len(t1["active"]) > 0
    # rounds 2 and 3, each from the device's own state just before the round
    for _ in range(2):
        a.step(15)
        before = a.topology()
        _, vel = a.read_root()
        a.step(1)
        after = a.topology()
        o.set_topology(before["block_slot"], before["slot_to_block"], before["free_list"], before["free_count"])
        o.refine_from_vel(vel)
        ro = o.read()
        assert np.array_equal(after["criterion"], ro["criterion"])
        topo_equal(after, ro)
    a.close()
    o.close()


@pytest.mark.parametrize("iface", [0, 1], ids=["interp", "explode"])
@pytest.mark.parametrize("bounceback", [False, True])
def test_macro_steps_match_fp64_oracle(lbm, oracle, bounceback, iface):
    s, cfg = make(lbm, bounceback=bounceback, iface=iface)
    a = lbm.Amr2D(cfg)
    a.write_root(s["f"], s["vel"])
    o = oracle.Amr2D(cfg)
    o.write_root(s["f"].astype(np.float64), s["vel"].astype(np.float64))
    n = 20  # refine rounds at macro-steps 0 and 16
    a.step(n)
    o.step(n)
    ro = o.read()
    t = a.topology()
    topo_equal(t, ro)
    f0, vel0 = a.read_root()
    f1, vel1 = a.read_pool()
    rel = lambda x, y: np.linalg.norm(x - y) / np.linalg.norm(y)
    assert rel(vel0, ro["vel0"]) <= U_TOL
    assert rel(f0, ro["f0"]) <= 1e-6
    act = t["active"]
    fb2 = cfg.rb * 2 + 4
    idx = np.concatenate([np.arange(s_ * fb2 * fb2, (s_ + 1) * fb2 * fb2) for s_ in act])
    assert rel(vel1[idx], ro["vel1"][idx]) <= U_TOL
    F = a.forces()
    Fo = ro["force"]
    scale = max(abs(Fo[0]), abs(Fo[1]), 1e-3)
    assert abs(F[0] - Fo[0]) <= F_TOL * scale and abs(F[1] - Fo[1]) <= F_TOL * scale
    assert F[3] == 0 and Fo[3] == 0
    assert abs(Fo[0]) > 1e-3  # the cylinder feels a drag
    a.close()
    o.close()


def test_body_is_fully_refined_and_pool_is_conservative(lbm, oracle):
    s, cfg = make(lbm)
    a = lbm.Amr2D(cfg)
    a.write_root(s["f"], s["vel"])
    a.step(1)
    t = a.topology()
    # every root block within the margin of the body is refined
    nbx = cfg.nx // cfg.rb
    for b in range(len(t["block_slot"])):
        bx, by = b % nbx, b // nbx
        cx, cy = bx * cfg.rb + cfg.rb / 2 - 0.5, by * cfg.rb + cfg.rb / 2 - 0.5
        if np.hypot(cx - 64, cy - 64) < cfg.body.a:
            assert t["block_slot"][b] >= 0
    # active count = 4 x refined root blocks, slots granted from the top of the free list
    assert len(t["active"]) % 4 == 0
    assert a.cell_updates() == cfg.nx * cfg.ny + len(t["active"]) * (2 * cfg.rb) ** 2 * 2
    a.close()


def test_pool_exhaustion_stays_coarse(lbm, oracle):
    s, cfg = make(lbm, max_slots=8)   # room for two quads only
    a = lbm.Amr2D(cfg)
    a.write_root(s["f"], s["vel"])
    a.step(1)
    t = a.topology()
    assert len(t["active"]) == 8 and t["free_count"] == 0
    o = oracle.Amr2D(cfg, fp32=True)
    o.refine_from_vel(s["vel"])
    topo_equal(t, o.read())
    a.step(5)
    f0, _ = a.read_root()
    assert np.isfinite(f0).all()
    a.close()


def test_explode_and_interp_interfaces_agree_on_drag(lbm):
    """The two couplings are different discretisations of one flow: after the
    start-up the drag of the refined cylinder agrees to a few per cent."""
    drags = []
    for iface in (0, 1):
        s, cfg = make(lbm, W=512, H=256, r=16.0, iface=iface)
        a = lbm.Amr2D(cfg)
        a.write_root(s["f"], s["vel"])
        a.step(3000)
        drags.append(a.forces()[0])
        f0, _ = a.read_root()
        assert np.isfinite(f0).all()
        a.close()
    print("drag interp %.5f explode %.5f" % tuple(drags))
    assert abs(drags[1] - drags[0]) <= 0.05 * abs(drags[0])


def test_manual_refine_rounds_equal_automatic_ones(lbm):
    """refineRound called by hand at the same macro-steps as the automatic
    schedule (every 16, from step 0) gives the same run, bit for bit."""
    s, cfg = make(lbm)
    runs = []
    for manual in (False, True):
        a = lbm.Amr2D(cfg)
        a.write_root(s["f"], s["vel"])
        if manual:
            a.set_auto_refine(False)
            for _ in range(3):
                a.refine_round()
                a.step(16)
        else:
            a.step(48)
        f, vel = a.read_root()
        runs.append((f, a.topology(), a.forces()))
        a.close()
    (f0, t0, F0), (f1, t1, F1) = runs
    assert np.array_equal(f0, f1)
    assert np.array_equal(t0["block_slot"], t1["block_slot"]) and np.array_equal(t0["active"], t1["active"])
    assert np.array_equal(F0, F1)


@pytest.mark.parametrize("bounceback", [False, True])
def test_fused_macro_step_equals_six_launches(lbm, oracle, bounceback):
    """The interp macro-step as one cooperative launch (the default) gives the
    six-launch form's bits: root and pool populations and velocity, force,
    topology, over 40 macro-steps and three refine rounds."""
    s, cfg = make(lbm, bounceback=bounceback)
    out = []
    for fused in (True, False):
        a = lbm.Amr2D(cfg)
        a.set_fused(fused)
        assert a.fused == fused
        a.write_root(s["f"], s["vel"])
        a.step(40)
        a.sync()
        f0, v0 = a.read_root()
        f1, v1 = a.read_pool()
        out.append((f0, v0, f1, v1, a.forces(), a.topology()))
        a.close()
    (f0a, v0a, f1a, v1a, Fa, ta), (f0b, v0b, f1b, v1b, Fb, tb) = out
    assert np.array_equal(f0a, f0b) and np.array_equal(v0a, v0b)
    fb2 = (cfg.rb * 2 + 4) ** 2
    idx = np.concatenate([np.arange(k * fb2, (k + 1) * fb2) for k in ta["active"]])
    assert np.array_equal(f1a.reshape(9, -1)[:, idx], f1b.reshape(9, -1)[:, idx])
    assert np.array_equal(v1a[idx], v1b[idx])
    assert np.array_equal(Fa, Fb)
    assert np.array_equal(ta["block_slot"], tb["block_slot"]) and np.array_equal(ta["active"], tb["active"])
