"""Version-7 snapshots of a 2D AMR session (main-cylinder-amr.js
debugSnapshotSave / debugSnapshotLoad), in the reference's own validation
protocol (tools/validate-snapshot-roundtrip.js):

* round trip: step 2N from the seed; separately step N, save, load into a
  FRESH session, step N more -- the two end states are bit-identical (N
  spans refine rounds, so the restored allocator is exercised);
* stale control: loading a capture from a different step changes the end
  state, so the load is load-bearing;
* refusals: another grid size, a pre-7 capture, a level 1 allocated per
  block, a topology whose maps disagree.

The layout checks (root tile order, payload encoding) run on the CPU.
"""
import copy
import json

import numpy as np
import pytest


def rootCellIndex(W, H, rb, gx, gy):
    side = 2 * rb
    nbx = W // side
    slot = (gy // side) * nbx + gx // side
    return slot * side * side + (gy % side) * side + (gx % side)


def test_root_order_is_the_reference_tile_layout(lbm):
    from getting_air_b200 import snapshot as S
    W, H, rb = 64, 32, 4
    order = S.root_order(W, H, rb)
    for gy in range(H):
        for gx in range(W):
            assert order[rootCellIndex(W, H, rb, gx, gy)] == gy * W + gx
    with pytest.raises(S.SnapshotError):
        S.root_order(60, 32, 4)


def test_payload_round_trip(lbm):
    from getting_air_b200 import snapshot as S
    a = np.random.default_rng(0).standard_normal(37).astype(np.float32)
    assert np.array_equal(S._unb64(S._b64(a), 37), a)
    with pytest.raises(S.SnapshotError):
        S._unb64(S._b64(a), 36)


def session(lbm, iface=0):
    from getting_air_b200 import scenarios as sc
    s = sc.cylinder_amr(W=256, H=128, r=10.0, centre=(64.0, 64.0), u0=0.08, re=100.0)
    cfg = lbm.amr2d_config(256, 128, iface=iface, **s["kw"])
    a = lbm.Amr2D(cfg)
    a.write_root(s["f"], s["vel"])
    return a


def fingerprint(a):
    f0, v0 = a.read_root()
    f1, _ = a.read_pool()
    t = a.topology()
    return f0, f1, t["block_slot"], t["slot_to_block"], a.forces()


def same(x, y):
    return all(np.array_equal(p, q) for p, q in zip(x, y))


@pytest.mark.gpu
@pytest.mark.parametrize("iface", [0, 1], ids=["interp", "explode"])
def test_round_trip_mid_run_is_bit_identical(lbm, iface):
    from getting_air_b200 import snapshot as S
    N = 40  # refine rounds at macro-steps 0, 16, 32, 48, 64
    ref = session(lbm, iface)
    ref.step(2 * N)
    want = fingerprint(ref)
    ref.close()
    a = session(lbm, iface)
    a.step(N)
    snap = S.loads(S.dumps(S.save_amr2d(a, params={"R": 10.0, "U0": 0.08, "RE": 100.0})))
    a.close()
    assert snap["formatVersion"] == 7 and snap["step"] == N
    b = session(lbm, iface)
    b.step(3)  # a different state, to be overwritten
    S.load_amr2d(b, snap)
    assert b.macro_step == N
    b.step(N)
    assert same(fingerprint(b), want)
    # stale control: a capture from another step gives another end state
    c = session(lbm, iface)
    c.step(N - 8)
    stale = S.save_amr2d(c)
    c.close()
    d = session(lbm, iface)
    S.load_amr2d(d, stale)
    d.step(N)
    assert not same(fingerprint(d), want)
    b.close()
    d.close()


@pytest.mark.gpu
def test_incompatible_captures_are_refused(lbm):
    from getting_air_b200 import snapshot as S
    a = session(lbm)
    a.step(20)
    snap = S.save_amr2d(a)
    for mutate, words in [
        (lambda s: s.update(W=512), "session is"),
        (lambda s: s.update(formatVersion=6), "dense grid"),
        (lambda s: s["pools"][1].update(quadAlloc=False), "per block"),
        (lambda s: s["pools"][1].update(MAX_FINE_BLOCKS=8), "does not match"),
        (lambda s: s["root"].update(cellsPerSlot=64), "does not match"),
    ]:
        bad = copy.deepcopy(snap)
        mutate(bad)
        with pytest.raises(S.SnapshotError, match=words):
            S.load_amr2d(a, bad)
    bad = copy.deepcopy(snap)
    bs = bad["pools"][1]["blockSlot"]
    used = [i for i, v in enumerate(bs) if v >= 0]
    bs[used[0]] = bs[used[1]]  # two blocks claim one slot: the maps are no longer inverse
    with pytest.raises(lbm.LbmError, match="inverse"):
        S.load_amr2d(a, bad)
    a.close()
