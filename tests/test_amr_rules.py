"""The AMR host rules against the reference's own known answers
(tools/test-amr2d.js) and properties; pure functions, no GPU."""
import numpy as np
import pytest


def test_dc_factors_known_answers(lbm):
    # tools/test-amr2d.js:1330: post-collision factor at tau_c = 0.8 (tau_f = 1.1)
    assert abs(lbm.dc_rescale_c2f(0.8, 1.1) - (-0.25)) < 1e-12
    for tc in [0.51, 0.55, 0.6, 0.7, 0.8, 0.9, 1.2, 1.7, 2.5]:   # TAU_CASES, :1297
        tf = 2 * tc - 0.5
        assert abs(lbm.dc_rescale_c2f(tc, tf) * lbm.dc_rescale_f2c(tc, tf) - 1) <= 2 * np.finfo(float).eps


def test_tau_chain(lbm):
    assert lbm.tau_at_level(0.596, 0) == 0.596
    assert abs(lbm.tau_at_level(0.596, 1) - 0.692) < 1e-15
    assert abs(lbm.tau_at_level(0.8, 2) - (2 * (2 * 0.8 - 0.5) - 0.5)) < 1e-15
    # level m is exactly singular at tau0 = 0.5 + 2^-(m+1)
    assert lbm.tau_chain_singularity(0.75, 2) == 1
    assert lbm.tau_chain_singularity(1.0, 2) == 0
    assert lbm.tau_chain_singularity(0.596, 2) is None


def test_amr_singular_tau_is_refused_before_device_work(lbm):
    cfg = lbm.amr2d_config(64, 32, tau=0.75, body=dict(shape="ellipse", centre=(16, 16, 0), a=4, b=4))
    with pytest.raises(lbm.LbmError, match="0/0"):
        lbm.Amr2D(cfg)
    cfg = lbm.amr2d_config(60, 32, tau=0.6, body=dict(shape="ellipse", centre=(16, 16, 0), a=4, b=4))
    with pytest.raises(lbm.LbmError, match="multiples of 2"):
        lbm.Amr2D(cfg)
    cfg = lbm.amr2d_config(64, 32, tau=0.6, max_slots=6, body=dict(shape="ellipse", centre=(16, 16, 0), a=4, b=4))
    with pytest.raises(lbm.LbmError, match="multiple of 4"):
        lbm.Amr2D(cfg)


def test_grant_known_answers(lbm):
    # tools/test-amr2d.js:1462-1468 "grant pops down from the top of the stack"
    r = lbm.grant_assignment([5, 2, 9], 4)
    assert [g[0] for g in r["granted"]] == [2, 5, 9]
    assert [g[1] for g in r["granted"]] == [3, 2, 1]
    assert r["refused"] == [] and r["free_count"] == 1
    # :1469-1475 "a starved pool starves the HIGHEST ids"
    r = lbm.grant_assignment([8, 1, 5, 3, 9], 2)
    assert [g[0] for g in r["granted"]] == [1, 3] and r["refused"] == [5, 8, 9] and r["free_count"] == 0
    # :1476-1481 empty pool
    r = lbm.grant_assignment([4, 1], 0)
    assert r["granted"] == [] and r["refused"] == [1, 4] and r["free_count"] == 0
    # :1451-1461 invariant under arrival order
    ref = lbm.grant_assignment([41, 7, 19, 3, 28], 6)
    for perm in ([3, 7, 19, 28, 41], [41, 28, 19, 7, 3], [19, 3, 41, 28, 7]):
        assert lbm.grant_assignment(perm, 6) == ref


def test_release_known_answers(lbm):
    # tools/test-amr2d.js:1488-1493
    r = lbm.release_assignment([12, 3, 7], 5)
    assert [w[0] for w in r["writes"]] == [3, 7, 12]
    assert [w[1] for w in r["writes"]] == [5, 6, 7]
    assert r["free_count"] == 8
    g = lbm.grant_assignment([6, 2, 11], 5)
    back = lbm.release_assignment([x[0] for x in g["granted"]], g["free_count"])
    assert back["free_count"] == 5
    assert sorted(x[1] for x in g["granted"]) == sorted(x[1] for x in back["writes"])


def test_active_slot_list(lbm):
    assert lbm.active_slot_list([-1, 4, -1, 0, 9, -1]) == [1, 3, 4]
    assert lbm.active_slot_list([-1, -1]) == []


def brute_cascade(wants, levels, nbx1, nby1):
    """Independent restatement of the closure's fixed point: quad-complete at
    m >= 2, and every 9-neighbour's parent present at m-1."""
    sets = [None] + [set(map(tuple, np.argwhere(np.asarray(wants[m]).reshape(nby1 << (m - 1), nbx1 << (m - 1)))))
                     for m in range(1, levels)]
    changed = True
    while changed:
        changed = False
        for m in range(levels - 1, 1, -1):
            W, H = nbx1 << (m - 1), nby1 << (m - 1)
            for (by, bx) in list(sets[m]):
                for q in range(4):
                    c = ((by >> 1) * 2 + (q >> 1), (bx >> 1) * 2 + (q & 1))
                    if c not in sets[m]:
                        sets[m].add(c); changed = True
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        ny, nx = (by + dy) % H, (bx + dx) % W
                        p = (ny >> 1, nx >> 1)
                        if m - 1 >= 2:
                            for q in range(4):
                                c = ((p[0] >> 1) * 2 + (q >> 1), (p[1] >> 1) * 2 + (q & 1))
                                if c not in sets[m - 1]:
                                    sets[m - 1].add(c); changed = True
                        elif p not in sets[m - 1]:
                            sets[m - 1].add(p); changed = True
    return sets


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_cascade21_closure(lbm, seed):
    rng = np.random.default_rng(seed)
    levels, nbx1, nby1 = 4, 6, 4
    wants = [None] + [(rng.random((nby1 << (m - 1)) * (nbx1 << (m - 1))) < 0.05).astype(np.uint8)
                      for m in range(1, levels)]
    closed, added = lbm.cascade21(wants, levels, nbx1, nby1)
    ref = brute_cascade(wants, levels, nbx1, nby1)
    for m in range(1, levels):
        got = set(map(tuple, np.argwhere(closed[m].reshape(nby1 << (m - 1), nbx1 << (m - 1)))))
        assert got == ref[m], m
    # idempotent: closing a closed set adds nothing
    again, added2 = lbm.cascade21(closed, levels, nbx1, nby1)
    assert added2 == 0 and all((again[m] == closed[m]).all() for m in range(1, levels))
    # minimal: everything added was forced (present in the brute-force closure)
    assert added == sum(len(ref[m]) for m in range(1, levels)) - sum(int(w.sum()) for w in wants[1:])
