"""GPU tests of the batched form: every domain of a batch must evolve exactly
as the same domain in its own dense session (same per-cell code), whatever
the tile shape, with or without the captured graph, and the autotuner must
leave the state untouched."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mixed_3d(lbm, q=19, storage="fp32"):
    from getting_air_b200 import scenarios as sc
    s1 = sc.sphere(n=6, dims=(36, 24, 20), u0=0.05, re=30, q=q, force=(1e-6, 0, 0), storage=storage)
    s2 = sc.sphere(n=8, dims=(40, 28, 30), u0=0.04, re=40, q=q, bounceback=False, storage=storage)
    kw3 = dict(tau=0.7, wall=(0, 1, 1), force=(1e-5, 0, 0), storage=storage)
    doms = [(s1["dims"], s1["kw"], s1["mac"]), (s2["dims"], s2["kw"], s2["mac"]),
            ((17, 13, 11), kw3, sc.uniform_macro(17 * 13 * 11, (0.02, 0, 0)))]
    return doms


def run_pair(lbm, oracle, q, doms, nsteps, tiling=None):
    cfgs = [lbm.config_from(q, d, **kw) for d, kw, _ in doms]
    b = lbm.Batch(cfgs)
    if tiling:
        b.set_tiling(*tiling)
    f0s = []
    for k, (d, kw, mac) in enumerate(doms):
        f0 = oracle.init_eq(q, mac, fp32=True).astype(np.float32)
        f0s.append(f0)
        b.write_f(k, f0)
    b.step(nsteps)
    got = [(b.read_f(k), b.read_mac(k)) for k in range(len(doms))]
    gf = b.forces()
    b.close()
    want, wf = [], []
    for k, (d, kw, mac) in enumerate(doms):
        s = lbm.Solver(cfgs[k])
        s.write_f(f0s[k])
        s.step(nsteps)
        want.append((s.read_f(), s.read_mac()))
        wf.append(s.forces())
        s.close()
    return got, want, gf, np.array(wf)


@pytest.mark.parametrize("tiling", [None, (128, 1, 2), (256, 8, 16)])
def test_batch_equals_dense_sessions_3d(lbm, oracle, tiling):
    got, want, gf, wf = run_pair(lbm, oracle, 19, mixed_3d(lbm), 7, tiling)
    for (f, m), (wf_, wm) in zip(got, want):
        assert np.array_equal(f, wf_)
        assert np.array_equal(m, wm)
    # same per-cell f32 contributions, FP64 sums over different partitions
    assert np.allclose(gf, wf, rtol=1e-10, atol=1e-12 * np.abs(wf).max())
    assert abs(gf[0, 0]) > 0 and abs(gf[1, 0]) > 0


def test_batch_q27_and_graph_path(lbm, oracle):
    # 37 steps: two captured 16-step graphs plus 5 single launches.
    got, want, gf, wf = run_pair(lbm, oracle, 27, mixed_3d(lbm, q=27), 37)
    for (f, m), (wf_, wm) in zip(got, want):
        assert np.array_equal(f, wf_) and np.array_equal(m, wm)


def test_batch_d2q9_tgv_and_channel(lbm, oracle):
    from getting_air_b200 import scenarios as sc
    w = lbm.lattice_tables(9)["w"]
    doms = sc.batched_domains(count=6, seed=7, nmin=16, nmax=96)
    cfgs = [lbm.config_from(9, d["dims"], **d["kw"]) for d in doms]
    b = lbm.Batch(cfgs)
    f0 = [sc.seed_domain(d, w) for d in doms]
    for k in range(len(doms)):
        b.write_f(k, f0[k])
    b.step(20)
    for k, d in enumerate(doms):
        s = lbm.Solver(cfgs[k])
        s.write_f(f0[k])
        s.step(20)
        assert np.array_equal(b.read_f(k), s.read_f())
        s.close()
    b.close()


def test_autotune_keeps_state(lbm, oracle):
    doms = mixed_3d(lbm)
    cfgs = [lbm.config_from(19, d, **kw) for d, kw, _ in doms]
    b = lbm.Batch(cfgs)
    for k, (d, kw, mac) in enumerate(doms):
        b.init_macro(k, mac)
    before = [b.read_f(k) for k in range(3)]
    ms = b.autotune(2)
    assert ms > 0
    assert b.tiling()[0] in (128, 256)
    for k in range(3):
        assert np.array_equal(b.read_f(k), before[k])
    b.close()


def test_batch_packed_storage_matches_dense(lbm, oracle):
    got, want, _, _ = run_pair(lbm, oracle, 19, mixed_3d(lbm, storage="bf16"), 5)
    for (f, m), (wf_, wm) in zip(got, want):
        assert np.array_equal(f, wf_)



@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16"])
def test_batch_d2q9_general_and_lean_tiles_equal_dense(lbm, oracle, storage):
    """A D2Q9 batch whose tiles split between the two kernels of a step: a
    cylinder (bounce-back body, sponge, force region: the general kernel)
    beside a Couette channel with moving walls, a forced channel and a
    periodic domain in uniform flow (the lean kernel). Each domain's
    populations and mac equal the same domain stepped alone as a dense
    session, to the bit, in every storage; the cylinder's force is the same
    FP64 sum over a different partition of the same cell contributions."""
    from getting_air_b200 import scenarios as sc
    cyl = sc.cylinder2d(W=96, H=48, r=6.0)
    doms = [((96, 48, 1), dict(cyl["kw"]), cyl["mac"]),
            ((64, 40, 1), dict(tau=0.7, sponge_w=0.0, wall=(0, 1, 0), wall_u=(0.03, -0.02)),
             sc.uniform_macro(64 * 40)),
            ((80, 72, 1), dict(tau=0.62, sponge_w=0.0, wall=(0, 1, 0), force=(2e-6, 0.0, 0.0)),
             sc.uniform_macro(80 * 72)),
            ((48, 48, 1), dict(tau=0.8, sponge_w=0.0), sc.uniform_macro(48 * 48, (0.02, -0.01, 0.0)))]
    doms = [(d, dict(kw, storage=storage), m) for d, kw, m in doms]
    got, want, gf, wf = run_pair(lbm, oracle, 9, doms, 12)
    for (f, m), (wf_, wm) in zip(got, want):
        assert np.array_equal(f, wf_)
        assert np.array_equal(m, wm)
    assert np.allclose(gf, wf, rtol=1e-10, atol=1e-12 * np.abs(wf).max())
    assert abs(wf[0][0]) > 0
