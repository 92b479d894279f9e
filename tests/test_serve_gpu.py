"""GPU tests of the serving form: a solve's result is the same alone and in
a mix (bit-identical to a dense session), admission respects the HBM budget,
and oversized requests are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mix(lbm):
    from getting_air_b200 import scenarios as sc
    reqs = sc.serving_stream(count=6, seed=5, nmin=16, nmax=40, steps=(20, 60))
    out = []
    for r in reqs:
        out.append((r["id"], lbm.config_from(r["q"], r["dims"], **r["kw"]), r["steps"]))
    # a diffuse-coupling D2Q9 cylinder in the same server
    from getting_air_b200 import scenarios as sc2
    c = sc2.cylinder2d(W=64, H=32, r=5.0, bounceback=False)
    out.append((99, lbm.config_from(9, c["dims"], **c["kw"]), 33))
    return out


def drain(srv, ids):
    got = {}
    for _ in range(10000):
        for r in srv.poll(16):
            got[r["id"]] = r
        if set(got) >= set(ids):
            return got
    raise AssertionError("server did not finish")


def test_results_same_alone_and_in_mix(lbm):
    reqs = mix(lbm)
    srv = lbm.Server(2 << 30)
    for rid, cfg, steps in reqs:
        srv.submit(rid, cfg, steps)
    got = drain(srv, [r[0] for r in reqs])
    for rid, cfg, steps in reqs:
        f, mac = srv.read(rid, cfg)
        alone = lbm.Solver(cfg)
        # the server's default seed, in the same f32 arithmetic
        ux, uy = np.float32(cfg.sponge_u[0]), np.float32(cfg.sponge_u[1])
        uz = np.float32(0) if cfg.q == 9 else np.float32(cfg.sponge_u[2])
        rho = np.float32(1) - (ux * ux + uy * uy + uz * uz) * np.float32(1.5)
        seed = np.tile(np.array([rho, ux, uy, uz], np.float32), (cfg.nx * cfg.ny * cfg.nz, 1))
        alone.init_macro(seed)
        alone.step(steps)
        assert got[rid]["steps"] == steps
        assert np.array_equal(f, alone.read_f()), rid
        assert np.array_equal(mac, alone.read_mac()), rid
        want = alone.forces()
        assert np.allclose(got[rid]["forces"], want, rtol=1e-10, atol=1e-12 * max(np.abs(want).max(), 1e-30))
        alone.close()
        srv.release(rid)
    assert srv.stats()["bytes_used"] == 0
    srv.close()


def test_budget_admission_queues_and_completes(lbm):
    reqs = mix(lbm)
    # room for the largest solve and a little more, so the others queue
    need = [2 * c.q * c.nx * c.ny * c.nz * 4 + 16 * c.nx * c.ny * c.nz for _, c, _ in reqs]
    srv = lbm.Server(int(max(need) * 1.3) + (1 << 20))
    for rid, cfg, steps in reqs:
        srv.submit(rid, cfg, steps)
    saw_queue = False
    done = {}
    for _ in range(10000):
        st = srv.stats()
        saw_queue |= st["queued"] > 0 and st["resident"] > 0
        assert st["bytes_used"] <= st["budget"]
        for r in srv.poll(8):
            done[r["id"]] = r
            srv.release(r["id"])
        if len(done) == len(reqs):
            break
    assert len(done) == len(reqs) and saw_queue
    # FIFO admission: admits happen in submission order
    admits = [done[rid]["admit_s"] for rid, _, _ in reqs]
    assert admits == sorted(admits)
    srv.close()


def test_oversized_request_is_refused(lbm):
    srv = lbm.Server(8 << 20)
    cfg = lbm.config_from(19, (64, 64, 64))
    with pytest.raises(lbm.LbmError, match="budget"):
        srv.submit(1, cfg, 10)
    srv.close()


def test_amr_solves_same_alone_and_in_mix(lbm):
    """Two-level AMR requests beside dense ones: each AMR result equals an
    lbm_amr3d session of the same config, bit for bit (L0 f and mac, force),
    and its hierarchy lives inside the server's arena."""
    from getting_air_b200 import scenarios as sc
    reqs = sc.serving_stream(count=8, seed=11, nmin=16, nmax=40, steps=(10, 30), amr_frac=0.5)
    assert {r["levels"] for r in reqs} == {1, 2}
    cfgs = {r["id"]: sc.serving_config(lbm, r) for r in reqs}
    srv = lbm.Server(2 << 30)
    for r in reqs:
        if r["levels"] == 2:
            srv.submit_amr3d(r["id"], cfgs[r["id"]], r["steps"])
        else:
            srv.submit(r["id"], cfgs[r["id"]], r["steps"])
    st = srv.stats()
    got = drain(srv, [r["id"] for r in reqs])
    used = srv.stats()["bytes_used"]
    amr_bytes = sum(lbm.amr3d_device_bytes(cfgs[r["id"]]) for r in reqs if r["levels"] == 2)
    assert used >= amr_bytes
    for r in reqs:
        rid, cfg, steps = r["id"], cfgs[r["id"]], r["steps"]
        f, mac = srv.read(rid, cfg)
        root = cfg.root if r["levels"] == 2 else cfg
        ux, uy, uz = (np.float32(v) for v in root.sponge_u)
        rho = np.float32(1) - (ux * ux + uy * uy + uz * uz) * np.float32(1.5)
        seed = np.tile(np.array([rho, ux, uy, uz], np.float32), (root.nx * root.ny * root.nz, 1))
        if r["levels"] == 2:
            alone = lbm.Amr3D(cfg)
            alone.init_macro(seed)
            alone.step(steps)
            af, amac = alone.read_coarse()
        else:
            alone = lbm.Solver(cfg)
            alone.init_macro(seed)
            alone.step(steps)
            af, amac = alone.read_f(), alone.read_mac()
        assert got[rid]["steps"] == steps
        assert np.array_equal(f, af), rid
        assert np.array_equal(mac, amac), rid
        want = alone.forces()
        assert np.array_equal(np.array(got[rid]["forces"]), np.array(want)), rid
        alone.close()
        srv.release(rid)
    assert srv.stats()["bytes_used"] == 0
    srv.close()


def test_amr_budget_refusal_and_queueing(lbm):
    from getting_air_b200 import scenarios as sc
    r = sc.serving_stream(count=1, seed=3, nmin=32, nmax=32, amr_frac=1.0)[0]
    cfg = sc.serving_config(lbm, r)
    need = lbm.amr3d_device_bytes(cfg)
    srv = lbm.Server(need // 2)
    with pytest.raises(lbm.LbmError, match="budget"):
        srv.submit_amr3d(1, cfg, 5)
    srv.close()
    # room for one at a time: the second queues until the first is released
    srv = lbm.Server(need + (need // 2))
    srv.submit_amr3d(1, cfg, 5)
    srv.submit_amr3d(2, cfg, 5)
    first = drain(srv, [1])
    assert srv.stats()["queued"] == 1
    srv.release(1)
    drain(srv, [2])
    srv.release(2)
    srv.close()


def test_shortest_work_first_with_a_resident_cap(lbm):
    """Policy 1 admits the least cells x steps first; the resident-cell cap
    holds the rest back while the device is busy; results are unchanged."""
    from getting_air_b200 import scenarios as sc
    reqs = sc.serving_stream(count=6, seed=9, nmin=16, nmax=40, steps=(10, 40))
    cfgs = {r["id"]: lbm.config_from(r["q"], r["dims"], **r["kw"]) for r in reqs}
    work = {r["id"]: int(np.prod(r["dims"])) * r["steps"] for r in reqs}
    biggest = max(int(np.prod(r["dims"])) for r in reqs)
    srv = lbm.Server(2 << 30)
    srv.set_policy("sjf", biggest)
    for r in reqs:
        srv.submit(r["id"], cfgs[r["id"]], r["steps"])
    held_back = False
    done = {}
    for _ in range(10000):
        for d in srv.poll(8):
            done[d["id"]] = d
        st = srv.stats()
        held_back |= st["resident"] > 0 and st["queued"] > 0
        if len(done) == len(reqs):
            break
    assert len(done) == len(reqs)
    # admitted in ascending total work (ties keep submission order)
    order = sorted(done, key=lambda i: done[i]["admit_s"])
    assert [work[i] for i in order] == sorted(work.values())
    # 2 GiB would hold all six at once: the cap is what queued some
    assert held_back
    for r in reqs:
        f, mac = srv.read(r["id"], cfgs[r["id"]])
        alone = lbm.Solver(cfgs[r["id"]])
        ux, uy, uz = (np.float32(v) for v in cfgs[r["id"]].sponge_u)
        rho = np.float32(1) - (ux * ux + uy * uy + uz * uz) * np.float32(1.5)
        alone.init_macro(np.tile(np.array([rho, ux, uy, uz], np.float32), (int(np.prod(r["dims"])), 1)))
        alone.step(r["steps"])
        assert np.array_equal(f, alone.read_f())
        alone.close()
        srv.release(r["id"])
    srv.close()


def test_large_requests_on_their_own_streams_equal_sessions(lbm):
    """Dense requests of 64^3 cells and up run the dense session's own step
    on their own streams beside the tile launches of the small ones: f, mac
    and the force are the session's, bit for bit (the same kernels and the
    same force-sum order)."""
    from getting_air_b200 import scenarios as sc
    reqs = sc.serving_stream(count=5, seed=21, nmin=24, nmax=80, steps=(20, 50))
    big = [dict(r, dims=(64, 64, 64)) for r in reqs[:1]]
    big[0]["kw"] = dict(big[0]["kw"], body=dict(big[0]["kw"]["body"], centre=(21, 32, 32)))
    reqs = big + reqs[1:]
    cfgs = {r["id"]: lbm.config_from(r["q"], r["dims"], **r["kw"]) for r in reqs}
    assert sum(int(np.prod(r["dims"])) >= 1 << 18 for r in reqs) >= 1
    srv = lbm.Server(4 << 30)
    for r in reqs:
        srv.submit(r["id"], cfgs[r["id"]], r["steps"])
    got = drain(srv, [r["id"] for r in reqs])
    for r in reqs:
        cfg = cfgs[r["id"]]
        f, mac = srv.read(r["id"], cfg)
        alone = lbm.Solver(cfg)
        ux, uy, uz = (np.float32(v) for v in cfg.sponge_u)
        rho = np.float32(1) - (ux * ux + uy * uy + uz * uz) * np.float32(1.5)
        alone.init_macro(np.tile(np.array([rho, ux, uy, uz], np.float32), (int(np.prod(r["dims"])), 1)))
        alone.step(r["steps"])
        assert np.array_equal(f, alone.read_f()), r["id"]
        assert np.array_equal(mac, alone.read_mac()), r["id"]
        want = np.array(alone.forces())
        if int(np.prod(r["dims"])) >= 1 << 18:
            assert np.array_equal(np.array(got[r["id"]]["forces"]), want), r["id"]
        else:
            assert np.allclose(got[r["id"]]["forces"], want, rtol=1e-10, atol=1e-12 * max(np.abs(want).max(), 1e-30))
        alone.close()
        srv.release(r["id"])
    assert srv.stats()["bytes_used"] == 0
    srv.close()
