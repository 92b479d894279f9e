"""GPU parity of the dense fused step, force and totals against the oracle.

Every case starts the GPU and the oracle from the same f32 populations
(written through lbm_write_f), advances both, and compares:

* velocity: relative L2 error <= U_TOL against the FP64 oracle;
* density:  relative L2 error <= RHO_TOL;
* force/torque of the last step: |gpu - oracle| <= F_TOL * max(|F|, 1e-3);
* topology-like integers (non-finite counts): exactly equal.

The GPU computes in f32 with fused multiply-adds, the FP64 oracle in
double; over tens of steps the two stay within ~1e-6 in these norms, so the
tolerances below leave an order of magnitude of headroom while still
catching any single wrong link, weight or sign (those produce errors of
1e-3 or more).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U_TOL = 1e-5
RHO_TOL = 1e-6
F_TOL = 1e-4


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def seed_random(q, n, rng, amp=0.03):
    mac = np.zeros((n, 4))
    mac[:, 0] = 1 + 0.01 * rng.standard_normal(n)
    mac[:, 1:] = amp * rng.standard_normal((n, 3))
    if q == 9:
        mac[:, 3] = 0
    return mac


def both(lbm, oracle, q, dims, kw, nsteps, mac=None, f0=None, fp32_oracle=False):
    s = lbm.Solver.create(q, dims, **kw)
    if f0 is None:
        f0 = oracle.init_eq(q, mac, fp32=True).astype(np.float32)
    s.write_f(f0)
    s.step(nsteps)
    g_f = s.read_f().astype(np.float64)
    g_mac = s.read_mac().astype(np.float64)
    g_force = s.forces()
    o_f, o_mac, o_forces = oracle.run(s.cfg, f0.astype(np.float64), nsteps, fp32=fp32_oracle)
    s.close()
    return (g_f, g_mac, g_force), (o_f, o_mac, o_forces[-1])


def check(g, o, u_tol=U_TOL, rho_tol=RHO_TOL, f_tol=F_TOL, forces=True):
    g_f, g_mac, g_force = g
    o_f, o_mac, o_force = o
    assert np.isfinite(g_f).all()
    eu = rel_l2(g_mac[:, 1:4], o_mac[:, 1:4])
    er = rel_l2(g_mac[:, 0], o_mac[:, 0])
    assert eu <= u_tol, f"u relL2 {eu:.3e}"
    assert er <= rho_tol, f"rho relL2 {er:.3e}"
    if forces:
        scale = max(np.abs(o_force[:6]).max(), 1e-3)
        assert np.abs(g_force - o_force[:6]).max() <= f_tol * scale, (g_force, o_force[:6])


@pytest.mark.parametrize("q", [19, 27])
def test_periodic_random_field(lbm, oracle, q):
    # White noise (rho +-1 %, u +-0.03 per cell) is the worst case for f32
    # cancellation in the moments; its stated bound is 5e-5.
    dims = (20, 12, 10)
    rng = np.random.default_rng(q)
    mac = seed_random(q, np.prod(dims), rng)
    g, o = both(lbm, oracle, q, dims, dict(tau=0.7), 12, mac=mac)
    check(g, o, u_tol=5e-5, forces=False)
    # the f32 oracle too (the reference's operation order, no FMA on the CPU side)
    g2, o2 = both(lbm, oracle, q, dims, dict(tau=0.7), 12, mac=mac, fp32_oracle=True)
    check(g2, o2, u_tol=5e-5, forces=False)


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("bb", [1, 0], ids=["bounceback", "penalty"])
def test_sphere_with_sponge_and_body_force(lbm, oracle, q, bb):
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40, q=q, bounceback=bool(bb),
                  force=(2e-6, 0.0, 0.0))
    g, o = both(lbm, oracle, q, s["dims"], s["kw"], 25, mac=s["mac"])
    check(g, o)
    assert abs(o[2][0]) > 1e-3  # the body does feel a force


def test_moving_sphere_swept_term(lbm, oracle):
    kw = dict(tau=0.6, has_body=1, use_bounceback=1,
              body=dict(shape="sphere", centre=(15.3, 12.2, 11.7), a=4.0, v=(0.02, -0.01, 0.0),
                        w=(0.0, 0.0, 0.01)))
    dims = (32, 24, 24)
    mac = seed_random(19, np.prod(dims), np.random.default_rng(3), amp=0.01)
    g, o = both(lbm, oracle, 19, dims, kw, 6, mac=mac)
    check(g, o)


@pytest.mark.parametrize("shape", ["roundbox", "spheroid"])
def test_rotated_bodies(lbm, oracle, shape):
    c, s_ = np.cos(0.3), np.sin(0.3)
    body = dict(shape=shape, centre=(16.4, 12.1, 12.6), a=5.0, b=3.0, c=2.5 if shape == "roundbox" else 7.0,
                r=0.8, quat=(c, 0.0, s_ * 0.6, s_ * 0.8))
    kw = dict(tau=0.65, has_body=1, use_bounceback=1, body=body, sponge_w=4.0, sponge_u=(0.03, 0, 0))
    dims = (36, 24, 24)
    from getting_air_b200 import scenarios as sc
    mac = sc.uniform_macro(int(np.prod(dims)), (0.03, 0, 0))
    g, o = both(lbm, oracle, 19, dims, kw, 15, mac=mac)
    check(g, o)


def test_duct_walls(lbm, oracle):
    # Seeded with a uniform stream so the walls shear a flow of O(0.02):
    # started from rest, |u| after 30 steps is O(1e-4) and a relative norm
    # would measure f32 rounding of f (~1e-8) against a vanishing velocity.
    from getting_air_b200 import scenarios as sc
    dims = (16, 20, 18)
    kw = dict(tau=0.8, wall=(0, 1, 1), force=(1e-5, 0, 0))
    mac = sc.uniform_macro(int(np.prod(dims)), (0.02, 0.0, 0.0))
    g, o = both(lbm, oracle, 19, dims, kw, 30, mac=mac)
    check(g, o, forces=False)
    g32, o32 = both(lbm, oracle, 19, dims, kw, 30, mac=mac, fp32_oracle=True)
    check(g32, o32, forces=False)
    # the walls slow the flow next to them
    u = g[1][:, 1].reshape(dims[2], dims[1], dims[0])
    assert u[:, 0, :].mean() < u[:, dims[1] // 2, :].mean()


@pytest.mark.parametrize("bb", [1, 0], ids=["bounceback", "penalty"])
def test_d2q9_cylinder(lbm, oracle, bb):
    from getting_air_b200 import scenarios as sc
    s = sc.cylinder2d(W=96, H=48, r=6.0, u0=0.05, tau=0.6, bounceback=bool(bb))
    g, o = both(lbm, oracle, 9, s["dims"], s["kw"], 40, mac=s["mac"])
    check(g, o)


def test_d2q9_ellipse_and_couette(lbm, oracle):
    body = dict(shape="ellipse", centre=(30.3, 20.7, 0), a=8.0, b=2.0, theta=0.4)
    kw = dict(tau=0.7, has_body=1, use_bounceback=1, body=body, wall=(0, 1, 0), wall_u=(0.0, 0.04),
              sponge_w=0.0)
    dims = (64, 40, 1)
    from getting_air_b200 import scenarios as sc
    mac = sc.uniform_macro(64 * 40, (0.02, 0.0, 0.0))
    g, o = both(lbm, oracle, 9, dims, kw, 30, mac=mac)
    check(g, o)


def test_d2q9_tgv_analytic_gate_on_gpu(lbm, oracle):
    """benchmarks/tgv.json dense-N64: relL2 <= 1e-2 against the exact field."""
    from getting_air_b200 import scenarios as sc
    N, u0, tau = 64, 0.04, 0.8
    w = lbm.lattice_tables(9)["w"]
    s = lbm.Solver.create(9, (N, N, 1), tau=tau, sponge_w=0.0)
    s.write_f(sc.tgv2d_f(N, u0, tau, w))
    _, _, _, td = sc.tgv2d_field(N, u0, tau)
    steps = round(1.5 * td)
    s.step(steps)
    m = s.read_mac().astype(np.float64)
    ax, ay, _, _ = sc.tgv2d_field(N, u0, tau, t=steps)
    err = np.sqrt(((m[:, 1] - ax) ** 2 + (m[:, 2] - ay) ** 2).sum() / (ax ** 2 + ay ** 2).sum())
    assert err <= 1e-2
    s.close()


@pytest.mark.parametrize("q", [9, 19, 27])
def test_totals_match_oracle(lbm, oracle, q):
    dims = (24, 16, 1 if q == 9 else 12)
    rng = np.random.default_rng(11)
    mac = seed_random(q, int(np.prod(dims)), rng)
    f0 = oracle.init_eq(q, mac, fp32=True).astype(np.float32)
    s = lbm.Solver.create(q, dims, tau=0.7, sponge_w=0.0)
    s.write_f(f0)
    t = s.totals()
    o = oracle.totals(q, f0.astype(np.float64))
    got = np.array([t[k] for k in ("mass", "px", "py", "pz", "rho_min", "rho_max", "max_u", "nonfinite")])
    assert np.allclose(got[:4], o[:4], rtol=1e-12, atol=1e-12)
    assert np.array_equal(got[4:6], o[4:6])  # min/max of the same per-cell f64 sums
    assert abs(got[6] - o[6]) <= 1e-14 and got[7] == o[7] == 0
    s.close()


def test_forces_async_matches_sync(lbm, oracle):
    # Pinned memory takes the kernel copy, pageable memory the copy engine;
    # every entry equals the force read synchronously after the same step.
    import torch
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40)
    runs = {}
    for kind in ("pinned", "pageable", "sync"):
        sol = lbm.Solver.create(19, s["dims"], **s["kw"])
        sol.init_macro(s["mac"])
        if kind == "pinned":
            t = torch.zeros((5, 6), dtype=torch.float64).pin_memory()
            hist, ptr = t.numpy(), lambda k: t[k].data_ptr()
        else:
            hist = np.zeros((5, 6))
            ptr = lambda k: hist[k].ctypes.data
        for k in range(5):
            sol.step(1)
            if kind == "sync":
                hist[k] = sol.forces()
            else:
                sol.forces_async(ptr(k))
        sol.sync()
        if kind == "pinned":
            assert np.array_equal(hist[4], sol.forces())
        runs[kind] = hist.copy()
        sol.close()
    assert np.array_equal(runs["pinned"], runs["sync"])
    assert np.array_equal(runs["pageable"], runs["sync"])
    assert not np.array_equal(runs["sync"][0], runs["sync"][4])


def test_totals_count_nonfinite_cells(lbm, oracle):
    dims = (16, 12, 10)
    f0 = oracle.init_eq(19, seed_random(19, 1920, np.random.default_rng(2)), fp32=True).astype(np.float32)
    f0[3, 17] = np.nan
    f0[5, 400] = np.inf
    s = lbm.Solver.create(19, dims)
    s.write_f(f0)
    assert s.totals()["nonfinite"] == 2
    s.close()


def test_write_read_roundtrip_and_determinism(lbm, oracle):
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40)
    f0 = oracle.init_eq(19, s["mac"], fp32=True).astype(np.float32)
    runs = []
    for _ in range(2):
        sol = lbm.Solver.create(19, s["dims"], **s["kw"])
        sol.write_f(f0)
        assert np.array_equal(sol.read_f(), f0)
        sol.step(7)
        runs.append((sol.read_f(), sol.forces()))
        sol.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


def test_step_in_pieces_equals_one_call(lbm, oracle):
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40)
    f0 = oracle.init_eq(19, s["mac"], fp32=True).astype(np.float32)
    a = lbm.Solver.create(19, s["dims"], **s["kw"])
    b = lbm.Solver.create(19, s["dims"], **s["kw"])
    a.write_f(f0)
    b.write_f(f0)
    a.step(9)
    for _ in range(3):
        b.step(3)
    assert np.array_equal(a.read_f(), b.read_f())
    assert np.array_equal(a.read_mac(), b.read_mac())
    assert np.array_equal(a.forces(), b.forces())
    buf = np.full((a.ncells, 4), np.nan, np.float32)
    assert a.read_mac(out=buf) is buf and np.array_equal(buf, b.read_mac())
    with pytest.raises(ValueError):
        a.read_mac(out=np.empty((a.ncells, 4), np.float64))
    a.close()
    b.close()


def test_chained_force_sums_equal_per_step_sums(lbm, oracle):
    """Within one step(n) each step's force partials are summed by the next
    step's first block, the last step's by a sum launched after it, with the
    partials alternating between two sets: an even count ends on the second
    set. The last force equals the one of n calls of step(1), whichever set
    the call ended on."""
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40)
    f0 = oracle.init_eq(19, s["mac"], fp32=True).astype(np.float32)
    a = lbm.Solver.create(19, s["dims"], **s["kw"])
    c = lbm.Solver.create(19, s["dims"], **s["kw"])
    a.write_f(f0)
    c.write_f(f0)
    a.step(8)
    for _ in range(8):
        c.step(1)
    assert np.array_equal(a.read_f(), c.read_f())
    assert np.array_equal(a.forces(), c.forces())
    a.step(3)
    c.step(2)
    c.step(1)
    assert np.array_equal(a.forces(), c.forces())
    a.close()
    c.close()


def test_init_macro_matches_oracle_init(lbm, oracle):
    rng = np.random.default_rng(5)
    dims = (16, 8, 8)
    mac = seed_random(27, 1024, rng).astype(np.float32)
    s = lbm.Solver.create(27, dims)
    s.init_macro(mac)
    f = s.read_f().astype(np.float64)
    o = oracle.init_eq(27, mac.astype(np.float64), fp32=True)
    # the device contracts multiply-adds, the f32 oracle rounds each: 1 ulp
    assert np.abs(f - o).max() <= 2 ** -24 * np.abs(o).max() * 2
    s.close()


@pytest.mark.parametrize("storage", ["fp16", "bf16"])
def test_packed_storage_error_is_bounded(lbm, oracle, storage):
    """16-bit storage holds (f - feq(1, U_far)) * scale: the round trip is
    within the 16-bit quantum of that deviation, and the velocity after 200
    steps stays within the stated bound of the FP64 oracle (1e-4 for FP16,
    1e-3 for BF16, the packed forms' accuracy target)."""
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40, storage=storage)
    f0 = oracle.init_eq(19, s["mac"], fp32=True).astype(np.float32)
    sol = lbm.Solver.create(19, s["dims"], **s["kw"])
    sol.write_f(f0)
    back = sol.read_f()
    t = lbm.lattice_tables(19)
    eu = t["ex"] * 0.05
    off = (t["w"] * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * 0.05 ** 2)).astype(np.float32)[:, None]
    quantum = 2.0 ** -11 if storage == "fp16" else 2.0 ** -8
    assert (np.abs(back - f0) <= quantum * np.abs(f0 - off) * 1.0001 + 2.0 ** -34).all()
    sol.step(200)
    m = sol.read_mac().astype(np.float64)
    _, om, _ = oracle.run(sol.cfg, back.astype(np.float64), 200)
    err = rel_l2(m[:, 1:4], om[:, 1:4])
    assert err <= (1e-4 if storage == "fp16" else 1e-3), err
    sol.close()



@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16"])
def test_raw_planes_give_an_exact_restart(lbm, oracle, storage):
    """lbm_read_f_raw / lbm_write_f_raw move the stored planes verbatim, so a
    second session restarted from them continues bit for bit (a decode and
    re-encode through the f32 wire format would re-quantise)."""
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40, storage=storage, force=(1e-6, 0.0, 0.0))
    a = lbm.Solver.create(19, s["dims"], **s["kw"])
    a.init_macro(s["mac"])
    a.step(7)
    raw = a.read_f_raw()
    assert raw.dtype == (np.float32 if storage == "fp32" else np.uint16)
    b = lbm.Solver.create(19, s["dims"], **s["kw"])
    b.write_f_raw(raw)
    assert np.array_equal(b.read_f_raw(), raw)
    a.step(5)
    b.step(5)
    assert np.array_equal(a.read_f_raw(), b.read_f_raw())
    assert np.array_equal(a.read_mac(), b.read_mac())
    assert np.array_equal(a.forces(), b.forces())
    a.close()
    b.close()
