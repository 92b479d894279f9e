"""The reference's analytic and literature physics gates, run on B200.

* benchmarks/channel.json: plane Poiseuille (force-driven) and Couette
  (moving wall) flow between halfway-bounce-back walls, steady u(y) against
  the exact profile (tools/lib/channel-metrics.js analyticProfile), relative
  L2 within each case's l2_tol;
* benchmarks/cylinder.json with the dense cylinder page's configuration
  (main-cylinder.js at res 9, bounce-back): Cd (and St for the shedding case)
  inside the literature bands, and close to what the reference's own dense
  bounce-back run recorded (benchmarks/results/cylinder-bounceback-2026-07-11.json:
  Re 20 Cd 2.180; Re 100 Cd 1.327, St 0.1614). The window sizing and the
  Strouhal estimator follow tools/lib/cylinder-metrics.js.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHANNEL_CASES = [("poiseuille", 16, 5, 0.01), ("poiseuille", 16, 10, 0.01), ("poiseuille", 32, 10, 0.005),
                 ("poiseuille", 32, 20, 0.005), ("couette", 16, 5, 0.01), ("couette", 16, 10, 0.01),
                 ("couette", 32, 10, 0.005), ("couette", 32, 20, 0.005)]


@pytest.mark.parametrize("mode,H,re,tol", CHANNEL_CASES)
def test_channel_steady_profile(lbm, mode, H, re, tol):
    tau = 0.8
    nu = (tau - 0.5) / 3.0
    umax = re * nu / H
    force = 8 * nu * umax / (H * H) if mode == "poiseuille" else 0.0
    wall_u = umax if mode == "couette" else 0.0
    W = 8
    s = lbm.Solver.create(9, (W, H, 1), tau=tau, wall=(0, 1, 0), wall_u=(0.0, wall_u), force=(force, 0.0, 0.0),
                          sponge_w=0.0)
    mac = np.zeros((W * H, 4), np.float32)
    mac[:, 0] = 1.0
    s.init_macro(mac)
    prev = None
    for block in range(200):          # blocks of 1024 steps, at most 204800 steps
        s.step(1024)
        u = s.read_mac()[:, 1].reshape(H, W).mean(axis=1).astype(np.float64)
        if prev is not None and np.linalg.norm(u - prev) <= 1e-6 * max(np.linalg.norm(u), 1e-30):
            break
        prev = u
    y = np.arange(H) + 0.5
    exact = force / (2 * nu) * y * (H - y) if mode == "poiseuille" else wall_u * y / H
    l2 = np.linalg.norm(u - exact) / np.linalg.norm(exact)
    print(f"{mode} H={H} Re={re}: {1024 * (block + 1)} steps, L2rel {l2:.3e}")
    assert l2 <= tol
    s.close()


def run_cylinder(lbm, re, case_st):
    import torch
    from getting_air_b200 import scenarios as sc
    c = sc.cylinder_page(res=9, re=re, bounceback=True)
    D, u0 = c["D"], c["u0"]
    rnd = lambda n: int(np.ceil(n / 64) * 64)
    transient = rnd(40 * D / u0)
    measure = rnd(15 * D / (case_st * u0)) if case_st else rnd(5 * D / u0)
    total = transient + measure
    s = lbm.Solver.create(9, c["dims"], **c["kw"])
    s.write_f(c["f"])
    nsamp = total // 64
    hist = torch.zeros((nsamp, 6), dtype=torch.float64).pin_memory()
    for k in range(nsamp):
        s.step(64)
        s.forces_async(hist[k].data_ptr())
    s.sync()
    h = hist.numpy()
    scale = 2.0 / (u0 * u0 * D)
    rows = [((k + 1) * 64, h[k, 0] * scale, h[k, 1] * scale) for k in range(nsamp)]
    s.close()
    return sc.cylinder_analyze(rows, transient, D, u0)


# (Re, literature Cd, Cd band, literature St, St band, recorded Cd, recorded St)
CYLINDER_CASES = [(20.0, 2.05, 0.15, None, None, 2.179687508032657, None),
                  (40.0, 1.52, 0.12, None, None, 1.6230468463618308, None),
                  (100.0, 1.35, 0.15, 0.165, 0.015, 1.326993803887924, 0.16137494128289825),
                  (200.0, 1.34, 0.15, 0.197, 0.015, 1.3691375122472504, 0.19727216751079932)]


@pytest.mark.parametrize("re,cd,cd_tol,st,st_tol,ref_cd,ref_st", CYLINDER_CASES, ids=lambda v: str(v))
def test_cylinder_gates(lbm, re, cd, cd_tol, st, st_tol, ref_cd, ref_st):
    r = run_cylinder(lbm, re, st)
    print(f"Re {re:g}: {r}")
    assert abs(r["cd"] - cd) <= cd_tol
    # the same configuration as the reference's recorded dense bounce-back run
    assert abs(r["cd"] - ref_cd) <= 2e-3 * ref_cd
    if st is not None:
        assert abs(r["st"] - st) <= st_tol
        assert abs(r["st"] - ref_st) <= 0.02 * ref_st


# The reference's recorded two-level AMR bounce-back run of the same page
# (main-cylinder-amr.js at res 9, levels 2): (Re, Cd, St), and its recorded
# dense Cd for the same Re.
AMR_RECORDED = [(20.0, 2.003906120080501, None, 2.179687508032657),
                (100.0, 1.285, 0.16394208475416622, 1.326993803887924)]


@pytest.mark.parametrize("re,ref_cd,ref_st,dense_cd", AMR_RECORDED, ids=lambda v: str(v))
def test_amr2d_cylinder_gates(lbm, re, ref_cd, ref_st, dense_cd):
    """The 2D AMR cylinder page (root 512^2 in 16^2 root tiles, RB 8, one 2:1
    level by vorticity and geometry, bounce-back): Cd / St inside the
    literature bands, St close to the reference's recorded AMR run, and Cd
    within 3 % of the dense result (the recorded AMR Cd sits 3-8 % below the
    recorded dense one; this build's fine level reproduces the dense drag,
    which a 1024^2 dense run confirms is resolution-converged: Cd 2.1779 at
    Re 20)."""
    from getting_air_b200 import scenarios as sc
    W = 512
    r = W / 48.0
    s = sc.cylinder_amr(W=W, H=W, r=r, centre=(W / 2.0, W / 2.0), u0=0.04, re=re, bounceback=True)
    cfg = lbm.amr2d_config(W, W, **s["kw"])
    a = lbm.Amr2D(cfg)
    a.write_root(s["f"], s["vel"])
    D, u0 = 2 * r, 0.04
    rnd = lambda n: int(np.ceil(n / 64) * 64)
    st_lit = {20.0: None, 100.0: 0.165}[re]
    transient = rnd(40 * D / u0)
    measure = rnd(15 * D / (st_lit * u0)) if st_lit else rnd(5 * D / u0)
    rows = []
    scale = 2.0 / (u0 * u0 * D)
    for k in range((transient + measure) // 64):
        a.step(64)
        f = a.forces()
        rows.append(((k + 1) * 64, f[0] * scale, f[1] * scale))
    a.close()
    res = sc.cylinder_analyze(rows, transient, D, u0)
    print(f"AMR Re {re:g}: {res}")
    cd_lit, cd_tol = {20.0: (2.05, 0.15), 100.0: (1.35, 0.15)}[re]
    assert abs(res["cd"] - cd_lit) <= cd_tol
    assert abs(res["cd"] - dense_cd) <= 0.03 * dense_cd
    if st_lit:
        assert abs(res["st"] - st_lit) <= 0.015
        assert abs(res["st"] - ref_st) <= 0.02 * ref_st
