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
