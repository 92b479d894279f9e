"""Free bodies on the GPU: the device integrator and the force -> physics ->
step loop against the oracle.

* spin: the fluid load switched off (NO_FLUID_FORCE), so the device
  trajectory must follow the host twin of stepFreeBody step for step -- the
  reference's own GPU-vs-host check of d3_physics.wgsl (its `spin` scenario);
* coupled: a sphere and a rotating rounded box, each free in a flow, against
  the oracle's coupled loop (force pass on f_t at P_t, integrate, step at
  P_t+1). The GPU's force is f32 summed in FP64, the oracle's FP64, so the
  trajectories agree to ~1e-6 relative over these horizons; the tolerances
  below leave a decade of headroom and still catch a one-step lag of the
  pose (a relative error of ~1e-2 in the displacement);
* pinned: a free body with `pinned` set moves nowhere and records the same
  load as the prescribed-pose session.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def flow(q, dims, u0, seed, amp=0.005):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims))
    mac = np.zeros((n, 4))
    mac[:, 0] = 1.0
    mac[:, 1] = u0
    mac[:, 1:] += amp * rng.standard_normal((n, 3))
    return mac


def test_spin_without_fluid_load_follows_host_twin(lbm, oracle):
    dims = (64, 48, 48)
    body = lbm.make_body("roundbox", (31.6, 24.2, 23.7), a=8.0, b=4.0, c=1.5, r=0.3,
                         w=(0.003, 0.004, 0.002))
    kw = dict(tau=0.6, has_body=1, use_bounceback=1, body=body)
    s = lbm.Solver.create(19, dims, **kw)
    s.init_macro(flow(19, dims, 0.0, 1))
    opts = lbm.body_opts(no_fluid_force=1, v_max=math.inf, o_max=math.inf)
    st = lbm.body_state(body, density=1.0)
    s.set_free_body(st, opts)
    s.step(40)
    dev = s.body_state().as_dict()
    host = lbm.body_advance(lbm.body_state(body, density=1.0), opts, 40).as_dict()
    for k in ("x", "q", "v", "L", "omega", "d"):
        assert np.allclose(dev[k], host[k], rtol=1e-12, atol=1e-14), (k, dev[k], host[k])
    assert dev["steps"] == 40
    # the load was measured and recorded all the same
    assert np.abs(dev["torque"]).max() > 0
    assert np.allclose(dev["force"], s.forces()[:3], rtol=0, atol=0)
    s.close()


def coupled(lbm, oracle, q, dims, kw, body, density, opts, nsteps, seed):
    mac = flow(q, dims, 0.03, seed)
    f0 = oracle.init_eq(q, mac, fp32=True).astype(np.float32)
    s = lbm.Solver.create(q, dims, body=body, **kw)
    s.write_f(f0)
    s.set_free_body(lbm.body_state(body, density), opts)
    traj = []
    for _ in range(nsteps):
        s.step(1)
        d = s.body_state().as_dict()
        traj.append(np.concatenate([d["x"], d["v"], d["L"], d["omega"], d["q"]]))
    g_mac = s.read_mac().astype(np.float64)
    g_force = s.forces()
    ost = oracle.body_make(body, density)
    _, o_mac, o_forces, o_traj = oracle.run_free(s.cfg, f0.astype(np.float64), nsteps, ost, opts)
    s.close()
    return np.array(traj), o_traj, g_mac, o_mac, g_force, o_forces[-1, :6]


def check_coupled(res, x0):
    g_traj, o_traj, g_mac, o_mac, g_force, o_force = res
    disp_g = g_traj[:, 0:3] - x0
    disp_o = o_traj[:, 0:3] - x0
    scale = max(np.abs(disp_o).max(), 1e-6)
    assert np.abs(disp_g - disp_o).max() <= 1e-3 * scale, (disp_g[-1], disp_o[-1])
    vs = max(np.abs(o_traj[:, 3:6]).max(), 1e-9)
    assert np.abs(g_traj[:, 3:6] - o_traj[:, 3:6]).max() <= 1e-3 * vs
    Ls = max(np.abs(o_traj[:, 6:9]).max(), 1e-9)
    assert np.abs(g_traj[:, 6:9] - o_traj[:, 6:9]).max() <= 1e-3 * Ls
    assert np.abs(g_traj[:, 12:16] - o_traj[:, 12:16]).max() <= 1e-6
    assert rel_l2(g_mac[:, 1:4], o_mac[:, 1:4]) <= 2e-5
    fs = max(np.abs(o_force).max(), 1e-3)
    assert np.abs(g_force - o_force).max() <= 1e-3 * fs


def test_free_sphere_in_flow_matches_oracle(lbm, oracle):
    body = lbm.make_body("sphere", (20.3, 16.2, 15.8), a=4.0)
    kw = dict(tau=0.6, has_body=1, use_bounceback=1, force=(1e-6, 0.0, 0.0))
    opts = lbm.body_opts(gravity=(0.0, -2e-5, 0.0))
    res = coupled(lbm, oracle, 19, (48, 32, 32), kw, body, 1.5, opts, 30, 5)
    check_coupled(res, np.float32([20.3, 16.2, 15.8]).astype(float))
    assert np.abs(res[1][-1, 3:6]).max() > 1e-5  # the body did move


@pytest.mark.parametrize("bb", [1, 0], ids=["bounceback", "penalty"])
def test_free_rotating_box_matches_oracle(lbm, oracle, bb):
    body = lbm.make_body("roundbox", (24.4, 16.1, 15.7), a=6.0, b=3.0, c=2.0, r=0.5,
                         quat=(math.cos(0.2), 0.0, 0.0, math.sin(0.2)), w=(0.0, 0.0, 0.01))
    kw = dict(tau=0.62, has_body=1, use_bounceback=bb, chi_eps=1.5)
    opts = lbm.body_opts(o_max=0.05)
    res = coupled(lbm, oracle, 27 if bb else 19, (48, 32, 32), kw, body, 1.2, opts, 20, 9)
    check_coupled(res, np.float32([24.4, 16.1, 15.7]).astype(float))


def test_pinned_free_body_matches_prescribed_pose(lbm, oracle):
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40, force=(1e-6, 0.0, 0.0))
    a = lbm.Solver.create(19, s["dims"], **s["kw"])
    b = lbm.Solver.create(19, s["dims"], **s["kw"])
    a.init_macro(s["mac"])
    b.init_macro(s["mac"])
    b.set_free_body(lbm.body_state(b.cfg.body, 1.0), lbm.body_opts(pinned=1))
    for _ in range(3):
        a.step(4)
        b.step(4)
        fa, fb = a.forces(), b.forces()
        assert np.allclose(fa, fb, rtol=1e-12, atol=1e-14 * np.abs(fa).max())
    assert np.allclose(a.read_f(), b.read_f(), rtol=0, atol=1e-7)
    st = b.body_state().as_dict()
    assert st["steps"] == 12
    assert np.array_equal(st["x"], np.array([b.cfg.body.cx, b.cfg.body.cy, b.cfg.body.cz], float))
    assert np.allclose(st["force"], fb[:3], rtol=0, atol=0)
    # back to the prescribed pose
    b.set_free_body(None)
    a.step(2)
    b.step(2)
    assert np.allclose(a.forces(), b.forces(), rtol=1e-12, atol=1e-14 * np.abs(fa).max())
    a.close()
    b.close()


def test_free_body_refused_where_unsupported(lbm):
    s = lbm.Solver.create(9, (32, 16, 1), tau=0.6)
    body = lbm.make_body("sphere", (5, 5, 5), a=2.0)
    with pytest.raises(lbm.LbmError):
        s.set_free_body(lbm.body_state(body), lbm.body_opts())
    s.close()
    s = lbm.Solver.create(19, (16, 16, 16), tau=0.6)  # no body
    with pytest.raises(lbm.LbmError):
        s.set_free_body(lbm.body_state(body), lbm.body_opts())
    with pytest.raises(lbm.LbmError):
        s.body_state()
    s.close()
