"""The two-relaxation-time collision on the CPU: the host rules, the
refusals, and the oracle's restatement (plans/TRT.md sec 8.0-8.1).

* tau_- = 1/2 + Lambda / (tau_+ - 1/2) and Lambda = (tau_+ - 1/2)(tau_- - 1/2)
  are inverse, and Lambda is the same at every level of the tau ladder
  (tau_f = 2 tau_c - 1/2 doubles tau_+ - 1/2);
* TRT is refused in D2Q9 (the 2D solver stays BGK), with Lambda <= 0, and in
  AMR hierarchies (whose transfers rescale one relaxation time);
* the oracle's TRT step conserves mass and momentum (the forcing adds
  exactly F per cell), and with Lambda = 3/16 halfway bounce-back walls carry
  a plane Poiseuille flow to the exact parabola, which BGK at the same tau
  misses by a slip that depends on tau: the test that an even/odd swap or a
  wrong sign in the delta form fails.
"""
import numpy as np
import pytest


def test_tau_minus_and_lambda_are_inverse(lbm):
    for tau in (0.51, 0.56, 0.6, 0.8, 1.3):
        for lam in (1 / 12, 3 / 16, 1 / 4):
            tm = lbm.trt_tau_minus(tau, lam)
            assert abs(lbm.trt_lambda(tau, tm) - lam) < 1e-14
    # constant down a 3-level ladder: tau_- per level from the same Lambda
    for m in range(3):
        tp = lbm.tau_at_level(0.55, m)
        assert abs(lbm.trt_lambda(tp, lbm.trt_tau_minus(tp, 3 / 16)) - 3 / 16) < 1e-14
    # the reference's card target: tau_+ = 0.5087 gives tau_- near 22 at L0
    assert abs(lbm.trt_tau_minus(0.5087, 3 / 16) - 22.05) < 0.01


def test_trt_refusals(lbm):
    cfg = lbm.config_from(9, (16, 16), trt=1, trt_lambda=0.1875)
    with pytest.raises(lbm.LbmError, match="3D"):
        lbm.Solver(cfg)
    for lam in (0.0, -1.0, float("nan")):
        with pytest.raises(lbm.LbmError, match="trt_lambda"):
            lbm.Solver(lbm.config_from(19, (8, 8, 8), trt=1, trt_lambda=lam))
    with pytest.raises(lbm.LbmError, match="trt must be"):
        lbm.Solver(lbm.config_from(19, (8, 8, 8), trt=2, trt_lambda=0.1875))
    acfg = lbm.amr3d_config(19, (32, 32, 32), refine="all", trt=1, trt_lambda=0.1875)
    with pytest.raises(lbm.LbmError, match="AMR") as ei:
        lbm.Amr3D(acfg)
    assert ei.value.code == lbm.ENOTSUP


def _poiseuille(lbm, oracle, trt, tau=0.8, N=16, steps=6000, q=19):
    nu = (tau - 0.5) / 3
    g = 1e-4
    kw = dict(tau=tau, wall=(0, 1, 0), force=(g, 0.0, 0.0), sponge_w=0.0)
    if trt:
        kw.update(trt=1, trt_lambda=3 / 16)
    cfg = lbm.config_from(q, (4, N, 4), **kw)
    n = 4 * N * 4
    mac = np.zeros((n, 4))
    mac[:, 0] = 1.0
    f0 = oracle.init_eq(q, mac)
    _, m, _ = oracle.run(cfg, f0, steps)
    u = m[:, 1].reshape(4, N, 4)[0, :, 0]
    y = np.arange(N)
    exact = g / (2 * nu) * (y + 0.5) * (N - 0.5 - y)
    return float(np.linalg.norm(u - exact) / np.linalg.norm(exact)), m


def test_oracle_trt_magic_lambda_makes_bounce_back_poiseuille_exact(lbm, oracle):
    e_trt, _ = _poiseuille(lbm, oracle, True)
    e_bgk, _ = _poiseuille(lbm, oracle, False)
    assert e_trt < 1e-5, e_trt
    assert e_bgk > 1e-3, e_bgk


def test_oracle_trt_conserves_mass_and_adds_the_force(lbm, oracle):
    # The odd relaxation changes neither mass nor the momentum input: one
    # step of TRT moves the totals exactly as one step of BGK does (the f32
    # weights' second moments are not exactly 1/3 in f64, so neither step
    # conserves mass to the last bit; the two agree to rounding), and the
    # momentum grows by F per cell. (The momentum of the odd equilibrium,
    # 3 rho sum w e (e.u), is rho u only up to the f32 weights' rounding, so
    # relaxing it at another rate moves the total momentum by ~1e-8 here.)
    rng = np.random.default_rng(7)
    dims = (12, 10, 8)
    n = int(np.prod(dims))
    mac = np.zeros((n, 4))
    mac[:, 0] = 1 + 0.01 * rng.standard_normal(n)
    mac[:, 1:] = 0.03 * rng.standard_normal((n, 3))
    F = (2e-5, -1e-5, 3e-5)
    for q in (19, 27):
        base = dict(tau=0.55, force=F, sponge_w=0.0)
        f0 = oracle.init_eq(q, mac)
        t0 = oracle.totals(q, f0)
        tb = oracle.totals(q, oracle.run(lbm.config_from(q, dims, **base), f0, 1)[0])
        tt = oracle.totals(q, oracle.run(lbm.config_from(q, dims, trt=1, trt_lambda=3 / 16, **base), f0, 1)[0])
        assert abs(tt[0] - tb[0]) < 1e-12
        for k in range(3):
            assert abs(tt[1 + k] - tb[1 + k]) < 1e-7
            assert abs((tt[1 + k] - t0[1 + k]) - n * F[k]) < 1e-7
        # and the fields differ: the odd moments relaxed at another rate
        fb = oracle.run(lbm.config_from(q, dims, **base), f0, 1)[0]
        ft = oracle.run(lbm.config_from(q, dims, trt=1, trt_lambda=3 / 16, **base), f0, 1)[0]
        assert np.abs(ft - fb).max() > 1e-6
