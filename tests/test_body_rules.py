"""The rigid-body integrator's host twin (lbm_body_advance, the code the
device runs after each force pass of a free body) against the oracle's FP64
restatement of d3-body.mjs stepFreeBody, and the reference's own checks of
that integrator (tools/test-d3-body.js, part C): exact |L| conservation,
energy to truncation order, the intermediate-axis flip, stable major/minor
spins, the textbook linear trajectory, direction-preserving clamps and the
planar projection. CPU only.
"""
import math
import zlib

import numpy as np
import pytest

import oracle


def qrot(q, v):
    """Rotate v by unit quaternion q = (w, x, y, z)."""
    w, x, y, z = q
    u = np.array([x, y, z])
    v = np.asarray(v, float)
    return v + 2 * np.cross(u, np.cross(u, v) + w * v)


def omega_from_L(q, ib, L):
    qc = np.array([q[0], -q[1], -q[2], -q[3]])
    lb = qrot(qc, L)
    return qrot(q, lb / ib)


def energy(st):
    d = st.as_dict()
    return 0.5 * float(np.dot(d["L"], omega_from_L(d["q"], d["ibody"], d["L"])))


def box(lbm, a, b, c, omega=(0, 0, 0), quat=(1, 0, 0, 0), density=1.0):
    body = lbm.make_body("roundbox", (0, 0, 0), a=a, b=b, c=c, r=0.0, quat=quat)
    body.wx, body.wy, body.wz = omega
    return lbm.body_state(body, density)


FREE = dict(v_max=math.inf, o_max=math.inf)


def test_inertia_and_volume(lbm):
    s = lbm.body_state(lbm.make_body("sphere", (0, 0, 0), a=3.0), density=5 / (4 / 3 * math.pi * 27))
    assert math.isclose(s.mass, 5.0, rel_tol=1e-12)
    assert np.allclose(s.as_dict()["ibody"], 0.4 * 5 * 9, rtol=1e-12)
    b = box(lbm, 2, 3, 4, density=5 / 192.0)
    I = b.as_dict()["ibody"]
    assert np.allclose(I, [5 * (6 ** 2 + 8 ** 2) / 12, 5 * (4 ** 2 + 8 ** 2) / 12, 5 * (4 ** 2 + 6 ** 2) / 12],
                       rtol=1e-12)
    sp = lbm.body_state(lbm.make_body("spheroid", (0, 0, 0), a=3.0, c=5.0))
    m = sp.mass
    assert math.isclose(m, 4 / 3 * math.pi * 9 * 5, rel_tol=1e-12)
    assert np.allclose(sp.as_dict()["ibody"], [m * 34 / 5, m * 34 / 5, 2 * m * 9 / 5], rtol=1e-12)
    # a thin square plate has I_zz ~ 2 I_xx
    p = box(lbm, 12, 12, 0.75).as_dict()["ibody"]
    assert p[2] > 1.9 * p[0]


def test_make_state_L_matches_omega(lbm):
    ax = np.array([1.0, 1.0, 0.0]) / math.sqrt(2)
    q = (math.cos(0.2), *(ax * math.sin(0.2)))
    s = box(lbm, 4, 3, 1, omega=(0.01, -0.02, 0.03), quat=q).as_dict()
    w = omega_from_L(s["q"], s["ibody"], s["L"])
    assert np.allclose(w, np.float32([0.01, -0.02, 0.03]), rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("shape", ["sphere", "spheroid", "roundbox"])
@pytest.mark.parametrize("mode", ["free", "clamped", "planar", "pinned", "no_fluid", "window"])
def test_host_twin_matches_oracle(lbm, shape, mode):
    rng = np.random.default_rng(zlib.crc32(f"{shape}/{mode}".encode()))
    body = lbm.make_body(shape, (10.3, 20.1, 5.5), a=6.0, b=3.0, c=2.0, r=0.5,
                         quat=(math.cos(0.3), 0.0, math.sin(0.3), 0.0), v=(0.01, -0.02, 0.005),
                         w=(0.003, -0.001, 0.002))
    kw = dict(FREE, gravity=(1e-4, -2e-4, 0.0))
    if mode == "clamped":
        kw.update(v_max=0.05, o_max=0.004)
    elif mode == "planar":
        kw["planar"] = 1
    elif mode == "pinned":
        kw["pinned"] = 1
    elif mode == "no_fluid":
        kw["no_fluid_force"] = 1
    elif mode == "window":
        kw["wrap"] = (32.0, 0.0, 24.0)
    opts = lbm.body_opts(**kw)
    a = lbm.body_state(body, density=1.3)
    b = oracle.body_make(body, density=1.3)
    assert np.allclose(np.array(a.L[:]), np.array(b.L[:]), rtol=1e-14, atol=0)
    for k in range(200):
        F = rng.standard_normal(3) * 50.0
        T = rng.standard_normal(3) * 400.0
        lbm.body_advance(a, opts, 1, F, T)
        oracle.body_step(b, opts, 1, F, T)
    da, db = a.as_dict(), b.as_dict()
    for key in ("x", "q", "v", "L", "omega", "d", "force", "torque"):
        assert np.allclose(da[key], db[key], rtol=1e-12, atol=1e-12 * (np.abs(db[key]).max() + 1e-30)), key
    assert da["steps"] == db["steps"] == 200
    if mode == "pinned":
        assert np.array_equal(da["x"], np.float32([10.3, 20.1, 5.5]).astype(float))
    if mode == "planar":
        assert da["v"][2] == 0.0 and da["L"][0] == 0.0 and da["L"][1] == 0.0
    if mode == "window":
        assert 0 <= da["x"][0] < 32 and 0 <= da["x"][2] < 24


def test_free_body_conserves_L_exactly_and_energy_to_truncation(lbm):
    s = box(lbm, 6, 4, 1, omega=(0.02, 0.01, 0.005))
    L0 = np.linalg.norm(s.as_dict()["L"])
    E0 = energy(s)
    lbm.body_advance(s, lbm.body_opts(**FREE), 20000)
    d = s.as_dict()
    assert abs(np.linalg.norm(d["L"]) - L0) <= 1e-12 * L0
    assert abs(energy(s) - E0) / E0 < 0.02
    assert abs(np.linalg.norm(d["q"]) - 1) < 1e-9


def _min_alignment(lbm, s, axis, steps=400000, every=100):
    opts = lbm.body_opts(**FREE)
    a0 = qrot(s.as_dict()["q"], axis)
    lo = 1.0
    for _ in range(steps // every):
        lbm.body_advance(s, opts, every)
        lo = min(lo, float(np.dot(qrot(s.as_dict()["q"], axis), a0)))
    return lo


def test_intermediate_axis_flips(lbm):
    # Roundbox 6x3x1: I_xx < I_yy < I_zz, so y is the intermediate axis.
    s = box(lbm, 6, 3, 1, omega=(1e-4, 0.02, 1e-4))
    I = s.as_dict()["ibody"]
    assert I[0] < I[1] < I[2]
    assert _min_alignment(lbm, s, [0, 1, 0]) < -0.9


@pytest.mark.parametrize("axis", [[1, 0, 0], [0, 0, 1]], ids=["minor", "major"])
def test_stable_axes_do_not_flip(lbm, axis):
    om = [0.02 * c + (1e-4 if i == 1 else 0.0) for i, c in enumerate(axis)]
    s = box(lbm, 6, 3, 1, omega=om)
    assert _min_alignment(lbm, s, axis) > 0.9


def test_constant_force_gives_textbook_trajectory(lbm):
    s = lbm.body_state(lbm.make_body("sphere", (0, 0, 0), a=2.0))
    g = -1e-4
    n = 1000
    lbm.body_advance(s, lbm.body_opts(gravity=(0.0, g, 0.0), **FREE), n)
    d = s.as_dict()
    assert abs(d["v"][1] - n * g) <= 1e-12 * abs(n * g)
    assert abs(d["x"][1] - g * n * (n + 1) / 2) <= abs(g) * 1e-6


def test_clamps_keep_direction(lbm):
    s = lbm.body_state(lbm.make_body("sphere", (0, 0, 0), a=2.0, v=(0.3, 0.4, 0.0)))
    lbm.body_advance(s, lbm.body_opts(v_max=0.1, o_max=math.inf))
    v = s.as_dict()["v"]
    assert abs(np.linalg.norm(v) - 0.1) <= 1e-7  # v came in as f32
    assert abs(v[0] / v[1] - float(np.float32(0.3)) / float(np.float32(0.4))) <= 1e-12


def test_planar_projection_is_exact(lbm):
    th = 2 * math.pi / 3
    ax = np.ones(3) / math.sqrt(3)
    q = (math.cos(th / 2), *(ax * math.sin(th / 2)))
    s = box(lbm, 16, 40, 2, quat=q, density=2.7)
    u = box(lbm, 16, 40, 2, quat=q, density=2.7)
    op = lbm.body_opts(gravity=(1e-3, 0.0, 0.0), planar=1, **FREE)
    ou = lbm.body_opts(gravity=(1e-3, 0.0, 0.0), **FREE)
    for i in range(50):
        F = [math.sin(i), math.cos(2 * i), 0.7 * math.sin(3 * i)]
        T = [0.2 * math.cos(i), 0.1 * math.sin(i), 0.05 * math.cos(4 * i)]
        lbm.body_advance(s, op, 1, F, T)
        lbm.body_advance(u, ou, 1, [F[0], F[1], 0.0], [0.0, 0.0, T[2]])
        d = s.as_dict()
        assert d["v"][2] == 0.0 and d["L"][0] == 0.0 and d["L"][1] == 0.0
        assert d["omega"][0] == 0.0 and d["omega"][1] == 0.0
    d, e = s.as_dict(), u.as_dict()
    assert abs(d["v"][0] - e["v"][0]) <= 1e-15 and abs(d["v"][1] - e["v"][1]) <= 1e-15
    assert abs(d["L"][2] - e["L"][2]) <= 1e-15
    assert np.allclose(d["q"], e["q"], atol=1e-12)


def test_invalid_state_is_refused(lbm):
    with pytest.raises(lbm.LbmError):
        lbm.body_state(lbm.make_body("sphere", (0, 0, 0), a=-1.0))
    s = lbm.BodyState()
    with pytest.raises(lbm.LbmError):
        lbm.body_advance(s, lbm.body_opts())
