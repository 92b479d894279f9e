"""The Q-criterion of the 3D manager's field test, on the CPU oracle.

The closed-form cases follow tools/test-d3-criterion.js: uniform flow has
Q = 0, pure shear has Q = 0 exactly (the reason the criterion is Q and not
|omega|), solid-body rotation has Q = omega^2, Q is a frame invariant, and the
centred-difference stencil converges at second order on a Taylor-Green cell.
The per-cell f32 stencil (common_d3_criterion.wgsl qAt) and the per-block
dilated max (reduceQ) are checked against numpy restatements here.
"""
import math

import numpy as np
import pytest

import oracle


def grad_at(u, p, h):
    """J[i][j] = du_i/dx_j by centred differences (d3-criterion.mjs gradU)."""
    J = np.zeros((3, 3))
    for j in range(3):
        pp, pm = list(p), list(p)
        pp[j] += h
        pm[j] -= h
        up, um = u(pp), u(pm)
        for i in range(3):
            J[i][j] = (up[i] - um[i]) / (2 * h)
    return J


def test_uniform_flow_has_no_q():
    J = grad_at(lambda p: [0.05, -0.02, 0.01], [1, 2, 3], 1)
    assert abs(oracle.q_of_grad(J)) <= 1e-12


@pytest.mark.parametrize("gamma", [0.001, 0.05, 1, 17.5, 100])
def test_pure_shear_is_exactly_zero(gamma):
    J = grad_at(lambda p: [gamma * p[1], 0, 0], [0, 0, 0], 1)
    assert abs(oracle.q_of_grad(J)) <= 1e-12 * max(1, gamma * gamma)


@pytest.mark.parametrize("w", [0.01, 0.5, 3])
def test_solid_body_rotation_is_omega_squared(w):
    J = grad_at(lambda p: [-w * p[1], w * p[0], 0], [0, 0, 0], 1)
    assert abs(oracle.q_of_grad(J) - w * w) <= 1e-10 * max(1, w * w)


def test_q_is_a_frame_invariant():
    w = 0.25
    qz = oracle.q_of_grad(grad_at(lambda p: [-w * p[1], w * p[0], 0], [0, 0, 0], 1))
    qx = oracle.q_of_grad(grad_at(lambda p: [0, -w * p[2], w * p[1]], [0, 0, 0], 1))
    assert abs(qz - qx) <= 1e-12


def test_stencil_converges_at_second_order():
    k, A = 0.3, 1.0

    def u(p):
        return [A * math.sin(k * p[0]) * math.cos(k * p[1]), -A * math.cos(k * p[0]) * math.sin(k * p[1]), 0]

    def exact(p):
        return (A * k) ** 2 * (math.sin(k * p[0]) ** 2 * math.sin(k * p[1]) ** 2
                               - math.cos(k * p[0]) ** 2 * math.cos(k * p[1]) ** 2)

    p = [0.7, 1.3, 2.1]
    assert abs(exact(p)) > 1e-3
    errs = [abs(oracle.q_of_grad(grad_at(u, p, h)) - exact(p)) for h in (0.4, 0.2, 0.1)]
    for a, b in zip(errs, errs[1:]):
        assert 3.2 < a / b < 4.8


def test_normalised_threshold_is_scale_free():
    w, D, U = 0.1, 16, 0.05
    q1 = oracle.q_of_grad(grad_at(lambda p: [-w * p[1], w * p[0], 0], [0, 0, 0], 1))
    q2 = oracle.q_of_grad(grad_at(lambda p: [-2 * w * p[1], 2 * w * p[0], 0], [0, 0, 0], 1))
    assert abs(q2 / q1 - 4) <= 1e-9
    assert abs((q1 / (U / D) ** 2) / (q2 / (2 * U / D) ** 2) - 1) <= 1e-9


def _mac(u):
    """(nz, ny, nx, 3) velocity -> (nz, ny, nx, 4) [rho = 1, u] in f32."""
    m = np.ones(u.shape[:3] + (4,), np.float32)
    m[..., 1:] = u
    return m


def _q_numpy(mac):
    """qAt in numpy f32, operation for operation."""
    u = mac[..., 1:].astype(np.float32)
    half = np.float32(0.5)
    J = [None] * 3  # J[j][..., i] = du_i/dx_j; the x axis is the last array axis
    for j, ax in enumerate((2, 1, 0)):
        J[j] = (np.roll(u, -1, axis=ax) - np.roll(u, 1, axis=ax)) * half
    s2 = np.zeros(u.shape[:3], np.float32)
    om2 = np.zeros(u.shape[:3], np.float32)
    for i in range(3):
        for j in range(3):
            a, b = J[j][..., i], J[i][..., j]
            S, O = half * (a + b), half * (a - b)
            s2 = s2 + S * S
            om2 = om2 + O * O
    return half * (om2 - s2)


def test_lattice_stencil_matches_numpy_bit_for_bit():
    rng = np.random.default_rng(7)
    u = (rng.standard_normal((6, 10, 8, 3)) * 0.03).astype(np.float32)
    mac = _mac(u)
    assert np.array_equal(oracle.q_cells(mac), _q_numpy(mac))


def test_lattice_shear_is_zero_and_rotation_is_positive():
    n = 16
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    shear = np.stack([0.002 * y, 0 * y, 0 * y], -1).astype(np.float32)
    q = oracle.q_cells(_mac(shear))
    # exact zero away from the periodic seam in y
    assert np.all(q[:, 1:-1, :] == 0)
    w = 0.003
    rot = np.stack([-w * (y - n / 2), w * (x - n / 2), 0 * x], -1).astype(np.float32)
    q = oracle.q_cells(_mac(rot))[:, 1:-1, 1:-1]
    assert np.allclose(q, w * w, rtol=1e-4)


def test_taylor_green_lattice_q_matches_analytic():
    n, A = 64, 0.05
    k = 2 * np.pi / n
    x = np.broadcast_to(np.arange(n)[None, None, :], (4, n, n)).astype(np.float64)
    y = np.broadcast_to(np.arange(n)[None, :, None], (4, n, n)).astype(np.float64)
    u = np.stack([A * np.sin(k * x) * np.cos(k * y), -A * np.cos(k * x) * np.sin(k * y), 0 * x], -1)
    q = oracle.q_cells(_mac(u.astype(np.float32)))
    exact = (A * k) ** 2 * (np.sin(k * x) ** 2 * np.sin(k * y) ** 2 - np.cos(k * x) ** 2 * np.cos(k * y) ** 2)
    # centred differences scale Q by sinc-like factors of order (k h)^2 / 6
    assert np.max(np.abs(q - exact)) <= 0.01 * (A * k) ** 2


def _block_q_numpy(q, rb, lead):
    nz, ny, nx = q.shape
    nb = (nx // rb, ny // rb, nz // rb)
    out = np.zeros(nb[::-1], np.float32)
    for bz in range(nb[2]):
        for by in range(nb[1]):
            for bx in range(nb[0]):
                idx = []
                for b in (bx, by, bz):
                    lo = np.float32(b * rb) - np.float32(lead)
                    hi = lo + np.float32(rb) + np.float32(2) * np.float32(lead)
                    idx.append(np.arange(int(np.floor(lo)), int(np.ceil(hi))))
                sub = q[np.ix_(idx[2] % nz, idx[1] % ny, idx[0] % nx)]
                out[bz, by, bx] = sub.max()
    return out.reshape(-1)


def _vortex_mac(dims, seed=3):
    """A periodic field with a few vortex cores and noise, [rho, u] f32."""
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    u = np.zeros((nz, ny, nx, 3))
    for _ in range(3):
        cx, cy, cz = rng.uniform(0, nx), rng.uniform(0, ny), rng.uniform(0, nz)
        w = rng.uniform(0.005, 0.02)
        dx = (x - cx + nx / 2) % nx - nx / 2
        dy = (y - cy + ny / 2) % ny - ny / 2
        dz = (z - cz + nz / 2) % nz - nz / 2
        g = np.exp(-(dx * dx + dy * dy + dz * dz) / 8.0)
        u[..., 0] += -w * dy * g
        u[..., 1] += w * dx * g
    u += rng.standard_normal(u.shape) * 1e-4
    u[..., 0] += 0.03
    return _mac(u.astype(np.float32))


@pytest.mark.parametrize("lead", [0.0, 0.5, 1.25, 3.0])
def test_block_max_over_the_dilated_box(lbm, lead):
    dims, rb = (24, 16, 20), 4
    c = lbm.amr3d_config(19, dims, refine="box", rb=rb, tau=0.6)
    mac = _vortex_mac(dims)
    o = oracle.Amr3D(c, fp32=True)
    o.seed(mac.reshape(-1, 4).astype(np.float64))
    got = o.block_q(lead)
    want = _block_q_numpy(_q_numpy(mac), rb, lead)
    assert np.array_equal(got, want)
    # the dilation never lowers a block's max
    if lead:
        assert np.all(got >= o.block_q(0.0))


def test_q_config_refusals(lbm):
    # a field criterion on a static set is refused, as main-3d.js refuses it
    c = lbm.amr3d_config(19, (16, 16, 16), refine="body", rb=4, tau=0.6, q_abs=1e-5, has_body=1,
                         use_bounceback=1, body=dict(shape="sphere", centre=(8, 8, 8), a=3))
    with pytest.raises(lbm.LbmError):
        lbm.Amr3D(c)
    for bad in (dict(q_abs=-1.0), dict(q_abs=float("nan")), dict(q_lead=-0.5), dict(q_hyst=float("inf"))):
        kw = dict(q_abs=1e-5, dynamic=1)
        kw.update(bad)
        c = lbm.amr3d_config(19, (16, 16, 16), refine="body", rb=4, tau=0.6, has_body=1, use_bounceback=1,
                             body=dict(shape="sphere", centre=(8, 8, 8), a=3), **kw)
        with pytest.raises(lbm.LbmError):
            lbm.Amr3D(c)
