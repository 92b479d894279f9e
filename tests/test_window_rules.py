"""The moving window's host rules (CPU).

The scalar maps follow tools/test-d3-window.js: identity on an unwindowed
axis, nearest image within half a period, the body held in its anchor cell at
every position it reaches, windowCoord a bijection of the buffer onto [0, n),
a zero offset at the anchor, and per-axis vector forms. Then the refusals
main-3d.js makes before a windowed run starts, and two oracle properties of a
windowed step: it is bit-identical to the unwindowed step while the body sits
in its anchor cell, and shifting the body (with the field) along the window
axis shifts the result -- the sponge follows the body.
"""
import math

import numpy as np
import pytest

import oracle


def test_window_spec_parsing(lbm):
    assert lbm.window_axes("x") == (1, 0, 0)
    assert lbm.window_axes("zy") == (0, 1, 1)
    assert lbm.window_axes("xyz") == (1, 1, 1)
    assert lbm.window_axes("all") == (1, 1, 1)
    assert lbm.window_axes("0") == (0, 0, 0)
    assert lbm.window_axes("none") == (0, 0, 0)
    assert lbm.window_axes(None) == (0, 0, 0)
    for bad in ("w", "xq"):
        with pytest.raises(ValueError, match="expected some of xyz"):
            lbm.window_axes(bad)


def test_every_map_is_the_identity_without_a_window():
    for v in (-7.25, 0.0, 3.5, 191.0, 1e6):
        assert oracle.win_wrap_delta(v, 0) == v
        assert oracle.win_coord(v, 0, 0) == v
        assert oracle.win_wrap_position(v, 0) == v
        assert oracle.win_offset(v, 17, 0) == 0
    assert oracle.win_wrap_delta(5, -192) == 5


def test_wrap_delta_takes_the_nearest_image():
    n = 192
    for d, want in ((10, 10), (-10, -10), (191, -1), (-191, 1), (200, 8), (-200, -8), (95.5, 95.5), (96.5, -95.5)):
        assert oracle.win_wrap_delta(d, n) == want
    for d in np.linspace(-600, 600, 241):
        assert abs(oracle.win_wrap_delta(d, n)) <= n / 2 + 1e-9
    # the half period: round half to even, either equidistant image
    assert abs(oracle.win_wrap_delta(96, n)) == 96


def test_the_window_holds_the_body_at_the_anchor():
    n, anchor = 192, 168
    c, v = 168.3, 0.37
    for k in range(2000):
        off = oracle.win_offset(c, anchor, n)
        w = oracle.win_coord(c, off, n)
        assert anchor <= w < anchor + 1, k
        c = oracle.win_wrap_position(c + v, n)


def test_window_coord_is_a_bijection_of_the_buffer():
    n = 48
    for off in (-100, -17, 0, 5, 47, 48, 131):
        seen = set()
        for b in range(n):
            w = oracle.win_coord(b, off, n)
            assert 0 <= w < n and w == int(w) and w not in seen
            seen.add(w)
        assert len(seen) == n


def test_offset_is_zero_at_the_anchor():
    n, anchor = 192, 40
    for frac in (0.0, 0.25, 0.5, 0.999):
        assert oracle.win_offset(anchor + frac, anchor, n) == 0
    for b in (0, 37, 191):
        assert oracle.win_coord(b, 0, n) == b


def test_wrap_position_from_either_side():
    n = 64
    assert oracle.win_wrap_position(64.25, n) == 0.25
    assert oracle.win_wrap_position(-0.25, n) == 63.75
    assert oracle.win_wrap_position(-64.5, n) == 63.5
    assert oracle.win_wrap_position(10, n) == 10


def test_vector_forms_are_per_axis():
    wrap = (192, 0, 72)
    assert [oracle.win_wrap_delta(d, n) for d, n in zip((189, 189, 69), wrap)] == [-3, 189, -3]
    assert [oracle.win_offset(10.5, 4, n) for n in wrap] == [6, 0, 6]
    assert [oracle.win_wrap_position(c, n) for c, n in zip((200, 200, 80), wrap)] == [8, 200, 8]


def _wcfg(lbm, dims=(48, 24, 24), **kw):
    base = dict(tau=0.6, has_body=1, use_bounceback=1, sponge_w=4.0, sponge_u=(0.0, 0.0, 0.0),
                body=dict(shape="sphere", centre=(20.25, 11.5, 12.0), a=4.0, v=(0.1, 0.0, 0.0)), window="x")
    base.update(kw)
    return lbm.config_from(19, dims, **base)


def test_anchor_defaults_to_the_body_cell(lbm):
    c = _wcfg(lbm)
    assert tuple(c.window) == (1, 0, 0)
    assert tuple(c.win_anchor) == (20, 11, 12)


@pytest.mark.parametrize("bad,msg", [
    (dict(has_body=0), "body to follow"),
    (dict(wall=(1, 0, 0)), "periodic axis"),
    (dict(sponge_w=0.0), "sponge"),
])
def test_window_refusals(lbm, bad, msg):
    c = _wcfg(lbm, **bad)
    with pytest.raises(lbm.LbmError, match=msg):
        lbm.Solver(c)


def test_window_refused_in_2d_and_batches(lbm):
    c = lbm.config_from(9, (64, 32, 1), tau=0.6, has_body=1, sponge_w=4.0,
                        body=dict(shape="ellipse", centre=(20.0, 16.0, 0.0), a=4.0, b=2.0), window=(1, 0, 0),
                        win_anchor=(20, 16, 0))
    with pytest.raises(lbm.LbmError, match="3D"):
        lbm.Solver(c)
    with pytest.raises(lbm.LbmError, match="dense sessions"):
        lbm.Batch([_wcfg(lbm)])


def _seed(dims, seed=1):
    n = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    mac = np.zeros((n, 4))
    mac[:, 0] = 1.0 + 1e-3 * rng.standard_normal(n)
    mac[:, 1:] = 0.01 * rng.standard_normal((n, 3))
    return mac


def test_windowed_step_starts_bit_identical(lbm):
    dims = (48, 24, 24)
    mac = _seed(dims)
    out = []
    for win in ("x", "0"):
        c = _wcfg(lbm, window=win, win_anchor=(20, 11, 12))
        f = oracle.init_eq(19, mac, fp32=True)
        f, m, F = oracle.run(c, f, 3, fp32=True)
        out.append((f, m, F))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][2], out[1][2])


def test_windowed_step_is_translation_invariant_along_the_window(lbm):
    # the body and the field shifted by k cells along x with the same anchor:
    # the sponge band follows the body, so the result is the shifted result,
    # here with the shifted body straddling the periodic seam
    dims = (48, 24, 24)
    mac = _seed(dims, 4).reshape(dims[2], dims[1], dims[0], 4)
    k = 25
    res = []
    for shift in (0, k):
        c = _wcfg(lbm, body=dict(shape="sphere", centre=(20.25 + shift, 11.5, 12.0), a=4.0, v=(0.1, 0.0, 0.0)),
                  win_anchor=(20, 11, 12))
        m = np.roll(mac, shift, axis=2).reshape(-1, 4)
        f = oracle.init_eq(19, m, fp32=True)
        f, mm, F = oracle.run(c, f, 3, fp32=True)
        res.append((f.reshape(19, dims[2], dims[1], dims[0]), F))
    assert np.array_equal(np.roll(res[0][0], k, axis=3), res[1][0])
    assert np.allclose(res[0][1], res[1][1], rtol=1e-9, atol=1e-12)
