"""The headless views' rules on the CPU oracle (common_d3_tree_sample.wgsl,
common_d3_resample.wgsl, common_d3_render_slice.wgsl).

* a volume at h = 1 aligned to the origin is a copy of the L0 field (the
  reference's own check of the resample);
* the finest level wins: voxels inside a refined block at h = 1/2 are the
  tile's interior cells one to one, never a ring cell; outside they repeat
  the L0 cell, and the level map says which;
* the slice picture: quarter turns are rotations of the image, the signed
  ramps put positive normal velocity and counter-clockwise rotation on the
  warm side, a uniform field is one colour;
* the PNG writer round-trips.
"""
import importlib
import math

import numpy as np
import pytest

import oracle

GH = 2


def field(dims, seed=0):
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims))
    mac = np.empty((n, 4), np.float32)
    mac[:, 0] = 1 + 0.01 * rng.standard_normal(n)
    mac[:, 1:] = 0.05 * rng.standard_normal((n, 3))
    return mac


def hierarchy(dims, rb, refined, seed=1):
    """A level-1 pool over the listed blocks: interior cells carry a value
    keyed to the global fine index, ring cells NaN."""
    nb = [d // rb for d in dims]
    fb = 2 * rb + 2 * GH
    block_slot = -np.ones(int(np.prod(nb)), np.int32)
    for s, (bx, by, bz) in enumerate(refined):
        block_slot[(bz * nb[1] + by) * nb[0] + bx] = s
    macp = np.full((len(refined), fb, fb, fb, 4), np.nan, np.float32)
    for s, (bx, by, bz) in enumerate(refined):
        for fz in range(2 * rb):
            for fy in range(2 * rb):
                for fx in range(2 * rb):
                    gx, gy, gz = bx * 2 * rb + fx, by * 2 * rb + fy, bz * 2 * rb + fz
                    key = (gz * 2 * dims[1] + gy) * 2 * dims[0] + gx
                    macp[s, fz + GH, fy + GH, fx + GH] = (1.0 + key * 1e-6, key * 1e-5, -key * 1e-5, 0.5)
    return block_slot, macp.reshape(-1, 4), fb


def test_unit_volume_is_a_copy_of_l0():
    dims = (12, 8, 6)
    mac = field(dims)
    out, lvl = oracle.tree_resample(mac, dims, (0, 0, 0), dims, (1, 1, 1))
    assert np.array_equal(out[:, :3], mac[:, 1:]) and np.array_equal(out[:, 3], mac[:, 0])
    assert not lvl.any()
    # a shifted origin wraps periodically
    out2, _ = oracle.tree_resample(mac, dims, (3, 0, 0), dims, (1, 1, 1))
    m = mac.reshape(dims[2], dims[1], dims[0], 4)
    assert np.array_equal(out2.reshape(dims[2], dims[1], dims[0], 4)[..., 3], np.roll(m[..., 0], -3, axis=2))


def test_finest_level_wins_and_never_reads_a_ring():
    dims, rb = (16, 8, 8), 4
    refined = [(1, 0, 0), (2, 1, 1)]
    mac = field(dims, 2)
    bs, macp, fb = hierarchy(dims, rb, refined)
    shape = tuple(2 * d for d in dims)
    out, lvl = oracle.tree_resample(mac, dims, (-0.25, -0.25, -0.25), shape, (0.5, 0.5, 0.5), levels=1, macp=macp,
                                    block_slot=bs, rb=rb, fb=fb)
    assert np.isfinite(out).all()
    out = out.reshape(shape[2], shape[1], shape[0], 4)
    lvl = lvl.reshape(shape[2], shape[1], shape[0])
    m = mac.reshape(dims[2], dims[1], dims[0], 4)
    for gz in range(shape[2]):
        for gy in range(shape[1]):
            for gx in range(shape[0]):
                b = (gx // (2 * rb), gy // (2 * rb), gz // (2 * rb))
                if b in refined:
                    key = (gz * 2 * dims[1] + gy) * 2 * dims[0] + gx
                    assert lvl[gz, gy, gx] == 1
                    assert out[gz, gy, gx, 0] == np.float32(key * 1e-5)
                else:
                    assert lvl[gz, gy, gx] == 0
                    assert np.array_equal(out[gz, gy, gx, :3], m[gz // 2, gy // 2, gx // 2, 1:])


def test_slice_quarter_turns_rotate_the_picture():
    dims = (12, 10, 6)
    mac = field(dims, 3)
    kw = dict(u_scale=0.1, v_scale=0.05)
    for mode in (0, 1, 2):
        imgs = {}
        for rot in range(4):
            a, b = dims[0], dims[1]
            w, h = (a, b) if rot % 2 == 0 else (b, a)
            imgs[rot] = oracle.tree_slice(mac, dims, 2, 3, mode, rot, w, h, **kw)
        for rot in range(1, 4):
            assert np.array_equal(imgs[rot], np.rot90(imgs[0], -rot)), (mode, rot)


def test_slice_signed_ramps():
    dims = (8, 8, 8)
    n = 512
    mac = np.zeros((n, 4), np.float32)
    mac[:, 0] = 1
    mac[:, 3] = 0.02  # +z velocity: the normal of a z slice
    img = oracle.tree_slice(mac, dims, 2, 4, 2, 0, 8, 8, 0.05, 0.01)
    assert (img == img[0, 0]).all() and img[0, 0, 0] > img[0, 0, 2]  # warm
    mac[:, 3] = -0.02
    img = oracle.tree_slice(mac, dims, 2, 4, 2, 0, 8, 8, 0.05, 0.01)
    assert img[0, 0, 2] > img[0, 0, 0]  # cool
    # solid-body rotation about z, counter-clockwise: positive vorticity
    z, y, x = np.meshgrid(np.arange(8), np.arange(8), np.arange(8), indexing="ij")
    w = 0.002
    mac = np.zeros((8, 8, 8, 4), np.float32)
    mac[..., 0] = 1
    mac[..., 1] = -w * (y - 3.5)
    mac[..., 2] = w * (x - 3.5)
    img = oracle.tree_slice(mac.reshape(-1, 4), dims, 2, 4, 1, 0, 8, 8, 0.05, 0.004)
    inner = img[2:6, 2:6]
    assert (inner[..., 0] > inner[..., 2]).all()


def test_png_round_trip(lbm):
    image = importlib.import_module("getting_air_b200.image")
    rng = np.random.default_rng(0)
    img = rng.integers(0, 256, (7, 5, 4), dtype=np.uint8)
    data = image.png_bytes(img)
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    assert np.array_equal(image.read_png(data), img)
