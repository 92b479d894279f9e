"""Host rules of the 3D hierarchy (CPU): the refinement predicates against
the oracle's restatement, resolveSource against the independent global-fine
route (tools/test-d3-amr.js's own check), pool geometry, and the refusals
lbm_amr3d_create makes before touching the GPU.
"""
import itertools

import numpy as np
import pytest

import oracle

GHOST = 2


@pytest.mark.parametrize("mode", ["body", "box", "bar", "slab", "all"])
def test_refine_sets_match_oracle(lbm, mode):
    c = lbm.amr3d_config(19, (48, 32, 40), refine=mode, tau=0.6, has_body=1, use_bounceback=1,
                         body=dict(shape="sphere", centre=(17.3, 15.8, 20.2), a=5.5))
    want = lbm.amr3d_refine_blocks(c)
    o = oracle.Amr3D(c)
    assert np.array_equal(o.block_slot >= 0, want > 0)
    # slots in ascending block id
    assert np.array_equal(o.slot_to_block, np.flatnonzero(want))
    assert o.slots == int(want.sum()) > 0


def test_body_refinement_covers_the_margin_at_cell_granularity(lbm):
    # every L0 cell within `margin` of the body sits in a refined block
    # (checkGeometryCoverage), on a rotated rounded box the corner sample
    # of a block would miss
    body = dict(shape="roundbox", centre=(24.2, 16.3, 15.9), a=7.0, b=2.0, c=1.2, r=0.3,
                quat=(0.9238795, 0.0, 0.3826834, 0.0))
    c = lbm.amr3d_config(19, (48, 32, 32), refine="body", margin=2.0, tau=0.6, has_body=1,
                         use_bounceback=1, body=body)
    want = lbm.amr3d_refine_blocks(c).reshape(8, 8, 12)
    b = c.root.body
    q = np.array([b.qw, b.qx, b.qy, b.qz], float)
    z, y, x = np.meshgrid(np.arange(32), np.arange(32), np.arange(48), indexing="ij")
    d = np.stack([x - b.cx, y - b.cy, z - b.cz], -1).astype(float)
    # world -> body: rotate by the conjugate quaternion
    w, u = q[0], -q[1:]
    pb = d + 2 * np.cross(u, np.cross(u, d) + w * d)
    h = np.array([b.a - b.r, b.b - b.r, b.c - b.r])
    qd = np.abs(pb) - h
    phi = np.linalg.norm(np.maximum(qd, 0), axis=-1) + np.minimum(qd.max(-1), 0) - b.r
    near = phi <= 2.0
    blocks = want[z // 4, y // 4, x // 4]
    assert near.sum() > 0
    assert (blocks[near] > 0).all()


def test_pool_geometry(lbm):
    c = lbm.amr3d_config(19, (16, 16, 16), refine="all", tau=0.8)
    assert 2 * c.rb + 2 * GHOST == 12
    c.rb = 5
    with pytest.raises(lbm.LbmError):
        lbm.Amr3D(c)  # 16 is not a multiple of 5


def to_global(rb, b, local):
    return [b[a] * 2 * rb + (local[a] - GHOST) for a in range(3)]


def from_global(rb, dims, g):
    n = [2 * d for d in dims]
    w = [((g[a] % n[a]) + n[a]) % n[a] for a in range(3)]
    blk = [w[a] // (2 * rb) for a in range(3)]
    return blk, [w[a] - blk[a] * 2 * rb + GHOST for a in range(3)]


def test_resolve_source_agrees_with_global_fine_route(lbm):
    rb, dims = 4, (16, 12, 8)
    nb = [d // rb for d in dims]
    rng = np.random.default_rng(4)
    block_slot = np.where(rng.random(int(np.prod(nb))) < 0.5, 0, -1).astype(np.int32)
    block_slot[block_slot >= 0] = np.arange((block_slot >= 0).sum())
    fb = 2 * rb + 2 * GHOST
    e19 = [d for d in itertools.product((-1, 0, 1), repeat=3) if sum(map(abs, d)) <= 2]
    checked = 0
    for bid in np.flatnonzero(block_slot >= 0)[:6]:
        b = [bid % nb[0], (bid // nb[0]) % nb[1], bid // (nb[0] * nb[1])]
        for loc in itertools.product(range(GHOST, GHOST + 2 * rb), repeat=3):
            for e in e19:
                src = [loc[a] - e[a] for a in range(3)]
                slot, fx, fy, fz = lbm.resolve_source(rb, nb, block_slot, b, src)
                gb, gl = from_global(rb, dims, to_global(rb, b, src))
                if gb == b:
                    assert slot == -1 and [fx, fy, fz] == src
                else:
                    owner = block_slot[(gb[2] * nb[1] + gb[1]) * nb[0] + gb[0]]
                    if owner < 0:
                        assert slot == -2
                    else:
                        # a source resolved into a neighbour lands in that tile's interior
                        assert slot == owner and [fx, fy, fz] == gl
                        assert all(GHOST <= v < GHOST + 2 * rb for v in (fx, fy, fz))
                checked += 1
    assert checked > 10000


def test_invalid_configs_are_refused_before_any_gpu_work(lbm):
    c = lbm.amr3d_config(9, (16, 16, 1), refine="all", tau=0.8)
    with pytest.raises(lbm.LbmError, match="D3Q19 or D3Q27"):
        lbm.Amr3D(c)
    c = lbm.amr3d_config(19, (16, 16, 16), refine="body", tau=0.8)
    with pytest.raises(lbm.LbmError, match="needs a body"):
        lbm.Amr3D(c)
    c = lbm.amr3d_config(19, (16, 16, 16), refine="all", tau=1.0)
    with pytest.raises(lbm.LbmError, match="tau = 1"):
        lbm.Amr3D(c)
    c = lbm.amr3d_config(19, (16, 16, 16), refine="all", tau=0.8, storage="fp16")
    with pytest.raises(lbm.LbmError):
        lbm.Amr3D(c)


def test_oracle_amr3d_is_conservative_in_fp64():
    """The restatement itself: with no body and no forcing, the explode /
    coalesce interface moves mass and momentum between the levels without
    creating them -- after the one-time start-up offset (the reference's
    readInterfaceDiag observation), the L0 totals stay put."""
    import math
    import sys
    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent))
    from conftest import load_package
    lbm = load_package()
    N = 16
    c = lbm.amr3d_config(19, (N, N, N), refine="bar", tau=0.8)
    o = oracle.Amr3D(c)
    k = 2 * math.pi / N
    z, y, x = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    u0 = 0.04
    ux = u0 * (np.sin(k * z) + np.cos(k * y))
    uy = u0 * (np.sin(k * x) + np.cos(k * z))
    uz = u0 * (np.sin(k * y) + np.cos(k * x))
    mac = np.stack([1 - 1.5 * (ux ** 2 + uy ** 2 + uz ** 2), ux, uy, uz], -1).reshape(-1, 4)
    o.seed(mac.astype(np.float32).astype(np.float64))
    o.step(2)
    m1 = o.read()[1]
    o.step(10)
    m2 = o.read()[1]
    tot = lambda m: np.array([np.sum(m[:, 0] - 1), *np.sum(m[:, :1] * m[:, 1:4], 0)])
    d = tot(m2) - tot(m1)
    assert abs(d[0]) < 1e-4 and np.abs(d[1:]).max() < 1e-5, d
