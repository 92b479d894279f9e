"""The z-slab exchange on the host, as the ranks run it: 2 and 3 gloo ranks
(one process each, 127.0.0.1), each holding a slab of a random population
field between ghost planes, exchange the populations that cross their z
faces with getting_air_b200.slab.exchange (downward to the rank below,
upward to the rank above, periodic ring) and pull-stream their planes. The
gathered result must equal the whole field streamed periodically, bit for
bit; the FP64 sum and max over ranks must be the serial ones.

The crossing populations are selected here as the library selects them (the
ez = -1 directions of the first plane, ez = +1 of the last, in ascending
direction order), so this checks the plumbing -- slab bounds, ring order,
send/receive pairing and tags -- that the GPU path shares.
"""
import importlib.util
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _slab_module():
    spec = importlib.util.spec_from_file_location("slab_under_test", ROOT / "getting-air_b200" / "slab.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _tables(q):
    sys.path.insert(0, str(ROOT))
    import oracle
    return oracle.tables(q)


def _stream(f, t, dims, ghosts=False):
    """Pull streaming of Q x (nz, ny, nx) planes; periodic in x, y, and in z
    unless the z neighbours come from ghost planes (first and last plane)."""
    q = f.shape[0]
    out = np.empty_like(f)
    for i in range(q):
        g = np.roll(f[i], shift=(int(t["ex"][i]), int(t["ey"][i])), axis=(2, 1))
        out[i] = np.roll(g, shift=int(t["ez"][i]), axis=0)
    return out[:, 1:-1] if ghosts else out


def _rank_main(rank, world, port, q, out):
    import datetime
    import os
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    slab = _slab_module()
    t = _tables(q)
    nx, ny, nz = 5, 4, 11
    rng = np.random.default_rng(1234)            # the same global field on every rank
    glob = rng.standard_normal((q, nz, ny, nx))
    z0, k = slab.split(nz, world)[rank]
    local = np.zeros((q, k + 2, ny, nx))
    local[:, 1:-1] = glob[:, z0:z0 + k]
    down = [i for i in range(q) if t["ez"][i] == -1]
    up = [i for i in range(q) if t["ez"][i] == 1]
    send_lo = torch.tensor(local[down, 1])        # leaves through the bottom face
    send_hi = torch.tensor(local[up, k])          # leaves through the top face
    recv_lo, recv_hi = torch.empty_like(send_hi), torch.empty_like(send_lo)
    slab.exchange(send_lo, send_hi, recv_lo, recv_hi, rank, world)
    local[up, 0] = recv_lo.numpy()                # the slab below's upward populations
    local[down, k + 1] = recv_hi.numpy()          # the slab above's downward populations
    mine = _stream(local, t, None, ghosts=True)
    total = slab._sum_over_ranks(np.array([float(rank + 1), 0.5]), world)
    biggest = slab._max_over_ranks(float(rank) * 2.0, world)
    parts = [None] * world
    dist.all_gather_object(parts, (z0, mine))
    dist.destroy_process_group()
    if rank == 0:
        whole = _stream(glob, t, None)
        ok = all(np.array_equal(m, whole[:, a:a + m.shape[1]]) for a, m in parts)
        out.put((ok, sorted(a for a, _ in parts), total.tolist(), biggest))


@pytest.mark.parametrize("world,q", [(2, 19), (3, 27)])
def test_gloo_ranks_exchange_slab_halos(world, q):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q, out)) for r in range(world)]
    for p in procs:
        p.start()
    ok, starts, total, biggest = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slab = _slab_module()
    assert ok
    assert starts == [z0 for z0, _ in slab.split(11, world)]
    assert total == [sum(range(1, world + 1)), 0.5 * world]
    assert biggest == 2.0 * (world - 1)


def test_split_and_ring():
    slab = _slab_module()
    assert slab.split(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert slab.neighbours(0, 3) == (2, 1) and slab.neighbours(2, 3) == (1, 0)
    with pytest.raises(ValueError):
        slab.split(2, 3)
