"""The benchmark's multi-rank plumbing on the host: two gloo ranks (the
contract's torchrun layout, one process per rank, 127.0.0.1 rendezvous).

* `barrier` and `max_over_ranks` give every rank the maximum over ranks;
* the reference arm runs on rank 0 only: rank 1 returns at once, without
  touching the oracle.
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import importlib.util
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    bench.barrier(world)
    got = bench.max_over_ranks(10.0 + 5.0 * rank, world)
    # the reference arm: only rank 0 works; rank 1 must return without the oracle
    ran_oracle = False
    if rank != 0:
        class Args:
            steps, warmup = 1, 3
        before = set(sys.modules)
        bench.run_reference(Args())
        ran_oracle = any(m == "oracle" or m.startswith("oracle.") for m in set(sys.modules) - before)
    bench.barrier(world)
    dist.destroy_process_group()
    out.put((rank, got, ran_oracle))


def test_two_gloo_ranks_agree_on_the_max_and_rank1_skips_the_reference():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    assert res[1][2] is False
