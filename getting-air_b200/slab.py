"""One dense 3D domain split into z-slabs, one per GPU (one process per GPU).

The reference steps one domain on one device; this is the multi-GPU form of
its dense step. Each rank holds planes [z0, z0 + nz) of the domain in a slab
session (lbm_create_slab): the physics is the whole domain's, and only the
populations that cross a z face move between ranks -- 5 of D3Q19's 19 (9 of
D3Q27's 27) per face per step, one plane each. Per step:

    pack      (the slab's first plane's downward and last plane's upward
               populations into two device buffers)
    exchange  (downward buffer to the rank below, upward to the rank above;
               z is periodic, so the ranks form a ring) over torch.distributed
               point-to-point: NCCL over NVLink between GPUs
    unpack    (the neighbours' buffers into the ghost planes)
    step

The body force and the conserved totals are each slab's share, summed in
FP64 over the ranks (all_reduce). Cell by cell the result is the one-domain
step's, bit for bit; the summed force differs from the one-domain sum only
in the order of its FP64 additions.
"""
from __future__ import annotations

import numpy as np


def split(nz: int, world: int) -> list[tuple[int, int]]:
    """(z0, planes) of each rank: nz planes in world contiguous slabs, the
    first nz % world one plane deeper."""
    if world < 1 or nz < world:
        raise ValueError(f"cannot split {nz} planes over {world} ranks")
    base, extra = divmod(nz, world)
    out, z0 = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((z0, k))
        z0 += k
    return out


def neighbours(rank: int, world: int) -> tuple[int, int]:
    """(below, above): z is periodic, so the slabs form a ring."""
    return (rank - 1) % world, (rank + 1) % world


def exchange(send_lo, send_hi, recv_lo, recv_hi, rank: int, world: int, group=None):
    """Sends send_lo to the rank below (into its recv_hi) and send_hi to the
    rank above (into its recv_lo), receiving the same from them. The tensors
    live where the backend moves them (CUDA for NCCL, host for gloo). With
    one rank the slab is its own neighbour on both sides."""
    if world == 1:
        recv_hi.copy_(send_lo)
        recv_lo.copy_(send_hi)
        return
    import torch.distributed as dist
    below, above = neighbours(rank, world)
    # tag 0: downward (my send_lo -> below's recv_hi); tag 1: upward. Between
    # one pair of ranks the operations match in the order posted, which is
    # the same order on every rank.
    ops = [dist.P2POp(dist.isend, send_lo, below, group, 0), dist.P2POp(dist.irecv, recv_hi, above, group, 0),
           dist.P2POp(dist.isend, send_hi, above, group, 1), dist.P2POp(dist.irecv, recv_lo, below, group, 1)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()


class SlabDomain:
    """This rank's slab of the domain `cfg` describes, on the current GPU.

    `step(n)` runs n exchange-and-step rounds; `forces()` and `totals()`
    return the whole domain's values (every rank gets them)."""

    def __init__(self, lbm, cfg, rank: int, world: int, group=None):
        import torch
        self.lbm, self.rank, self.world, self.group = lbm, rank, world, group
        self.z0, self.nz = split(cfg.nz, world)[rank]
        self.solver = lbm.Solver(cfg, slab=(self.z0, self.nz))
        nb = self.solver.halo_bytes()
        self.bufs = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(4)]
        self.stream = torch.cuda.current_stream()
        self.solver.set_stream(self.stream.cuda_stream)

    def close(self):
        self.solver.close()

    def exchange(self):
        send_lo, send_hi, recv_lo, recv_hi = self.bufs
        self.solver.pack(send_lo.data_ptr(), send_hi.data_ptr())
        exchange(send_lo, send_hi, recv_lo, recv_hi, self.rank, self.world, self.group)
        self.solver.unpack(recv_lo.data_ptr(), recv_hi.data_ptr())

    def step(self, n: int = 1):
        for _ in range(n):
            self.exchange()
            self.solver.step(1)

    def forces(self) -> np.ndarray:
        return _sum_over_ranks(np.asarray(self.solver.forces(), np.float64), self.world, self.group)

    def totals(self) -> dict:
        t = self.solver.totals()
        s = _sum_over_ranks(np.array([t["mass"], t["px"], t["py"], t["pz"], t["nonfinite"]], np.float64),
                            self.world, self.group)
        lo = -_max_over_ranks(-t["rho_min"], self.world, self.group)
        hi = _max_over_ranks(t["rho_max"], self.world, self.group)
        um = _max_over_ranks(t["max_u"], self.world, self.group)
        return {"mass": s[0], "px": s[1], "py": s[2], "pz": s[3], "rho_min": lo, "rho_max": hi, "max_u": um,
                "nonfinite": s[4]}


def _device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def _sum_over_ranks(v: np.ndarray, world: int, group=None) -> np.ndarray:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor(v, dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def _max_over_ranks(x: float, world: int, group=None) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
