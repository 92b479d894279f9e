"""Benchmark of the dense lattice-Boltzmann hot path on B200.

Workload: D3Q19 dense flow past a pinned sphere, 256 x 128 x 128 cells,
sphere r = 16 at (96, 64, 64), inlet/sponge u = 0.05, tau = 0.56, Ladd
bounce-back with local rho_w, ALBC sponge (width 16) toward the freestream,
uniform Guo body force F_x = 1e-6, FP32 storage, drag/lift summed in FP64
every step. A "step" is one fused stream-collide-force pass over the whole
grid (4,194,304 lattice updates). Inputs are synthetic (uniform freestream
seed, as the reference's sphere scenario does); f is 2 x 319 MB, larger than
L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica of the workload on its
own GPU (weak scaling, no data-path collective); the timed region is
bracketed by a barrier and a device synchronize, and the reported time is
the maximum over ranks. `--impl reference` times the CPU restatement of the
reference's arithmetic (the reference itself is WGSL that cannot run here)
on this host's cores; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
BYTES_PER_LU = {("d3q19", "fp32"): 152, ("d3q19", "fp16"): 76, ("d3q19", "bf16"): 76,
                ("d3q27", "fp32"): 216, ("d3q27", "fp16"): 108, ("d3q27", "bf16"): 108}
DIMS = (256, 128, 128)


def load_package():
    if "getting_air_b200" in sys.modules:
        return sys.modules["getting_air_b200"]
    pkg = ROOT / "getting-air_b200"
    spec = importlib.util.spec_from_file_location("getting_air_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["getting_air_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def scenarios():
    """The scenario builders (pure Python: synthetic inputs from formulas),
    loaded from their file on their own, so that the reference arm, which
    runs the oracle alone, maps none of the product's native code."""
    name = "_lbm_scenarios"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, ROOT / "getting-air_b200" / "scenarios.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def workload(storage="fp32", dims=DIMS, n=32, q=19):
    return scenarios().sphere(n=n, dims=dims, u0=0.05, tau=0.56, q=q, bounceback=True,
                              force=(1e-6, 0.0, 0.0), storage=storage)


def config_key(storage="fp32"):
    """The workload's description; identical in both arms (no arm-specific keys)."""
    return {"workload": "D3Q19 dense sphere 256x128x128 r=16 tau=0.56 u0=0.05 bounce-back+sponge+Guo force, "
                        "FP64 drag/lift every step",
            "lattice": "D3Q19", "dims": list(DIMS), "cells": int(np.prod(DIMS)), "storage": storage,
            "l2": "inputs larger than L2 (2 x 319 MB f buffers), no flush"}


# ---- clocks ------------------------------------------------------------------

REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x40: "sw_thermal_slowdown",
           0x80: "hw_thermal_slowdown", 0x100: "hw_power_brake_slowdown", 0x2: "applications_clocks_setting"}


class ClockSampler:
    """Samples the SM clock and clock-event reasons of this rank's GPU via NVML."""

    def __init__(self, torch_dev: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(torch_dev).uuid)
            for i in range(pynvml.nvmlDeviceGetCount()):
                h = pynvml.nvmlDeviceGetHandleByIndex(i)
                u = pynvml.nvmlDeviceGetUUID(h)
                u = u.decode() if isinstance(u, bytes) else u
                if u.replace("GPU-", "") == uuid.replace("GPU-", ""):
                    self._h = h
            if self._h is None:
                self._h = pynvml.nvmlDeviceGetHandleByIndex(0)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._nv = pynvml
        except Exception as e:  # NVML missing: report no clocks rather than guess
            self.error = repr(e)

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(0.05)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._h is not None:
            self._t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


# ---- peaks / profiles -----------------------------------------------------------

def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel: str):
    """DRAM bytes per launch recorded from an ncu capture, if one is committed."""
    p = ROOT / "profiles" / f"{kernel}.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":", 1)[1])
    return None


# ---- distributed plumbing ----------------------------------------------------

def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """The maximum of x over the ranks (NCCL on the GPU, or gloo on the host)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- our arm -------------------------------------------------------------------

def time_device(lbm, wl, steps, warmup, world):
    """Device-resident throughput: K fused steps, CUDA events on the session stream."""
    import torch
    s = lbm.Solver.create(wl["q"], wl["dims"], **wl["kw"])
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        s.init_macro(wl["mac"])
        s.step(warmup)
        s.sync()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize()
        with ClockSampler(torch.cuda.current_device()) as clk:
            start.record(stream)
            s.step(steps)
            end.record(stream)
            torch.cuda.synchronize()
        barrier(world)
    total_ms = start.elapsed_time(end)
    # The stream runs one step kernel per step (each also sums the previous
    # step's force partials) and one force-sum launch after the last:
    # total / steps bounds the step kernel's mean duration from above.
    launch_ms = [total_ms / steps]
    forces = s.forces()
    totals = s.totals()
    s.close()
    return total_ms, launch_ms, clk.summary(), forces, totals


def time_e2e(lbm, wl, steps, warmup, world):
    """Through the C ABI with host buffers: upload the seed from pinned host
    memory, K steps each followed by a queued 48-byte device->host copy of
    that step's drag/lift into a pinned history buffer, and the final
    macroscopic field read back to host memory. Wall clock around it all."""
    import torch
    mac_host = torch.from_numpy(np.ascontiguousarray(wl["mac"], np.float32)).pin_memory()
    out_host = torch.empty_like(mac_host).pin_memory()
    hist = torch.zeros((steps, 6), dtype=torch.float64).pin_memory()
    mac_np, out_np = mac_host.numpy(), out_host.numpy()
    s = lbm.Solver.create(wl["q"], wl["dims"], **wl["kw"])
    s.init_macro(mac_np)
    s.step(warmup)
    s.sync()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.init_macro(mac_np)
    for k in range(steps):
        s.step(1)
        s.forces_async(hist[k].data_ptr())
    s.sync()
    s.read_mac(out=out_np)
    t1 = time.perf_counter()
    s.close()
    ms = max_over_ranks((t1 - t0) * 1e3, world)
    h2d = mac_np.nbytes / steps
    d2h = (out_np.nbytes + 6 * 8 * steps) / steps
    return ms, h2d, d2h


def time_batched(lbm, steps, warmup, world, plain_steps=20):
    """Batched form (512 D2Q9 domains, log-uniform 64^2..512^2, seeded) in one
    persistent graph-captured launch per step after autotuning the tile
    shape, against the plain form: the same domains as 512 dense sessions
    stepped one launch each."""
    import torch
    from getting_air_b200 import scenarios as sc
    doms = sc.batched_domains(count=512, seed=12345)
    w = lbm.lattice_tables(9)["w"]
    cfgs = [lbm.config_from(9, d["dims"], **d["kw"]) for d in doms]
    seeds = [sc.seed_domain(d, w) for d in doms]
    cells = sum(int(np.prod(d["dims"])) for d in doms)
    b = lbm.Batch(cfgs)
    for k, f0 in enumerate(seeds):
        b.write_f(k, f0)
    tune_ms = b.autotune(3)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    b.step(max(warmup, 34))   # builds the captured graphs of both buffer parities
    b.sync()
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    a.record(stream)
    b.step(steps)
    z.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(a.elapsed_time(z), world)
    tiling = b.tiling()
    b.close()
    batched = {"mlups": cells * steps * world / (ms * 1e-3) / 1e6, "ms_per_step": ms / steps,
               "domains": len(doms), "cells": cells, "tiling": {"threads": tiling[0], "cells_per_thread": tiling[1],
                                                              "ctas_per_sm": tiling[2]},
               "autotune_best_ms": tune_ms, "gbs": 72 * cells / (ms / steps * 1e-3) / 1e9,
               # the lean kernel takes every tile here; domains with a body
               # or a force region would add the general kernel's launch
               "launches_per_step": 1 + int(any(c.has_body for c in cfgs)), "graph_steps": 16}
    sols = []
    for cfg, f0 in zip(cfgs, seeds):
        s = lbm.Solver(cfg)
        s.write_f(f0)
        sols.append(s)
    for s in sols:
        s.step(warmup)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(plain_steps):
        for s in sols:
            s.step(1)
    torch.cuda.synchronize()
    pms = max_over_ranks((time.perf_counter() - t0) * 1e3, world)
    for s in sols:
        s.close()
    plain = {"mlups": cells * plain_steps * world / (pms * 1e-3) / 1e6, "ms_per_step": pms / plain_steps,
             "launches_per_step": len(doms), "timing": "host wall clock around device-synchronised loop"}
    return batched, plain


def time_amr(lbm, steps, warmup, world):
    """2D AMR cylinder (1024 x 256 root in 16 x 16 root blocks, r = 20 at
    (256, 128), u0 = 0.08, Re = 100, one 2:1 level by vorticity + geometry,
    refine every 16, drag/lift every macro-step). MLUPS counts the
    reference's cellUpdatesPerMacroStep (amr2d.mjs:558) at each step's
    topology."""
    import torch
    from getting_air_b200 import scenarios as sc
    s = sc.cylinder_amr(W=1024, H=256, r=20.0, centre=(256.0, 128.0), u0=0.08, re=100.0)
    cfg = lbm.amr2d_config(1024, 256, **s["kw"])
    a = lbm.Amr2D(cfg)
    stream = torch.cuda.Stream()
    a.set_stream(stream.cuda_stream)
    a.write_root(s["f"], s["vel"])
    a.step(max(warmup, 16))
    a.sync()
    updates = 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    ev0.record(stream)
    chunk = 16
    done = 0
    counts = []
    while done < steps:
        k = min(chunk, steps - done)
        a.step(k)
        done += k
        counts.append((k, a.cell_updates()))   # topology changes only at refine rounds
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    updates = sum(k * c for k, c in counts)
    f = a.forces()
    t = a.topology()
    a.close()
    return {"mlups": updates * world / (ms * 1e-3) / 1e6, "ms_per_macro_step": ms / steps,
            "cell_updates_per_macro_step": updates / steps, "active_tiles": int(len(t["active"])),
            "drag": f[0], "lift": f[1],
            "cd_startup_transient": 2 * f[0] / (s["u0"] ** 2 * 2 * s["r"]),
            "cd_note": f"after {max(warmup, 16) + steps} macro-steps from an impulsive start: a start-up transient, "
                       "not a settled Cd (settled cylinder drag is checked against the reference's recorded runs "
                       "by the physics tests)",
            "timing": "CUDA events around the macro-steps; topology readback between 16-step chunks"}


def time_amr3d(lbm, steps, warmup, world):
    """3D AMR sphere (sphere-amr-Re20-D16: D = 16 pinned sphere at (48, 64, 64)
    in 192 x 128 x 128, u0 = 0.05, Re = 20, the blocks within 2 cells of it
    refined, RB = 4). MLUPS counts L0 cells outside the refined blocks plus
    two substeps of every refined interior cell per macro-step."""
    import torch
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=16, u0=0.05, re=20)
    cfg = lbm.amr3d_config(19, s["dims"], refine="body", margin=2.0, **s["kw"])
    a = lbm.Amr3D(cfg)
    stream = torch.cuda.Stream()
    a.set_stream(stream.cuda_stream)
    a.init_macro(s["mac"])
    a.step(max(warmup, 3))
    a.sync()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    ev0.record(stream)
    a.step(steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    upd = a.cell_updates()
    f = a.forces()
    out = {"mlups": upd * steps * world / (ms * 1e-3) / 1e6, "ms_per_macro_step": ms / steps,
           "cell_updates_per_macro_step": upd, "tiles": a.slots,
           "cd_startup_transient": f[0] / (0.5 * 0.05 ** 2 * s["area"]),
           "cd_note": f"after {max(warmup, 3) + steps} macro-steps from an impulsive start: a start-up transient, "
                      "not the settled Cd (2.94 for this case, checked by the sphere-AMR physics test)",
           "timing": "CUDA events around the macro-steps (graph-launched), pool force every macro-step"}
    a.close()
    return out


def time_amr3d_served_request(lbm, steps, warmup):
    """The largest two-level AMR request of the served stream (a 180^3
    rounded box, RB = 4, blocks within 2 cells refined) stepped alone as a
    session: CUDA events around `steps` graph-launched macro-steps."""
    import torch
    from getting_air_b200 import scenarios as sc
    reqs = [r for r in sc.serving_stream(count=48, seed=2024, rate=200.0, amr_frac=0.25) if r["levels"] == 2]
    r = max(reqs, key=lambda x: int(np.prod(x["dims"])) * x["steps"])
    a = lbm.Amr3D(sc.serving_config(lbm, r))
    stream = torch.cuda.Stream()
    a.set_stream(stream.cuda_stream)
    a.init_macro(sc.uniform_macro(int(np.prod(r["dims"])), (0.05, 0.0, 0.0)))
    a.step(max(warmup, 3))
    a.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    a.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out = {"request": {"id": r["id"], "q": r["q"], "dims": list(r["dims"]), "body": r["kw"]["body"]["shape"]},
           "tiles": a.slots, "ms_per_macro_step": ms, "cell_updates_per_macro_step": a.cell_updates(),
           "mlups": a.cell_updates() / (ms * 1e-3) / 1e6}
    a.close()
    return out


# The served form admits the least work first, with about two of the largest
# (192^3) requests' worth of cells resident: enough to keep the GPU busy, so
# short requests do not share it with every long one. Measured on this
# stream (pipelined ticks): 7.7 GLUPS at p50 3.2 s, against 7.9 GLUPS at
# p50 8.8 s with no cap.
SERVE_RESIDENT_CELLS = 16 << 20


def time_served(lbm, world, count=48, budget_gb=48, policy="sjf", max_resident_cells=SERVE_RESIDENT_CELLS):
    """Serving: a seeded Poisson stream (200 req/s) of D3Q19/D3Q27 sphere or
    rounded-box solves, N^3 with N log-uniform in [32, 192], 500-2000 steps,
    a quarter of them two-level AMR solves (blocks near the body refined),
    admitted by HBM budget into one device arena and batched continuously.
    Latency = completion - arrival on the host clock. Against it, the plain
    form: the same requests one after another as single sessions (FIFO).
    Work = lattice updates (an AMR macro-step counts its L0 cells outside
    refined blocks plus two substeps of every fine cell)."""
    import torch
    from getting_air_b200 import scenarios as sc
    reqs = sc.serving_stream(count=count, seed=2024, rate=200.0, amr_frac=0.25)
    cfgs = {r["id"]: sc.serving_config(lbm, r) for r in reqs}

    def submit(srv, r):
        if r["levels"] == 2:
            srv.submit_amr3d(r["id"], cfgs[r["id"]], r["steps"])
        else:
            srv.submit(r["id"], cfgs[r["id"]], r["steps"])
    # warm the kernels of both lattices
    w = lbm.Server(1 << 30)
    for k, q in enumerate((19, 27)):
        w.submit(k, lbm.config_from(q, (32, 32, 32), **reqs[0]["kw"] | {"body": dict(shape="sphere", centre=(10, 16, 16), a=4)}), 4)
    while len(w.poll(4)) < 2 and w.stats()["resident"]:
        pass
    w.close()
    srv = lbm.Server(int(budget_gb * (1 << 30)))
    srv.set_policy(policy, max_resident_cells)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    nxt, done, lat = 0, {}, {}
    while len(done) < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt]["t"] <= now:
            submit(srv, reqs[nxt])
            nxt += 1
        st = srv.stats()
        if st["resident"] == 0 and st["queued"] == 0:
            if nxt < len(reqs):
                time.sleep(max(0.0, reqs[nxt]["t"] - (time.perf_counter() - t0)))
            continue
        for r in srv.poll(64):
            tdone = time.perf_counter() - t0
            done[r["id"]] = r
            lat[r["id"]] = tdone - reqs[r["id"]]["t"]
            srv.release(r["id"])
    total = time.perf_counter() - t0
    work = srv.stats()["lattice_updates"]
    srv.close()
    L = np.array(sorted(lat.values()))
    served = {"mlups": work / total / 1e6, "wall_s": total, "requests": len(reqs),
              "amr_requests": sum(r["levels"] == 2 for r in reqs),
              "lattice_updates": work, "p50_latency_ms": 1e3 * float(np.percentile(L, 50)),
              "p99_latency_ms": 1e3 * float(np.percentile(L, 99)), "budget_gb": budget_gb,
              "arrivals": "Poisson 200/s, seed 2024", "admission": f"{policy}, at most {max_resident_cells} resident cells",
              "timing": "host wall clock, first arrival to last completion"}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plat = []
    for r in reqs:
        now = time.perf_counter() - t0
        if now < r["t"]:
            time.sleep(r["t"] - now)
        s = lbm.Amr3D(cfgs[r["id"]]) if r["levels"] == 2 else lbm.Solver(cfgs[r["id"]])
        s.init_macro(sc.uniform_macro(int(np.prod(r["dims"])), (0.05, 0.0, 0.0)))
        s.step(r["steps"])
        s.forces()
        s.close()
        plat.append(time.perf_counter() - t0 - r["t"])
    ptotal = time.perf_counter() - t0
    P = np.array(plat)
    plain = {"mlups": work / ptotal / 1e6, "wall_s": ptotal, "p50_latency_ms": 1e3 * float(np.percentile(P, 50)),
             "p99_latency_ms": 1e3 * float(np.percentile(P, 99)),
             "timing": "host wall clock; requests one after another as single sessions"}
    return served, plain


ACCURACY_STEPS = 100


def packed_accuracy(lbm, steps=ACCURACY_STEPS):
    """Error of each storage form against the FP64 oracle on the headline
    workload itself (256 x 128 x 128), from the same f32 start: velocity and
    density relative L2 and drag after `steps` steps. (The same comparison,
    with its bounds, is a GPU test.)"""
    import oracle
    wl = workload("fp32")
    cfg = lbm.config_from(19, wl["dims"], **wl["kw"])
    f0 = oracle.init_eq(19, wl["mac"], fp32=True).astype(np.float32)
    t0 = time.perf_counter()
    _, om, of = oracle.run(cfg, f0.astype(np.float64), steps)
    t_oracle = time.perf_counter() - t0
    out = {"case": f"the headline sphere 256x128x128, {steps} steps from the same f32 start; FP64 oracle on "
                   f"the host ({t_oracle:.0f} s)"}
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    for st in ("fp32", "fp16", "bf16"):
        sol = lbm.Solver(lbm.config_from(19, wl["dims"], **(wl["kw"] | {"storage": st})))
        sol.write_f(f0)
        sol.step(steps)
        m = sol.read_mac().astype(np.float64)
        fx = sol.forces()[0]
        sol.close()
        out[st] = {"u_rel_l2": rel(m[:, 1:4], om[:, 1:4]), "rho_rel_l2": rel(m[:, 0], om[:, 0]),
                   "drag_rel": abs(fx - of[-1, 0]) / abs(of[-1, 0])}
    return out


def oracle_steps(wl, nsteps, f=None):
    """nsteps of the oracle's f32 path (the reference's shader arithmetic in
    its operation order, OpenMP over this host's cores) on a workload, from
    the equilibrium seed or from f. Returns (f, forces, seconds)."""
    import oracle
    from oracle import abi
    cfg = abi.config_from(19, wl["dims"], **wl["kw"])
    if f is None:
        f = oracle.init_eq(19, wl["mac"], fp32=True)
    t0 = time.perf_counter()
    f, _, forces = oracle.run(cfg, f, nsteps, fp32=True)
    return f, forces, time.perf_counter() - t0


def host_cores():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def cpu_baseline(seconds=10.0):
    """The oracle's f32 path on this host's cores, on the headline workload
    itself (256 x 128 x 128): a two-step probe sizes a sample of about
    `seconds` of CPU work, which is then timed as one call."""
    wl = workload()
    f, _, t2 = oracle_steps(wl, 2)
    k = max(2, int(round(seconds / max(t2 / 2, 1e-3))))
    _, _, dt = oracle_steps(wl, k, f)
    cells = int(np.prod(wl["dims"]))
    return {"value": cells * k / dt / 1e6, "unit": "MLUPS", "cores": host_cores(), "kind": "port",
            "sample": f"the headline 256x128x128 workload, {k} steps incl. the force pass ({dt:.1f} s), "
                      "oracle f32 mode (the reference's WGSL arithmetic restated in C++), OpenMP"}


def run_ours(args):
    import torch
    lbm = load_package()
    world, rank, local = dist_setup(args.gpus)
    wl = workload("fp32")
    cells = int(np.prod(wl["dims"]))
    total_ms, launch_ms, clocks, forces, totals = time_device(lbm, wl, args.steps, args.warmup, world)
    t_max = max_over_ranks(total_ms, world)
    kern_ms = max_over_ranks(statistics.mean(launch_ms), world)
    value = cells * args.steps * world / (t_max * 1e-3) / 1e6
    e2e_ms, h2d, d2h = time_e2e(lbm, wl, args.steps, args.warmup, world)
    e2e_value = cells * args.steps * world / (e2e_ms * 1e-3) / 1e6

    # Packed storage forms on the same workload (device-resident, same timing).
    forms = {}
    if not args.skip_forms:
        peak = hbm_peak()[0]
        for q, st in ((19, "fp16"), (19, "bf16"), (27, "fp32"), (27, "fp16")):
            tm, lm, _, fo, _ = time_device(lbm, workload(st, q=q), args.steps, args.warmup, world)
            tm = max_over_ranks(tm, world)
            gbs = BYTES_PER_LU[(f"d3q{q}", st)] * cells / (statistics.mean(lm) * 1e-3) / 1e9
            forms[st if q == 19 else f"d3q27_{st}"] = {
                "mlups": cells * args.steps * world / (tm * 1e-3) / 1e6, "ms_per_step": tm / args.steps,
                "gbs": gbs, "frac_of_measured_hbm": gbs / peak,
                "algorithmic_bytes_per_lu": BYTES_PER_LU[(f"d3q{q}", st)], "fx_last": fo[0]}
        forms["batched"], forms["batched_plain"] = time_batched(lbm, args.steps, args.warmup, world)
        forms["amr2d_cylinder"] = time_amr(lbm, args.steps, args.warmup, world)
        forms["amr3d_sphere"] = time_amr3d(lbm, args.steps, args.warmup, world)
        forms["served"], forms["served_plain"] = time_served(lbm, world)
        if rank == 0:
            forms["accuracy_vs_fp64"] = packed_accuracy(lbm)
    peak, peak_kind = hbm_peak()
    achieved = BYTES_PER_LU[("d3q19", "fp32")] * cells / (kern_ms * 1e-3) / 1e9
    traffic = profiled_traffic("d3q19_sphere_step")
    line = {
        "metric": "MLUPS (D3Q19 dense sphere step, FP32) and % of HBM roofline",
        "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (uniform freestream seed, sphere scenario)",
        "config": config_key("fp32"),
        "replicas": world,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                     else "fallback 6650 GB/s",
                     "algorithmic_bytes_per_lu": 152, "kernel": "d3_step<19,float>",
                     "kernel_ms": kern_ms},
        "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms / args.steps},
        "gpu_launches": args.steps + 1,  # a step kernel per step, a force sum after the last
        "clocks": clocks,
        "forms": forms,
        "drag_lift_last_step": {"fx": forces[0], "fy": forces[1], "fz": forces[2],
                                "after_steps": args.warmup + args.steps},
        "mass_excess": totals["mass"],
    }
    if rank == 0:
        if world == 1 and not args.skip_cpu:
            line["cpu_baseline"] = cpu_baseline(args.cpu_seconds)
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    """The reference's arithmetic on the host cores: the reference is WGSL
    that cannot run here (no WebGPU, no graphics stack), so its stand-in is
    the oracle's f32 restatement of it, configured through the oracle's own
    ABI mirror (no product library is loaded). W untimed and K timed full
    steps of the headline workload from the same seed as our arm; under
    torchrun rank 0 alone runs and prints."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = workload("fp32")
    cells = int(np.prod(wl["dims"]))
    f, _, _ = oracle_steps(wl, args.warmup)
    _, forces, dt = oracle_steps(wl, args.steps, f)
    value = cells * args.steps / dt / 1e6
    cores = host_cores()
    last = forces[-1] if len(forces) else np.zeros(8)
    line = {
        "impl": "reference",
        "metric": "MLUPS (D3Q19 dense sphere step, FP32) and % of HBM roofline",
        "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (uniform freestream seed, sphere scenario)",
        "config": config_key("fp32"),
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": cores, "kind": "port",
                         "sample": f"the full 256x128x128 workload, {args.steps} timed steps after "
                                   f"{args.warmup} untimed, incl. the force pass; the reference's WGSL cannot "
                                   "run here (no WebGPU), so this is the oracle's f32 restatement of it"},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "drag_lift_last_step": {"fx": float(last[0]), "fy": float(last[1]), "fz": float(last[2]),
                                "after_steps": args.warmup + args.steps},
    }
    print(json.dumps(line), flush=True)


def run_form(args):
    """One side form alone, one GPU: the same timing as inside the full run."""
    lbm = load_package()
    world, rank, local = dist_setup(1)
    if args.form in ("fp32", "fp16", "bf16", "d3q27_fp32", "d3q27_fp16"):
        q = 27 if args.form.startswith("d3q27") else 19
        st = args.form.split("_")[-1]
        if args.dims:
            dims = tuple(int(v) for v in args.dims.split(","))
            wl = workload(st, dims=dims, n=max(4, round(32 * dims[0] / DIMS[0])), q=q)
        else:
            wl = workload(st, q=q)
        cells = int(np.prod(wl["dims"]))
        tm, lm, _, fo, _ = time_device(lbm, wl, args.steps, args.warmup, world)
        out = {"mlups": cells * args.steps / (tm * 1e-3) / 1e6, "ms_per_step": tm / args.steps}
    elif args.form == "accuracy":
        out = packed_accuracy(lbm)
    elif args.form == "batched":
        out = dict(zip(("batched", "batched_plain"), time_batched(lbm, args.steps, args.warmup, world)))
    elif args.form == "amr2d_cylinder":
        out = time_amr(lbm, args.steps, args.warmup, world)
    elif args.form == "amr3d_sphere":
        out = time_amr3d(lbm, args.steps, args.warmup, world)
    elif args.form == "amr3d_served":
        out = time_amr3d_served_request(lbm, args.steps, args.warmup)
    else:
        out = dict(zip(("served", "served_plain"), time_served(lbm, world)))
    print(json.dumps({"form": args.form, "steps": args.steps, "warmup": args.warmup, **out}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--skip-forms", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--form", choices=("fp32", "fp16", "bf16", "d3q27_fp32", "d3q27_fp16", "batched", "amr2d_cylinder",
                                       "amr3d_sphere", "amr3d_served", "served", "accuracy"),
                    help="run one of the side forms alone (for profiling) and print its JSON line")
    ap.add_argument("--dims", type=str, default=None,
                    help="with --form fp32/fp16/bf16: a smaller sphere domain NX,NY,NZ (profiling captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.form:
        run_form(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
