"""Version-7 snapshots of a 2D AMR session: checkpoint, resume, and
interchange with the reference's captures.

The layout is main-cylinder-amr.js debugSnapshotSave / debugSnapshotLoad
(:1524-1705) and amr2d-gpu.mjs encodeRootCapture / readRootCapture /
restoreRootCapture (:514-632): a JSON object

    formatVersion  7
    W, H, step     root grid and the macro-step counter (refine schedule)
    root           level 0 as a RINGLESS tile pool: tiles of 2*RB x 2*RB root
                   cells, tile-major (amr2d.mjs rootCellIndex), f as 9 planes
                   of f32, velocity as [ux, uy] f32 per cell, both base64
    pools[1]       level 1: RB, GHOST, FB, MAX_FINE_BLOCKS, NBLOCKS, NBX, NBY,
                   blockSlot, slotToBlock, parentSlot, quadrant, quadAlloc,
                   freeList (quad indices), freeCount, fB64, velB64
    cardState      the body's CardState (common_geometry.wgsl), 26 f32
    params, numLevels

The session keeps level 0 as a dense row-major grid; this module permutes
between the two orders. Loading refuses what the reference refuses: another
grid size, a pre-7 capture (level 0 as a dense grid), a level 1 allocated per
block rather than per quad, and pool shapes that do not match the session.
"""
from __future__ import annotations

import base64
import json

import numpy as np

FORMAT_VERSION = 7
GHOST = 2

CARD_FIELDS = ("cx", "cy", "theta", "vx", "vy", "omega", "fx", "fy", "tz", "mass", "i_body", "g_eff", "a", "b",
               "v_max", "o_max", "cx_old", "cy_old", "th_old", "tau", "y_total", "x_total", "off_x", "off_y",
               "off_x_old", "off_y_old")


class SnapshotError(ValueError):
    pass


def _b64(a: np.ndarray) -> str:
    return base64.b64encode(np.ascontiguousarray(a, "<f4").tobytes()).decode("ascii")


def _unb64(s: str, n: int) -> np.ndarray:
    a = np.frombuffer(base64.b64decode(s), "<f4")
    if a.size != n:
        raise SnapshotError(f"payload holds {a.size} floats, expected {n}")
    return a.astype(np.float32)


def root_order(W: int, H: int, rb: int) -> np.ndarray:
    """For each root-pool cell (tile-major, tiles of 2*rb), the dense row-major
    cell it holds (amr2d.mjs rootCellIndex composed with the row-major grid)."""
    side = 2 * rb
    if W % side or H % side:
        raise SnapshotError(f"domain {W}x{H} does not divide into {side}-cell root tiles")
    nbx = W // side
    gy, gx = np.divmod(np.arange(W * H), W)
    pool = ((gy // side) * nbx + gx // side) * side * side + (gy % side) * side + (gx % side)
    order = np.empty(W * H, np.int64)
    order[pool] = np.arange(W * H)
    return order


def save_amr2d(a, params: dict | None = None) -> dict:
    """Captures a session (lbm.Amr2D) at its current macro-step."""
    cfg = a.cfg
    W, H, rb = a.W, a.H, a.rb
    side = 2 * rb
    order = root_order(W, H, rb)
    f0, v0 = a.read_root()
    f1, v1 = a.read_pool()
    t = a.topology()
    b = cfg.body
    card = {k: 0.0 for k in CARD_FIELDS}
    card.update(cx=b.cx, cy=b.cy, theta=b.theta, vx=b.vx, vy=b.vy, omega=b.wz, a=b.a, b=b.b, tau=cfg.tau,
                cx_old=b.cx, cy_old=b.cy, th_old=b.theta)
    F = a.forces()
    card.update(fx=F[0], fy=F[1], tz=F[2])
    nroot = (W // side) * (H // side)
    root = {"level": 0, "MAX_FINE_BLOCKS": nroot, "NBLOCKS": nroot, "NBX": W // side, "NBY": H // side,
            "cellsPerSlot": side * side, "fB64": _b64(f0[:, order]), "velB64": _b64(v0[order])}
    slots = a.slots
    pool = {"level": 1, "RB": rb, "GHOST": GHOST, "FB": a.fb, "MAX_FINE_BLOCKS": slots,
            "NBLOCKS": a.nbx * a.nby, "NBX": a.nbx, "NBY": a.nby,
            "blockSlot": t["block_slot"].tolist(), "slotToBlock": t["slot_to_block"].tolist(),
            "quadAlloc": True, "parentSlot": a.parent_slots().tolist(),
            "quadrant": (np.arange(slots) % 4).tolist(),
            "freeList": t["free_list"].tolist(), "freeCount": int(t["free_count"]),
            "fB64": _b64(f1), "velB64": _b64(v1)}
    return {"formatVersion": FORMAT_VERSION, "root": root, "W": W, "H": H, "step": a.macro_step,
            "cardState": [float(np.float32(card[k])) for k in CARD_FIELDS],
            "params": dict(params or {}), "numLevels": 2, "pools": [None, pool]}


def load_amr2d(a, snap: dict) -> None:
    """Restores a capture into a session of the same shape (lbm.Amr2D)."""
    W, H, rb = a.W, a.H, a.rb
    if snap.get("W") != W or snap.get("H") != H:
        raise SnapshotError(f"snapshot is {snap.get('W')}x{snap.get('H')}, session is {W}x{H}")
    if not (snap.get("formatVersion", 0) >= FORMAT_VERSION) or not isinstance(snap.get("pools"), list):
        raise SnapshotError(f"formatVersion {snap.get('formatVersion', '?')} carries level 0 as a dense grid; "
                            "version 7 carries it as `root` -- re-capture the snapshot")
    side = 2 * rb
    root = snap.get("root")
    nroot = (W // side) * (H // side)
    if not root:
        raise SnapshotError("snapshot has no level 0 (`root`)")
    if root["MAX_FINE_BLOCKS"] != nroot or root["NBLOCKS"] != nroot or root["cellsPerSlot"] != side * side:
        raise SnapshotError(f"snapshot root (slots={root['MAX_FINE_BLOCKS']}, blocks={root['NBLOCKS']}, "
                            f"cellsPerSlot={root['cellsPerSlot']}) does not match this session's "
                            f"(slots={nroot}, blocks={nroot}, cellsPerSlot={side * side})")
    if snap.get("numLevels", 2) != 2 or len(snap["pools"]) < 2 or snap["pools"][1] is None:
        raise SnapshotError("this session has exactly one pool level")
    pool = snap["pools"][1]
    if not pool.get("quadAlloc"):
        raise SnapshotError("level 1 was allocated per block; this session allocates quads, and a free list of "
                            "block indices would hand out overlapping quads")
    if (pool["RB"], pool["FB"], pool["MAX_FINE_BLOCKS"], pool["NBLOCKS"]) != (rb, a.fb, a.slots, a.nbx * a.nby):
        raise SnapshotError(f"snapshot level 1 (RB={pool['RB']}, FB={pool['FB']}, slots={pool['MAX_FINE_BLOCKS']}, "
                            f"blocks={pool['NBLOCKS']}) does not match this session's (RB={rb}, FB={a.fb}, "
                            f"slots={a.slots}, blocks={a.nbx * a.nby})")
    n0 = W * H
    order = root_order(W, H, rb)
    f0p = _unb64(root["fB64"], 9 * n0).reshape(9, n0)
    v0p = _unb64(root["velB64"], 2 * n0).reshape(n0, 2)
    f0 = np.empty_like(f0p)
    v0 = np.empty_like(v0p)
    f0[:, order] = f0p
    v0[order] = v0p
    n1 = a.slots * a.fb * a.fb
    f1 = _unb64(pool["fB64"], 9 * n1).reshape(9, n1)
    v1 = _unb64(pool["velB64"], 2 * n1).reshape(n1, 2)
    fl = np.zeros(a.slots // 4, np.int32)
    src = np.asarray(pool["freeList"], np.int32)[: a.slots // 4]
    fl[: src.size] = src
    a.write_topology(pool["blockSlot"], pool["slotToBlock"], pool["parentSlot"], fl, int(pool["freeCount"]))
    a.write_root(f0, v0)
    a.write_pool(f1, v1)
    a.macro_step = int(snap.get("step", 0))
    card = dict(zip(CARD_FIELDS, snap.get("cardState", [])))
    if card:
        from . import make_body
        b = a.cfg.body
        body = make_body("ellipse", (card["cx"], card["cy"], 0.0), a=b.a, b=b.b, theta=card["theta"],
                         v=(card["vx"], card["vy"], 0.0), w=(0.0, 0.0, card["omega"]))
        a.set_body(body)


def dumps(snap: dict) -> str:
    return json.dumps(snap)


def loads(text: str) -> dict:
    return json.loads(text)
