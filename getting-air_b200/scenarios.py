"""Synthetic inputs: the reference's scenario seeds, restated.

* :func:`sphere` -- d3-scenarios.mjs:350-389 (`SCENARIOS.sphere`): domain
  12D x 8D x 8D unless dims are given, centre (3D, NY/2, NZ/2), tau from Re,
  sponge width max(6, round(D/2)) toward (u0, 0, 0), uniform seed
  rho = 1 - |u|^2 / (2 cs^2) (seedMacro3, d3-scenarios.mjs:245-261).
* :func:`tgv2d_field` -- main-tgv.js:69-89 analyticField: the exact decaying
  Taylor-Green field with its O(Ma^2) density term; :func:`tgv2d_f` seeds f
  at equilibrium in f64 and rounds to f32 (main-tgv.js:136 initF).
* :func:`cylinder2d` -- the pinned-cylinder crossflow of the 2D cylinder
  pages: circle of radius r, sponge toward (u0, 0).
* :func:`mulberry32` -- the seeded generator the reference uses for
  perturbations (d3-scenarios.mjs:207-215).
"""
from __future__ import annotations

import math

import numpy as np

CS2 = 1.0 / 3.0


def nu_from_tau(tau: float) -> float:
    return CS2 * (tau - 0.5)


def tau_from_nu(nu: float) -> float:
    return nu / CS2 + 0.5


def mulberry32(seed: int):
    s = seed & 0xFFFFFFFF

    def imul(a, b):
        return (a * b) & 0xFFFFFFFF

    def nxt():
        nonlocal s
        s = (s + 0x6D2B79F5) & 0xFFFFFFFF
        t = imul(s ^ (s >> 15), 1 | s)
        t = ((t + imul(t ^ (t >> 7), 61 | t)) & 0xFFFFFFFF) ^ t
        return ((t ^ (t >> 14)) & 0xFFFFFFFF) / 4294967296.0

    return nxt


def uniform_macro(ncells: int, u=(0.0, 0.0, 0.0)) -> np.ndarray:
    ux, uy, uz = u
    mac = np.empty((ncells, 4), np.float32)
    mac[:, 0] = np.float32(1 - (ux * ux + uy * uy + uz * uz) / (2 * CS2))
    mac[:, 1], mac[:, 2], mac[:, 3] = ux, uy, uz
    return mac


def sphere(n: int = 16, u0: float = 0.05, re: float = 100.0, tau: float | None = None,
           dims=None, q: int = 19, bounceback: bool = True, force=(0.0, 0.0, 0.0),
           storage: str = "fp32") -> dict:
    """Flow past a pinned sphere of diameter n (cells). Returns solver kwargs + seed."""
    if tau is None:
        nu = u0 * n / re
        tau = tau_from_nu(nu)
    d = list(dims) if dims is not None else [round(12 * n), round(8 * n), round(8 * n)]
    R = n / 2
    body = dict(shape="sphere", centre=(3 * n, d[1] / 2, d[2] / 2), a=R)
    kw = dict(tau=float(tau), has_body=1, use_bounceback=int(bounceback), body=body,
              sponge_w=float(max(6, round(n / 2))), sponge_u=(u0, 0.0, 0.0), force=tuple(force),
              storage=storage)
    return {"q": q, "dims": tuple(d), "kw": kw, "mac": uniform_macro(d[0] * d[1] * d[2], (u0, 0, 0)),
            "area": math.pi * R * R, "u0": u0}


def tgv2d_field(N: int, u0: float, tau: float, t: float = 0.0):
    """Analytic TGV (ux, uy, rho) on an N x N periodic box at time t, f64."""
    k = 2 * math.pi / N
    nu = nu_from_tau(tau)
    td = 1.0 / (nu * (k * k + k * k))
    x = np.arange(N)[None, :].astype(np.float64)
    y = np.arange(N)[:, None].astype(np.float64)
    dec, dec2 = math.exp(-t / td), math.exp(-2 * t / td)
    ux = -u0 * np.cos(k * x) * np.sin(k * y) * dec
    uy = u0 * np.sin(k * x) * np.cos(k * y) * dec
    p = -(u0 * u0 / 4) * (np.cos(2 * k * x) + np.cos(2 * k * y)) * dec2
    rho = 1 + p / CS2
    return ux.ravel(), uy.ravel(), rho.ravel(), td


def tgv2d_f(N: int, u0: float, tau: float, w) -> np.ndarray:
    """Equilibrium seed (9 x N^2, f32) from the analytic t=0 field."""
    ux, uy, rho, _ = tgv2d_field(N, u0, tau)
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], np.float64)
    ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], np.float64)
    f = np.empty((9, N * N), np.float32)
    usq = ux * ux + uy * uy
    for i in range(9):
        eu = ex[i] * ux + ey[i] * uy
        f[i] = (float(w[i]) * rho * (1 + eu * 3 + eu * eu * 4.5 - usq * 1.5)).astype(np.float32)
    return f


def cylinder2d(W: int = 256, H: int = 128, r: float = 10.0, u0: float = 0.05, tau: float = 0.6,
               centre=None, bounceback: bool = True, sponge_w: float = 8.0) -> dict:
    cx, cy = centre if centre is not None else (W / 4, H / 2)
    body = dict(shape="ellipse", centre=(cx, cy, 0.0), a=r, b=r)
    kw = dict(tau=float(tau), has_body=1, use_bounceback=int(bounceback), body=body,
              sponge_w=float(sponge_w), sponge_u=(u0, 0.0, 0.0))
    return {"q": 9, "dims": (W, H, 1), "kw": kw, "mac": uniform_macro(W * H, (u0, 0, 0))}


def cylinder_page(res: int = 9, re: float = 100.0, u0: float = 0.04, blockage: float = 24.0, upstream: float = 12.0,
                  bounceback: bool = True, perturb: float = 0.02, seed: int = 12345, k_eps: float = 1.5) -> dict:
    """The dense 2D cylinder page's configuration (main-cylinder.js): a square
    W = H = 2^res domain, R = W / (2 blockage) at (upstream * 2R, H/2), tau from
    Re on the diameter (tau = 0.5 + 3 nu, nu = u0 D / Re), sponge width 4
    toward (u0, 0), SOLID_EQ, bounce-back or the chi penalty with K_EPS, and
    the seed of initF: every cell at feq(1, u0, uy) with a per-cell
    transverse uy = (rng * 2 - 1) * perturb * u0 from mulberry32(seed)."""
    W = H = 1 << res
    R = W / (2.0 * blockage)
    D = 2.0 * R
    nu = u0 * D / re
    tau = float(np.float32(0.5 + 3.0 * nu))
    rng = mulberry32(seed)
    n = W * H
    uy = np.array([(rng() * 2 - 1) * perturb * u0 for _ in range(n)], np.float64)
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], np.float64)
    ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], np.float64)
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    f = np.empty((9, n), np.float32)
    usq = u0 * u0 + uy * uy
    for i in range(9):
        eu = ex[i] * u0 + ey[i] * uy
        f[i] = (w[i] * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * usq)).astype(np.float32)
    body = dict(shape="ellipse", centre=(upstream * D, H / 2.0, 0.0), a=R, b=R)
    kw = dict(tau=tau, has_body=1, use_bounceback=int(bounceback), chi_eps=k_eps, solid_eq=1, body=body,
              sponge_w=4.0, sponge_u=(u0, 0.0, 0.0))
    return {"q": 9, "dims": (W, H, 1), "kw": kw, "f": f, "u0": u0, "D": D, "re": re}


def cylinder_analyze(history, transient: int, D: float, u0: float) -> dict:
    """Cd mean over the post-transient samples and St from the zero crossings
    of the mean-removed Cl (linear interpolation), as tools/lib/cylinder-
    metrics.js analyze(); history rows are (step, Cd, Cl)."""
    win = [r for r in history if r[0] > transient]
    cd = float(np.mean([r[1] for r in win]))
    cl = np.array([r[2] for r in win])
    c = cl - cl.mean()
    cross = []
    for i in range(1, len(c)):
        if c[i - 1] < 0 <= c[i]:
            a, b = win[i - 1][0], win[i][0]
            cross.append(a + (-c[i - 1] / (c[i] - c[i - 1])) * (b - a))
    st = None
    if len(cross) >= 3:
        period = float(np.mean(np.diff(cross)))
        st = D / period / u0
    return {"cd": cd, "st": st, "samples": len(win), "crossings": len(cross)}


def batched_domains(count: int = 512, seed: int = 12345, nmin: int = 64, nmax: int = 512,
                    tau_range=(0.55, 0.9), u0: float = 0.04):
    """The batched D2Q9 workload: `count` square domains with N = round(nmin *
    (nmax/nmin)^U), U uniform on [0, 1) from mulberry32(seed), tau uniform in
    tau_range, alternating a periodic Taylor-Green vortex (amplitude u0) and
    a plane Poiseuille channel (walls on y, body force for a peak of u0).
    Returns a list of dicts: q, dims, kw (Solver keywords), kind, and a seed
    ('f' for TGV, 'mac' for the channel)."""
    rng = mulberry32(seed)
    out = []
    ratio = nmax / nmin
    for k in range(count):
        n = int(round(nmin * ratio ** rng()))
        tau = tau_range[0] + (tau_range[1] - tau_range[0]) * rng()
        tau = float(np.float32(tau))
        if k % 2 == 0:
            out.append({"q": 9, "dims": (n, n, 1), "kind": "tgv", "u0": u0,
                        "kw": dict(tau=tau, sponge_w=0.0)})
        else:
            nu = nu_from_tau(tau)
            g = 8.0 * nu * u0 / (n * n)      # plane Poiseuille: u_max = g H^2 / (8 nu)
            out.append({"q": 9, "dims": (n, n, 1), "kind": "channel", "u0": u0,
                        "kw": dict(tau=tau, sponge_w=0.0, wall=(0, 1, 0), force=(g, 0.0, 0.0))})
    return out


def seed_domain(dom, w) -> np.ndarray:
    """Initial f (9 x N^2, f32) for a batched_domains entry."""
    n = dom["dims"][0]
    if dom["kind"] == "tgv":
        return tgv2d_f(n, dom["u0"], dom["kw"]["tau"], w)
    # channel: fluid at rest, rho = 1 (f_i = w_i), driven by the body force
    return np.repeat(np.asarray(w, np.float32)[:, None], n * n, axis=1)


def cylinder_amr(W: int = 1024, H: int = 256, r: float = 20.0, centre=(256.0, 128.0), u0: float = 0.08,
                 re: float = 100.0, perturb: float = 0.02, seed: int = 12345, bounceback: bool = False,
                 max_slots=None) -> dict:
    """The 2D AMR cylinder: root W x H, circle of radius r, tau from Re on the
    diameter, sponge (width 4) toward (u0, 0), diffuse (chi) coupling unless
    bounceback, and the reference's seed (main-cylinder-amr.js:803-830):
    every root cell at feq(1, u0, uy) with uy = (rng*2-1) * perturb * u0 from
    mulberry32(seed), the same (u0, uy) as the initial root velocity."""
    nu = u0 * 2 * r / re
    tau = float(np.float32(tau_from_nu(nu)))
    rng = mulberry32(seed)
    n = W * H
    uy = np.array([(rng() * 2 - 1) * perturb * u0 for _ in range(n)], np.float64)
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], np.float64)
    ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], np.float64)
    w = np.array([0.44444444775581360, 0.11111111193895340, 0.11111111193895340, 0.11111111193895340,
                  0.11111111193895340, 0.027777777984738350, 0.027777777984738350, 0.027777777984738350,
                  0.027777777984738350])
    f = np.empty((9, n), np.float32)
    usq = u0 * u0 + uy * uy
    for i in range(9):
        eu = ex[i] * u0 + ey[i] * uy
        f[i] = (w[i] * (1 + eu * 3 + eu * eu * 4.5 - usq * 1.5)).astype(np.float32)
    vel = np.stack([np.full(n, u0), uy], 1).astype(np.float32)
    kw = dict(tau=tau, use_bounceback=int(bounceback), sponge_w=4.0, sponge_u=(u0, 0.0),
              body=dict(shape="ellipse", centre=(centre[0], centre[1], 0.0), a=r, b=r))
    if max_slots is not None:
        kw["max_slots"] = max_slots
    return {"dims": (W, H), "kw": kw, "f": f, "vel": vel, "u0": u0, "r": r}


def serving_stream(count: int = 48, seed: int = 2024, rate: float = 200.0, nmin: int = 32, nmax: int = 192,
                   steps=(500, 2000), amr_frac: float = 0.0):
    """Seeded Poisson stream of 3D obstacle solves: arrival times with mean
    rate `rate`/s, cubic domains N^3 with N log-uniform in [nmin, nmax],
    D3Q19 or D3Q27, a pinned sphere (radius N/8) or rounded box (half-extent
    N/8), bounce-back, sponge (width max(6, N/16)) toward u0 = 0.05 along x,
    tau uniform in [0.55, 0.7], steps uniform in the given range. A fraction
    `amr_frac` are two-level AMR solves (levels = 2, RB = 4, the blocks near
    the body refined, N rounded to a multiple of 4; steps are macro-steps).
    Returns a list of dicts: t (arrival, s), q, dims, kw (Solver keywords),
    steps, levels."""
    rng = mulberry32(seed)
    amr_rng = mulberry32(seed ^ 0x5EED)
    t = 0.0
    out = []
    for k in range(count):
        t += -math.log(1.0 - rng()) / rate
        n = int(round(nmin * (nmax / nmin) ** rng()))
        levels = 2 if amr_rng() < amr_frac else 1
        if levels == 2:
            n = max(16, 4 * (n // 4))
        q = 19 if rng() < 0.5 else 27
        box = rng() < 0.5
        tau = float(np.float32(0.55 + 0.15 * rng()))
        nsteps = int(steps[0] + (steps[1] - steps[0]) * rng())
        a = n / 8.0
        centre = (round(n / 3), n / 2, n / 2)
        body = (dict(shape="roundbox", centre=centre, a=a, b=a, c=a, r=a / 4) if box else
                dict(shape="sphere", centre=centre, a=a))
        kw = dict(tau=tau, has_body=1, use_bounceback=1, body=body, sponge_w=float(max(6, n // 16)),
                  sponge_u=(0.05, 0.0, 0.0))
        out.append({"t": t, "q": q, "dims": (n, n, n), "kw": kw, "steps": nsteps, "id": k, "levels": levels})
    return out


def serving_config(lbm, r):
    """The request's config: an lbm_config, or for levels = 2 an
    lbm_amr3d_config refining the blocks within 2 cells of the body."""
    if r.get("levels", 1) == 2:
        return lbm.amr3d_config(r["q"], r["dims"], refine="body", rb=4, margin=2.0, **r["kw"])
    return lbm.config_from(r["q"], r["dims"], **r["kw"])
