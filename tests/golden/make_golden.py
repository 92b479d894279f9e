"""Generates the golden fixtures under tests/golden/ from the reference tree.

Reads the reference's checked-in files AS TEXT (nothing of the reference is
executed; its JavaScript cannot run here):

* lattice.json   -- the velocity sets, weights (f32 bit patterns) and opp
                    tables parsed out of the generated WGSL
                    (shaders/common_lattice.wgsl, common_d3q19_lattice.wgsl,
                    common_d3q27_lattice.wgsl), plus the properties
                    tools/test-lattice-2d.js / test-lattice-3d.js assert.
* fpack.json     -- every `f32ToF16Bits(expr) === 0x....` known answer in
                    tools/test-f-pack.js, with expr evaluated to a number.
* benchmarks.json -- the analytic gates of benchmarks/tgv.json (cases and
                    tolerances) used by the physics tests.

Usage: python tests/golden/make_golden.py <path of the reference checkout>
"""
from __future__ import annotations

import json
import math
import re
import struct
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def f32_bits(x: float) -> int:
    return struct.unpack("<I", struct.pack("<f", x))[0]


def parse_array(src: str, name: str):
    m = re.search(r"const\s+%s\s*=\s*array<(\w+),\s*(\d+)>\(([^)]*)\)" % name, src, re.S)
    if not m:
        raise ValueError(name)
    items = [s.strip() for s in m.group(3).replace("\n", " ").split(",") if s.strip()]
    if m.group(1) == "f32":
        return [float(s.rstrip("f")) for s in items]
    return [int(s.rstrip("u")) for s in items]


def lattice(ref: Path) -> dict:
    out = {}
    for q, fname in ((9, "common_lattice.wgsl"), (19, "common_d3q19_lattice.wgsl"),
                     (27, "common_d3q27_lattice.wgsl")):
        src = (ref / "shaders" / fname).read_text()
        ex, ey = parse_array(src, "ex"), parse_array(src, "ey")
        ez = parse_array(src, "ez") if q != 9 else [0] * 9
        wt = parse_array(src, "wt")
        opp = parse_array(src, "opp")
        out[str(q)] = {
            "source": f"shaders/{fname}",
            "ex": ex, "ey": ey, "ez": ez, "opp": opp,
            "w_bits": [f32_bits(w) for w in wt],
        }
    out["properties"] = {
        "d2q9_sum_minus_1_range": [0.0, 7.4507e-9],   # tools/test-lattice-2d.js:103
        "d2q9_velocity_drift": 0.0,                     # tools/test-lattice-2d.js:72-83
        "d3_weight_sum": 1.0,                           # tools/test-lattice-3d.js (exact sum)
        "max_ulp_tweak": 4,                             # tools/test-lattice-2d.js:117
    }
    return out


def fpack(ref: Path) -> list:
    src = (ref / "tools" / "test-f-pack.js").read_text()
    env = {"Math": None}
    q = 2.0 ** -24

    def js_eval(expr: str) -> float:
        e = expr.replace("Math.pow", "pow").replace("Infinity", "math.inf")
        return float(eval(e, {"__builtins__": {}}, {"pow": pow, "math": math, "q": q}))

    cases = []
    for m in re.finditer(r"assert\.strictEqual\(f32ToF16Bits\(([^;]*?)\),\s*(0x[0-9a-fA-F]+)\)", src):
        expr, bits = m.group(1).strip(), int(m.group(2), 16)
        v = js_eval(expr)
        line = src[: m.start()].count("\n") + 1
        cases.append({"expr": expr, "value": v, "neg_zero": expr.strip() == "-0",
                      "bits": bits, "line": line})
    return cases


def benchmarks(ref: Path) -> dict:
    tgv = json.loads((ref / "benchmarks" / "tgv.json").read_text())
    return {"tgv": {"source": "benchmarks/tgv.json",
                    "cases": [c for c in tgv["cases"] if "levels" not in c]}}


def main(ref: Path):
    (HERE / "lattice.json").write_text(json.dumps(lattice(ref), indent=1) + "\n")
    (HERE / "fpack.json").write_text(json.dumps(fpack(ref), indent=1) + "\n")
    (HERE / "benchmarks.json").write_text(json.dumps(benchmarks(ref), indent=1) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(Path(sys.argv[1]))
