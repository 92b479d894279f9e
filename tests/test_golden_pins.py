"""Pins the oracle (and the library's pure tables) to the reference's own
known answers, read out of the reference tree into tests/golden/ by
tests/golden/make_golden.py.

* lattice tables: the generated WGSL literals (common_lattice.wgsl:20-37,
  common_d3q19_lattice.wgsl:26-52, common_d3q27_lattice.wgsl:26-57) bit for
  bit, and the properties tools/test-lattice-2d.js:72-196 and
  tools/test-lattice-3d.js:126-277 assert;
* binary16 encoding: every known answer in tools/test-f-pack.js:29-77.
"""
import json
import math
import struct
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
LAT = json.loads((GOLD / "lattice.json").read_text())
FPACK = json.loads((GOLD / "fpack.json").read_text())


def bits(x):
    return struct.unpack("<I", struct.pack("<f", float(x)))[0]


@pytest.mark.parametrize("q", [9, 19, 27])
def test_oracle_tables_equal_reference_wgsl(oracle, q):
    g = LAT[str(q)]
    t = oracle.tables(q)
    assert t["ex"].tolist() == g["ex"]
    assert t["ey"].tolist() == g["ey"]
    assert t["ez"].tolist() == g["ez"]
    assert t["opp"].tolist() == g["opp"]
    assert [bits(w) for w in t["w"]] == g["w_bits"]


@pytest.mark.parametrize("q", [9, 19, 27])
def test_library_tables_equal_reference_wgsl(lbm, q):
    g = LAT[str(q)]
    t = lbm.lattice_tables(q)
    assert t["ex"].tolist() == g["ex"] and t["ey"].tolist() == g["ey"] and t["ez"].tolist() == g["ez"]
    assert t["opp"].tolist() == g["opp"]
    assert [bits(w) for w in t["w"]] == g["w_bits"]


def exact_sum(ws):
    return sum(Fraction(float(w)) for w in ws)


def test_d2q9_weight_properties(oracle):
    w = oracle.tables(9)["w"]
    lo, hi = LAT["properties"]["d2q9_sum_minus_1_range"]
    s = exact_sum(w) - 1
    assert lo <= float(s) <= hi
    # 2 w1 + 8 w2 - w0 == 0 exactly: zero velocity drift through a collision.
    assert 2 * Fraction(float(w[1])) + 8 * Fraction(float(w[5])) - Fraction(float(w[0])) == 0


@pytest.mark.parametrize("q", [19, 27])
def test_d3_weights_sum_to_exactly_one(oracle, q):
    assert exact_sum(oracle.tables(q)["w"]) == 1


@pytest.mark.parametrize("q", [9, 19, 27])
def test_moments_and_opp(oracle, q):
    t = oracle.tables(q)
    e = np.stack([t["ex"], t["ey"], t["ez"]], 1).astype(np.float64)
    w = t["w"].astype(np.float64)
    d = 2 if q == 9 else 3
    assert abs(w.sum() - 1) < 2e-8
    for a in range(d):
        assert abs((w * e[:, a]).sum()) == 0
        assert abs((w * e[:, a] ** 2).sum() - 1 / 3) < 3e-8
        assert abs((w * e[:, a] ** 4).sum() - 1 / 3) < 3e-8
    for i in range(q):
        o = t["opp"][i]
        assert t["opp"][o] == i
        assert (e[o] == -e[i]).all()
    if q == 19:
        t27 = oracle.tables(27)
        assert (t27["ex"][:19] == t["ex"]).all() and (t27["ey"][:19] == t["ey"]).all()
        assert (t27["ez"][:19] == t["ez"]).all()


def test_mutated_table_is_caught(oracle):
    """A transposed opp (the reference's highest-consequence bug) fails the check."""
    t = oracle.tables(19)
    opp = t["opp"].copy()
    opp[[1, 3]] = opp[[3, 1]]
    e = np.stack([t["ex"], t["ey"], t["ez"]], 1)
    assert not all((e[opp[i]] == -e[i]).all() for i in range(19))


def _f32(v):
    return float(np.float32(v)) if math.isfinite(v) or math.isinf(v) else v


@pytest.mark.parametrize("case", FPACK, ids=[c["expr"] for c in FPACK])
def test_f16_known_answers_oracle(oracle, case):
    v = -0.0 if case["neg_zero"] else _f32(case["value"])
    assert oracle.f16_bits(v) == case["bits"]


@pytest.mark.parametrize("case", FPACK, ids=[c["expr"] for c in FPACK])
def test_f16_known_answers_library(lbm, case):
    v = -0.0 if case["neg_zero"] else _f32(case["value"])
    assert lbm.f32_to_f16_bits(v) == case["bits"]


def test_f16_decode_inverts_encode(lbm):
    # Every finite binary16 pattern round-trips (tools/test-f-pack.js:100-107).
    for b in list(range(0, 0x7C00, 7)) + list(range(0x8000, 0xFC00, 11)) + [0x7BFF, 0x03FF, 0x0400]:
        assert lbm.f32_to_f16_bits(lbm.f16_bits_to_f32(b)) == b


def test_f16_library_matches_numpy_rne(lbm):
    rng = np.random.default_rng(7)
    vals = (rng.standard_normal(4000) * 10.0 ** rng.integers(-8, 5, 4000)).astype(np.float32)
    want = vals.astype(np.float16).view(np.uint16)
    got = np.array([lbm.f32_to_f16_bits(float(v)) for v in vals], np.uint16)
    assert (got == want).all()
