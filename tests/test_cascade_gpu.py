"""The 2:1 cascade closure on the device (amr_cascade.wgsl completeQuads and
balance, one deepest-first sweep) against the host rule lbm_cascade21 and
the brute-force fixed point, on seeded want sets that violate the
invariant, at 3 to 5 levels, with blocks on the periodic seam."""
import numpy as np
import pytest

from test_amr_rules import brute_cascade

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("levels,seed", [(3, 1), (4, 2), (4, 3), (5, 4)])
def test_device_cascade_equals_host_rule(lbm, levels, seed):
    rng = np.random.default_rng(seed)
    nbx1, nby1 = 6, 4
    wants = [None] + [(rng.random((nby1 << (m - 1)) * (nbx1 << (m - 1))) < 0.04).astype(np.uint8)
                      for m in range(1, levels)]
    # a deepest-level block on the corner of the seam
    wants[levels - 1][0] = 1
    host, added_h = lbm.cascade21(wants, levels, nbx1, nby1)
    dev, added_d = lbm.cascade21_device(wants, levels, nbx1, nby1)
    assert added_d == added_h > 0
    for m in range(1, levels):
        assert np.array_equal(dev[m], host[m]), m
    ref = brute_cascade(wants, levels, nbx1, nby1)
    for m in range(1, levels):
        got = set(map(tuple, np.argwhere(dev[m].reshape(nby1 << (m - 1), nbx1 << (m - 1)))))
        assert got == ref[m], m
    # a closed set is a fixed point on the device too
    again, added2 = lbm.cascade21_device(dev, levels, nbx1, nby1)
    assert added2 == 0 and all(np.array_equal(again[m], dev[m]) for m in range(1, levels))
