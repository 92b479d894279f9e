"""The allocation-free step (lbm_step_noalloc) against the ordinary session
step: same populations, mac field and body force on two calls in a row.

It exists for callers that cannot call cudaMalloc (hosts that own all device
memory, loops that must not take cudaMalloc/cudaFree's implicit device
synchronisation); its reduction scratch is a fixed array inside the library,
shared by every call. The device buffers below belong to the test (the
caller), not to the library. This file is collected last, so a run that
stops at the first failure has already run every other test; it also passes
alone in a fresh process, where its first call performs the one-time
scratch address lookup.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_step_matches_session_step_twice(lbm, oracle):
    import torch
    from getting_air_b200 import scenarios as sc
    s = sc.sphere(n=8, dims=(48, 32, 32), u0=0.05, re=40, force=(1e-6, 0.0, 0.0))
    cfg = lbm.config_from(19, s["dims"], **s["kw"])
    n = int(np.prod(s["dims"]))
    f0 = oracle.init_eq(19, s["mac"], fp32=True).astype(np.float32)
    sol = lbm.Solver(cfg)
    sol.write_f(f0)
    a = torch.from_numpy(f0).cuda()
    b = torch.empty_like(a)
    mac = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    force = torch.zeros(8, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        lbm.step_noalloc(cfg, a.data_ptr(), b.data_ptr(), mac.data_ptr(), force.data_ptr(), stream)
        torch.cuda.synchronize()
        sol.step(1)
        assert np.array_equal(b.cpu().numpy(), sol.read_f())
        assert np.array_equal(mac.cpu().numpy(), sol.read_mac())
        want = sol.forces()
        got = force.cpu().numpy()[:6]
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
        assert abs(got[0]) > 0
        a, b = b, a
    sol.close()


def test_noalloc_step_refuses_oversized_force_region(lbm):
    # A body spanning most of a large grid needs more force partials than the
    # fixed scratch holds: refused before anything is launched. The buffers
    # are NULL on purpose: the size check comes first, and without it the
    # call still stops at the NULL-buffer check (EINVAL), never at a launch.
    cfg = lbm.config_from(19, (64, 2000, 2000), tau=0.6, has_body=1, use_bounceback=1,
                          body=dict(shape="sphere", centre=(32, 1000, 1000), a=900.0))
    with pytest.raises(lbm.LbmError, match="fixed scratch") as ei:
        lbm.step_noalloc(cfg, 0, 0, None, 8)
    assert ei.value.code == lbm.ENOSPC
    with pytest.raises(lbm.LbmError, match="distinct device buffers"):
        lbm.step_noalloc(lbm.config_from(19, (8, 8, 8)), 0, 0)
