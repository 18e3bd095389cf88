"""The allocation-free max-change entry point (gatt_max_change_noalloc) against the
max-change gatt_step reports, on two calls in a row.

gatt_max_change_noalloc serves callers that cannot call cudaMalloc (graph capture in
progress, host callbacks, an external allocator owning device memory): its accumulators
live in a static device array shared by all calls, which it clears at the start of each
call.  Two consecutive calls on different data therefore each return their own maxima.
This file is collected last so a stop-at-first-failure run has executed every other test.
"""
import ctypes

import numpy as np
import pytest

from gatt_dns_b200 import case as cs

pytestmark = pytest.mark.gpu

KEYS = ("U", "V", "W", "R", "E")


def _device(flow):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(flow[k].ravel(order="F"))).cuda() for k in KEYS]


def _noalloc(lib, sets_a, sets_b, n, nvar=5):
    nsets = len(sets_a)
    a = (ctypes.c_void_p * (nsets * nvar))(*[t.data_ptr() for s in sets_a for t in s])
    b = (ctypes.c_void_p * (nsets * nvar))(*[t.data_ptr() for s in sets_b for t in s])
    out = np.zeros(nsets * nvar)
    rc = lib.gatt_max_change_noalloc(nsets, nvar, n, a, b, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
    return rc, out.reshape(nsets, nvar)


def test_no_alloc_max_change_matches_step_on_two_calls(cuda_lib):
    import torch
    from gatt_dns_b200.solver import GattDNS
    c = cs.periodic_box(n=24)
    f0 = cs.random_flow(c, seed=21, amp=0.05)
    dt = 0.25 * c.cfl_dt(f0["U"], f0["V"], f0["W"], 1.0)
    g = GattDNS(c)
    g.upload(f0)
    states, steps = [f0], []
    for s in range(2):
        steps.append(g.step(s * dt, dt)[0])
        states.append(g.download())
    g.close()
    torch.cuda.synchronize()
    dev = [_device(st) for st in states]
    # call 1: step 1's new state against its start; call 2: step 2 -- the second call
    # must not see the first call's (larger) maxima left in the shared scratch
    for s in range(2):
        rc, mc = _noalloc(cuda_lib, [dev[s + 1]], [dev[s]], c.npts)
        assert rc == 0
        assert np.allclose(mc[0], steps[s], rtol=1e-12, atol=0.0), (s, mc[0], steps[s])
    assert not np.allclose(steps[0], steps[1], rtol=1e-3)
    # several sets in one call give the per-set maxima
    rc, mc = _noalloc(cuda_lib, [dev[1], dev[2]], [dev[0], dev[1]], c.npts)
    assert rc == 0
    assert np.allclose(mc, np.vstack(steps), rtol=1e-12, atol=0.0)


def test_no_alloc_rejects_requests_beyond_its_scratch(cuda_lib):
    import torch
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    sets = [[x] * 5 for _ in range(33)]  # 165 accumulators > 160
    rc, _ = _noalloc(cuda_lib, sets, sets, 8)
    assert rc == 2
    assert b"160" in cuda_lib.gatt_last_error()
    rc, mc = _noalloc(cuda_lib, sets[:32], sets[:32], 8)
    assert rc == 0 and np.all(mc == 0.0)
