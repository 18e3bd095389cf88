"""The allocation-free max-change entry point (gatt_max_change_noalloc) against the
max-change gatt_step reports, on two calls in a row.

gatt_max_change_noalloc serves callers that cannot call cudaMalloc (a host application
whose own allocator owns all device memory): its accumulators live in a static device
array shared by all calls, which it clears at the start of each call.  Two consecutive calls on different data therefore each return their own maxima.
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


def test_no_alloc_refuses_a_capturing_stream(cuda_lib):
    """The call synchronises its stream and returns host values, so on a stream that is
    being captured it must return GATT_ERR_STATE (6) before enqueuing anything."""
    import torch
    x = torch.ones(64, dtype=torch.float64, device="cuda")
    y = torch.zeros(64, dtype=torch.float64, device="cuda")
    rc, mc = _noalloc(cuda_lib, [[x]], [[y]], 64, nvar=1)  # first call: address set-up
    assert rc == 0 and mc[0, 0] == 1.0
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        graph.capture_begin()
        try:
            a = (ctypes.c_void_p * 1)(x.data_ptr())
            b = (ctypes.c_void_p * 1)(y.data_ptr())
            out = np.zeros(1)
            rc = cuda_lib.gatt_max_change_noalloc(1, 1, 64, a, b, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                  ctypes.c_void_p(s.cuda_stream))
        finally:
            graph.capture_end()
    assert rc == 6
    assert b"captured" in cuda_lib.gatt_last_error()
    rc, mc = _noalloc(cuda_lib, [[x]], [[y]], 64, nvar=1)  # still usable afterwards
    assert rc == 0 and mc[0, 0] == 1.0
