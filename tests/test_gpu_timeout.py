"""The pipelined line solver's bounded waits: a self-test sweep whose copy barriers expect
more bytes than arrive must give up, report GATT_ERR_TIMEOUT at the next synchronisation,
and leave the context usable (a normal line solve afterwards matches the oracle)."""
import numpy as np
import pytest

from gatt_dns_b200 import case as cs

pytestmark = pytest.mark.gpu

GATT_ERR_TIMEOUT = 5


def test_pipeline_wait_gives_up_and_context_survives(cuda_lib, oracle_lib):
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    c = cs.periodic_box(n=32)
    f = cs.solenoidal_turbulence(c, seed=3)
    with GattDNS(c) as g:
        g.upload(f)
        rc = g.lib.gatt_selftest_pipeline_timeout(g.h)
        assert rc == GATT_ERR_TIMEOUT, (rc, g.lib.gatt_last_error().decode())
        assert "gave up" in g.lib.gatt_last_error().decode()
        # the flag was cleared and the context still solves lines correctly
        g.synchronize()
        a = g.calc_derivs(f["U"], 1)
        b = Oracle(c).calc_derivs(f["U"], 1)
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-12
