"""The host time loop (main.F90:192-533) and the flow files (exportFlow / importFlow).

CPU: flow-file round trip, wall NaNs, naming, log columns, the CFL rate.  GPU: the loop on
the device context and on an oracle-backed stand-in with the same interface export the same
flows (1e-10) and the same log."""
import os

import numpy as np
import pytest

from gatt_dns_b200 import case as cs
from gatt_dns_b200 import timeloop as tl


def test_flow_file_round_trip(tmp_path):
    c = cs.lid_driven(n=16)
    f = cs.random_flow(c, seed=1)
    wall = np.zeros((c.nx, c.ny, c.nz), dtype=bool)
    wall[0, 0, 0] = True
    p = tl.flow_path(str(tmp_path), 7)
    assert os.path.basename(p) == "flow_0000000007.mat"
    assert os.path.basename(tl.flow_path("x", -1)) == "flow_-000000001.mat"
    tl.write_flow(p, f, 0.25, inside_wall=wall)
    g, t = tl.read_flow(p, (c.nx, c.ny, c.nz))
    assert t == 0.25
    for k in tl.KEYS:
        assert np.array_equal(g[k][~wall], f[k][~wall])
    assert g["U"][0, 0, 0] == 0.0 and g["R"][0, 0, 0] == 1.0 and g["E"][0, 0, 0] == 1.0


def test_log_line_and_cfl_rate():
    line = tl.log_line(3, 10, 0.5, 1e-3, 0.45, [1e-3, 2e-3, 0.0, 4e-4, 5e-5], [[0.0, 1.0, 2.0, 3.0, 4.0]])
    cols = line.split("\t")
    assert len(cols) == 10 + 5 and cols[0].strip() == "3" and cols[1].strip() == "10" and cols[10] == "0"
    c = cs.lid_driven(n=16)
    f = cs.random_flow(c, seed=2)
    vmax = [float(np.max(np.abs(f[k]))) for k in ("U", "V", "W")]
    assert abs(0.5 / tl.cfl_rate(c, vmax) - c.cfl_dt(f["U"], f["V"], f["W"], 0.5)) < 1e-15


class _OracleContext:
    """The part of GattDNS the loop uses, on the CPU oracle."""

    def __init__(self, case, flow):
        from oracle import Oracle
        self.case = case
        self.o = Oracle(case)
        self.st = self.o.new_state(flow)

    def max_velocity(self):
        return np.array([[float(np.max(np.abs(self.st[k]))) for k in ("U", "V", "W")]])

    def step(self, t, dt):
        return np.array([self.o.step(self.st, t, dt)])

    def download(self):
        return {k: self.st[k].copy() for k in tl.KEYS}


@pytest.mark.gpu
def test_loop_matches_oracle_loop(cuda_lib, oracle_lib, tmp_path):
    from gatt_dns_b200.solver import GattDNS
    c = cs.lid_driven(n=32)
    f = cs.uniform_flow(c)
    g = GattDNS(c)
    g.upload(f)
    g.apply_bound_cond(0.0)
    f0 = g.download()
    dg, do = tmp_path / "gpu", tmp_path / "oracle"
    dg.mkdir()
    do.mkdir()
    kw = dict(time_control=2, dtmax=1.0, max_cfl=0.5, qtimes=0.01, tmax=0.03, tracked=[(16, 16, 1)])
    rg = tl.run(g, folder=str(dg), **kw)
    ro = tl.run(_OracleContext(c, f0), folder=str(do), **kw)
    g.close()
    assert rg[1:] == ro[1:] and abs(rg[0] - ro[0]) < 1e-12
    saved = sorted(x for x in os.listdir(dg) if x.startswith("flow_"))
    assert saved == sorted(x for x in os.listdir(do) if x.startswith("flow_")) and len(saved) >= 2
    # a save interval cut short by tmax is numbered but not exported (as in main.F90)
    for n in range(1, len(saved) + 1):
        a, ta = tl.read_flow(tl.flow_path(str(dg), n), (c.nx, c.ny, c.nz))
        b, tb = tl.read_flow(tl.flow_path(str(do), n), (c.nx, c.ny, c.nz))
        assert abs(ta - tb) < 1e-12
        for k in tl.KEYS:
            assert np.max(np.abs(a[k] - b[k])) <= 1e-10 * max(1.0, np.max(np.abs(b[k]))), (n, k)
    lg = (dg / "log.txt").read_text().splitlines()
    lo = (do / "log.txt").read_text().splitlines()
    assert len(lg) == len(lo) == rg[1]
    assert [x.split("\t")[:2] for x in lg] == [x.split("\t")[:2] for x in lo]
