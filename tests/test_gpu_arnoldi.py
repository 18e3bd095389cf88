"""GPU parity of the Jacobian-free Arnoldi driver (gatt_arnoldi).

* batched vs sequential: nbatch problems in one context give the same Hessenberg matrices,
  bit for bit, as each problem run alone (the batch only shares launches);
* against the oracle's restatement of calcInstability.m:304-400 (oracle/arnoldi.py).  The
  finite-difference quotient (UP - UM)/(eps*sqrt(N)) divides the 1e-12-level step
  differences by eps*sqrt(N), so the tests take eps = 1e-4 and compare H to 1e-6.
"""
import numpy as np
import pytest

from gatt_dns_b200 import case as cs

pytestmark = pytest.mark.gpu

H_TOL = 1e-6


def disturbances(case, nb, seed):
    """Seeded Gaussian disturbances in U and V (amplitude 1e-6)."""
    rng = np.random.default_rng(seed)
    s = (case.nx, case.ny, case.nz)
    out = []
    for _ in range(nb):
        d = {k: np.zeros(s, order="F") for k in ("U", "V", "W", "R", "E")}
        d["U"][...] = 1e-6 * rng.standard_normal(s)
        d["V"][...] = 1e-6 * rng.standard_normal(s)
        out.append(d)
    return out


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def box():
    c = cs.periodic_box(n=16)
    return c, cs.solenoidal_turbulence(c, seed=1234)


@pytest.fixture(scope="module")
def lid():
    c = cs.lid_driven(n=24)
    base = cs.uniform_flow(c)
    # flow region: interior nodes (walls and the lid excluded, as calcInstability.m:137-141
    # drops points outside the flow)
    region = np.zeros((c.nx, c.ny, c.nz), dtype=bool)
    region[1:-1, 1:-1, :] = True
    return c, base, region


def test_batched_equals_sequential(cuda_lib, box):
    from gatt_dns_b200.solver import GattDNS
    c, base = box
    nb, m, nsteps, dt = 3, 4, 6, 0.01
    v0 = disturbances(c, nb, seed=4321)
    with GattDNS(c, nbatch=nb) as g:
        Hb = g.arnoldi(base, v0, m, nsteps, dt, eps=1e-7)
    for b in range(nb):
        with GattDNS(c, nbatch=1) as g1:
            Hs = g1.arnoldi(base, [v0[b]], m, nsteps, dt, eps=1e-7)[0]
        assert np.array_equal(Hb[b], Hs), (b, rel(Hb[b], Hs))
    # a Hessenberg matrix with a positive subdiagonal
    assert np.all(np.triu(Hb[0], -1)[: m + 1, :m] == Hb[0])
    assert np.all(np.diag(Hb[0], -1) > 0)


def test_box_against_oracle(cuda_lib, oracle_lib, box):
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    from oracle.arnoldi import arnoldi as oracle_arnoldi
    c, base = box
    m, nsteps, dt, eps = 4, 6, 0.01, 1e-4
    v0 = disturbances(c, 2, seed=7)
    with GattDNS(c, nbatch=2) as g:
        H = g.arnoldi(base, v0, m, nsteps, dt, eps=eps)
    o = Oracle(c)
    for b in range(2):
        Ho = oracle_arnoldi(o, c, base, v0[b], m, nsteps, dt, eps)
        assert rel(H[b], Ho) < H_TOL, (b, rel(H[b], Ho))
        # Ritz values of the leading block agree as well
        ev, evo = np.linalg.eigvals(H[b, :m, :m]), np.linalg.eigvals(Ho[:m, :m])
        ev, evo = ev[np.argsort(-np.abs(ev))], evo[np.argsort(-np.abs(evo))]
        assert np.max(np.abs(ev - evo)) < H_TOL * np.max(np.abs(evo))


def test_lid_region_against_oracle(cuda_lib, oracle_lib, lid):
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    from oracle.arnoldi import arnoldi as oracle_arnoldi
    c, base, region = lid
    m, nsteps, dt, eps = 3, 5, 2e-3, 1e-4
    v0 = disturbances(c, 1, seed=11)
    with GattDNS(c, nbatch=1) as g:
        H = g.arnoldi(base, v0, m, nsteps, dt, eps=eps, region=region)[0]
        z = g.arnoldi_vector(0, 1)
    Ho = oracle_arnoldi(Oracle(c), c, base, v0[0], m, nsteps, dt, eps, region=region)
    assert rel(H, Ho) < H_TOL, rel(H, Ho)
    # basis vectors vanish outside the region and are unit vectors over it
    for k in ("U", "V", "R", "E"):
        assert np.all(z[k][~region] == 0.0)
    assert abs(sum(float(np.sum(z[k] ** 2)) for k in ("U", "V", "R", "E")) - 1.0) < 1e-12


def test_bad_arguments(cuda_lib, box):
    from gatt_dns_b200.solver import GattDNS
    from gatt_dns_b200._lib import GattError
    c, base = box
    with GattDNS(c, nbatch=1) as g:
        v0 = disturbances(c, 1, seed=1)
        with pytest.raises(GattError):
            g.arnoldi(base, v0, 0, 2, 0.01)
        with pytest.raises(GattError):
            g.arnoldi(base, v0, 2, 2, 0.01, eps=-1.0)
        with pytest.raises(GattError):
            g.arnoldi(base, v0, 2, 2, 0.01, region=np.zeros((c.nx, c.ny, c.nz), dtype=bool))
