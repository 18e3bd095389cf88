"""The CPU oracle (restatement of derivs.F90 / nseq.F90 / timeIntegration.F90 / main.F90)
checked against closed-form answers, since the reference provides no golden outputs.
"""
import math

import numpy as np
import pytest

from gatt_dns_b200 import case as cs
from gatt_dns_b200 import matrices as mx


@pytest.fixture(scope="module")
def box():
    from oracle import Oracle
    c = cs.periodic_box(n=32)
    return c, Oracle(c)


def _mesh(c):
    return np.meshgrid(c.X, c.Y, c.Z, indexing="ij")


def sl4_modified_wavenumber(kh):
    cl, cr, _, _ = mx.finite_difference_coefficients("SL4")
    return (2 * cr[1] * math.sin(kh) + 2 * cr[2] * math.sin(2 * kh)) / (1 + 2 * cl[1] * math.cos(kh))


@pytest.mark.parametrize("k", [1, 3, 7])
def test_periodic_derivative_equals_modified_wavenumber(box, oracle_lib, k):
    """On a uniform periodic grid a compact scheme maps sin(kx) exactly to k'(k) cos(kx)."""
    c, o = box
    X, Y, Z = _mesh(c)
    h = c.X[1] - c.X[0]
    kp = sl4_modified_wavenumber(k * h) / h
    for d, coord in enumerate((X, Y, Z)):
        F = np.asfortranarray(np.sin(k * coord))
        dF = o.calc_derivs(F, d + 1)
        assert np.max(np.abs(dF - kp * np.cos(k * coord))) < 5e-12


@pytest.mark.parametrize("k", [2, 9, 16])
def test_periodic_filter_equals_transfer_function(box, oracle_lib, k):
    c, o = box
    X, _, _ = _mesh(c)
    h = c.X[1] - c.X[0]
    lhs, rhs, _, _ = mx.spatial_filter_coefficients(0.49)
    w = k * h
    T = (rhs[0] + 2 * sum(rhs[n] * math.cos(n * w) for n in range(1, 6))) / (1 + 2 * 0.49 * math.cos(w))
    F = np.asfortranarray(np.cos(k * X + 0.3))
    Ff = o.calc_derivs(F, 1, "filter")
    assert np.max(np.abs(Ff - T * F)) < 1e-12


def test_uniform_state_is_steady(box, oracle_lib):
    c, o = box
    f = cs.uniform_flow(c, U0=0.3)
    k = o.nseq(f)
    for key in ("U", "V", "W", "R", "E"):
        assert np.max(np.abs(k[key])) < 1e-12


def test_periodic_mass_is_conserved(box, oracle_lib):
    """dR = -div(rho u) discretised with the periodic compact scheme integrates to ~0."""
    c, o = box
    f = cs.solenoidal_turbulence(c, seed=3)
    st = o.new_state(f)
    m0 = np.sum(st["R"])
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.3)
    for s in range(3):
        o.step(st, s * dt, dt)
    assert abs(np.sum(st["R"]) - m0) / m0 < 1e-12


def test_lid_driven_bcs(oracle_lib):
    from oracle import Oracle
    c = cs.lid_driven(n=24)
    o = Oracle(c)
    f = o.apply_bound_cond(cs.uniform_flow(c))
    # lid profile U0 (1 - (2 xi - 1)^18)^2 on the top row, zero on the other walls
    xi = (c.X - c.X[0]) / (c.X[-1] - c.X[0])
    assert np.allclose(f["U"][:, -1, 0], (1 - (2 * xi - 1) ** 18) ** 2, atol=1e-14)
    assert np.all(f["U"][:, 0, 0] == 0) and np.all(f["U"][0, :-1, 0] == 0)
    # pressure at rest stays P0 = (gamma-1) E0: R = 1 everywhere
    assert np.allclose(f["R"], 1.0, atol=1e-13)


def test_divergence_is_reported(oracle_lib):
    from oracle import Oracle
    c = cs.lid_driven(n=16)
    o = Oracle(c)
    f = cs.uniform_flow(c)
    f["E"][5, 5, 0] = np.nan
    st = o.new_state(f)
    mc = o.step(st, 0.0, 1e-3)
    assert np.isnan(mc).any()
