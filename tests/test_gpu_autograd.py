"""The tangent-linear and adjoint entry points driven through torch.autograd.

tests/gatt_autograd.py wraps ``gatt_rhs_jvp`` / ``gatt_rhs_vjp`` and ``gatt_jvp`` /
``gatt_vjp`` as the forward- and reverse-mode rules of two torch.autograd.Functions (a test
harness only).  Through them:
* ``torch.autograd.gradcheck`` (fast mode, reverse and forward mode) against torch's own
  central differences of the nonlinear C-ABI path;
* the dot-product test <J v, w> = <v, J^T w> with J v from a forward-mode dual and J^T w from
  ``torch.autograd.grad``;
* the tangent of a multi-step run against the reference's Jacobian-free linearisation,
  B = (Phi(q + eps sqrt(N) zeta) - Phi(q)) / (eps sqrt(N)) with eps = 1e-7 and its central
  form (calcInstability.m:353-390);
* the gradient of J = 1/2 sum(u^2 + v^2 + w^2) after the run, from ``backward()``, against a
  Richardson-extrapolated central difference.
Tolerances: dot products 1e-10 relative; gradcheck 1e-6 relative (central differences of
step 1e-6 along a unit direction); first-order linearisation O(eps sqrt(N)) = 1e-4 relative,
central (step 1e-4) 1e-6; gradient 1e-6.
"""
import numpy as np
import pytest
import torch
import torch.autograd.forward_ad as fwAD

from gatt_dns_b200 import case as cs
from gatt_autograd import RHS, Steps

pytestmark = pytest.mark.gpu

NSTEPS, EVERY = 4, 2


def _state(name):
    if name == "box":
        c = cs.periodic_box(n=16)
        q = cs.solenoidal_turbulence(c, seed=1234)
    else:
        c = cs.boundary_layer(nx=48, ny=32, nz=16)
        q = cs.blasius_flow(c)
        r = cs.random_flow(c, seed=3, amp=0.01)
        for k in ("U", "V", "W"):
            q[k] = q[k] + r[k]
    rng = np.random.default_rng(3)
    q = {k: np.array(v, copy=True) for k, v in q.items()}
    q["R"] = q["R"] * (1.0 + 0.01 * rng.standard_normal(q["R"].shape))
    q["E"] = q["E"] * (1.0 + 0.01 * rng.standard_normal(q["E"].shape))
    return c, q


@pytest.fixture(scope="module", params=["box", "bl"])
def setup(request, cuda_lib):
    from gatt_dns_b200.solver import GattDNS
    c, q = _state(request.param)
    g = GattDNS(c)
    q0 = torch.from_numpy(g._pack(q))
    dt = 0.25 * c.cfl_dt(q["U"], q["V"], q["W"], 1.0)
    yield c, g, q0, dt
    g.close()


def _rand(n, seed):
    return torch.from_numpy(np.random.default_rng(seed).standard_normal(n))


def test_gradcheck_rhs(setup):
    c, g, q0, _ = setup
    q = q0.clone().requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x: RHS.apply(x, g), (q,), eps=1e-6, atol=1e-5, rtol=1e-6,
                                    fast_mode=True, check_forward_ad=True, check_undefined_grad=False)


def test_gradcheck_steps(setup):
    c, g, q0, dt = setup
    q = q0.clone().requires_grad_(True)
    assert torch.autograd.gradcheck(lambda x: Steps.apply(x, g, NSTEPS, 0.0, dt, EVERY), (q,), eps=1e-6,
                                    atol=1e-6, rtol=1e-6, fast_mode=True, check_forward_ad=True,
                                    check_undefined_grad=False)


@pytest.mark.parametrize("which", ["rhs", "steps"])
def test_dot_product_through_autograd(setup, which):
    c, g, q0, dt = setup
    n = q0.numel()
    v, w = _rand(n, 5), _rand(n, 6)
    f = (lambda x: RHS.apply(x, g)) if which == "rhs" else (lambda x: Steps.apply(x, g, NSTEPS, 0.0, dt, EVERY))
    with fwAD.dual_level():
        jv = fwAD.unpack_dual(f(fwAD.make_dual(q0, v))).tangent
    q = q0.clone().requires_grad_(True)
    (jtw,) = torch.autograd.grad(f(q), q, w)
    a, b = float(torch.dot(jv, w)), float(torch.dot(v, jtw))
    assert abs(a - b) < 1e-10 * max(abs(a), abs(b)), (which, a, b)


def test_tangent_against_jacobian_free_linearisation(setup):
    """J zeta of the run against calcInstability.m's finite difference of two nonlinear runs,
    first order (eps = 1e-7, the instability analysis' default) and central."""
    c, g, q0, dt = setup
    n = q0.numel()
    zeta = _rand(n, 8)
    zeta = zeta / torch.linalg.norm(zeta)
    with fwAD.dual_level():
        jz = fwAD.unpack_dual(Steps.apply(fwAD.make_dual(q0, zeta), g, NSTEPS, 0.0, dt, EVERY)).tangent
    h = 1e-7 * np.sqrt(n)
    base = Steps.apply(q0, g, NSTEPS, 0.0, dt, EVERY)
    plus = Steps.apply(q0 + h * zeta, g, NSTEPS, 0.0, dt, EVERY)
    b1 = (plus - base) / h
    scale = float(torch.max(torch.abs(jz)))
    assert float(torch.max(torch.abs(b1 - jz))) < 1e-4 * scale
    h2 = 1e-4
    minus = Steps.apply(q0 - h2 * zeta, g, NSTEPS, 0.0, dt, EVERY)
    plus2 = Steps.apply(q0 + h2 * zeta, g, NSTEPS, 0.0, dt, EVERY)
    b2 = (plus2 - minus) / (2 * h2)
    assert float(torch.max(torch.abs(b2 - jz))) < 1e-6 * scale


def test_energy_gradient_by_backward(setup):
    """dJ/dq0 . d from backward() against a central difference of J along the unit direction
    d, Richardson extrapolated over steps h and h/2; J differences come from the field
    differences (J itself is a large sum whose rounding would swamp a difference of it)."""
    c, g, q0, dt = setup
    npts = c.nx * c.ny * c.nz
    vel = slice(0, 3 * npts)

    def energy(x):
        y = Steps.apply(x, g, NSTEPS, 0.0, dt, EVERY)
        return 0.5 * torch.sum(y[vel] ** 2)

    q = q0.clone().requires_grad_(True)
    energy(q).backward()
    d = _rand(q0.numel(), 9)
    d = d / torch.linalg.norm(d)

    def fd(h):
        with torch.no_grad():
            up = Steps.apply(q0 + h * d, g, NSTEPS, 0.0, dt, EVERY)[vel]
            um = Steps.apply(q0 - h * d, g, NSTEPS, 0.0, dt, EVERY)[vel]
        return float(torch.sum((up - um) * (up + um))) / (4 * h)

    h = 1e-4
    rich = (4.0 * fd(h / 2) - fd(h)) / 3.0
    an = float(torch.dot(q.grad, d))
    assert abs(an - rich) < 1e-6 * abs(an), (an, rich)
