"""GPU tests of the tangent-linear and adjoint (gatt_rhs_jvp / gatt_rhs_vjp / gatt_jvp / gatt_vjp).

Checks, on the 3-D periodic box and on a 3-D cavity channel with walls, corners and open-top
lists (the boundary program's tangent and its taped adjoint):
* transposed line operators: <L x, y> = <x, L^T y> per direction, derivative and filter;
* tangent of the RHS and of the step against central finite differences of the nonlinear
  GPU path (the Jacobian-free linearisation of calcInstability.m:353-390) and of the CPU
  oracle's step;
* dot-product tests <J v, w> = <v, J^T w> for the RHS and for several checkpointed steps;
* the gradient of J = 1/2 sum(u^2 + v^2 + w^2) after the steps against finite differences.
Tolerances: dot-product tests 1e-10 relative (both sides are one rounding-level apart);
central differences with h = 1e-4 relative to the field scale, O(h^2) truncation: 1e-6.
"""
import numpy as np
import pytest

from gatt_dns_b200 import case as cs

pytestmark = pytest.mark.gpu

KEYS = ("U", "V", "W", "R", "E")
DOT_TOL = 1e-10
FD_TOL = 1e-6


def dot(a, b):
    return float(sum(np.sum(a[k] * b[k]) for k in KEYS))


def axpy(a, x, y):
    return {k: a * x[k] + y[k] for k in KEYS}


def rel_err(a, b):
    num = max(float(np.max(np.abs(a[k] - b[k]))) for k in KEYS)
    den = max(float(np.max(np.abs(b[k]))) for k in KEYS)
    return num / den


def rand_flow(case, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    s = (case.nx, case.ny, case.nz)
    return {k: scale * rng.standard_normal(s) for k in KEYS}


_CASES = {}


def _case(name):
    if name not in _CASES:
        if name == "box":
            c = cs.periodic_box(n=16)
            q = cs.solenoidal_turbulence(c, seed=1234)
        elif name == "bl":
            # boundary layer: inflow Dirichlet, outflow pressure Dirichlet, open top, plate
            c = cs.boundary_layer(nx=48, ny=32, nz=16)
            q = cs.blasius_flow(c)
        else:
            # walls with isothermal Dirichlet and pressure Neumann lists, adiabatic corners,
            # an open top with null second derivatives: every op of the boundary program
            c = cs.cavity_channel(nx=24, ny=20, nz=8, adiabatic_corners=True)
            q = cs.random_flow(c, seed=5, amp=0.05)
        # a thermodynamic perturbation so that every variable's derivative path is exercised
        rng = np.random.default_rng(3)
        q = {k: np.array(v, copy=True) for k, v in q.items()}
        q["R"] = q["R"] * (1.0 + 0.01 * rng.standard_normal(q["R"].shape))
        q["E"] = q["E"] * (1.0 + 0.01 * rng.standard_normal(q["E"].shape))
        _CASES[name] = (c, q)
    return _CASES[name]


@pytest.fixture(scope="module", params=["box", "cavity3d", "bl"])
def box(request):
    return _case(request.param)


def test_transposed_line_operators(cuda_lib, box):
    from gatt_dns_b200.solver import GattDNS
    c, _ = box
    rng = np.random.default_rng(1)
    s = (c.nx, c.ny, c.nz)
    with GattDNS(c) as g:
        for d in (1, 2, 3):
            for kind in ("deriv", "filter"):
                x, y = rng.standard_normal(s), rng.standard_normal(s)
                lhs = float(np.sum(g.calc_derivs(x, d, kind) * y))
                rhs = float(np.sum(x * g.calc_derivs(y, d, kind + "_T")))
                assert abs(lhs - rhs) < DOT_TOL * abs(lhs), (d, kind, lhs, rhs)
    lid = cs.lid_driven(n=24)  # non-periodic lines with boundary stencils
    with GattDNS(lid) as g:
        s = (lid.nx, lid.ny, lid.nz)
        for d in (1, 2):
            for kind in ("deriv", "filter"):
                x, y = rng.standard_normal(s), rng.standard_normal(s)
                lhs = float(np.sum(g.calc_derivs(x, d, kind) * y))
                rhs = float(np.sum(x * g.calc_derivs(y, d, kind + "_T")))
                assert abs(lhs - rhs) < DOT_TOL * abs(lhs), ("lid", d, kind, lhs, rhs)


def test_rhs_tangent_against_differences(cuda_lib, box):
    from gatt_dns_b200.solver import GattDNS
    c, q = box
    v = rand_flow(c, 5, 1.0)
    h = 1e-4
    with GattDNS(c) as g:
        jv = g.rhs_jvp(q, v)
        fp = g.nseq(axpy(h, v, q))
        fm = g.nseq(axpy(-h, v, q))
    fd = {k: (fp[k] - fm[k]) / (2 * h) for k in KEYS}
    assert rel_err(jv, fd) < FD_TOL, rel_err(jv, fd)


def test_rhs_dot_product(cuda_lib, box):
    from gatt_dns_b200.solver import GattDNS
    c, q = box
    v, w = rand_flow(c, 6), rand_flow(c, 7)
    with GattDNS(c) as g:
        jv = g.rhs_jvp(q, v)
        jtw = g.rhs_vjp(q, w)
    a, b = dot(jv, w), dot(v, jtw)
    assert abs(a - b) < DOT_TOL * abs(a), (a, b)


def _dt(c, q):
    return c.cfl_dt(q["U"], q["V"], q["W"], 0.5)


def test_step_tangent_against_differences(cuda_lib, oracle_lib, box):
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    c, q = box
    dt, nsteps, h = _dt(c, q), 3, 1e-4
    v = rand_flow(c, 8)
    with GattDNS(c) as g:
        g.upload(q)
        jv = g.jvp(v, nsteps, 0.0, dt)
        out = {}
        for sgn in (1, -1):
            g.upload(axpy(sgn * h, v, q))
            g.run(nsteps, 0.0, dt)
            out[sgn] = g.download()
    fd = {k: (out[1][k] - out[-1][k]) / (2 * h) for k in KEYS}
    assert rel_err(jv, fd) < FD_TOL, rel_err(jv, fd)
    # the same linearisation through the CPU oracle's step
    o = Oracle(c)
    res = {}
    for sgn in (1, -1):
        st = o.new_state(axpy(sgn * h, v, q))
        t = 0.0
        for _ in range(nsteps):
            o.step(st, t, dt)
            t += dt
        res[sgn] = {k: st[k].copy() for k in KEYS}
    fdo = {k: (res[1][k] - res[-1][k]) / (2 * h) for k in KEYS}
    assert rel_err(jv, fdo) < FD_TOL, rel_err(jv, fdo)


@pytest.mark.parametrize("nsteps,every", [(1, 1), (5, 2), (6, 3)])
def test_step_dot_product_checkpointed(cuda_lib, box, nsteps, every):
    from gatt_dns_b200.solver import GattDNS
    c, q = box
    dt = _dt(c, q)
    v, w = rand_flow(c, 9), rand_flow(c, 10)
    with GattDNS(c) as g:
        g.upload(q)
        jv = g.jvp(v, nsteps, 0.0, dt)
        g.upload(q)
        jtw = g.vjp(w, nsteps, 0.0, dt, checkpoint_every=every)
        end = g.download()
        g.upload(q)
        g.run(nsteps, 0.0, dt)
        ref_end = g.download()
    a, b = dot(jv, w), dot(v, jtw)
    assert abs(a - b) < DOT_TOL * abs(a), (a, b)
    # the state is left at the end of the forward run
    assert rel_err(end, ref_end) == 0.0


def test_energy_gradient(cuda_lib, box):
    """dJ/dq0 for J = 1/2 sum(u^2 + v^2 + w^2) after the steps, against differences."""
    from gatt_dns_b200.solver import GattDNS
    c, q = box
    dt, nsteps, h = _dt(c, q), 4, 1e-4
    v = rand_flow(c, 11)

    def J(g, q0):
        g.upload(q0)
        g.run(nsteps, 0.0, dt)
        f = g.download()
        return 0.5 * float(np.sum(f["U"] ** 2 + f["V"] ** 2 + f["W"] ** 2)), f

    with GattDNS(c) as g:
        _, fN = J(g, q)
        lamN = {"U": fN["U"], "V": fN["V"], "W": fN["W"], "R": 0 * fN["R"], "E": 0 * fN["E"]}
        g.upload(q)
        grad = g.vjp(lamN, nsteps, 0.0, dt, checkpoint_every=2)
        jp, _ = J(g, axpy(h, v, q))
        jm, _ = J(g, axpy(-h, v, q))
    fd = (jp - jm) / (2 * h)
    ad = dot(grad, v)
    assert abs(ad - fd) < FD_TOL * abs(fd), (ad, fd)
