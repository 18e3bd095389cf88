"""GPU tests of the tangent-linear and adjoint on 2-D cases and on cases with SFD.

In 2-D the entry points run the 3-D data flow without a z direction (W components zero);
with SFD the step maps the state and the mean, and the step vectors carry both (keys mU ...
mE).  Cases: the 2-D lid-driven cavity (wall lists, corners, the moving-lid disturbance),
a 2-D and a 3-D cavity channel with SFD on a buffer ramp, and the 2-D boundary layer over a
cavity (free-slip upstream wall, break point, SFD in the buffer zones: the config-3 base-flow
problem), and 2-D and 3-D boundary layers that start downstream of the leading edge (holdInlet
on the inflow plane, with the density held in 3-D; a periodicSine strip on the plate).  Checks as in test_gpu_tangent.py: RHS and step tangents against central finite
differences of the nonlinear path (state and mean perturbed together), dot-product tests of
the checkpointed adjoint, and the gradient of J = 1/2 sum(u^2 + v^2 + w^2).
Tolerances: dot-product tests 1e-10 relative; central differences with h = 1e-4: 1e-6 (the
gradient: Richardson-extrapolated central differences, 1e-6).
"""
import numpy as np
import pytest

from gatt_dns_b200 import case as cs

pytestmark = pytest.mark.gpu

KEYS = ("U", "V", "W", "R", "E")
MKEYS = ("mU", "mV", "mW", "mR", "mE")
DOT_TOL = 1e-10
FD_TOL = 1e-6

_CASES = {}


def _case(name):
    if name not in _CASES:
        if name == "lid":
            c = cs.lid_driven(n=24)
            q = cs.random_flow(c, seed=5, amp=0.05)
        elif name == "cavity2d_sfd":
            c = cs.cavity_channel(nx=24, ny=20, nz=1, sfd={"X": 0.05, "Delta": 10.0, "buffer": 6})
            q = cs.random_flow(c, seed=5, amp=0.05)
        elif name == "cavity3d_sfd":
            c = cs.cavity_channel(nx=24, ny=20, nz=8, adiabatic_corners=True,
                                  sfd={"X": 0.05, "Delta": 10.0, "buffer": 6})
            q = cs.random_flow(c, seed=5, amp=0.05)
        elif name in ("bl_hold", "bl_hold3d"):
            if name == "bl_hold":
                c = cs.boundary_layer_isothermal(40, 28, 1, x_range=(0.5, 4.0))
            else:
                c = cs.boundary_layer_isothermal(24, 24, 8, x_range=(0.5, 3.0))
                c.bc.disturbances[0]["par"] = [1.0]  # hold the density too
            c = cs.periodic_sine_strip(c, 6, 14)
            q = cs.blasius_flow(c)
            r = cs.random_flow(c, seed=5, amp=0.01)
            for k in ("U", "V", "W"):
                q[k] = q[k] + r[k]
        else:
            c = cs.boundary_layer_cavity(nx=64, ny=40, buffers=((6, 5), (0, 6)))
            q = cs.blasius_flow(c)
            r = cs.random_flow(c, seed=5, amp=0.01)
            for k in ("U", "V"):
                q[k] = q[k] + r[k]
        rng = np.random.default_rng(3)
        q = {k: np.array(v, copy=True) for k, v in q.items()}
        q["R"] = q["R"] * (1.0 + 0.01 * rng.standard_normal(q["R"].shape))
        q["E"] = q["E"] * (1.0 + 0.01 * rng.standard_normal(q["E"].shape))
        if not c.is3d:
            q["W"] = np.zeros_like(q["W"])
        # the SFD mean: the state, slightly off (so that the relaxation acts)
        m = None
        if c.sfd_type:
            m = {k: q[k] * (1.0 + 0.02 * rng.standard_normal(q[k].shape)) for k in KEYS}
            if not c.is3d:
                m["W"] = np.zeros_like(m["W"])
        _CASES[name] = (c, q, m)
    return _CASES[name]


@pytest.fixture(scope="module", params=["lid", "cavity2d_sfd", "cavity3d_sfd", "bl_cavity", "bl_hold", "bl_hold3d"])
def case(request):
    return _case(request.param)


def rand_vec(c, seed, with_mean):
    rng = np.random.default_rng(seed)
    s = (c.nx, c.ny, c.nz)
    v = {k: rng.standard_normal(s) for k in KEYS}
    if with_mean:
        v.update({mk: rng.standard_normal(s) for mk in MKEYS})
    if not c.is3d:
        v["W"] = np.zeros(s)
        if with_mean:
            v["mW"] = np.zeros(s)
    return v


def dot(a, b):
    return float(sum(np.sum(a[k] * b[k]) for k in a if k in b))


def rel_err(a, b, keys):
    num = max(float(np.max(np.abs(a[k] - b[k]))) for k in keys)
    den = max(float(np.max(np.abs(b[k]))) for k in keys)
    return num / den


def _dt(c, q):
    return c.cfl_dt(q["U"], q["V"], q["W"], 0.5)


def _prime(g, c, q, m):
    """holdInlet: the first boundary-condition call keeps the unperturbed inflow plane."""
    if any(d["type"] == "holdInlet" for d in c.bc.disturbances):
        _start(g, q, m)
        g.apply_bound_cond(0.0)


def _start(g, q, m, v=None, h=0.0):
    """Upload state (and mean) q + h v."""
    g.upload({k: q[k] + h * v[k] for k in KEYS} if v is not None else q)
    if m is not None:
        g.upload_mean({k: m[k] + h * v["m" + k] for k in KEYS} if v is not None else m)


def test_rhs_tangent_and_dot_product(cuda_lib, case):
    from gatt_dns_b200.solver import GattDNS
    c, q, _ = case
    v, w = rand_vec(c, 5, False), rand_vec(c, 6, False)
    h = 1e-4
    keys = KEYS if c.is3d else ("U", "V", "R", "E")
    with GattDNS(c) as g:
        jv = g.rhs_jvp(q, v)
        fp = g.nseq({k: q[k] + h * v[k] for k in KEYS})
        fm = g.nseq({k: q[k] - h * v[k] for k in KEYS})
        jtw = g.rhs_vjp(q, w)
    fd = {k: (fp[k] - fm[k]) / (2 * h) for k in keys}
    assert rel_err(jv, fd, keys) < FD_TOL, rel_err(jv, fd, keys)
    if not c.is3d:
        assert np.all(jv["W"] == 0.0) and np.all(jtw["W"] == 0.0)
    a, b = dot(jv, w), dot(v, jtw)
    assert abs(a - b) < DOT_TOL * abs(a), (a, b)


def test_step_tangent_against_differences(cuda_lib, case):
    from gatt_dns_b200.solver import GattDNS
    c, q, m = case
    sfd = m is not None
    dt, nsteps, h = _dt(c, q), 3, 1e-4
    v = rand_vec(c, 8, sfd)
    keys = (KEYS if c.is3d else ("U", "V", "R", "E"))
    with GattDNS(c) as g:
        _prime(g, c, q, m)
        _start(g, q, m)
        jv = g.jvp(v, nsteps, 0.0, dt)
        out = {}
        for sgn in (1, -1):
            _start(g, q, m, v, sgn * h)
            g.run(nsteps, 0.0, dt)
            out[sgn] = g.download()
            if sfd:
                out[sgn].update({"m" + k: x for k, x in g.download_mean().items()})
    allk = keys + (tuple("m" + k for k in keys) if sfd else ())
    fd = {k: (out[1][k] - out[-1][k]) / (2 * h) for k in allk}
    assert rel_err(jv, fd, allk) < FD_TOL, rel_err(jv, fd, allk)


@pytest.mark.parametrize("nsteps,every", [(1, 1), (5, 2)])
def test_step_dot_product_checkpointed(cuda_lib, case, nsteps, every):
    from gatt_dns_b200.solver import GattDNS
    c, q, m = case
    sfd = m is not None
    dt = _dt(c, q)
    v, w = rand_vec(c, 9, sfd), rand_vec(c, 10, sfd)
    with GattDNS(c) as g:
        _prime(g, c, q, m)
        _start(g, q, m)
        jv = g.jvp(v, nsteps, 0.0, dt)
        _start(g, q, m)
        jtw = g.vjp(w, nsteps, 0.0, dt, checkpoint_every=every)
        end = g.download()
        _start(g, q, m)
        g.run(nsteps, 0.0, dt)
        ref_end = g.download()
    a, b = dot(jv, w), dot(v, jtw)
    assert abs(a - b) < DOT_TOL * abs(a), (a, b)
    for k in KEYS:
        assert np.array_equal(end[k], ref_end[k]), k  # left at the end of the forward run


def test_energy_gradient(cuda_lib, case):
    """dJ/dq0 . v from the adjoint against a central difference of J along v, Richardson
    extrapolated over steps h and h/2 (these cases are strongly nonlinear: the plain central
    difference at h = 1e-4 is off by ~1e-4 relative, an h^2 term that the extrapolation
    removes); J differences are formed from the field differences, not from two large sums."""
    from gatt_dns_b200.solver import GattDNS
    c, q, m = case
    sfd = m is not None
    dt, nsteps = _dt(c, q), 4
    v = rand_vec(c, 11, sfd)
    vel = ("U", "V", "W") if c.is3d else ("U", "V")

    def final(g, vv=None, hh=0.0):
        _start(g, q, m, vv, hh)
        g.run(nsteps, 0.0, dt)
        return g.download()

    def fd(g, h):
        up, um = final(g, v, h), final(g, v, -h)
        return float(sum(np.sum((up[k] - um[k]) * (up[k] + um[k])) for k in vel)) / (4 * h)

    with GattDNS(c) as g:
        _prime(g, c, q, m)
        fN = final(g)
        z = np.zeros_like(fN["R"])
        lamN = {"U": fN["U"], "V": fN["V"], "W": fN["W"] if c.is3d else z, "R": z, "E": z}
        if sfd:
            lamN.update({mk: z for mk in MKEYS})
        _start(g, q, m)
        grad = g.vjp(lamN, nsteps, 0.0, dt, checkpoint_every=2)
        h = 1e-4
        rich = (4.0 * fd(g, h / 2) - fd(g, h)) / 3.0
    ad = dot(grad, v)
    assert abs(ad - rich) < FD_TOL * abs(rich), (ad, rich)


def test_sfd_step_needs_the_mean(cuda_lib):
    """gatt_jvp / gatt_vjp on an SFD case before the mean exists: GATT_ERR_STATE."""
    from gatt_dns_b200.solver import GattDNS
    from gatt_dns_b200._lib import GattError
    c = cs.cavity_channel(nx=24, ny=20, nz=8, sfd={"X": 0.05, "Delta": 10.0, "buffer": 6})
    with GattDNS(c) as g:
        f = cs.uniform_flow(c)
        g.upload(f)
        with pytest.raises(GattError) as e:
            g.jvp(rand_vec(c, 1, True), 1, 0.0, 1e-3)
        assert e.value.code == 6
