"""The CPU oracle against the reference's own Fortran (golden vectors).

tests/golden/reference_<case>.npz were made by tests/golden/make_reference_golden.py, which
runs the reference's unmodified derivs.F90, nseq.F90 and timeIntegration.F90 (and the
lid-driven disturbance) through a Fortran-subset translator on small cases (periodic box,
3-D and 2-D cavity channels with SFD, lid-driven cavity, boundary layer over a cavity, 2-D
and 3-D boundary layers with holdInlet and a periodicSine strip): the
line solves of every direction and kind, the right-hand side, the boundary conditions, the
filters with and without the blend, and one time step as main.F90 sequences it, with each
of its three integrators and with the reference's forcings.  Here the oracle runs the same
cases on the same inputs and must agree to 1e-12 relative (max-norm per field; the
translated Fortran evaluates every expression in the reference's operation order, so the
only differences are the oracle's own evaluation order where it fuses loops).
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12


def _load(name):
    import sys
    sys.path.insert(0, GOLD)
    import make_reference_golden as mk
    case = mk.golden_cases()[name]
    z = np.load(os.path.join(GOLD, "reference_%s.npz" % name))
    assert str(z["checksum"]) == mk.matrices_checksum(case), "case builder changed: regenerate the fixtures"
    return mk, case, z


def rel(a, b):
    s = np.max(np.abs(b))
    return float(np.max(np.abs(np.asarray(a) - b)) / (s if s > 0 else 1.0))


NAMES = ["box", "cavity3d", "cavity2d", "lid", "bl_cavity", "turb_box", "cavity2d_dpdx", "bl_hold", "bl_hold3d"]


def prime_hold(o, case, z, flow):
    """holdInlet keeps what the first applyBoundCond saw: the generator's first call was on
    the seeded flow at t (main.F90:112 makes it on the initial state), so make it here too."""
    if any(d["type"] == "holdInlet" for d in case.bc.disturbances):
        o.apply_bound_cond(flow, float(z["t"]))


@pytest.mark.parametrize("name", NAMES)
def test_line_solves_match_reference(oracle_lib, name):
    import oracle
    mk, case, z = _load(name)
    o = oracle.Oracle(case)
    F = z["F"]
    for d in range(1, 4 if case.is3d else 3):
        for kind in ("deriv", "filter"):
            assert rel(o.calc_derivs(F, d, kind), z["%s_%d" % (kind, d)]) < TOL, (name, d, kind)


@pytest.mark.parametrize("name", NAMES)
def test_rhs_matches_reference(oracle_lib, name):
    import oracle
    mk, case, z = _load(name)
    o = oracle.Oracle(case)
    flow = {k: z["flow_" + k] for k in ("U", "V", "W", "R", "E")}
    out = o.nseq(flow)
    for k in (("U", "V", "W", "R", "E") if case.is3d else ("U", "V", "R", "E")):
        assert rel(out[k], z["rhs_" + k]) < TOL, (name, k)


@pytest.mark.parametrize("name", NAMES)
def test_boundary_conditions_match_reference(oracle_lib, name):
    import oracle
    mk, case, z = _load(name)
    o = oracle.Oracle(case)
    flow = {k: z["flow_" + k] for k in ("U", "V", "W", "R", "E")}
    out = o.apply_bound_cond(flow, float(z["t"]))
    for k in ("U", "V", "W", "R", "E"):
        assert rel(out[k], z["bc_" + k]) < TOL, (name, k)


@pytest.mark.parametrize("name", NAMES)
def test_filters_match_reference(oracle_lib, name):
    import oracle
    mk, case, z = _load(name)
    o = oracle.Oracle(case)
    flow = {k: z["flow_" + k] for k in ("U", "V", "W", "R", "E")}
    for blend, key in ((-1.0, "filter_"), (0.3, "filterblend_")):
        out = o.apply_filters(flow, blend)
        for k in (("U", "V", "W", "R", "E") if case.is3d else ("U", "V", "R", "E")):
            assert rel(out[k], z[key + k]) < TOL, (name, blend, k)


@pytest.mark.parametrize("name", NAMES)
def test_time_step_matches_reference(oracle_lib, name):
    import oracle
    mk, case, z = _load(name)
    o = oracle.Oracle(case)
    flow = {k: z["flow_" + k] for k in ("U", "V", "W", "R", "E")}
    prime_hold(o, case, z, flow)
    st = o.new_state(flow)
    mc = o.step(st, float(z["t"]), float(z["dt"]))
    for k in ("U", "V", "W", "R", "E"):
        got = st["Wnew"] if (k == "W" and not case.is3d) else st[k]
        assert rel(got, z["step_" + k]) < TOL, (name, k)
    assert np.allclose(mc, z["step_maxchange"], rtol=1e-10, atol=1e-14), (name, mc, z["step_maxchange"])
    if case.sfd_type > 0:
        for k in ("U", "V", "W", "R", "E"):
            if k == "W" and not case.is3d:
                continue
            assert rel(st["m" + k], z["step_mean_" + k]) < TOL, (name, k)


@pytest.mark.parametrize("scheme", [2, 3])
@pytest.mark.parametrize("name", ["box", "cavity2d", "lid", "bl_cavity", "turb_box", "bl_hold", "bl_hold3d"])
def test_euler_and_ssprk3_steps_match_reference(oracle_lib, name, scheme):
    """timeStepping 2 (EULER_2D/3D) and 3 (SSPRK3_2D/3D) in the same main-loop step."""
    import dataclasses
    import oracle
    mk, case, z = _load(name)
    case = dataclasses.replace(case, time_stepping=scheme)
    key = {2: "euler_", 3: "ssprk3_"}[scheme]
    o = oracle.Oracle(case)
    flow = {k: z["flow_" + k] for k in ("U", "V", "W", "R", "E")}
    prime_hold(o, case, z, flow)
    st = o.new_state(flow)
    mc = o.step(st, float(z["t"]), float(z["dt"]))
    for k in ("U", "V", "W", "R", "E"):
        got = st["Wnew"] if (k == "W" and not case.is3d) else st[k]
        assert rel(got, z[key + k]) < TOL, (name, scheme, k)
    assert np.allclose(mc, z[key + "maxchange"], rtol=1e-10, atol=1e-14), (name, scheme, mc)
