"""GPU parity: the CUDA path through the C-ABI against the CPU oracle on the same inputs.

Tolerances (FP64; the kernels keep the reference's per-line operation order, so the
differences are rounding only):
* one line solve or one RHS evaluation: 1e-12 relative (max-norm per field)
* one time step: 1e-12 relative; 100 steps: 1e-9 relative
"""
import numpy as np
import pytest

from gatt_dns_b200 import case as cs

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
STEP_TOL = 1e-12
LONG_TOL = 1e-9
KEYS = ("U", "V", "W", "R", "E")


def rel(a, b):
    s = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (s if s > 0 else 1.0))


def fields(case):
    return KEYS if case.is3d else ("U", "V", "R", "E")


_CASES = {}


def get_case(name):
    if name not in _CASES:
        if name == "box":
            _CASES[name] = cs.periodic_box(n=32)
        elif name == "box_aniso":
            _CASES[name] = cs.periodic_box(nxyz=(40, 24, 16))
        elif name == "lid":
            _CASES[name] = cs.lid_driven(n=48)
        elif name == "lid_tanh":
            _CASES[name] = cs.lid_driven(nxy=(40, 36), mesh_type="tanh")
        elif name == "cavity2d":
            _CASES[name] = cs.cavity_channel(nx=48, ny=40, nz=1, sfd={"X": 0.05, "Delta": 10.0, "buffer": 8})
        elif name == "cavity3d":
            _CASES[name] = cs.cavity_channel(nx=24, ny=20, nz=8, adiabatic_corners=True,
                                             sfd={"X": 0.05, "Delta": 10.0, "buffer": 6})
        elif name == "box64":
            _CASES[name] = cs.periodic_box(n=64)
        elif name == "lid64":
            _CASES[name] = cs.lid_driven(n=64)
        elif name == "cavity3d_32":
            _CASES[name] = cs.cavity_channel(nx=32, ny=32, nz=16, adiabatic_corners=True,
                                             sfd={"X": 0.05, "Delta": 10.0, "buffer": 6})
        elif name == "bl":
            _CASES[name] = cs.boundary_layer(nx=48, ny=32, nz=16)
        elif name == "bl_cavity":
            _CASES[name] = cs.boundary_layer_cavity(nx=96, ny=48, buffers=((8, 6), (0, 8)))
        elif name == "long_x":
            _CASES[name] = cs.lid_driven(nxy=(900, 12))
        elif name == "lid_x400":
            # 400-point x lines: 25 row blocks, the wide pipelined solver
            _CASES[name] = cs.lid_driven(nxy=(400, 16))
        elif name == "lid_y300":
            # 300-point y lines: padded to 304, two tensor boxes of 152 rows, 19 row blocks
            _CASES[name] = cs.lid_driven(nxy=(16, 300))
        elif name == "box_y288":
            _CASES[name] = cs.periodic_box(nxyz=(16, 288, 8))
        elif name == "box_x400":
            _CASES[name] = cs.periodic_box(nxyz=(400, 16, 8))
        elif name == "box_yz32":
            # y and z lines of equal length (one launch) and a partial x tile (24 of 32 lanes)
            _CASES[name] = cs.periodic_box(nxyz=(24, 32, 32))
        elif name == "box_ragged":
            # 5040 points: the last 256-point chunk of the tensor-copy assembly is partial
            _CASES[name] = cs.periodic_box(nxyz=(20, 18, 14))
        elif name == "box_odd":
            # 5187 points (odd): the assembly takes the thread-load kernel
            _CASES[name] = cs.periodic_box(nxyz=(21, 19, 13))
    return _CASES[name]


def flow_for(case, seed=5):
    return cs.random_flow(case, seed=seed, amp=0.05)


@pytest.fixture(scope="module")
def libs(cuda_lib, oracle_lib):
    return cuda_lib, oracle_lib


def pair(name):
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    c = get_case(name)
    return c, GattDNS(c), Oracle(c)


@pytest.mark.parametrize("name", ["box", "box_aniso", "box64", "lid", "lid64", "lid_tanh", "cavity2d", "cavity3d",
                                  "cavity3d_32", "long_x", "lid_x400", "box_x400", "lid_y300", "box_y288"])
@pytest.mark.parametrize("kind", ["deriv", "filter"])
@pytest.mark.parametrize("solver", ["pipe", "reg", "tile"])
def test_line_solves(libs, monkeypatch, name, kind, solver):
    """The three line-solve kernel families (register rows fed by the TMA ring, register rows
    loaded from global memory, shared-memory tile) against the oracle; GATT_SWEEP is read
    when matrices are set."""
    monkeypatch.setenv("GATT_SWEEP", solver)
    c, g, o = pair(name)
    rng = np.random.default_rng(11)
    F = np.asfortranarray(rng.standard_normal((c.nx, c.ny, c.nz)))
    for d in range(1, 4 if c.is3d else 3):
        a = g.calc_derivs(F, d, kind)
        b = o.calc_derivs(F, d, kind)
        assert rel(a, b) < RHS_TOL, (name, kind, d, rel(a, b))
    g.close()


@pytest.mark.parametrize("name", ["box", "box_aniso", "box64", "box_yz32", "lid", "lid64", "lid_tanh", "cavity2d",
                                  "cavity3d", "cavity3d_32", "bl", "bl_cavity"])
def test_rhs(libs, name):
    c, g, o = pair(name)
    f = flow_for(c)
    a, b = g.nseq(f), o.nseq(f)
    for k in fields(c):
        assert rel(a[k], b[k]) < RHS_TOL, (name, k, rel(a[k], b[k]))
    g.close()


@pytest.mark.parametrize("name", ["lid", "cavity2d", "cavity3d"])
def test_boundary_conditions(libs, name):
    c, g, o = pair(name)
    f = flow_for(c, seed=9)
    g.upload(f)
    g.apply_bound_cond(0.0)
    a = g.download()
    b = o.apply_bound_cond(f)
    for k in KEYS:
        assert rel(a[k], b[k]) < 1e-14, (name, k)
    g.close()


@pytest.mark.parametrize("name", ["box", "lid", "cavity3d"])
def test_filter_in_place(libs, name):
    c, g, o = pair(name)
    f = flow_for(c, seed=4)
    for blend in (-1.0, 0.3):
        g.upload(f)
        g.apply_filters(blend)
        a = g.download()
        b = o.apply_filters(f, blend)
        for k in fields(c):
            assert rel(a[k], b[k]) < RHS_TOL, (name, blend, k)
    g.close()


@pytest.mark.parametrize("name", ["box", "box_aniso", "box64", "lid", "lid64", "lid_tanh", "cavity2d", "cavity3d",
                                  "cavity3d_32", "bl", "bl_cavity", "box_ragged", "box_odd", "lid_x400", "box_x400",
                                  "lid_y300", "box_y288"])
def test_step(libs, name):
    c, g, o = pair(name)
    f = flow_for(c, seed=2)
    dt = 0.25 * c.cfl_dt(f["U"], f["V"], f["W"], 1.0)
    g.upload(f)
    st = o.new_state(f)
    for s in range(3):
        mg = g.step(s * dt, dt)[0]
        mo = o.step(st, s * dt, dt)
        assert np.allclose(mg, mo, rtol=1e-10, atol=1e-15), (name, s, mg, mo)
    a = g.download()
    for k in KEYS:
        assert rel(a[k], st[k]) < STEP_TOL * 10, (name, k, rel(a[k], st[k]))
    if c.sfd_type:
        m = g.download_mean()
        for k in fields(c):
            assert rel(m[k], st["m" + k]) < STEP_TOL * 10
    if not c.is3d:
        assert rel(g.download_wnew(), st["Wnew"]) < 1e-14
    assert g.kernel_launches() > 0
    g.close()


@pytest.mark.parametrize("scheme", [2, 3])
@pytest.mark.parametrize("name", ["box", "cavity3d", "lid", "bl_cavity", "box_ragged"])
def test_euler_and_ssprk3_match_oracle(libs, name, scheme):
    """timeStepping 2 (Euler) and 3 (SSPRK3): three steps against the oracle, and the
    tangent-linear and adjoint steps refused (they are RK4's)."""
    import dataclasses
    from gatt_dns_b200 import _lib
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    c = dataclasses.replace(get_case(name), time_stepping=scheme)
    g, o = GattDNS(c), Oracle(c)
    f = flow_for(c, seed=4)
    dt = 0.1 * c.cfl_dt(f["U"], f["V"], f["W"], 1.0)
    g.upload(f)
    st = o.new_state(f)
    for s in range(3):
        mg = g.step(s * dt, dt)[0]
        mo = o.step(st, s * dt, dt)
        assert np.allclose(mg, mo, rtol=1e-10, atol=1e-15), (name, scheme, s, mg, mo)
    a = g.download()
    for k in fields(c):
        assert rel(a[k], st[k]) < STEP_TOL * 10, (name, scheme, k, rel(a[k], st[k]))
    if c.sfd_type:
        m = g.download_mean()
        for k in fields(c):
            assert rel(m[k], st["m" + k]) < STEP_TOL * 10
    with pytest.raises(_lib.GattError):
        g.jvp(g.download(), 1, 0.0, dt)
    g.close()


@pytest.mark.parametrize("scheme", [1, 2, 3])
@pytest.mark.parametrize("nz", [1, 8])
def test_hold_inlet_and_periodic_sine_match_oracle(libs, nz, scheme):
    """holdInlet on the inflow plane (the density held in 3-D) and a periodicSine strip on the
    plate of a boundary layer that starts downstream of the leading edge: the first
    gatt_apply_bc keeps the inflow values, then 25 steps from t0 = 0.3 (RK4, Euler, SSPRK3:
    the sine's stage times come from the step parameters on the device) against the oracle.
    Stepping before that first call is refused, and so is a call after the held boxes change
    until gatt_apply_bc runs again."""
    import dataclasses
    from gatt_dns_b200 import _lib
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    if nz == 1:
        c = cs.boundary_layer_isothermal(48, 32, 1, x_range=(0.5, 4.0))
    else:
        c = cs.boundary_layer_isothermal(32, 24, 8, x_range=(0.5, 3.0))
        c.bc.disturbances[0]["par"] = [1.0]
    c = dataclasses.replace(cs.periodic_sine_strip(c, 8, 20, omega=9.0, amp=0.03), time_stepping=scheme)
    f = cs.blasius_flow(c)
    r = cs.random_flow(c, seed=8, amp=0.01)
    for k in ("U", "V", "W", "R"):
        f[k] = f[k] + r[k]
    dt = 0.2 * c.cfl_dt(f["U"], f["V"], f["W"], 1.0)
    t0 = 0.3
    g, o = GattDNS(c), Oracle(c)
    g.upload(f)
    with pytest.raises(_lib.GattError) as e:
        g.step(t0, dt)
    assert e.value.code == 6  # GATT_ERR_STATE
    g.apply_bound_cond(t0)
    fo = o.apply_bound_cond(f, t0)
    a0 = g.download()
    for k in KEYS:
        assert rel(a0[k], fo[k]) < STEP_TOL, k
    st = o.new_state(fo)
    mg = g.run(25, t0, dt)[0]
    t = t0
    for s in range(25):
        mo = o.step(st, t, dt)
        t = t + dt
    assert np.allclose(mg, mo, rtol=1e-9, atol=1e-15), (mg, mo)
    a = g.download()
    for k in fields(c):
        assert rel(a[k], st[k]) < LONG_TOL, (k, rel(a[k], st[k]))
    held = ("U", "V", "W", "E") + (("R",) if nz > 1 else ())
    for k in held:  # the inflow plane is the first call's, bit for bit
        assert np.array_equal(a[k][0], a0[k][0]), k
    g.close()


@pytest.mark.parametrize("name", ["turb_box", "cavity2d_dpdx", "turb_box_multi"])
def test_forcings_match_oracle(libs, name):
    """runForcings: turbulenceGenerator over the whole box, pressureGradient on part of the
    2-D cavity channel, and two forcings on sub-boxes; two batch members with different
    flows (their box sums differ), three steps against the oracle; the tangent-linear and
    adjoint refused."""
    from gatt_dns_b200 import _lib
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    if name == "turb_box":
        c = cs.turbulence_box(nxyz=(32, 24, 16))
    elif name == "turb_box_multi":
        c = cs.turbulence_box(nxyz=(24, 20, 16))
        c.forcings = [{"type": "turbulenceGenerator", "ind": [3, 20, 1, 20, 2, 15], "par": [0.5, c.forcings[0]["par"][1]]},
                      {"type": "pressureGradient", "ind": [1, 24, 5, 12, 1, 16], "par": [0.02]}]
    else:
        c = get_case("cavity2d")
        import dataclasses
        c = dataclasses.replace(c, forcings=[{"type": "pressureGradient", "ind": [3, 40, 2, 39, 1, 1], "par": [0.008]}])
    g, o = GattDNS(c, nbatch=2), Oracle(c)
    fa, fb = flow_for(c, seed=6), flow_for(c, seed=7)
    dt = 0.1 * c.cfl_dt(fa["U"], fa["V"], fa["W"], 1.0)
    g.upload(fa, 0)
    g.upload(fb, 1)
    if c.sfd_type:
        g.upload_mean(fa, 0)
        g.upload_mean(fb, 1)
    sa, sb = o.new_state(fa), o.new_state(fb)
    for s in range(3):
        mg = g.step(s * dt, dt)
        ma, mb = o.step(sa, s * dt, dt), o.step(sb, s * dt, dt)
        # turbulence forcing: box sums added in another order (see test_gpu_reference_golden)
        tol = 1e-8 if name.startswith("turb") else 1e-10
        assert np.allclose(mg[0], ma, rtol=tol, atol=1e-15), (name, s, mg[0], ma)
        assert np.allclose(mg[1], mb, rtol=tol, atol=1e-15), (name, s, mg[1], mb)
    for b, st in ((0, sa), (1, sb)):
        a = g.download(b)
        for k in fields(c):
            assert rel(a[k], st[k]) < STEP_TOL * 10, (name, b, k, rel(a[k], st[k]))
    with pytest.raises(_lib.GattError):
        g.jvp(g.download(0), 1, 0.0, dt)
    g.close()


def test_lid_driven_100_steps(libs):
    c, g, o = pair("lid")
    f = cs.uniform_flow(c)
    f = o.apply_bound_cond(f)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    g.upload(f)
    st = o.new_state(f)
    for s in range(100):
        o.step(st, s * dt, dt)
    mg = g.run(100, 0.0, dt)[0]
    a = g.download()
    for k in ("U", "V", "R", "E"):
        assert rel(a[k], st[k]) < LONG_TOL, (k, rel(a[k], st[k]))
    assert np.all(np.isfinite(mg))
    g.close()


def _long_case(name):
    """Cases for the 100-step comparison (each stable over the run on its grid)."""
    if name == "box":
        c = cs.periodic_box(n=32)
        return c, cs.solenoidal_turbulence(c, seed=7)
    if name == "bl":
        c = cs.boundary_layer(nx=128, ny=64, nz=8, buffers=((10, 8), (0, 10)))
    elif name == "bl_cavity3d":
        c = cs.boundary_layer_cavity(nx=160, ny=64, nz=8, buffers=((10, 8), (0, 10)))
    else:
        c = cs.boundary_layer_cavity(nx=96, ny=48, buffers=((8, 6), (0, 8)))
    f = cs.blasius_flow(c)
    if c.is3d:  # a small spanwise-varying disturbance so that every direction carries work
        r = cs.random_flow(c, seed=3, amp=0.01)
        for k in ("U", "V", "W"):
            f[k] = np.asfortranarray(f[k] + r[k])
    return c, f


@pytest.mark.parametrize("name", ["box", "bl", "bl_cavity3d", "bl_cavity"])
def test_100_steps(libs, name):
    """100 RK4 steps at CFL 0.5 against the oracle at 1e-9: the 3-D periodic turbulence box,
    the 3-D boundary layer with its free-slip upstream wall and break point, the 3-D and
    2-D boundary layers over a cavity with SFD in the buffer zones."""
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    c, f = _long_case(name)
    o = Oracle(c)
    f = o.apply_bound_cond(f, 0.0)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    st = o.new_state(f)
    for s in range(100):
        mo = o.step(st, s * dt, dt)
    g = GattDNS(c)
    g.upload(f)
    mg = g.run(100, 0.0, dt)[0]
    a = g.download()
    assert np.all(np.isfinite(mg))
    assert np.allclose(mg, mo, rtol=1e-7, atol=1e-14), (name, mg, mo)
    for k in fields(c):
        assert rel(a[k], st[k]) < LONG_TOL, (name, k, rel(a[k], st[k]))
    if c.sfd_type:
        m = g.download_mean()
        for k in fields(c):
            assert rel(m[k], st["m" + k]) < LONG_TOL, (name, "mean", k)
    g.close()


def test_batched_members_match_single_runs(libs):
    from gatt_dns_b200.solver import GattDNS
    c = get_case("box")
    fa, fb = flow_for(c, seed=1), flow_for(c, seed=2)
    dt = 0.2 * c.cfl_dt(fa["U"], fa["V"], fa["W"], 1.0)
    gb = GattDNS(c, nbatch=2)
    gb.upload(fa, 0)
    gb.upload(fb, 1)
    mc = gb.run(3, 0.0, dt)
    outs = [gb.download(0), gb.download(1)]
    for i, f in enumerate((fa, fb)):
        g1 = GattDNS(c)
        g1.upload(f)
        m1 = g1.run(3, 0.0, dt)[0]
        o1 = g1.download()
        assert np.array_equal(m1, mc[i])
        for k in KEYS:
            assert np.array_equal(o1[k], outs[i][k])
        g1.close()
    gb.close()


@pytest.mark.parametrize("name", ["box", "cavity3d", "bl", "box_ragged"])
def test_assembly_paths_agree(libs, monkeypatch, name):
    """The tensor-copy-fed assembly and the thread-load assembly (GATT_PW=plain, read when a
    context is created) run the same arithmetic: the states after three steps (batch of two,
    every RK stage mode) are equal bit for bit."""
    from gatt_dns_b200.solver import GattDNS
    c = get_case(name)
    fa, fb = flow_for(c, seed=3), flow_for(c, seed=4)
    dt = 0.2 * c.cfl_dt(fa["U"], fa["V"], fa["W"], 1.0)
    out = {}
    for mode in ("pipe", "plain"):
        if mode == "plain":
            monkeypatch.setenv("GATT_PW", "plain")
        g = GattDNS(c, nbatch=2)
        g.upload(fa, 0)
        g.upload(fb, 1)
        mc = g.run(3, 0.0, dt)
        out[mode] = (mc, g.download(0), g.download(1))
        g.close()
    assert np.array_equal(out["pipe"][0], out["plain"][0])
    for i in (1, 2):
        for k in KEYS:
            assert np.array_equal(out["pipe"][i][k], out["plain"][i][k]), (name, i, k)


@pytest.mark.parametrize("name", ["box", "box64", "box_yz32", "box_aniso", "cavity3d", "bl"])
def test_merged_yz_sweeps_match_separate_launches(libs, monkeypatch, name):
    """The y and z derivative sweeps in one launch (the default where both directions' sets
    allow it) and in two launches (GATT_MERGE_YZ=0, read when a context is created) solve
    every line with the same arithmetic: states after three steps are equal bit for bit."""
    from gatt_dns_b200.solver import GattDNS
    c = get_case(name)
    fa, fb = flow_for(c, seed=3), flow_for(c, seed=4)
    dt = 0.2 * c.cfl_dt(fa["U"], fa["V"], fa["W"], 1.0)
    out = {}
    for mode in ("merged", "separate"):
        if mode == "separate":
            monkeypatch.setenv("GATT_MERGE_YZ", "0")
        g = GattDNS(c, nbatch=2)
        g.upload(fa, 0)
        g.upload(fb, 1)
        mc = g.run(3, 0.0, dt)
        out[mode] = (mc, g.download(0), g.download(1))
        g.close()
    assert np.array_equal(out["merged"][0], out["separate"][0])
    for i in (1, 2):
        for k in KEYS:
            assert np.array_equal(out["merged"][i][k], out["separate"][i][k]), (name, i, k)


@pytest.mark.parametrize("name", ["box", "box_aniso", "box_yz32", "cavity3d"])
def test_uniform_band_solver_matches_records(libs, monkeypatch, name):
    """Cyclic lines of one matrix type whose rows share one band run the solver that reads
    the band as launch constants; GATT_UBAND=0 (read when a context is created) keeps the
    per-row shared-memory records.  Same arithmetic: states after three steps are equal bit
    for bit, and line solves agree with the oracle either way."""
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    c = get_case(name)
    fa, fb = flow_for(c, seed=3), flow_for(c, seed=4)
    dt = 0.2 * c.cfl_dt(fa["U"], fa["V"], fa["W"], 1.0)
    rng = np.random.default_rng(13)
    F = np.asfortranarray(rng.standard_normal((c.nx, c.ny, c.nz)))
    o = Oracle(c)
    out = {}
    for mode in ("uniform", "records"):
        if mode == "records":
            monkeypatch.setenv("GATT_UBAND", "0")
        g = GattDNS(c, nbatch=2)
        for d in (1, 2, 3):
            for kind in ("deriv", "filter"):
                assert rel(g.calc_derivs(F, d, kind), o.calc_derivs(F, d, kind)) < RHS_TOL, (mode, d, kind)
        g.upload(fa, 0)
        g.upload(fb, 1)
        mc = g.run(3, 0.0, dt)
        out[mode] = (mc, g.download(0), g.download(1))
        g.close()
    assert np.array_equal(out["uniform"][0], out["records"][0])
    for i in (1, 2):
        for k in KEYS:
            assert np.array_equal(out["uniform"][i][k], out["records"][i][k]), (name, i, k)


@pytest.mark.parametrize("name", ["box", "box_aniso", "box_ragged", "lid64", "cavity3d"])
def test_x_tile_order_matches_tile_inner(libs, monkeypatch, name):
    """x tiles taken field-inner and last tile first (the default) or tile-inner from the
    first tile (GATT_X_ORDER=0, read when a context is created) solve every line with the
    same arithmetic: states after three steps are equal bit for bit."""
    from gatt_dns_b200.solver import GattDNS
    c = get_case(name)
    fa, fb = flow_for(c, seed=3), flow_for(c, seed=4)
    dt = 0.2 * c.cfl_dt(fa["U"], fa["V"], fa["W"], 1.0)
    out = {}
    for mode in ("field_inner", "tile_inner"):
        if mode == "tile_inner":
            monkeypatch.setenv("GATT_X_ORDER", "0")
        g = GattDNS(c, nbatch=2)
        g.upload(fa, 0)
        g.upload(fb, 1)
        mc = g.run(3, 0.0, dt)
        out[mode] = (mc, g.download(0), g.download(1))
        g.close()
    assert np.array_equal(out["field_inner"][0], out["tile_inner"][0])
    for i in (1, 2):
        for k in KEYS:
            assert np.array_equal(out["field_inner"][i][k], out["tile_inner"][i][k]), (name, i, k)


@pytest.mark.parametrize("env", ["GATT_VISC_V2", "GATT_FZ_REV", "GATT_X_COMPACT", "GATT_X_WSTORE", "GATT_FORK_X"])
@pytest.mark.parametrize("name", ["box", "box_ragged", "box_odd", "box_x400", "cavity3d", "lid", "cavity2d",
                                  "lid_x400", "bl_cavity"])
def test_stress_and_filter_order_variants_match(libs, monkeypatch, env, name):
    """The two-points-per-thread stress kernel, the reversed field order of every second
    filter direction, the compact shared-memory layout of the uniform-band x solver, the x
    tiles stored chunk by chunk by their warps, and the x sweeps beside the y (and z) sweeps
    and two filter field chains side by side on a second stream, in 3-D and 2-D (the defaults;
    box_x400 and lid_x400 take the global-memory line solver, whose scratch field each stream
    has its own of) against their
    plain forms (env var = 0): same arithmetic on every point and line, so states after three
    steps are equal bit for bit."""
    from gatt_dns_b200.solver import GattDNS
    c = get_case(name)
    f = flow_for(c, seed=3)
    dt = 0.2 * c.cfl_dt(f["U"], f["V"], f["W"], 1.0)
    out = {}
    for mode in ("default", "plain"):
        if mode == "plain":
            monkeypatch.setenv(env, "0")
        g = GattDNS(c)
        g.upload(f)
        mc = g.run(3, 0.0, dt)
        out[mode] = (mc, g.download())
        g.close()
    assert np.array_equal(out["default"][0], out["plain"][0])
    for k in KEYS:
        assert np.array_equal(out["default"][1][k], out["plain"][1][k]), (name, env, k)


@pytest.mark.parametrize("name", ["box", "box_yz32", "box_ragged"])
def test_max_change_in_filter_matches_kernel(libs, monkeypatch, name):
    """On cases where nothing follows the filter, its last sweep reduces the max-change in
    its epilogue; GATT_FUSE_MC=0 (read when a context is created) keeps the separate
    reduction kernel.  Both give the same max-change history and states, bit for bit."""
    from gatt_dns_b200.solver import GattDNS
    c = get_case(name)
    fa, fb = flow_for(c, seed=3), flow_for(c, seed=4)
    dt = 0.2 * c.cfl_dt(fa["U"], fa["V"], fa["W"], 1.0)
    out = {}
    for mode in ("fused", "kernel"):
        if mode == "kernel":
            monkeypatch.setenv("GATT_FUSE_MC", "0")
        g = GattDNS(c, nbatch=2)
        g.upload(fa, 0)
        g.upload(fb, 1)
        hist = [g.step(s * dt, dt) for s in range(3)]
        out[mode] = (hist, g.download(0), g.download(1))
        g.close()
    for s in range(3):
        assert np.array_equal(out["fused"][0][s], out["kernel"][0][s]), s
    for i in (1, 2):
        for k in KEYS:
            assert np.array_equal(out["fused"][i][k], out["kernel"][i][k]), (name, i, k)


@pytest.mark.parametrize("name", ["lid", "cavity3d", "bl", "bl_cavity"])
def test_boundary_program_cluster_matches_single_cta(libs, monkeypatch, name):
    """The boundary program run by a cluster of CTAs per member (cluster barriers between
    ops) and by one CTA per member (GATT_BC_CLUSTER=0, read when a context is created) give
    the same states after three steps, bit for bit."""
    from gatt_dns_b200.solver import GattDNS
    c = get_case(name)
    f = flow_for(c, seed=6)
    dt = 0.2 * c.cfl_dt(f["U"], f["V"], f["W"], 1.0)
    out = {}
    for mode in ("cluster", "cta"):
        if mode == "cta":
            monkeypatch.setenv("GATT_BC_CLUSTER", "0")
        g = GattDNS(c)
        g.upload(f)
        mc = g.run(3, 0.0, dt)
        out[mode] = (mc, g.download())
        g.close()
    assert np.array_equal(out["cluster"][0], out["cta"][0])
    for k in KEYS:
        assert np.array_equal(out["cluster"][1][k], out["cta"][1][k]), (name, k)


def test_full_size_box_one_step(libs):
    """128^3 periodic box: one step against the oracle, plus exact mass conservation."""
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    c = cs.periodic_box(n=128)
    f = cs.solenoidal_turbulence(c, seed=1234)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    g = GattDNS(c)
    g.upload(f)
    mg = g.step(0.0, dt)[0]
    a = g.download()
    o = Oracle(c)
    st = o.new_state(f)
    mo = o.step(st, 0.0, dt)
    assert np.allclose(mg, mo, rtol=1e-10)
    for k in KEYS:
        assert rel(a[k], st[k]) < STEP_TOL * 10, k
    m0 = np.sum(f["R"])
    mg2 = g.run(10, dt, dt)
    b = g.download()
    assert abs(np.sum(b["R"]) - m0) / m0 < 1e-12
    g.close()


def test_full_size_box_ten_steps(libs):
    """128^3 periodic box (the bench workload): ten steps against the oracle."""
    from gatt_dns_b200.solver import GattDNS
    from oracle import Oracle
    c = cs.periodic_box(n=128)
    f = cs.solenoidal_turbulence(c, seed=1234)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    g = GattDNS(c)
    g.upload(f)
    mg = g.run(10, 0.0, dt)[0]
    a = g.download()
    g.close()
    o = Oracle(c)
    st = o.new_state(f)
    for s in range(10):
        mo = o.step(st, s * dt, dt)
    assert np.allclose(mg, mo, rtol=1e-9)
    for k in KEYS:
        assert rel(a[k], st[k]) < 1e-10, (k, rel(a[k], st[k]))


def test_errors_are_reported(libs):
    import ctypes
    from gatt_dns_b200 import _lib
    from gatt_dns_b200.solver import GattDNS
    c = get_case("lid")
    g = GattDNS(c)
    L = g.lib
    m = c.mats[0]
    A, B, C, R = (np.asfortranarray(x) for x in (m.A, m.B.copy(), m.C, m.R))
    B[3, 0] = np.inf
    blocks = np.asfortranarray(m.blocks.astype(np.int32))
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    rc = L.gatt_set_matrices(g.h, 1, 0, 0, m.nRHS, m.nTypes, dp(A), dp(B), dp(C), None, dp(R), blocks.shape[0], ip(blocks))
    assert rc == 3  # GATT_ERR_BADCOEF
    B = np.asfortranarray(m.B)
    bad = blocks.copy()
    bad[0, 2] = bad[0, 2] - 1  # leaves a line uncovered
    rc = L.gatt_set_matrices(g.h, 1, 0, 0, m.nRHS, m.nTypes, dp(A), dp(B), dp(C), None, dp(R), bad.shape[0], ip(bad))
    assert rc == 2  # GATT_ERR_BADARG
    # a NaN in the state is reported as divergence (main.F90:433-438)
    f = cs.uniform_flow(c)
    f["E"][7, 7, 0] = np.nan
    g.upload(f)
    with pytest.raises(_lib.GattError) as e:
        g.step(0.0, 1e-3)
    assert e.value.code == 4
    g.close()


@pytest.mark.parametrize("name", ["box64", "cavity3d_32", "bl", "lid"])
def test_autotuned_configuration_matches_oracle(libs, name):
    """gatt_autotune may pick any kernel family and row-block partition per matrix set; the
    results must stay those of the oracle."""
    c, g, o = pair(name)
    choice = g.autotune(reps=2)
    ndir = 3 if c.is3d else 2
    assert all((d, k) in choice for d in range(1, ndir + 1) for k in (0, 1))
    for (d, k), (fam, P, us) in choice.items():
        assert fam in ("tile", "reg", "pipe") and P >= 1 and us > 0
    rng = np.random.default_rng(12)
    F = np.asfortranarray(rng.standard_normal((c.nx, c.ny, c.nz)))
    for d in range(1, ndir + 1):
        for kind in ("deriv", "filter"):
            assert rel(g.calc_derivs(F, d, kind), o.calc_derivs(F, d, kind)) < RHS_TOL, (name, d, kind)
    f = flow_for(c, seed=4)
    dt = 0.25 * c.cfl_dt(f["U"], f["V"], f["W"], 1.0)
    g.upload(f)
    st = o.new_state(f)
    g.step(0.0, dt)
    o.step(st, 0.0, dt)
    a = g.download()
    for k in KEYS:
        assert rel(a[k], st[k]) < STEP_TOL * 10, (name, k)
    g.close()
