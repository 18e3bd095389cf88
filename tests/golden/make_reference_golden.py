"""Writes tests/golden/reference_<case>.npz: the reference's own Fortran solver modules run on
small cases, through the Fortran-subset translator beside this script.

Run it where the reference tree is present (it reads ``source/Fortran/derivs.F90``,
``nseq.F90``, ``timeIntegration.F90``, ``holdInlet.F90`` and the disturbances
``source/disturbances/lidDrivenMovement.F90``, ``periodicSine.F90``, ``pressureGradient.F90``
and ``turbulenceGenerator.F90`` there, unmodified):

    python tests/golden/make_reference_golden.py [reference root [case names...]]

Each fixture holds, for one case built by ``gatt_dns_b200.case`` (the same builders the
tests use; a checksum of the coefficient arrays is stored so that a changed builder is
caught instead of compared): a seeded flow; the first-derivative and filter solves of a
seeded field in every direction (``calcDerivsX/Y/Z``, derivs.F90:9-110); the right-hand side
(``nseq2d`` / ``nseq3d``, nseq.F90:10-323); the boundary conditions (``applyBoundCond``,
nseq.F90:327-518); the filters with and without the blend (``applyFilters2D/3D``,
derivs.F90:303-552); and one time step as main.F90:306-418 sequences it (``RK4_2D/3D``, the
filters with dt/FilterCharTime, SFD, ``applyBoundCond`` at t + dt, maxChange), and on most
cases the same step with ``EULER_2D/3D`` and ``SSPRK3_2D/3D`` as the integrator.  The SFD
update and the maxChange reduction are main-program lines, restated here in numpy with
their line numbers; everything else is the reference's code.

Case coefficient arrays come from the repository's restatement of the MATLAB preprocessing
(there is no MATLAB here); the fixtures pin the solver modules, not the preprocessing.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "..", ".."))

import fortran_subset as fs  # noqa: E402
from gatt_dns_b200 import case as cs  # noqa: E402
from gatt_dns_b200 import fortran_io as fio  # noqa: E402

VARS = ("U", "V", "W", "P", "E")


def golden_cases():
    """name -> case; small enough for the translated Fortran to run in seconds.  Every
    non-periodic line is at least 2 nRHS - 1 = 21 points long: on shorter ones the
    reference's right-hand-side loops (derivs.F90:583-600) index past the line end (reads
    that the Fortran does not check and whose coefficients are zero)."""
    return {
        "box": cs.periodic_box(nxyz=(16, 12, 8)),
        "cavity3d": cs.cavity_channel(nx=24, ny=24, nz=8, adiabatic_corners=True,
                                      sfd={"X": 0.05, "Delta": 10.0, "buffer": 6}),
        "cavity2d": cs.cavity_channel(nx=24, ny=24, nz=1, sfd={"X": 0.05, "Delta": 10.0, "buffer": 6}),
        "lid": cs.lid_driven(n=24),
        # break point at the leading edge, free-slip wall upstream, three x matrix types,
        # buffer zones, SFD
        "bl_cavity": cs.boundary_layer_cavity(nx=48, ny=32, buffers=((6, 5), (0, 6))),
        # runForcings: turbulenceGenerator over the whole box (examples/turbulenceBox.m), and
        # pressureGradient on part of the 2-D cavity channel
        "turb_box": cs.turbulence_box(nxyz=(16, 12, 8)),
        "cavity2d_dpdx": _with_forcing(cs.cavity_channel(nx=24, ny=24, nz=1, sfd={"X": 0.05, "Delta": 10.0, "buffer": 6}),
                                       {"type": "pressureGradient", "ind": [3, 20, 2, 23, 1, 1], "par": [0.008]}),
        # a boundary layer whose mesh starts downstream of the leading edge: holdInlet keeps the
        # inflow plane (boundaryLayerIsothermal.m:53-66), and a periodicSine strip of V on the
        # plate (the blowing and suction of source/disturbances/periodicSine.F90)
        "bl_hold": _with_sine(cs.boundary_layer_isothermal(40, 28, 1, x_range=(0.5, 4.0))),
        # the same in 3-D with the density held too (holdInlet's holdDensity > 0.5)
        "bl_hold3d": _with_sine(_hold_density(cs.boundary_layer_isothermal(24, 24, 8, x_range=(0.5, 3.0))), i1=6, i2=14),
    }


def _with_sine(case, i1=10, i2=20):
    return cs.periodic_sine_strip(case, i1, i2, omega=7.0, amp=0.02)


def _hold_density(case):
    for d in case.bc.disturbances:
        if d["type"] == "holdInlet":
            d["par"] = [1.0]
    return case


def _with_forcing(case, f):
    case.forcings = [f]
    return case


# cases that also hold one Euler and one SSPRK3 step (timeIntegration.F90:158-336, 500-680)
SCHEME_CASES = ("box", "cavity2d", "lid", "bl_cavity", "turb_box", "bl_hold", "bl_hold3d")


def matrices_checksum(case):
    h = hashlib.sha256()
    for m in case.mats:
        if m is None:
            continue
        for a in (m.A, m.B, m.C, m.D, m.R, m.Af, m.Bf, m.Cf, m.Df, m.Rf, np.asarray(m.blocks)):
            h.update(np.ascontiguousarray(np.asarray(a, dtype=np.float64)).tobytes())
    return h.hexdigest()


def _emitted(writer, case):
    """The text the repository's emitter writes (gatt_dns_b200.fortran_io), so that the
    reference runs on the emitter's include files and the fixtures check the emitter too."""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "inc.F90")
        writer(case, path)
        return open(path).read()


def forcing_include(case):
    """runForcings2D/3D.F90 (writeFortranDisturbances.m:19-94, forcing = true), one rank."""
    return _emitted(fio.write_run_forcings_f90, case)


def disturbance_include(case):
    """runDisturbances.F90 (writeFortranDisturbances.m:19-94), one rank."""
    return _emitted(fio.write_run_disturbances_f90, case)


def reference(case, root):
    nx, ny, nz = case.nx, case.ny, case.nz
    src = os.path.join(root, "source")
    texts = [open(os.path.join(src, "Fortran", f)).read() for f in ("derivs.F90", "nseq.F90", "timeIntegration.F90")]
    for f in ("lidDrivenMovement", "periodicSine", "pressureGradient", "turbulenceGenerator"):
        texts.append(open(os.path.join(src, "disturbances", f + ".F90")).read())
    # holdInlet lives beside the solver (writeFortranDisturbances.m:108-113)
    texts.append(open(os.path.join(src, "Fortran", "holdInlet.F90")).read())
    one = np.array([1, 1, 1])
    size = np.array([nx, ny, nz])
    g = {"xstart": one, "ystart": one, "zstart": one, "xend": size, "yend": size, "zend": size,
         "xsize": size, "ysize": size, "zsize": size}

    def copy(a, b):  # one rank: every pencil holds the whole grid in the same index order
        b[...] = a

    ext = {"transpose_x_to_y": copy, "transpose_y_to_x": copy, "transpose_y_to_z": copy,
           "transpose_z_to_y": copy, "nrank": 0, "mpi_real8": 0, "mpi_int": 0, "mpi_sum": 0,
           "mpi_comm_world": 0}
    # the generator writes the forcing calls into the include of the case's dimension and
    # leaves the other one empty (writeFortranDisturbances.m:11-17)
    inc = {"rundisturbances.f90": disturbance_include(case),
           "runforcings3d.f90": forcing_include(case) if case.is3d else "",
           "runforcings2d.f90": "" if case.is3d else forcing_include(case)}
    fns, _, _ = fs.build(texts, g, ext, include_texts=inc)
    return fns


# ---- argument lists as main.F90 passes them -------------------------------------------------

def _f64(a):
    return np.array(a, dtype=np.float64, copy=True)


def _deriv_args(case, kind, dims):
    """Per-direction coefficient arguments of calcDerivs / nseq / RK4 (kind 0) or the
    filters (kind 1), in the reference's order: counts, blocks, nRHS, (A, B, C, R) per
    direction, D per direction, periodic flags."""
    ms = [case.mats[d] for d in dims]
    nb = [np.asarray(m.blocks).shape[0] for m in ms]
    blk = [np.asarray(m.blocks, dtype=np.int64) for m in ms]
    if kind == 0:
        nrhs = [m.nRHS for m in ms]
        abcr = [(_f64(m.A), _f64(m.B), _f64(m.C), _f64(m.R)) for m in ms]
        dd = [_f64(m.D) for m in ms]
    else:
        nrhs = [m.nRHSf for m in ms]
        abcr = [(_f64(m.Af), _f64(m.Bf), _f64(m.Cf), _f64(m.Rf)) for m in ms]
        dd = [_f64(m.Df) for m in ms]
    per = [int(m.periodic) for m in ms]
    return nb, blk, nrhs, abcr, dd, per


def _coef_list(case, kind):
    dims = (0, 1, 2) if case.is3d else (0, 1)
    nb, blk, nrhs, abcr, dd, per = _deriv_args(case, kind, dims)
    out = nb + blk + nrhs
    for t in abcr:
        out += list(t)
    return out + dd + per


def _bc_list(case):
    """neumannLength .. cAdiabatic of applyBoundCond (nseq.F90:327-334)."""
    bc = case.bc
    n, ind, dirs = [], [], []
    for kind in "dns":
        for V in VARS:
            a = bc.ind.get((kind, V))
            a = np.zeros((0, 6), dtype=np.int64) if a is None else np.asarray(a, dtype=np.int64).reshape(-1, 6)
            n.append(a.shape[0])
            ind.append(a)
    vals = [_f64(bc.val[V]) if V in bc.val else np.zeros(0) for V in VARS]
    for kind in "ns":
        for V in VARS:
            d = bc.dirs.get((kind, V))
            dirs.append(np.zeros(0, dtype=np.int64) if d is None else np.asarray(d, dtype=np.int64))
    nc1, nc2 = _f64(bc.neumannCoeffs), _f64(bc.neumann2Coeffs)
    cL = np.asarray(bc.cL, dtype=np.int64).reshape(-1, 6)
    cD = np.asarray(bc.cD, dtype=np.int64)
    cD = cD.reshape(cL.shape[0], 3) if cD.ndim != 2 else cD
    cA = np.asarray(bc.cAdiabatic, dtype=np.int64)
    return [nc1.size, nc2.size, nc1, nc2] + n + ind + vals + dirs + [cL.shape[0], cL, cD, cA]


def _phys(case):
    return [case.Re, case.Ma, case.Pr, case.gamma, case.T0]


# ---- runs -------------------------------------------------------------------------------

def run_derivs(fns, case, F):
    out = {}
    names = ("calcderivsx", "calcderivsy", "calcderivsz")
    for d in range(3 if case.is3d else 2):
        for kind, label in ((0, "deriv"), (1, "filter")):
            nb, blk, nrhs, abcr, dd, per = _deriv_args(case, kind, (d,))
            dF = np.zeros_like(F)
            fns[names[d]](F.copy(), dF, nb[0], blk[0], nrhs[0], *abcr[0], dd[0], per[0])
            out["%s_%d" % (label, d + 1)] = dF
    return out


def run_nseq(fns, case, flow):
    keys = ("U", "V", "W", "R", "E") if case.is3d else ("U", "V", "R", "E")
    ins = [flow[k].copy() for k in keys]
    outs = [np.zeros_like(flow["U"]) for _ in keys]
    fns["nseq3d" if case.is3d else "nseq2d"](*ins, *outs, *_phys(case), *_coef_list(case, 0))
    return {"rhs_" + k: o for k, o in zip(keys, outs)}


def run_bc(fns, case, flow, t):
    f = {k: flow[k].copy() for k in ("U", "V", "W", "R", "E")}
    fns["applyboundcond"](f["U"], f["V"], f["W"], f["R"], f["E"], case.gamma, t, *_bc_list(case))
    return {"bc_" + k: f[k] for k in f}


def run_filters(fns, case, flow, blend):
    keys = ("U", "V", "W", "R", "E") if case.is3d else ("U", "V", "R", "E")
    f = {k: flow[k].copy() for k in keys}
    fd = [int(x) for x in case.filterDirections[:3 if case.is3d else 2]]
    if case.is3d:
        fns["applyfilters3d"](*[f[k] for k in keys], *fd, *_coef_list(case, 1), blend)
    else:
        fns["applyfilters2d"](*[f[k] for k in keys], *fd, *_coef_list(case, 1), blend)
    return f


def run_step(fns, case, flow, t, dt, scheme="rk4", prefix="step_"):
    """main.F90:306-418 for one step: the time integrator (timeStepping 1 RK4, 2 EULER, 3
    SSPRK3), the filters, SFD, boundary conditions, maxChange."""
    U, V, W, R, E = (flow[k].copy() for k in ("U", "V", "W", "R", "E"))
    Un, Vn, Wn, Rn, En = (np.zeros_like(U) for _ in range(5))  # Wnew = 0 (main.F90:186)
    mean = {k: flow[k].copy() for k in ("U", "V", "W", "R", "E")}
    if case.is3d:
        fns[scheme + "_3d"](U, V, W, R, E, Un, Vn, Wn, Rn, En, t, dt, *_phys(case), *_coef_list(case, 0),
                            *_bc_list(case))
    else:
        fns[scheme + "_2d"](U, V, W, R, E, Un, Vn, Rn, En, t, dt, *_phys(case), *_coef_list(case, 0),
                            *_bc_list(case))
    # filters with dt/FilterCharTime (main.F90:358-377)
    new = {"U": Un, "V": Vn, "W": Wn, "R": Rn, "E": En}
    f = run_filters(fns, case, new, dt / case.filterCharTime)
    new.update(f)
    # SFD (main.F90:381-402, restated): the mean relaxes toward the new state, the new state
    # toward the mean with the region weight SFD_X (a field for type 2)
    if case.sfd_type > 0:
        X = case.sfd_chi if case.sfd_type == 2 else case.sfd_X
        keys = ("U", "V", "R", "E") + (("W",) if case.nz > 1 else ())
        for k in keys:
            if case.sfd_delta > 0:
                mean[k] = mean[k] + dt / case.sfd_delta * (new[k] - mean[k])
            new[k] = new[k] - dt * X * (new[k] - mean[k])
    b = run_bc(fns, case, new, t + dt)
    new = {k: b["bc_" + k] for k in ("U", "V", "W", "R", "E")}
    # maxChange (main.F90:413-418, restated)
    old = {"U": U, "V": V, "W": W, "R": R, "E": E}
    mc = np.array([np.max(np.abs(new[k] - old[k])) for k in ("U", "V", "W", "R", "E")])
    out = {prefix + k: new[k] for k in new}
    out[prefix + "maxchange"] = mc
    if case.sfd_type > 0:
        out.update({prefix + "mean_" + k: mean[k] for k in mean})
    return out


def make(name, case, root):
    fns = reference(case, root)
    flow = cs.random_flow(case, seed=11, amp=0.05)
    flow = {k: np.asarray(flow[k], dtype=np.float64).reshape(case.nx, case.ny, case.nz, order="F").copy()
            for k in ("U", "V", "W", "R", "E")}
    rng = np.random.default_rng(17)
    F = rng.standard_normal((case.nx, case.ny, case.nz))
    dt = 0.2 * case.cfl_dt(flow["U"], flow["V"], flow["W"], 1.0)
    t = 0.37
    rec = {"checksum": np.array(matrices_checksum(case)), "F": F, "t": np.array(t), "dt": np.array(dt)}
    rec.update({"flow_" + k: v for k, v in flow.items()})
    rec.update(run_derivs(fns, case, F))
    rec.update(run_nseq(fns, case, flow))
    rec.update(run_bc(fns, case, flow, t))
    rec.update({"filter_" + k: v for k, v in run_filters(fns, case, flow, -1.0).items()})
    rec.update({"filterblend_" + k: v for k, v in run_filters(fns, case, flow, 0.3).items()})
    rec.update(run_step(fns, case, flow, t, dt))
    if name in SCHEME_CASES:
        rec.update(run_step(fns, case, flow, t, dt, "euler", "euler_"))
        rec.update(run_step(fns, case, flow, t, dt, "ssprk3", "ssprk3_"))
    path = os.path.join(HERE, "reference_%s.npz" % name)
    np.savez_compressed(path, **rec)
    return path


if __name__ == "__main__":
    # make_reference_golden.py [reference root [case names...]]
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    only = set(sys.argv[2:])
    for name, case in golden_cases().items():
        if not only or name in only:
            print(make(name, case, root))
