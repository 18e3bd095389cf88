"""Read and write the generated Fortran include files of a reference case.

The reference MATLAB preprocessing writes ``<case>/bin/parameters.F90``, ``matrices.F90``,
``boundaryInfo.F90``, ``runDisturbances.F90`` and ``runForcings2D/3D.F90``
(``source/writeFortranParameters.m``,
``writeFortranMatrices.m``, ``writeFortranBoundaries.m``, ``writeFortranDisturbances.m``)
and compiles them into the solver.  This module parses those files into a
:class:`~gatt_dns_b200.case.Case` so an existing case directory drives the GPU path
unchanged, and writes the same text format (``%.20f`` values, ``reshape((/.../),shape(x))``
arrays) from a case, which makes the package a stand-alone coefficient emitter.
Only rank 0 of a ``select case(nrank)`` block is read: one GPU holds the whole grid.
"""
from __future__ import annotations

import re

import numpy as np

from . import matrices as mx
from .case import BoundaryInfo, Case

_NUM = r"[-+0-9.eEdD]+"


def _to_float(tok):
    return float(tok.strip().lower().replace("d", "e"))


def _rank0(text):
    """Text of `case(0)` in the first `select case(nrank)` block, plus the text after it."""
    m = re.search(r"select\s+case\s*\(\s*nrank\s*\)(.*?)end\s+select", text, re.S | re.I)
    if not m:
        return text, text
    body = m.group(1)
    parts = re.split(r"\n\s*case\s*\(\s*(\d+)\s*\)", body)
    r0 = ""
    for i in range(1, len(parts) - 1, 2):
        if parts[i] == "0":
            r0 = parts[i + 1]
            break
    return r0, text[m.end():]


def _parse_assignments(text):
    """name -> value for `x = reshape((/.../),shape(x))`, `x = (/.../)`, `x = number`,
    together with the allocate() shapes."""
    shapes = {}
    for m in re.finditer(r"allocate\(\s*(\w+)\s*\(([^)]*)\)\s*\)", text, re.I):
        shapes[m.group(1)] = tuple(int(v) for v in m.group(2).split(","))
    vals = {}
    for m in re.finditer(r"(\w+)\s*=\s*reshape\(\s*\(/(.*?)/\)\s*,\s*shape\(\s*\w+\s*\)\s*\)", text, re.S | re.I):
        vals[m.group(1)] = [t for t in m.group(2).replace("\n", "").split(",") if t.strip()]
    for m in re.finditer(r"^\s*(\w+)\s*=\s*\(/(.*?)/\)\s*$", text, re.M | re.S):
        vals.setdefault(m.group(1), [t for t in m.group(2).split(",") if t.strip()])
    for m in re.finditer(r"^\s*(\w+)\s*=\s*(" + _NUM + r")\s*$", text, re.M):
        vals.setdefault(m.group(1), m.group(2))
    return vals, shapes


def _array(vals, shapes, name, dtype=np.float64):
    raw = vals[name]
    conv = _to_float if dtype == np.float64 else (lambda t: int(t))
    a = np.array([conv(t) for t in raw], dtype=dtype)
    shp = shapes.get(name, (a.size,))
    return a.reshape(shp, order="F")


def _scalar(vals, name, conv=int):
    v = vals[name]
    return conv(v if isinstance(v, str) else v[0])


# ---------------------------------------------------------------------------
# parameters.F90
# ---------------------------------------------------------------------------

def read_parameters_f90(path):
    """Scalars of parameters.F90 (writeFortranParameters.m) as a dict."""
    out = {}
    for line in open(path):
        m = re.match(r"\s*(integer|real\*8|logical)[^:]*::\s*(\w+)\s*=\s*(.+)$", line, re.I)
        if not m:
            continue
        typ, name, val = m.group(1).lower(), m.group(2), m.group(3).strip()
        if val.startswith("(/"):
            out[name] = [_to_float(t) for t in val.strip("(/) ").split(",")]
        elif typ == "integer":
            out[name] = int(val)
        elif typ == "logical":
            out[name] = ".true." in val.lower()
        else:
            out[name] = _to_float(val)
    return out


# ---------------------------------------------------------------------------
# matrices.F90
# ---------------------------------------------------------------------------

def _fmt(v):
    return "%.20fd0" % v


def _write_matrix(f, name, a):
    flat = np.asarray(a, dtype=np.float64).ravel(order="F")
    f.write("    %s = reshape((/%s/),shape(%s))\n" % (name, ",".join(_fmt(v) for v in flat), name))


def write_matrices_f90(case: Case, path):
    """Write matrices.F90 for one rank in the layout of writeFortranMatrices.m:1-235."""
    dims = (case.nx, case.ny, case.nz)
    with open(path, "w") as f:
        f.write("    select case(nrank)\n        case(0)\n")
        for d, key in enumerate("XYZ"):
            m = case.mats[d]
            if m is None:
                continue
            b = np.asarray(m.blocks, dtype=np.int64)
            f.write("            nDerivBlocks%s = %d\n" % (key, b.shape[0]))
            f.write("            allocate(derivBlocks%s(%d,5))\n" % (key, b.shape[0]))
            f.write("            derivBlocks%s = reshape((/%s/),shape(derivBlocks%s))\n\n"
                    % (key, ",".join(str(v) for v in b.ravel(order="F")), key))
        f.write("    end select\n\n")
        for d, key in enumerate("XYZ"):
            f.write("    filter%s = %d\n" % (key, case.filterDirections[d]))
        for d, key in enumerate("xyz"):
            m = case.mats[d]
            if m is None:
                continue
            K, N = key.upper(), dims[d]
            f.write("    derivnRHS%s = %d\n" % (key, m.nRHS))
            f.write("    filternRHS%s = %d\n" % (key, m.nRHSf))
            for pre, nR in (("derivs", m.nRHS), ("filter", m.nRHSf)):
                f.write("    allocate(%sA%s(%d,%d))\n" % (pre, K, N - 1, m.nTypes))
                f.write("    allocate(%sB%s(%d,%d))\n" % (pre, K, N - m.periodic, m.nTypes))
                f.write("    allocate(%sC%s(%d,%d))\n" % (pre, K, N - 1, m.nTypes))
                f.write("    allocate(%sR%s(%d,%d,%d))\n\n" % (pre, K, N, 2 * nR - 1, m.nTypes))
            for pre, arrs in (("derivs", (m.A, m.B, m.C, m.R)), ("filter", (m.Af, m.Bf, m.Cf, m.Rf))):
                for letter, a in zip("ABCR", arrs):
                    _write_matrix(f, "%s%s%s" % (pre, letter, K), a)
            f.write("    periodic%s = %d\n\n" % (K, m.periodic))
            if m.periodic:
                f.write("    allocate(derivsD%s(%d,%d))\n" % (K, N, m.nTypes))
                f.write("    allocate(filterD%s(%d,%d))\n" % (K, N, m.nTypes))
                _write_matrix(f, "derivsD" + K, m.D)
                _write_matrix(f, "filterD" + K, m.Df)
        bc = case.bc
        for nm, arr in (("neumann", bc.neumannCoeffs), ("neumann2", bc.neumann2Coeffs)):
            f.write("\n    %sLength = %d\n" % (nm, len(arr)))
            f.write("    allocate(%sCoeffs(%d))\n" % (nm, len(arr)))
            f.write("    %sCoeffs = (/%s/)\n" % (nm, ",".join(_fmt(v) for v in arr)))
        f.write("    nTracked = 0\n")


def read_matrices_f90(path, nx, ny, nz):
    """Parse matrices.F90 into per-direction :class:`DirectionMatrices` and Neumann coefficients."""
    text = open(path).read()
    r0, rest = _rank0(text)
    bvals, bshapes = _parse_assignments(r0)
    vals, shapes = _parse_assignments(rest)
    mats = []
    for d, key in enumerate("XYZ"):
        if ("derivsA" + key) not in vals:
            mats.append(None)
            continue
        per = _scalar(vals, "periodic" + key)
        nR = _scalar(vals, "derivnRHS" + key.lower())
        nRf = _scalar(vals, "filternRHS" + key.lower())
        A, B, C, R = (_array(vals, shapes, "derivs%s%s" % (l, key)) for l in "ABCR")
        Af, Bf, Cf, Rf = (_array(vals, shapes, "filter%s%s" % (l, key)) for l in "ABCR")
        nT = B.shape[1]
        N = (nx, ny, nz)[d]
        D = _array(vals, shapes, "derivsD" + key) if per else np.zeros((N, nT))
        Df = _array(vals, shapes, "filterD" + key) if per else np.zeros((N, nT))
        blocks = _array(bvals, bshapes, "derivBlocks" + key, dtype=np.int64)
        mats.append(mx.DirectionMatrices(periodic=per, nTypes=nT, A=A, B=B, C=C, D=D, R=R, nRHS=nR,
                                         Af=Af, Bf=Bf, Cf=Cf, Df=Df, Rf=Rf, nRHSf=nRf, blocks=blocks))
    filt = tuple(_scalar(vals, "filter" + k) if ("filter" + k) in vals else 0 for k in "XYZ")
    n1 = _array(vals, shapes, "neumannCoeffs") if "neumannCoeffs" in vals else np.zeros(0)
    n2 = _array(vals, shapes, "neumann2Coeffs") if "neumann2Coeffs" in vals else np.zeros(0)
    return mats, filt, n1, n2


# ---------------------------------------------------------------------------
# boundaryInfo.F90 and runDisturbances.F90
# ---------------------------------------------------------------------------

_BVARS = ("U", "V", "W", "E", "P")


def write_boundary_info_f90(case: Case, path):
    """Write boundaryInfo.F90 for one rank (writeFortranBoundaries.m:1-190)."""
    bc = case.bc
    with open(path, "w") as f:
        f.write("    select case (nrank)\n        case (0)\n")
        for kind in "dns":
            for V in _BVARS:
                ind = bc.ind.get((kind, V))
                n = 0 if ind is None else ind.shape[0]
                f.write("            n%s%s = %d\n" % (V, kind, n))
                if n > 0:
                    f.write("            allocate(i%s%s(%d,6))\n" % (V, kind, n))
                    second = "v" if kind == "d" else "d"
                    f.write("            allocate(%s%s%s(%d))\n" % (second, V, kind, n))
                    f.write("            i%s%s = reshape((/%s/),shape(i%s%s))\n"
                            % (V, kind, ",".join(str(int(v)) for v in ind.ravel(order="F")), V, kind))
                    if kind == "d":
                        f.write("            v%sd = (/%s/)\n\n" % (V, ",".join(_fmt(v) for v in bc.val[V])))
                    else:
                        f.write("            d%s%s = (/%s/)\n\n"
                                % (V, kind, ",".join(str(int(v)) for v in bc.dirs[(kind, V)])))
                elif kind != "d":
                    f.write("            allocate(i%s%s(1,6))\n            allocate(d%s%s(1))\n\n" % (V, kind, V, kind))
        cN = bc.cL.shape[0]
        f.write("            cN = %d\n" % cN)
        f.write("            allocate(cL(%d,6))\n            allocate(cD(%d,3))\n            allocate(cAdiabatic(%d))\n"
                % (max(cN, 1), max(cN, 1), max(cN, 1)))
        if cN:
            f.write("            cL = reshape((/%s/),shape(cL))\n" % ",".join(str(int(v)) for v in bc.cL.ravel(order="F")))
            f.write("            cD = reshape((/%s/),shape(cD))\n" % ",".join(str(int(v)) for v in bc.cD.ravel(order="F")))
            f.write("            cAdiabatic = (/%s/)\n\n" % ",".join(str(int(v)) for v in bc.cAdiabatic))
        f.write("    end select\n")


def read_boundary_info_f90(path):
    text = open(path).read()
    r0, _ = _rank0(text)
    vals, shapes = _parse_assignments(r0)
    bi = BoundaryInfo()
    for kind in "dns":
        for V in _BVARS:
            n = _scalar(vals, "n%s%s" % (V, kind)) if ("n%s%s" % (V, kind)) in vals else 0
            if n == 0:
                continue
            shapes["i%s%s" % (V, kind)] = (n, 6)
            bi.ind[(kind, V)] = _array(vals, shapes, "i%s%s" % (V, kind), dtype=np.int64).astype(np.int32)
            if kind == "d":
                bi.val[V] = _array(vals, shapes, "v%sd" % V)
            else:
                bi.dirs[(kind, V)] = _array(vals, shapes, "d%s%s" % (V, kind), dtype=np.int64).astype(np.int32)
    cN = _scalar(vals, "cN") if "cN" in vals else 0
    if cN:
        shapes["cL"], shapes["cD"], shapes["cAdiabatic"] = (cN, 6), (cN, 3), (cN,)
        bi.cL = _array(vals, shapes, "cL", dtype=np.int64).astype(np.int32)
        bi.cD = _array(vals, shapes, "cD", dtype=np.int64).astype(np.int32)
        bi.cAdiabatic = _array(vals, shapes, "cAdiabatic", dtype=np.int64).astype(np.int32)
    return bi


def write_run_disturbances_f90(case: Case, path):
    """runDisturbances.F90 lines for the disturbances of a case (writeFortranDisturbances.m:35-90)."""
    with open(path, "w") as f:
        f.write("    select case (nrank)\n        case (0)\n")
        for d in case.bc.disturbances:
            i = [int(v) for v in d["ind"]]
            X = np.asarray(d["X"], dtype=np.float64)
            Y = case.Y[i[2] - 1:i[3]]
            Z = case.Z[i[4] - 1:i[5]]
            args = "%d,%d,%d,(/%s/),(/%s/),(/%s/),t" % (
                i[1] - i[0] + 1, i[3] - i[2] + 1, i[5] - i[4] + 1, ",".join(_fmt(v) for v in X),
                ",".join(_fmt(v) for v in Y), ",".join(_fmt(v) for v in Z))
            args += "".join(",%s(%d:%d,%d:%d,%d:%d)" % (v, i[0], i[1], i[2], i[3], i[4], i[5]) for v in d["var"])
            args += "".join("," + _fmt(p) for p in d["par"])
            f.write("            call %s(%s)\n" % (d["type"], args))
        f.write("    end select\n")


_FORCING_VARS = {"pressureGradient": "RU", "turbulenceGenerator": "UVWE"}


def write_run_forcings_f90(case: Case, path):
    """runForcings2D/3D.F90 lines for the forcings of a case (writeFortranDisturbances.m:35-90
    with forcing = true: no t; each variable's box, then its right-hand side's d<var>)."""
    with open(path, "w") as f:
        f.write("    select case (nrank)\n        case (0)\n")
        for d in getattr(case, "forcings", None) or []:
            i = [int(v) for v in d["ind"]]
            X, Y, Z = case.X[i[0] - 1:i[1]], case.Y[i[2] - 1:i[3]], case.Z[i[4] - 1:i[5]]
            args = "%d,%d,%d,(/%s/),(/%s/),(/%s/)" % (
                i[1] - i[0] + 1, i[3] - i[2] + 1, i[5] - i[4] + 1, ",".join(_fmt(v) for v in X),
                ",".join(_fmt(v) for v in Y), ",".join(_fmt(v) for v in Z))
            box = "(%d:%d,%d:%d,%d:%d)" % tuple(i)
            var = _FORCING_VARS[d["type"]]
            args += "".join(",%s%s" % (v, box) for v in var) + "".join(",d%s%s" % (v, box) for v in var)
            args += "".join("," + _fmt(p) for p in d["par"])
            f.write("            call %s(%s)\n" % (d["type"], args))
        f.write("    end select\n")


def read_run_forcings_f90(path):
    """Forcing calls of rank 0 (pressureGradient and turbulenceGenerator)."""
    text = open(path).read()
    if "case" not in text:
        return []
    r0, _ = _rank0(text)
    out = []
    for m in re.finditer(r"call\s+(\w+)\s*\((.*)\)\s*$", r0, re.M):
        name, args = m.group(1), m.group(2)
        if name not in _FORCING_VARS:
            continue
        boxes = list(re.finditer(r",d?[UVWRE]\((\d+):(\d+),(\d+):(\d+),(\d+):(\d+)\)", args))
        ind = np.array([int(boxes[0].group(k)) for k in range(1, 7)], dtype=np.int32)
        tail = args[boxes[-1].end():]
        par = [_to_float(t) for t in tail.split(",") if t.strip()]
        out.append(dict(type=name, ind=ind, par=par))
    return out


def read_run_disturbances_f90(path):
    """Disturbance calls of rank 0 (lidDrivenMovement, periodicSine, holdInlet)."""
    text = open(path).read()
    r0, _ = _rank0(text)
    out = []
    for m in re.finditer(r"call\s+(\w+)\s*\((.*)\)\s*$", r0, re.M):
        name, args = m.group(1), m.group(2)
        arrays = re.findall(r"\(/(.*?)/\)", args)
        X = np.array([_to_float(t) for t in arrays[0].split(",")])
        boxes = list(re.finditer(r",([UVWRE])\((\d+):(\d+),(\d+):(\d+),(\d+):(\d+)\)", args))
        var = "".join(b.group(1) for b in boxes)
        ind = np.array([int(boxes[0].group(k)) for k in range(2, 8)], dtype=np.int32)
        tail = args[boxes[-1].end():]
        par = [_to_float(t) for t in tail.split(",") if t.strip()]
        out.append(dict(type=name, var=var, ind=ind, X=X, par=par))
    return out


def case_from_fortran_dir(bin_dir, name="reference_case", sfd_chi=None):
    """Build a :class:`Case` from a reference ``<case>/bin`` directory (rank 0 of each file).

    The mesh coordinates are not in these files (they live in mesh.mat); X is taken from the
    disturbance calls when present and otherwise left as node indices (the GPU path only
    needs coordinates for disturbances).
    """
    import os
    p = read_parameters_f90(os.path.join(bin_dir, "parameters.F90"))
    nx, ny, nz = p["nx"], p["ny"], p["nz"]
    mats, filt, n1, n2 = read_matrices_f90(os.path.join(bin_dir, "matrices.F90"), nx, ny, nz)
    bc = read_boundary_info_f90(os.path.join(bin_dir, "boundaryInfo.F90"))
    bc.neumannCoeffs, bc.neumann2Coeffs = n1, n2
    rd = os.path.join(bin_dir, "runDisturbances.F90")
    if os.path.exists(rd):
        bc.disturbances = [d for d in read_run_disturbances_f90(rd)
                           if d["type"] in ("lidDrivenMovement", "periodicSine", "holdInlet")]
    forcings = []
    for nm in ("runForcings3D.F90", "runForcings2D.F90"):
        rf = os.path.join(bin_dir, nm)
        if os.path.exists(rf):
            forcings += read_run_forcings_f90(rf)
    dxmin = tuple(p.get("dxmin", [0.0, 0.0, 0.0]))
    c = Case(name=name, nx=nx, ny=ny, nz=nz, Re=p["Re"], Ma=p["Ma"], Pr=p["Pr"], gamma=p["gamma"], T0=p["T0"],
             X=np.arange(1, nx + 1, dtype=float), Y=np.arange(1, ny + 1, dtype=float),
             Z=np.arange(1, nz + 1, dtype=float), mats=mats, bc=bc, filterDirections=filt,
             filterCharTime=p.get("FilterCharTime", -1.0), dxmin=dxmin,
             time_stepping=int(p.get("timeStepping", 1)), forcings=forcings or None)
    sfd = p.get("SFD", 0)
    if sfd:
        c.sfd_type, c.sfd_delta, c.sfd_X = sfd, p.get("SFD_Delta", 0.0), p.get("SFD_X_val", 0.0)
        c.sfd_chi = sfd_chi
    return c


def write_parameters_f90(case: Case, path, dt=1.0, max_cfl=1.0):
    """The physics/grid part of parameters.F90 (writeFortranParameters.m:5-103)."""
    with open(path, "w") as f:
        f.write("    integer :: nx = %d\n    integer :: ny = %d\n    integer :: nz = %d\n\n" % (case.nx, case.ny, case.nz))
        for nm in ("Re", "Ma", "Pr", "T0", "gamma"):
            f.write("    real*8 :: %s = %s\n" % (nm, _fmt(getattr(case, nm))))
        f.write("\n    real*8 :: dtmax = %s\n    real*8 :: maxCFL = %s\n" % (_fmt(dt), _fmt(max_cfl)))
        f.write("    integer :: SFD = %d\n    real*8 :: SFD_Delta = %s\n    real*8 :: SFD_X_val = %s\n"
                % (case.sfd_type, _fmt(case.sfd_delta), _fmt(case.sfd_X)))
        f.write("    real*8 :: FilterCharTime = %s\n" % _fmt(case.filterCharTime))
        f.write("    real*8,dimension(3) :: dxmin = (/%s,%s,%s/)\n\n" % tuple(_fmt(v) for v in case.dxmin))
        f.write("    integer :: p_row = 1\n    integer :: p_col = 1\n")
        # writeFortranParameters.m:50-57: RK4 1, Euler 2, SSPRK3 3
        f.write("    integer :: timeStepping = %d\n" % int(getattr(case, "time_stepping", 1)))
