"""Case description consumed by the C-ABI: mesh, coefficient arrays, boundary lists.

A :class:`Case` holds exactly the data the generated Fortran include files carry
(``parameters.F90``, ``matrices.F90``, ``boundaryInfo.F90``, ``runDisturbances.F90``)
for one rank owning the whole grid.  The builders below restate the reference MATLAB
preprocessing for the workloads this package is measured on:

* :func:`periodic_box` -- ``source/boundaries/periodicBox.m`` (128^3 turbulence box)
* :func:`lid_driven` -- ``source/boundaries/lidDrivenFlow.m`` +
  ``source/disturbances/lidDrivenMovement.F90`` (2-D cavity)
* :func:`cavity_channel` -- the wall/corner machinery of ``source/findWallsForBoundaries.m``
  on a box with an open cavity (used for stretched-mesh, multi-type parity cases)

Mesh generation follows ``source/generateMesh.m`` (uniform, tanh, power; periodic
domain-size fix; buffer zones), boundary extraction ``source/findWallsForBoundaries.m``
and list assembly ``source/initBoundaries.m`` (one rank).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import matrices as mx

VARS = ("U", "V", "W", "P", "E")          # boundaryInfo.F90 variable letters
VAR_INDEX = {"U": 0, "V": 1, "W": 2, "P": 3, "R": 3, "E": 4}  # C-ABI numbering (P lists act on R)
DIR_CODE = {"xi": 1, "xf": 2, "yi": 3, "yf": 4, "zi": 5, "zf": 6}


# ---------------------------------------------------------------------------
# data model
# ---------------------------------------------------------------------------

@dataclass
class BoundaryInfo:
    """``boundaryInfo.F90`` for one rank: lists per (kind, variable).

    ``ind[(kind, var)]`` is an (n, 6) int array of 1-based [i1 i2 j1 j2 k1 k2];
    ``val[var]`` holds Dirichlet values; ``dirs[(kind, var)]`` Neumann directions 1..6.
    kind is 'd', 'n' or 's'; var is one of U V W P E.
    """
    ind: Dict[Tuple[str, str], np.ndarray] = field(default_factory=dict)
    val: Dict[str, np.ndarray] = field(default_factory=dict)
    dirs: Dict[Tuple[str, str], np.ndarray] = field(default_factory=dict)
    cL: np.ndarray = field(default_factory=lambda: np.zeros((0, 6), np.int32))
    cD: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    cAdiabatic: np.ndarray = field(default_factory=lambda: np.zeros((0,), np.int32))
    neumannCoeffs: np.ndarray = field(default_factory=lambda: np.zeros(0))
    neumann2Coeffs: np.ndarray = field(default_factory=lambda: np.zeros(0))
    # disturbances: dicts with keys type ('lidDrivenMovement', 'periodicSine', 'holdInlet'), var
    # (the variables in the reference call's order, e.g. 'U' or 'UVRWE'), ind (6,), X (box x
    # coords), par (list)
    disturbances: List[dict] = field(default_factory=list)

    def count(self, kind, var):
        a = self.ind.get((kind, var))
        return 0 if a is None else int(a.shape[0])


@dataclass
class Case:
    name: str
    nx: int
    ny: int
    nz: int
    Re: float
    Ma: float
    Pr: float
    gamma: float
    T0: float
    X: np.ndarray
    Y: np.ndarray
    Z: np.ndarray
    mats: List[Optional[mx.DirectionMatrices]]     # x, y, z (z is None in 2-D)
    bc: BoundaryInfo
    filterDirections: Tuple[int, int, int] = (1, 1, 1)
    filterCharTime: float = -1.0
    sfd_type: int = 0
    sfd_delta: float = 0.0
    sfd_X: float = 0.0
    sfd_chi: Optional[np.ndarray] = None
    # parameters.F90 timeStepping (main.F90:304-352): 1 RK4, 2 Euler, 3 SSPRK3
    time_stepping: int = 1
    # forcings of runForcings2D/3D.F90 (disturbances with forcing = true): dicts with
    # type ("pressureGradient" | "turbulenceGenerator"), ind (1-based box, 6 ints), par
    forcings: Optional[list] = None
    flowRegion: Optional[np.ndarray] = None
    dxmin: Tuple[float, float, float] = (0.0, 0.0, 0.0)

    @property
    def npts(self):
        return self.nx * self.ny * self.nz

    @property
    def is3d(self):
        return self.nz > 1

    @property
    def E0(self):
        return 1.0 / ((self.gamma ** 2 - self.gamma) * self.Ma ** 2)

    def cfl_dt(self, U, V, W, cfl):
        """dt for a target CFL from main.F90:206-212 (the caller-side time control)."""
        c = 1.0 / self.Ma
        v = (c + np.max(np.abs(U))) * self.dxmin[0] + (c + np.max(np.abs(V))) * self.dxmin[1]
        if self.is3d:
            v += (c + np.max(np.abs(W))) * self.dxmin[2]
        return cfl / v


# ---------------------------------------------------------------------------
# mesh (generateMesh.m subset)
# ---------------------------------------------------------------------------

def _buffer_zone(par):
    """calcBufferZone of generateMesh.m:249-288."""
    n = int(par["n"])
    if par["type"] == "exponential":
        if "ramp" not in par:
            xb = np.zeros(n)
            xb[0] = 1 + par["stretching"]
            for i in range(2, n + 1):
                xb[i - 1] = xb[i - 2] + (1 + par["stretching"]) ** i
            return xb
        delta = np.ones(n)
        for i in range(2, n + 1):
            st = 1 + min(1.0, i / par["ramp"]) * par["stretching"]
            delta[i - 1] = delta[i - 2] * st
        return np.cumsum(delta)
    if par["type"] == "sigmoid":
        xb = np.array([-10 + 12 * (i - 1) / (n - 1) for i in range(1, n + 1)])
        delta = 1.0 / (1.0 + np.exp(-1.0 * xb))
        delta = delta * par["stretching"] + 1
        return np.cumsum(delta)
    raise ValueError("unknown buffer type %r" % par["type"])


def _match_fixed(xp, fix_points):
    """generateMesh.m:186-207 with matchFixed = 2: move the nodes nearest to the fixed points
    onto them and shift the others by the pchip interpolant of those moves."""
    from scipy.interpolate import PchipInterpolator
    n = len(xp)
    fp = np.unique(np.concatenate([xp[[0, 1]], np.asarray(fix_points, dtype=np.float64), xp[[-2, -1]]]))
    fp = fp[np.isfinite(fp) & (fp >= xp[0]) & (fp <= xp[-1])]
    closest = np.argmin(np.abs(xp[:, None] - fp[None, :]), axis=0)
    for _ in range(n + 1):
        dup = np.nonzero(np.diff(closest) == 0)[0]
        if len(dup) == 0:
            break
        closest[dup] -= 1
    shift = PchipInterpolator(closest.astype(np.float64), xp[closest] - fp)(np.arange(n, dtype=np.float64))
    out = xp - shift
    out[closest] = fp
    return out


def _attractor_mesh(xi, xf, n, points=(), regions=()):
    """generateMesh.m:123-147 ('attractors'): node density 1 + sum of Gaussian attractors
    (point, strength, size) + sum of region ramps (strength times the squared pchip of
    0 0 1 1 0 0 over [a-1, a, b, c, d, d+1]), integrated on 100 n base points and inverted
    with a not-a-knot cubic spline, as interp1(..., 'spline') does."""
    from scipy.interpolate import CubicSpline, PchipInterpolator
    xb = np.linspace(xi, xf, 100 * n)
    eta = np.ones(100 * n)
    for (p, strength, size) in points:
        eta += strength * np.exp(-((xb - p) / size) ** 2)
    for reg in regions:
        pos = [float(v) for v in reg[:4]]
        if math.isinf(pos[1]):
            pos[0:2] = [xi - 2, xi - 1]
        if math.isinf(pos[2]):
            pos[2:4] = [xf + 1, xf + 2]
        pos = [pos[0] - 1] + pos + [pos[3] + 1]
        eta += reg[4] * PchipInterpolator(pos, [0, 0, 1, 1, 0, 0])(xb) ** 2
    eta = np.cumsum(eta)
    eta -= eta[0]
    eta = (n - 1) * eta / eta[-1] + 1
    eta[-1] = n
    return CubicSpline(eta, xb)(np.arange(1, n + 1, dtype=np.float64))


def generate_mesh(xi, xf, n, mtype="uniform", periodic=False, fix_periodic_domain_size=False,
                  par=2.0, local="b", power=2.0, buffer_i=None, buffer_f=None, fix_points=None,
                  attractor_points=(), attractor_regions=()):
    """Node coordinates of one direction (generateMesh.m:1-247); ``fix_points`` are matched
    as mesh.matchFixed = 2 does (points outside [xi, xf] are dropped, meshAddFixedPoints.m:54)."""
    buffer_i = dict(buffer_i or {"n": 0})
    buffer_f = dict(buffer_f or {"n": 0})
    if n == 1:
        mtype = "uniform"
    if periodic:
        buffer_i["n"] = 0
        buffer_f["n"] = 0
    added = False
    if periodic and fix_periodic_domain_size and n > 1:
        n = n + 1
        added = True
    ni, nf = int(buffer_i.get("n", 0)), int(buffer_f.get("n", 0))
    ntot = n + ni + nf
    if mtype == "uniform":
        xp = np.linspace(xi, xf, n)
    elif mtype == "power":
        xp = xi + (xf - xi) * np.linspace(0, 1, n) ** power
    elif mtype == "tanh":
        if local == "f":
            eta = np.tanh(np.linspace(0, par, n)); eta = eta / eta[-1]
        elif local == "i":
            eta = np.tanh(np.linspace(0, par, n)); eta = eta / eta[-1]; eta = 1 - eta[::-1]
        else:
            eta = np.tanh(np.linspace(-par, par, n)); eta = eta / eta[-1]; eta = (eta + 1) / 2
        xp = (xf - xi) * eta + xi
    elif mtype == "attractors":
        xp = _attractor_mesh(xi, xf, n, attractor_points, attractor_regions)
    else:
        raise ValueError("mesh type %r not restated" % mtype)
    if fix_points is not None and len(fix_points) and n > 1:
        xp = _match_fixed(xp, fix_points)
    X = np.zeros(ntot)
    X[ni:ni + n] = xp
    if ni > 0:
        base = X[ni + 1] - X[ni]
        xb = _buffer_zone(buffer_i) * base
        X[:ni] = X[ni] - xb[::-1]
    if nf > 0:
        base = X[ni + n - 1] - X[ni + n - 2]
        xb = _buffer_zone(buffer_f) * base
        X[ni + n:] = X[ni + n - 1] + xb
    if added:
        X = X[:-1]
    return X


# ---------------------------------------------------------------------------
# walls and corners (findWallsForBoundaries.m)
# ---------------------------------------------------------------------------

def _runs(v):
    """1-based (start, end) of the true runs of a boolean vector."""
    v = np.asarray(v, dtype=bool)
    if v.size == 0:
        return []
    d = np.diff(v.astype(np.int8))
    starts = ([1] if v[0] else []) + list(np.nonzero(d == 1)[0] + 2)
    ends = list(np.nonzero(d == -1)[0] + 1) + ([v.size] if v[-1] else [])
    return list(zip(starts, ends))


def find_walls_for_boundaries(flow_region):
    """Walls, corners and wall-interior boxes of a flow-region mask.

    Restates ``source/findWallsForBoundaries.m:1-329`` (including its thin-wall removal,
    which modifies the mask).  Returns (flowRegion, walls dict, corners dict, insideWalls).
    """
    fr = np.array(flow_region, dtype=bool, copy=True)
    nx, ny, nz = fr.shape
    if nx > 2:
        fr[1:-1] = fr[1:-1] | (fr[:-2] & fr[2:])
    if ny > 2:
        fr[:, 1:-1] = fr[:, 1:-1] | (fr[:, :-2] & fr[:, 2:])
    if nz > 2:
        fr[:, :, 1:-1] = fr[:, :, 1:-1] | (fr[:, :, :-2] & fr[:, :, 2:])
    f8 = fr.astype(np.int8)
    wF = np.zeros_like(fr); wF[:-1] = np.diff(f8, axis=0) == 1
    wB = np.zeros_like(fr); wB[1:] = np.diff(f8, axis=0) == -1
    wU = np.zeros_like(fr); wU[:, :-1] = np.diff(f8, axis=1) == 1
    wD = np.zeros_like(fr); wD[:, 1:] = np.diff(f8, axis=1) == -1
    wR = np.zeros_like(fr); wR[:, :, :-1] = np.diff(f8, axis=2) == 1
    wL = np.zeros_like(fr); wL[:, :, 1:] = np.diff(f8, axis=2) == -1

    def x_walls(wall):
        out = []
        for i in range(nx):
            lw = wall[i]  # (ny, nz)
            if not lw.any():
                continue
            starts = None
            kstart = 0
            for k in range(nz):
                if k == 0 or not starts:
                    starts = _runs(lw[:, k])
                    kstart = k
                if k == nz - 1 or np.any(lw[:, k] != lw[:, k + 1]):
                    for (s, e) in starts:
                        out.append([i + 1, i + 1, s, e, kstart + 1, k + 1])
                    starts = []
        return out

    def y_walls(wall):
        out = []
        for j in range(ny):
            lw = wall[:, j, :]  # (nx, nz)
            if not lw.any():
                continue
            starts = None
            kstart = 0
            for k in range(nz):
                if k == 0 or not starts:
                    starts = _runs(lw[:, k])
                    kstart = k
                if k == nz - 1 or np.any(lw[:, k] != lw[:, k + 1]):
                    for (s, e) in starts:
                        out.append([s, e, j + 1, j + 1, kstart + 1, k + 1])
                    starts = []
        return out

    def z_walls(wall):
        out = []
        for k in range(nz):
            lw = wall[:, :, k]  # (nx, ny)
            if not lw.any():
                continue
            starts = None
            istart = 0
            for i in range(nx):
                if i == 0 or not starts:
                    starts = _runs(lw[i, :])
                    istart = i
                if i == nx - 1 or np.any(lw[i, :] != lw[i + 1, :]):
                    for (s, e) in starts:
                        out.append([istart + 1, i + 1, s, e, k + 1, k + 1])
                    starts = []
        return out

    walls = {"front": x_walls(wF), "back": x_walls(wB), "up": y_walls(wU), "down": y_walls(wD),
             "right": z_walls(wR), "left": z_walls(wL)}
    # join adjacent walls in z (findWallsForBoundaries.m:181-205)
    for key in ("front", "back", "up", "down"):
        cw = [list(r) for r in walls[key]]
        done = False
        while not done:
            done = True
            merge = None
            for a in range(len(cw) - 1):
                for b in range(a + 1, len(cw)):
                    if cw[a][0:4] == cw[b][0:4] and cw[a][5] == cw[b][4] - 1:
                        merge = (a, b)
                        done = False
                if not done:
                    break
            if not done:
                cw[merge[0]][5] = cw[merge[1]][5]
                del cw[merge[1]]
        walls[key] = cw

    limits, dirs = [], []
    cm = [wF & wU, wF & wD, wB & wU, wB & wD]
    cdir = [[1, 1, 0], [1, -1, 0], [-1, 1, 0], [-1, -1, 0]]
    for i in range(nx):
        for j in range(ny):
            for m in range(4):
                for (s, e) in _runs(cm[m][i, j, :]):
                    limits.append([i + 1, i + 1, j + 1, j + 1, s, e]); dirs.append(cdir[m])
    cm = [wF & wR, wF & wL, wB & wR, wB & wL]
    cdir = [[1, 0, 1], [1, 0, -1], [-1, 0, 1], [-1, 0, -1]]
    for i in range(nx):
        for k in range(nz):
            for m in range(4):
                for (s, e) in _runs(cm[m][i, :, k]):
                    limits.append([i + 1, i + 1, s, e, k + 1, k + 1]); dirs.append(cdir[m])
    cm = [wU & wR, wU & wL, wD & wR, wD & wL]
    cdir = [[0, 1, 1], [0, 1, -1], [0, -1, 1], [0, -1, -1]]
    for j in range(ny):
        for k in range(nz):
            for m in range(4):
                for (s, e) in _runs(cm[m][:, j, k]):
                    limits.append([s, e, j + 1, j + 1, k + 1, k + 1]); dirs.append(cdir[m])
    cm3 = np.stack([wF & wU & wR, wF & wU & wL, wF & wD & wR, wF & wD & wL,
                    wB & wU & wR, wB & wU & wL, wB & wD & wR, wB & wD & wL], axis=3)
    cdir3 = [[1, 1, 1], [1, 1, -1], [1, -1, 1], [1, -1, -1], [-1, 1, 1], [-1, 1, -1], [-1, -1, 1], [-1, -1, -1]]
    idx = np.nonzero(cm3.ravel(order="F"))[0]
    I, J, K, M = np.unravel_index(idx, cm3.shape, order="F")
    for a in range(len(idx)):
        limits.append([I[a] + 1, I[a] + 1, J[a] + 1, J[a] + 1, K[a] + 1, K[a] + 1]); dirs.append(cdir3[M[a]])
    corners = {"limits": np.array(limits, dtype=np.int32).reshape(-1, 6),
               "dir": np.array(dirs, dtype=np.int32).reshape(-1, 3)}
    corners["adiabatic"] = np.zeros(corners["limits"].shape[0], dtype=np.int32)

    # regions completely inside walls (findWallsForBoundaries.m:291-329)
    iw = []
    is_wall = ~fr
    for k in range(nz):
        for j in range(ny):
            for (s, e) in _runs(is_wall[:, j, k]):
                iw.append([s, e, j + 1, j + 1, k + 1, k + 1])
    if iw:
        keys = [(r[0], r[1]) for r in iw]
        order_of_key = {}
        for kk in keys:
            order_of_key.setdefault(kk, len(order_of_key))
        ind = sorted(range(len(iw)), key=lambda r: order_of_key[keys[r]])  # stable
        iw = [iw[r] for r in ind]
    i = 0
    while i < len(iw) - 1:
        a, b = iw[i], iw[i + 1]
        if [a[0], a[1], a[4], a[5]] == [b[0], b[1], b[4], b[5]] and a[3] + 1 == b[2]:
            a[3] = b[3]; del iw[i + 1]
        else:
            i += 1
    i = 0
    while i < len(iw) - 1:
        a, b = iw[i], iw[i + 1]
        if a[0:4] == b[0:4] and a[5] + 1 == b[4]:
            a[5] = b[5]; del iw[i + 1]
        else:
            i += 1
    return fr, walls, corners, np.array(iw, dtype=np.int32).reshape(-1, 6)


def wall_boundary_list(walls, inside_walls, P0, E0, t_wall_relative=None):
    """The boundary list lidDrivenFlow.m builds from walls (:30-132): pressure Neumann on
    every wall face, Dirichlet p/u/v/w/e inside walls."""
    items = []
    for key, d in (("front", "xi"), ("back", "xf"), ("up", "yi"), ("down", "yf"), ("right", "zi"), ("left", "zf")):
        for w in walls[key]:
            items.append(("p", "neu", d, 0.0, list(w)))
    e_wall = E0 * t_wall_relative if t_wall_relative is not None else E0
    for w in inside_walls:
        w = list(w)
        items.append(("p", "dir", "yi", P0, w))
        items.append(("u", "dir", "yi", 0.0, w))
        items.append(("v", "dir", "yi", 0.0, w))
        items.append(("w", "dir", "yi", 0.0, w))
        items.append(("e", "dir", "yi", e_wall, w))
    return items


def init_boundaries(items, corners, neumann_coeffs, neumann2_coeffs):
    """Sort a boundary list into the per-variable arrays (initBoundaries.m:17-108, one rank)."""
    bi = BoundaryInfo()
    lists = {}
    for (var, typ, d, val, box) in items:
        kind = {"dir": "d", "neu": "n", "sec": "s"}[typ]
        V = var.upper()
        lists.setdefault((kind, V), []).append((box, val, DIR_CODE[d]))
    for (kind, V), rows in lists.items():
        bi.ind[(kind, V)] = np.array([r[0] for r in rows], dtype=np.int32).reshape(-1, 6)
        if kind == "d":
            bi.val[V] = np.array([r[1] for r in rows], dtype=np.float64)
        else:
            bi.dirs[(kind, V)] = np.array([r[2] for r in rows], dtype=np.int32)
    bi.cL = np.asarray(corners["limits"], dtype=np.int32).reshape(-1, 6)
    bi.cD = np.asarray(corners["dir"], dtype=np.int32).reshape(-1, 3)
    bi.cAdiabatic = np.asarray(corners["adiabatic"], dtype=np.int32).reshape(-1)
    bi.neumannCoeffs = np.asarray(neumann_coeffs, dtype=np.float64)
    bi.neumann2Coeffs = np.asarray(neumann2_coeffs, dtype=np.float64)
    return bi


# ---------------------------------------------------------------------------
# matrices for a case (makeMatrices.m + prepareThomas.m + getMatrixTypeBlocks.m)
# ---------------------------------------------------------------------------

def build_matrices(X, Y, Z, flow_region, periodic, fix_periodic, domain_ends, deriv="SL4", deriv_buffer="EX4",
                   filter_alpha=0.49, filter_borders="decentered", filter_border_flags=None,
                   buffers=None, metric="SL4", round_fortran=True, break_points=(None, None, None)):
    """Per-direction :class:`DirectionMatrices` for a case (``makeMatrices.m:1-155``);
    ``break_points`` restates ``mesh.x/y/z.breakPoint`` (``findDerivativeRegions.m:45-60``)."""
    nx, ny, nz = len(X), len(Y), len(Z)
    reg = mx.find_derivative_regions(flow_region, periodic, break_points)
    cl, cr, dl, dr = mx.finite_difference_coefficients(deriv)
    clb, crb, dlb, drb = mx.finite_difference_coefficients(deriv_buffer)
    fl, fr_, fdl, fdr = mx.spatial_filter_coefficients(filter_alpha, filter_borders)
    buffers = buffers or [{"i": {"n": 0}, "f": {"n": 0}}] * 3
    out = []
    coords = (X, Y, Z)
    for d, (n, key) in enumerate(zip((nx, ny, nz), "XYZ")):
        if n == 1:
            out.append(None)
            continue
        starts, ends = reg["derivStarts" + key], reg["derivEnds" + key]
        tmap = reg["typeMap" + key]
        clz, crz, clbz, crbz = cl, cr, clb, crb
        if d == 2 and nz == 4 and len(starts) == 1 and not starts[0] and not ends[0]:
            clz, crz = np.array([1.0]), np.array([0.0, math.pi / 4])
            clbz, crbz = clz, crz
        fclz, fcrz, fdlz, fdrz = fl, fr_, fdl, fdr
        if d == 2 and 1 < nz < 2 * len(fr_) - 1:
            fclz = fcrz = fdlz = fdrz = np.array([[1.0]])
        L, R = mx.make_matrices_each_direction(clz, crz, dl, dr, starts, ends, n, None)
        Lb, Rb = mx.make_matrices_each_direction(clbz, crbz, dlb, drb, starts, ends, n, buffers[d])
        fL, fR = mx.make_matrices_each_direction(fclz, fcrz, fdlz, fdrz, starts, ends, n, None)
        L, R = mx.add_buffer_to_matrix(L, Lb, R, Rb, n, buffers[d])
        mm = metric if not (d == 2 and nz == 4) else "SL4"
        L = mx.apply_metric(L, coords[d], periodic[d], fix_periodic[d], domain_ends[d], mm)
        flags = (filter_border_flags or {})
        # makeMatrices.m:90: `if numMethods.filterBorders` is true for any non-empty string
        if filter_borders:
            for side in ("Start", "End"):
                if flags.get("filterBorders%s%s" % (side, key), True) is False:
                    for t in range(len(fL)):
                        if side == "Start":
                            fL[t][0:5, :] = 0; fR[t][0:5, :] = 0
                            fL[t][0:5, 0:5] = np.eye(5); fR[t][0:5, 0:5] = np.eye(5)
                        else:
                            fL[t][-5:, :] = 0; fR[t][-5:, :] = 0
                            fL[t][-5:, -5:] = np.eye(5); fR[t][-5:, -5:] = np.eye(5)
        m = mx.prepare_thomas(L, R, fL, fR, tmap)
        blocks = mx.get_matrix_type_blocks(tmap, 1, 1)[0]
        m.blocks = blocks
        m = m.rounded() if round_fortran else m
        m.adj = mx.adjoint_sets(L, R, fL, fR, tmap)
        out.append(m)
    return out


def _dxmin(X, Y, Z):
    if len(Z) == 1:
        return (1 / np.min(np.diff(X)), 1 / np.min(np.diff(Y)), 0.0)
    return (1 / np.min(np.diff(X)), 1 / np.min(np.diff(Y)), 1 / np.min(np.diff(Z)))


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

def periodic_box(n=128, Re=1600.0, Ma=0.3, Pr=0.71, gamma=1.4, T0=300.0, filter_alpha=0.49, deriv="SL4",
                 nxyz=None, L=2 * math.pi):
    """Triply periodic box on [0, L)^3 (``source/boundaries/periodicBox.m``)."""
    nx, ny, nz = nxyz if nxyz else (n, n, n)
    X = generate_mesh(0, L, nx, periodic=True, fix_periodic_domain_size=True)
    Y = generate_mesh(0, L, ny, periodic=True, fix_periodic_domain_size=True)
    Z = generate_mesh(0, L, nz, periodic=True, fix_periodic_domain_size=True)
    fr = np.ones((nx, ny, nz), dtype=bool)
    fr, walls, corners, inside = find_walls_for_boundaries(fr)
    mats = build_matrices(X, Y, Z, fr, (True, True, nz > 1), (True, True, True), (L, L, L), deriv=deriv,
                          filter_alpha=filter_alpha)
    n1, n2 = mx.neumann_coefficients(6, 2)
    bc = init_boundaries(wall_boundary_list(walls, inside, 0.0, 0.0), corners,
                         mx.fortran_round(n1), mx.fortran_round(n2))
    return Case(name="periodic_box_%dx%dx%d" % (nx, ny, nz), nx=nx, ny=ny, nz=nz, Re=Re, Ma=Ma, Pr=Pr,
                gamma=gamma, T0=T0, X=X, Y=Y, Z=Z, mats=mats, bc=bc, flowRegion=fr, dxmin=_dxmin(X, Y, Z))


def turbulence_box(n=64, Re=1000.0, Ma=0.1, epsilon=1.0, L=1.0, nxyz=None, deriv="SL6", filter_alpha=0.499):
    """The forced turbulence box of ``examples/turbulenceBox.m``: a periodic box on [0, L)^3,
    SL6 derivatives, filter strength 0.499, and the ``turbulenceGenerator`` forcing over the
    whole domain with par = [epsilon, e0], e0 = 1/((gamma^2 - gamma) Ma^2)."""
    c = periodic_box(n=n, Re=Re, Ma=Ma, nxyz=nxyz, L=L, deriv=deriv, filter_alpha=filter_alpha)
    e0 = 1.0 / ((c.gamma ** 2 - c.gamma) * Ma ** 2)
    c.forcings = [{"type": "turbulenceGenerator", "ind": [1, c.nx, 1, c.ny, 1, c.nz], "par": [epsilon, e0]}]
    c.name = "turbulence_box_%dx%dx%d" % (c.nx, c.ny, c.nz)
    return c


def lid_driven(n=128, Re=1000.0, Ma=0.5, Pr=0.71, gamma=1.4, T0=300.0, filter_alpha=0.49, deriv="SL4",
               mesh_type="uniform", U0=1.0, nxy=None):
    """2-D lid-driven cavity on the unit square (``source/boundaries/lidDrivenFlow.m``).

    Numerics follow ``examples/lidDriven.m`` (filter borders 'reducedOrder' with the x
    start/end and y end rows left unfiltered, Neumann orders 6 and 2) with the SL4 scheme.
    """
    nx, ny = nxy if nxy else (n, n)
    X = generate_mesh(0, 1, nx, mtype=mesh_type, par=2.0)
    Y = generate_mesh(0, 1, ny, mtype=mesh_type, par=2.0)
    Z = generate_mesh(0, 1, 1, periodic=True, fix_periodic_domain_size=True)
    fr = np.ones((nx, ny, 1), dtype=bool)
    fr[[0, -1], :, :] = False
    fr[:, [0, -1], :] = False
    fr, walls, corners, inside = find_walls_for_boundaries(fr)
    E0 = 1.0 / ((gamma ** 2 - gamma) * Ma ** 2)
    P0 = (gamma - 1) * E0
    items = wall_boundary_list(walls, inside, P0, E0)
    n1, n2 = mx.neumann_coefficients(6, 2)
    bc = init_boundaries(items, corners, mx.fortran_round(n1), mx.fortran_round(n2))
    # lid: disturbance on y = 1 over the whole x range (examples/lidDriven.m:85-93)
    ind = np.array([1, nx, ny, ny, 1, 1], dtype=np.int32)
    bc.disturbances.append(dict(type="lidDrivenMovement", var="U", ind=ind,
                                X=mx.fortran_round(X[0:nx]), par=[U0]))
    flags = {"filterBordersStartX": False, "filterBordersEndX": False, "filterBordersEndY": False}
    mats = build_matrices(X, Y, Z, fr, (False, False, True), (False, False, True), (1.0, 1.0, 1.0),
                          deriv=deriv, filter_alpha=filter_alpha, filter_borders="reducedOrder",
                          filter_border_flags=flags)
    return Case(name="lid_driven_%dx%d" % (nx, ny), nx=nx, ny=ny, nz=1, Re=Re, Ma=Ma, Pr=Pr, gamma=gamma,
                T0=T0, X=X, Y=Y, Z=Z, mats=mats, bc=bc, flowRegion=fr, dxmin=_dxmin(X, Y, Z))


def cavity_channel(nx=96, ny=64, nz=1, Re=1000.0, Ma=0.5, Pr=0.71, gamma=1.4, T0=300.0, filter_alpha=0.49,
                   deriv="SL4", cavity=(0.3, 0.6, 0.35), adiabatic_corners=False, sfd=None):
    """A stretched 2-D/3-D box with walls at y-min and y-max, a rectangular cavity cut into
    the lower wall, and periodic x (and z): several matrix types per direction, corners,
    wall Neumann lists and an SFD buffer ramp -- the machinery the boundary-layer-over-cavity
    case exercises, in a size the CPU oracle runs in seconds."""
    X = generate_mesh(0, 1, nx, periodic=True, fix_periodic_domain_size=True)
    Y = generate_mesh(-0.5, 1, ny, mtype="tanh", par=1.5)
    Z = generate_mesh(0, 1, nz, periodic=True, fix_periodic_domain_size=True)
    x0, x1, depth_y = cavity
    fr = np.ones((nx, ny, nz), dtype=bool)
    # solid below y = 0 except the cavity x0 < x < x1
    solid = (Y[None, :, None] < 0) & ~((X[:, None, None] > x0) & (X[:, None, None] < x1))
    fr &= ~solid
    fr[:, [0, -1], :] = False
    fr, walls, corners, inside = find_walls_for_boundaries(fr)
    if adiabatic_corners:
        corners["adiabatic"][:] = 1
    E0 = 1.0 / ((gamma ** 2 - gamma) * Ma ** 2)
    P0 = (gamma - 1) * E0
    items = wall_boundary_list(walls, inside, P0, E0)
    # open top: null second derivative of u, v, e and Neumann pressure on the top row
    top = [1, nx, ny, ny, 1, nz]
    for v in ("u", "v", "e"):
        items.append((v, "sec", "yf", 0.0, list(top)))
    n1, n2 = mx.neumann_coefficients(6, 2)
    bc = init_boundaries(items, corners, mx.fortran_round(n1), mx.fortran_round(n2))
    mats = build_matrices(X, Y, Z, fr, (True, False, True), (True, False, True), (1.0, 1.0, 1.0),
                          deriv=deriv, filter_alpha=filter_alpha, filter_borders="decentered")
    case = Case(name="cavity_channel_%dx%dx%d" % (nx, ny, nz), nx=nx, ny=ny, nz=nz, Re=Re, Ma=Ma, Pr=Pr,
                gamma=gamma, T0=T0, X=X, Y=Y, Z=Z, mats=mats, bc=bc, flowRegion=fr, dxmin=_dxmin(X, Y, Z))
    if sfd:
        chi = np.ones((nx, ny, nz))
        nb = sfd.get("buffer", 8)
        for j in range(1, nb + 1):  # calcSFDregion.m:31-35 ramp on the y end
            chi[:, -j, :] *= 0.5 - 0.5 * math.cos(math.pi * (j - 1) / nb)
        chi = sfd["X"] * (1 - chi)
        case.sfd_type, case.sfd_delta, case.sfd_X = 2, sfd["Delta"], sfd["X"]
        case.sfd_chi = np.asfortranarray(chi)
    return case


def sfd_region(shape, buffers, X):
    """calcSFDregion.m:4-53 with applyX/Y/Z = 2: X * (1 - prod of 0.5 - 0.5 cos ramps over the
    buffer zones); buffers[d] = (n initial, n final) buffer nodes of direction d."""
    chi = np.ones(shape)
    for d, (ni, nf) in enumerate(buffers):
        for i in range(1, ni + 1):
            idx = [slice(None)] * 3
            idx[d] = i - 1
            chi[tuple(idx)] *= 0.5 - 0.5 * math.cos(math.pi * (i - 1) / ni)
        for i in range(1, nf + 1):
            idx = [slice(None)] * 3
            idx[d] = shape[d] - i
            chi[tuple(idx)] *= 0.5 - 0.5 * math.cos(math.pi * (i - 1) / nf)
    return np.asfortranarray(X * (1.0 - chi))


def boundary_layer_isothermal(nx, ny, nz=1, Re=1000.0, Ma=0.5, Pr=0.71, gamma=1.4, T0=300.0, filter_alpha=0.49,
                              deriv="SL4", cavity=None, buffers=((0, 0), (0, 0)), sfd=None, x_range=(-1.0, 5.0),
                              y_top=4.0, Lz=1.0, name=None):
    """Compressible boundary layer over an isothermal plate at y = 0, with an optional
    rectangular cavity of depth 1 at cavity = (x0, x1); 2-D (nz = 1) or spanwise periodic.

    The boundary set is boundaryLayerIsothermal.m's for mesh.X(1) < 0, in its order:
    * Dirichlet inflow u = 1, v = w = 0, e = E0 and pressure Neumann over the whole x = X(1)
      plane (:4-78), outflow null second derivatives with p = P0 (:80-138), outer flow null
      second derivatives (:141-201); z is periodic, so :203-315 add nothing;
    * the flow region: solid at and below the row nearest y = 0, the cavity carved out
      (:317-344), walls, corners and wall interiors from findWallsForBoundaries;
    * the free-slip wall (:362-369): every up-facing wall is moved to start at the first node
      with x >= 0, the plate row upstream of it becomes a wall of its own (the last up wall)
      and the x derivative and filter stencils are cut there (mesh.x.breakPoint, restated by
      findDerivativeRegions.m:45-60);
    * pressure Neumann on every wall (:371-405), u and w Neumann on the free-slip wall
      (:407-431), then p = P0, u = v = w = 0, e = E0 on every solid node (:433-497).

    Meshes follow parameters.m:84-147 ('attractors', matchFixed = 2, sigmoid buffer zones)
    scaled to this domain: in x a point attractor at the leading edge (the reference's
    domain starts there) and, with a cavity, a region of strength 3 around it; in y the
    region [-2D, -D/10, D/10, 2 delta99] of strength 12 with delta99 = 5 sqrt(xEnd / Re) at
    the outflow (D = 1 with a cavity, 0 without); fixed points (meshAddFixedPoints.m:3-10)
    at the leading edge and the cavity's edges and bottom.  The filter borders are those of
    parameters.m:182-186 (reduced order, no filter on the first and last five x nodes nor on
    the last five y nodes).  With ``sfd = (X, Delta)``, SFD type 2 on the buffer ramps
    (calcSFDregion.m).  nx, ny count all nodes, buffers included.
    """
    (bxi, bxf), (byi, byf) = buffers
    sig = lambda n, st: {"n": n, "type": "sigmoid", "stretching": st, "transition": 0.2}
    depth = 1.0 if cavity else 0.0
    xf_pts = (0.0,) + (tuple(cavity) if cavity else ())
    x_regions = [(cavity[0] - 0.5, cavity[0] - 0.25, cavity[1] + 0.25, cavity[1] + 0.5, 3.0)] if cavity else []
    X = generate_mesh(x_range[0], x_range[1], nx - bxi - bxf, mtype="attractors",
                      attractor_points=[(0.0, 2.0, 0.1)], attractor_regions=x_regions,
                      buffer_i=sig(bxi, 30) if bxi else None, buffer_f=sig(bxf, 15) if bxf else None,
                      fix_points=xf_pts)
    d99 = 5.0 * math.sqrt(x_range[1] / Re)
    Y = generate_mesh(-depth, y_top, ny - byi - byf, mtype="attractors",
                      attractor_regions=[(-2.0 * depth if depth else -2.0, -depth / 10 if depth else -1.0,
                                          depth / 10, 2.0 * d99, 12.0)],
                      buffer_i=sig(byi, 30) if byi else None, buffer_f=sig(byf, 30) if byf else None,
                      fix_points=(-depth, 0.0) if depth else (0.0,))
    if nz > 1:
        Z = generate_mesh(0.0, Lz, nz, periodic=True, fix_periodic_domain_size=True)
    else:
        Z = np.array([0.0])
    E0 = 1.0 / ((gamma ** 2 - gamma) * Ma ** 2)
    P0 = (gamma - 1) * E0
    items = []
    # inflow (:4-78): Dirichlet u, v, w, e when the mesh starts at x <= 0; otherwise the
    # holdInlet disturbance keeps the inflow plane at its first values (:53-66)
    inflow = [1, 1, 1, ny, 1, nz]
    hold = X[0] > 0
    if not hold:
        for v, val in (("u", 1.0), ("v", 0.0), ("w", 0.0), ("e", E0)):
            items.append((v, "dir", "xi", val, list(inflow)))
    items.append(("p", "neu", "xi", 0.0, list(inflow)))
    # outflow (:80-138) and outer flow (:141-201)
    outflow = [nx, nx, 1, ny, 1, nz]
    for v in ("u", "v", "w", "e"):
        items.append((v, "sec", "xf", 0.0, list(outflow)))
    items.append(("p", "dir", "xf", P0, list(outflow)))
    top = [1, nx, ny, ny, 1, nz]
    for v in ("u", "v", "w", "e", "p"):
        items.append((v, "sec", "yf", 0.0, list(top)))
    # flow region (:317-344): the plate, then the cavity (open intervals in x and y)
    fr = np.ones((nx, ny, nz), dtype=bool)
    wall_j = int(np.argmin(np.abs(Y))) + 1
    fr[:, :wall_j, :] = False
    if cavity:
        in_x = (X > cavity[0]) & (X < cavity[1])
        in_y = (Y > -depth) & (Y < 0.0)
        fr[np.ix_(in_x, in_y, np.ones(nz, dtype=bool))] = True
    fr, walls, corners, inside = find_walls_for_boundaries(fr)
    # free-slip wall and the break point (:362-369)
    break_x = None
    if X[0] < 0:
        first_pos = int(np.nonzero(X >= 0)[0][0]) + 1
        last_neg = int(np.nonzero(X < 0)[0][-1]) + 1
        j_plate = int(np.nonzero(Y >= 0)[0][0]) + 1
        up = [list(w) for w in walls["up"]]
        for w in up:
            w[0] = max(w[0], first_pos)
        up.append([1, last_neg, j_plate, j_plate, 1, nz])
        walls["up"] = up
        break_x = [[last_neg, j_plate, j_plate, 1, nz]]
    # pressure Neumann on every wall (:371-405)
    for key, d in (("front", "xi"), ("back", "xf"), ("up", "yi"), ("down", "yf"), ("right", "zi"), ("left", "zf")):
        for w in walls[key]:
            items.append(("p", "neu", d, 0.0, list(w)))
    # u and w Neumann on the free-slip wall, the last up wall (:407-431)
    if X[0] < 0:
        for v in ("u", "w"):
            items.append((v, "neu", "yi", 0.0, list(walls["up"][-1])))
    # every solid node (:433-497)
    for w in inside:
        w = list(w)
        items.append(("p", "dir", "yi", P0, w))
        for v in ("u", "v", "w"):
            items.append((v, "dir", "yi", 0.0, w))
        items.append(("e", "dir", "yi", E0, w))
    n1, n2 = mx.neumann_coefficients(6, 2)
    bc = init_boundaries(items, corners, mx.fortran_round(n1), mx.fortran_round(n2))
    if hold:  # par 0: the density is not held
        bc.disturbances.append(dict(type="holdInlet", var="UVRWE", ind=np.array(inflow, dtype=np.int32),
                                    X=np.asarray(X[:1], dtype=np.float64), par=[0.0]))
    bufs = [{"i": sig(bxi, 30) if bxi else {"n": 0}, "f": sig(bxf, 15) if bxf else {"n": 0}},
            {"i": sig(byi, 30) if byi else {"n": 0}, "f": sig(byf, 30) if byf else {"n": 0}},
            {"i": {"n": 0}, "f": {"n": 0}}]
    flags = {"filterBordersStartX": False, "filterBordersEndX": False, "filterBordersEndY": False}
    mats = build_matrices(X, Y, Z, fr, (False, False, True), (False, False, True),
                          (x_range[1], y_top, Lz), deriv=deriv, deriv_buffer="EX4", filter_alpha=filter_alpha,
                          filter_borders="reducedOrder", filter_border_flags=flags, buffers=bufs,
                          break_points=(break_x, None, None))
    case = Case(name=name or "bl_%dx%dx%d" % (nx, ny, nz), nx=nx, ny=ny, nz=nz, Re=Re, Ma=Ma, Pr=Pr, gamma=gamma,
                T0=T0, X=X, Y=Y, Z=Z, mats=mats, bc=bc, flowRegion=fr, dxmin=_dxmin(X, Y, Z))
    if sfd:
        case.sfd_type, case.sfd_X, case.sfd_delta = 2, sfd[0], sfd[1]
        case.sfd_chi = sfd_region((nx, ny, nz), ((bxi, bxf), (byi, byf), (0, 0)), sfd[0])
    return case


def add_disturbance(case: Case, dtype, var, ind, par):
    """Append a disturbance to the case (a flowType.disturb entry with active = true and
    forcing = false): dtype 'lidDrivenMovement', 'periodicSine' or 'holdInlet', var the
    variables of the call ('V', or 'UVRWE' for holdInlet), ind the 1-based box
    [i1 i2 j1 j2 k1 k2], par the parameters ([U0]; [omega, amplitude]; [holdDensity]).  The
    box's x coordinates come from the mesh, as writeFortranDisturbances.m:40-50 writes them."""
    ind = np.asarray(ind, dtype=np.int32)
    case.bc.disturbances.append(dict(type=dtype, var=var, ind=ind, X=np.asarray(case.X[ind[0] - 1:ind[1]], dtype=np.float64),
                                     par=[float(p) for p in par]))
    return case


def periodic_sine_strip(case: Case, i1, i2, omega=7.0, amp=0.02, var="V"):
    """A periodicSine disturbance (blowing and suction) of `var` on the plate row of a
    boundary layer, x nodes i1..i2, all z."""
    j = int(np.nonzero(np.asarray(case.Y) >= 0)[0][0]) + 1
    return add_disturbance(case, "periodicSine", var, [i1, i2, j, j, 1, case.nz], [omega, amp])


def boundary_layer_cavity(nx=800, ny=300, nz=1, buffers=((40, 30), (0, 40)), sfd=(0.02, 15.0), **kw):
    """Config 3: the 2-D boundary layer over a cavity of depth 1 and length 1 at 1 < x < 2,
    x in [-1, 5] and y in [-1, 4] (physical part), Re 1000, Ma 0.5, with the buffer zones of
    parameters.m:124-142 (inflow 40, outflow 30 and top 40 nodes in the full case), EX4
    derivatives inside them and SFD (X 0.02, Delta 15) on their ramps; see
    :func:`boundary_layer_isothermal`.  nz > 1 gives the spanwise-periodic 3-D version."""
    kw.setdefault("cavity", (1.0, 2.0))
    c = boundary_layer_isothermal(nx, ny, nz, buffers=buffers, sfd=sfd, **kw)
    c.name = "bl_cavity_%dx%d" % (nx, ny) + ("x%d" % nz if nz > 1 else "")
    return c


def boundary_layer(nx=400, ny=150, nz=64, **kw):
    """Config 5: the 3-D spanwise-periodic boundary layer over a flat plate (no cavity, no
    buffer zones, no SFD), x in [-1, 5], y in [0, 4], z in [0, 1); see
    :func:`boundary_layer_isothermal`."""
    return boundary_layer_isothermal(nx, ny, nz, name="boundary_layer_%dx%dx%d" % (nx, ny, nz), **kw)


def blasius_profile(eta_max=12.0, n=6001):
    """Blasius similarity solution f(eta), f'(eta): f''' + f f''/2 = 0, f(0) = f'(0) = 0,
    f'(inf) = 1, by RK4 shooting on f''(0).  It stands in for the compressible profile of
    calcCompressibleBL.m."""
    eta = np.linspace(0.0, eta_max, n)
    h = eta[1] - eta[0]

    def rhs(y):
        return np.array([y[1], y[2], -0.5 * y[0] * y[2]])

    def integrate(s):
        y = np.array([0.0, 0.0, s])
        out = np.zeros((n, 3))
        out[0] = y
        for i in range(1, n):
            k1 = rhs(y)
            k2 = rhs(y + 0.5 * h * k1)
            k3 = rhs(y + 0.5 * h * k2)
            k4 = rhs(y + h * k3)
            y = y + h / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
            out[i] = y
        return out

    lo, hi = 0.2, 0.5
    for _ in range(50):
        mid = 0.5 * (lo + hi)
        if integrate(mid)[-1, 1] > 1.0:
            hi = mid
        else:
            lo = mid
    sol = integrate(0.5 * (lo + hi))
    return eta, sol[:, 0], sol[:, 1]


def blasius_flow(case: Case):
    """generateInitialFlow.m:53-103 ('blasius', no blasiusFit): R = 1, E = E0, V = W = 0;
    U = 1 at x <= 0; at x > 0 the Blasius u(eta) with the momentum thickness
    theta = 0.664 sqrt(x / Re) (the table's eta scaled by theta / 0.664155), U = 0 below
    y = 0, U clipped at 1.  The Blasius table comes from RK4 shooting instead of ode45 and is
    interpolated linearly instead of by splines (differences of order 1e-7 in the initial
    field, which only seeds the run)."""
    eta_t, _, fp_t = blasius_profile()
    theta_bl = 0.664155332943009
    s = (case.nx, case.ny, case.nz)
    U = np.ones((case.nx, case.ny))
    for i, xi in enumerate(case.X):
        if xi > 0:
            theta = 0.664 * math.sqrt(xi / case.Re)
            u = np.interp(case.Y * theta_bl / theta, eta_t, fp_t, left=0.0, right=1.0)
            u[case.Y < 0] = 0.0
            U[i] = u
    U = np.minimum(U, 1.0)
    out = uniform_flow(case)
    out["U"] = np.asfortranarray(np.repeat(U[:, :, None], s[2], axis=2))
    return out


# ---------------------------------------------------------------------------
# initial flows (synthetic, seeded)
# ---------------------------------------------------------------------------

def uniform_flow(case: Case, U0=0.0):
    """generateInitialFlow.m:19-36 'uniform' (R = 1, E = E0, U = U0)."""
    s = (case.nx, case.ny, case.nz)
    return dict(U=np.full(s, U0, order="F"), V=np.zeros(s, order="F"), W=np.zeros(s, order="F"),
                R=np.ones(s, order="F"), E=np.full(s, case.E0, order="F"))


def solenoidal_turbulence(case: Case, seed=1234, k0=4.0, urms=1.0):
    """Random solenoidal velocity with E(k) ~ k^4 exp(-2 (k/k0)^2), unit-rms, R = 1, E = E0.

    Seeded synthetic stand-in for the turbulence-box initial condition (the reference has
    no such initializer; its example adds noise and a forcing).
    """
    nx, ny, nz = case.nx, case.ny, case.nz
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(nx, 1.0 / nx)
    ky = np.fft.fftfreq(ny, 1.0 / ny)
    kz = np.fft.rfftfreq(nz, 1.0 / nz)
    KX, KY, KZ = np.meshgrid(kx, ky, kz, indexing="ij")
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    k = np.sqrt(k2)
    amp = np.zeros_like(k)
    nz_ = k > 0
    spec = k ** 4 * np.exp(-2.0 * (k / k0) ** 2)
    amp[nz_] = np.sqrt(spec[nz_] / (4 * math.pi * k2[nz_]))
    comps = []
    for _ in range(3):
        ph = rng.uniform(0, 2 * math.pi, size=k.shape)
        comps.append(amp * np.exp(1j * ph))
    u, v, w = comps
    # project out the divergence
    with np.errstate(invalid="ignore", divide="ignore"):
        dot = (KX * u + KY * v + KZ * w) / np.where(k2 > 0, k2, 1)
    u = u - KX * dot; v = v - KY * dot; w = w - KZ * dot
    ax = (0, 1, 2)
    U = np.fft.irfftn(u, s=(nx, ny, nz), axes=ax)
    V = np.fft.irfftn(v, s=(nx, ny, nz), axes=ax)
    Wf = np.fft.irfftn(w, s=(nx, ny, nz), axes=ax)
    rms = math.sqrt(np.mean(U ** 2 + V ** 2 + Wf ** 2) / 3.0)
    U, V, Wf = U * urms / rms, V * urms / rms, Wf * urms / rms
    s = (nx, ny, nz)
    return dict(U=np.asfortranarray(U), V=np.asfortranarray(V), W=np.asfortranarray(Wf),
                R=np.ones(s, order="F"), E=np.full(s, case.E0, order="F"))


def random_flow(case: Case, seed=7, amp=0.05):
    """Smooth-ish random perturbation of the uniform state for parity tests."""
    rng = np.random.default_rng(seed)
    s = (case.nx, case.ny, case.nz)
    f = uniform_flow(case)
    for key, scale in (("U", 1.0), ("V", 1.0), ("W", 1.0 if case.is3d else 0.0), ("R", 0.2), ("E", 0.2 * case.E0)):
        noise = rng.standard_normal(s)
        # light smoothing so the field is resolved by the compact schemes
        for ax in range(3):
            if s[ax] > 2:
                noise = 0.25 * np.roll(noise, 1, ax) + 0.5 * noise + 0.25 * np.roll(noise, -1, ax)
        f[key] = np.asfortranarray(f[key] + amp * scale * noise)
    return f
