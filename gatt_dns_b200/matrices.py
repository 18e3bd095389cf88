"""Compact-scheme coefficient emitter (host preprocessing, numpy).

Restates the MATLAB preprocessing that produces the arrays the solver reads from
``matrices.F90``.  The CUDA kernels and the CPU oracle both consume exactly these
arrays, so kernel parity is an exact-input comparison.

Reference files restated here (paths within the GATT_DNS project):

* ``source/finiteDifferenceCoefficients.m:10-163`` -- SL4 / SL6 / SL6O3 / EX2 / EX4 stencils
* ``source/spatialFilterCoefficients.m:1-104``       -- Gaitonde 10th-order compact filter
* ``source/makeMatrices.m:158-342``                  -- dense LHS/RHS per direction and type,
  buffer-zone blending and the grid-stretching metric
* ``source/prepareThomas.m:1-172``                   -- Thomas factors, cyclic ``D`` row, RHS diagonals
* ``source/getMatrixTypeBlocks.m:1-102``             -- (type, line-range) block lists
* ``source/getDomainSlices.m:1-24``                  -- 2DECOMP-style slicing
* ``source/findDerivativeRegions.m:1-179``           -- per-line matrix type maps
* ``source/writeFortranMatrices.m:228-235``          -- the ``%.20f`` text rounding the solver sees

MATLAB's ``\\`` and ``inv`` are replaced by LAPACK through numpy; the two agree to a
few ulps, which is why the emitted arrays (not MATLAB) are the parity anchor.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "finite_difference_coefficients",
    "spatial_filter_coefficients",
    "make_matrices_each_direction",
    "add_buffer_to_matrix",
    "apply_metric",
    "prepare_thomas",
    "get_domain_slices",
    "get_matrix_type_blocks",
    "find_derivative_regions",
    "fortran_round",
    "DirectionMatrices",
    "neumann_coefficients",
]


def fortran_round(x):
    """Round values through the ``%.20f`` text the generated Fortran source carries.

    ``writeFortranMatrices.m:231`` prints every coefficient with ``'%.20fd0'``; the
    Fortran compiler then converts that decimal literal to the nearest double.
    """
    a = np.asarray(x, dtype=np.float64)
    flat = [float("%.20f" % v) for v in a.ravel(order="F")]
    return np.array(flat, dtype=np.float64).reshape(a.shape, order="F")


# ---------------------------------------------------------------------------
# Stencils
# ---------------------------------------------------------------------------

def finite_difference_coefficients(method: str):
    """Centered and decentered compact first-derivative stencils.

    Follows ``source/finiteDifferenceCoefficients.m:5-163``.  Returns
    ``(centeredLHS, centeredRHS, decenteredLHS, decenteredRHS)``; centered stencils
    start at the centre point and move right, decentered ones are the rows at the top
    of the matrix.
    """
    if method == "SL6":
        w = 1.8
        ma = np.array([[1, 1, 1, -2],
                       [1, 4, 9, -6],
                       [1, 16, 81, -10],
                       [math.sin(w), math.sin(2 * w) / 2, math.sin(3 * w) / 3, -2 * w * math.cos(w)]],
                      dtype=np.float64)
        mb = np.array([1, 0, 0, w], dtype=np.float64)
        c = np.linalg.solve(ma, mb)
        a, b, cc, alpha = c[0] / 2, c[1] / 4, c[2] / 6, c[3]
        cl = np.array([1.0, alpha])
        cr = np.array([0.0, a, b, cc])
        # border, first stage (finiteDifferenceCoefficients.m:37-61)
        ma = np.array([[1, 1, 1, 1, 1, 1, 0],
                       [0, 1, 2, 3, 4, 5, -1],
                       [0, 1, 4, 9, 16, 25, -2],
                       [0, 1, 8, 27, 64, 125, -3],
                       [0, 1, 16, 81, 256, 625, -4],
                       [0, 1, 32, 243, 1024, 3125, -5],
                       [0, 1, 64, 729, 4096, 15625, -6]], dtype=np.float64)
        mb = np.array([0, 1, 0, 0, 0, 0, 0], dtype=np.float64)
        c = np.linalg.solve(ma, mb)
        lhs1 = [1.0, c[6], 0.0, 0.0]
        rhs1 = [c[0], c[1], c[2], c[3], c[4], c[5]]
        # second stage (:63-74)
        ma = np.array([[-1, 2], [-1, 6]], dtype=np.float64)
        mb = np.array([-1, 0], dtype=np.float64)
        c = np.linalg.solve(ma, mb)
        a2, alpha2 = c[0] / 2, c[1]
        lhs2 = [alpha2, 1.0, alpha2, 0.0]
        rhs2 = [-a2, 0.0, a2, 0.0, 0.0, 0.0]
        # third stage = centered SL4 (:76-92)
        ma = np.array([[1, 0, -2 / 3], [0, 1, -4 / 3],
                       [math.sin(w), math.sin(2 * w) / 2, -2 * w * math.cos(w)]], dtype=np.float64)
        mb = np.array([4 / 3, -1 / 3, w], dtype=np.float64)
        c = np.linalg.solve(ma, mb)
        a3, b3, alpha3 = c[0] / 2, c[1] / 4, c[2]
        lhs3 = [0.0, alpha3, 1.0, alpha3]
        rhs3 = [-b3, -a3, 0.0, a3, b3, 0.0]
        return cl, cr, np.array([lhs1, lhs2, lhs3]), np.array([rhs1, rhs2, rhs3])

    if method == "SL6O3":
        c = [0.392465753424658, 1.565410958904110, 0.237260273972603, -0.017739726027397]
        alpha, a, b, cc = c
        cl = np.array([1.0, alpha])
        cr = np.array([0.0, a / 2, b / 4, cc / 6])
        alpha3, a3, b3 = 0.350978473581213, 1.567318982387476, 0.134637964774951
        pi = math.pi
        dl = np.array([[1, (3 * pi + 40) / (3 * pi + 8), 0, 0],
                       [1 / 4, 1, 1 / 4, 0],
                       [0, alpha3, 1, alpha3]], dtype=np.float64)
        dr = np.array([[-(13 * pi + 56) / (2 * (3 * pi + 8)), (15 * pi + 8) / (2 * (3 * pi + 8)),
                        -(3 * pi - 56) / (2 * (3 * pi + 8)), (pi - 8) / (2 * (3 * pi + 8)), 0],
                       [-3 / 4, 0, 3 / 4, 0, 0],
                       [-b3 / 4, -a3 / 2, 0, a3 / 2, b3 / 4]], dtype=np.float64)
        return cl, cr, dl, dr

    if method == "SL4":
        w = 1.8
        ma = np.array([[1, 0, -2 / 3], [0, 1, -4 / 3],
                       [math.sin(w), math.sin(2 * w) / 2, -2 * w * math.cos(w)]], dtype=np.float64)
        mb = np.array([4 / 3, -1 / 3, w], dtype=np.float64)
        c = np.linalg.solve(ma, mb)
        a, b, alpha = c[0] / 2, c[1] / 4, c[2]
        cl = np.array([1.0, alpha])
        cr = np.array([0.0, a, b])
        dl = np.array([[1, 3, 0], [1 / 4, 1, 1 / 4]], dtype=np.float64)
        dr = np.array([[-17 / 6, 3 / 2, 3 / 2, -1 / 6], [-3 / 4, 0, 3 / 4, 0]], dtype=np.float64)
        return cl, cr, dl, dr

    if method == "EX2":
        return (np.array([1.0]), np.array([0.0, 0.5]),
                np.array([[1.0]]), np.array([[-1.5, 2.0, -0.5]]))

    if method == "EX4":
        return (np.array([1.0]), np.array([0.0, 2 / 3, -1 / 12]),
                np.array([[1.0]]),
                np.array([[-25 / 12, 4, -3, 4 / 3, -1 / 4], [-1 / 2, 0, 1 / 2, 0, 0]], dtype=np.float64))

    raise ValueError("Finite differences method not implemented: %s" % method)


def spatial_filter_coefficients(alpha: float, filter_borders="decentered"):
    """Gaitonde & Visbal 10th-order compact filter stencils.

    Follows ``source/spatialFilterCoefficients.m:1-104`` (borders: ``decentered``,
    ``reducedOrder`` or ``off``; a logical ``True``/``False`` maps to decentered/off).
    """
    lhs = np.array([1.0, alpha])
    rhs = np.array([(193 + 126 * alpha) / 256, (105 + 302 * alpha) / 512, (-15 + 30 * alpha) / 128,
                    (45 - 90 * alpha) / 1024, (-5 + 10 * alpha) / 512, (1 - 2 * alpha) / 1024])
    if isinstance(filter_borders, (bool, np.bool_)):
        filter_borders = "decentered" if filter_borders else "off"
    a = alpha
    if filter_borders == "decentered":
        dl = np.array([[1.0, alpha]])
        ab = np.zeros((11, 5))
        ab[:, 4] = [(-1 + 2 * a) / 1024, (5 - 10 * a) / 512, (-45 + 90 * a) / 1024, (15 + 98 * a) / 128,
                    (407 + 210 * a) / 512, (63 + 130 * a) / 256, (-105 + 210 * a) / 512, (15 - 30 * a) / 128,
                    (-45 + 90 * a) / 1024, (5 - 10 * a) / 512, (-1 + 2 * a) / 1024]
        ab[:, 3] = [(1 - 2 * a) / 1024, (-5 + 10 * a) / 512, (45 + 934 * a) / 1024, (113 + 30 * a) / 128,
                    (105 + 302 * a) / 512, (-63 + 126 * a) / 256, (105 - 210 * a) / 512, (-15 + 30 * a) / 128,
                    (45 - 90 * a) / 1024, (-5 + 10 * a) / 512, (1 - 2 * a) / 1024]
        ab[:, 2] = [(-1 + 2 * a) / 1024, (5 + 502 * a) / 512, (979 + 90 * a) / 1024, (15 + 98 * a) / 128,
                    (-105 + 210 * a) / 512, (63 - 126 * a) / 256, (-105 + 210 * a) / 512, (15 - 30 * a) / 128,
                    (-45 + 90 * a) / 1024, (5 - 10 * a) / 512, (-1 + 2 * a) / 1024]
        ab[:, 1] = [(1 + 1022 * a) / 1024, (507 + 10 * a) / 512, (45 + 934 * a) / 1024, (-15 + 30 * a) / 128,
                    (105 - 210 * a) / 512, (-63 + 126 * a) / 256, (105 - 210 * a) / 512, (-15 + 30 * a) / 128,
                    (45 - 90 * a) / 1024, (-5 + 10 * a) / 512, (1 - 2 * a) / 1024]
        ab[:, 0] = [(1023 + 1 * a) / 1024, (5 + 507 * a) / 512, (-45 + 45 * a) / 1024, (15 - 15 * a) / 128,
                    (-105 + 105 * a) / 512, (63 - 63 * a) / 256, (-105 + 105 * a) / 512, (15 - 15 * a) / 128,
                    (-45 + 45 * a) / 1024, (5 - 5 * a) / 512, (-1 + 1 * a) / 1024]
        return lhs, rhs, dl, ab.T.copy()
    if filter_borders == "reducedOrder":
        dl = np.array([[1.0]])
        F2 = np.array([1 / 2 + a, 1 / 2 + a]) / np.array([1, 2])
        F4 = np.array([5 / 8 + 3 / 4 * a, 1 / 2 + a, -1 / 8 + 1 / 4 * a]) / np.array([1, 2, 2])
        F6 = np.array([11 / 16 + 5 / 8 * a, 15 / 32 + 17 / 16 * a, -3 / 16 + 3 / 8 * a, 1 / 32 - 1 / 16 * a]) / np.array([1, 2, 2, 2])
        F8 = np.array([93 / 128 + 70 / 128 * a, 7 / 16 + 18 / 16 * a, -7 / 32 + 14 / 32 * a, 1 / 16 - 1 / 8 * a,
                       -1 / 128 + 1 / 64 * a]) / np.array([1, 2, 2, 2, 2])
        dr = np.zeros((5, 9))
        dr[0, 0] = 1
        dr[1, 0:3] = F2[[1, 0, 1]]
        dr[2, 0:5] = F4[[2, 1, 0, 1, 2]]
        dr[3, 0:7] = F6[[3, 2, 1, 0, 1, 2, 3]]
        dr[4, 0:9] = F8[[4, 3, 2, 1, 0, 1, 2, 3, 4]]
        return lhs, rhs, dl, dr
    if filter_borders == "off":
        return lhs, rhs, np.eye(5), np.eye(5)
    raise ValueError("unknown filterBorders %r" % (filter_borders,))


def neumann_coefficients(neumann_order: int, neumann2_order: int):
    """Extrapolation weights for Neumann and null-second-derivative conditions.

    ``source/getBoundaryConditions.m:75-80``: one-sided difference stencils NC1/NC2 of the
    given orders, normalised so that ``u(1) = sum(c(i) * u(i+1))``.
    """
    nc1 = [[-1, 1], [-3 / 2, 2, -1 / 2], [-11 / 6, 3, -3 / 2, 1 / 3], [-25 / 12, 4, -3, 4 / 3, -1 / 4],
           [-137 / 60, 5, -5, 10 / 3, -5 / 4, 1 / 5], [-49 / 20, 6, -15 / 2, 20 / 3, -15 / 4, 6 / 5, -1 / 6]]
    nc2 = [[1, -2, 1], [2, -5, 4, -1], [35 / 12, -26 / 3, 19 / 2, -14 / 3, 11 / 12],
           [15 / 4, -77 / 6, 107 / 6, -13, 61 / 12, -5 / 6],
           [203 / 45, -87 / 5, 117 / 4, -254 / 9, 33 / 2, -27 / 5, 137 / 180],
           [469 / 90, -223 / 10, 879 / 20, -949 / 18, 41, -201 / 10, 1019 / 180, -7 / 10]]
    s1 = np.array(nc1[neumann_order - 1], dtype=np.float64)
    s2 = np.array(nc2[neumann2_order - 1], dtype=np.float64)
    return -s1[1:] / s1[0], -s2[1:] / s2[0]


# ---------------------------------------------------------------------------
# Dense matrices per direction
# ---------------------------------------------------------------------------

def make_matrices_each_direction(cl, cr, dl, dr, deriv_starts, deriv_ends, n, buffer_info=None):
    """Dense LHS/RHS per matrix type (``makeMatrices.m:158-263``).

    ``deriv_starts``/``deriv_ends`` are lists (one per type) of 1-based node indices at
    which a one-sided boundary stencil starts/ends.
    """
    cl = np.atleast_1d(np.asarray(cl, dtype=np.float64))
    cr = np.atleast_1d(np.asarray(cr, dtype=np.float64))
    dl = np.atleast_2d(np.asarray(dl, dtype=np.float64))
    dr = np.atleast_2d(np.asarray(dr, dtype=np.float64))
    if n != 1 and n < 2 * len(cr) - 1:
        raise ValueError("Mesh is not large enough for one of the stencils. It has %d nodes but the "
                         "stencil needs at least %d." % (n, 2 * len(cr) - 1))
    ntypes = len(deriv_starts)
    if n == 1:
        v = 0.0 if cr[0] == 0 else 1.0
        return [np.ones((1, 1)) for _ in range(ntypes)], [np.full((1, 1), v) for _ in range(ntypes)]

    rows = np.arange(n)
    lhs_base = np.diag(np.full(n, cl[0]))
    rhs_base = np.diag(np.full(n, cr[0]))
    invert = -1.0 if cr[0] == 0 else 1.0
    for i in range(1, len(cl)):
        lhs_base[rows, (rows + i) % n] = cl[i]
        lhs_base[rows, (rows - i) % n] = cl[i]
    for i in range(1, len(cr)):
        rhs_base[rows, (rows + i) % n] = cr[i]
        rhs_base[rows, (rows - i) % n] = invert * cr[i]

    deriv_starts = [list(np.atleast_1d(s).astype(int)) for s in deriv_starts]
    deriv_ends = [list(np.atleast_1d(e).astype(int)) for e in deriv_ends]
    if buffer_info is not None:
        bi, bf = buffer_info.get("i", {}), buffer_info.get("f", {})
        if bi.get("upwind", False):
            for t in range(ntypes):
                deriv_starts[t] = sorted(set(deriv_starts[t]) | set(range(1, bi["n"] + 1)), reverse=True)
        if bf.get("upwind", False):
            for t in range(ntypes):
                deriv_ends[t] = sorted(set(deriv_ends[t]) | set(n + 1 - k for k in range(1, bf["n"] + 1)))

    mL, nL = dl.shape
    mR, nR = dr.shape
    lhs_list, rhs_list = [], []
    for t in range(ntypes):
        L = lhs_base.copy()
        Rm = rhs_base.copy()
        for s in deriv_starts[t]:
            s0 = s - 1
            if s0 + max(mL, mR, nL, nR) > n:
                raise ValueError("boundary stencil starting at node %d does not fit in %d nodes" % (s, n))
            L[s0:s0 + mL, :] = 0
            Rm[s0:s0 + mR, :] = 0
            L[s0:s0 + mL, s0:s0 + nL] = dl
            Rm[s0:s0 + mR, s0:s0 + nR] = dr
        for e in deriv_ends[t]:
            if e - max(mL, mR, nL, nR) < 0:
                raise ValueError("boundary stencil ending at node %d does not fit" % e)
            L[e - mL:e, :] = 0
            Rm[e - mR:e, :] = 0
            L[e - mL:e, e - nL:e] = dl[::-1, ::-1]
            Rm[e - mR:e, e - nR:e] = invert * dr[::-1, ::-1]
        lhs_list.append(L)
        rhs_list.append(Rm)
    return lhs_list, rhs_list


def add_buffer_to_matrix(base_l, buf_l, base_r, buf_r, n, buffer_info):
    """Blend the buffer-zone scheme into the interior scheme (``makeMatrices.m:266-311``)."""
    ni = int(buffer_info["i"].get("n", 0))
    nf = int(buffer_info["f"].get("n", 0))
    nti = int(round(buffer_info["i"]["transition"] * ni)) if "transition" in buffer_info["i"] else ni
    ntf = int(round(buffer_info["f"]["transition"] * nf)) if "transition" in buffer_info["f"] else nf
    ni1, ni2 = ni - nti + 1, ni
    nf1 = n - nf + 1
    nf2 = nf1 + ntf - 1
    eta = np.ones(n)
    if ni > 0:
        eta[0:ni1] = 0
        eta[ni1 - 1:ni2] = 0.5 - 0.5 * np.cos(np.linspace(0, math.pi, ni2 - ni1 + 1))
    if nf > 0:
        eta[nf2 - 1:n] = 0
        eta[nf1 - 1:nf2] = 0.5 + 0.5 * np.cos(np.linspace(0, math.pi, nf2 - nf1 + 1))
    eta = np.sqrt(eta)
    new_l = [eta[:, None] * bl + (1 - eta)[:, None] * fl for bl, fl in zip(base_l, buf_l)]
    new_r = [eta[:, None] * br + (1 - eta)[:, None] * fr for br, fr in zip(base_r, buf_r)]
    return new_l, new_r


def apply_metric(lhs_list, X, periodic, fix_periodic_domain_size, xf, method="SL4"):
    """Scale LHS columns by dX/deta for stretched meshes (``makeMatrices.m:313-342``)."""
    X = np.asarray(X, dtype=np.float64).ravel()
    added = False
    if periodic and fix_periodic_domain_size and len(X) > 1:
        X = np.concatenate([X, [xf]])
        added = True
    n = len(X)
    if n == 1:
        return lhs_list
    cl, cr, dl, dr = finite_difference_coefficients(method)
    Lt, Rt = make_matrices_each_direction(cl, cr, dl, dr, [[1]], [[n]], n, None)
    dxdeta = np.linalg.solve(Lt[0], Rt[0] @ X)
    if added:
        dxdeta = dxdeta[:-1]
    return [L * dxdeta[None, :] for L in lhs_list]


# ---------------------------------------------------------------------------
# Thomas preparation
# ---------------------------------------------------------------------------

@dataclass
class DirectionMatrices:
    """The per-direction arrays ``matrices.F90`` declares (``writeFortranMatrices.m:73-110``).

    Shapes follow the Fortran allocations (column-major when flattened with order='F'):
    ``A,C: (N-1, nTypes)``, ``B: (N-periodic, nTypes)``, ``D: (N, nTypes)``,
    ``R: (N, 2*nRHS-1, nTypes)``; the ``f`` variants are the filter.
    """
    periodic: int
    nTypes: int
    A: np.ndarray
    B: np.ndarray
    C: np.ndarray
    D: np.ndarray
    R: np.ndarray
    nRHS: int
    Af: np.ndarray
    Bf: np.ndarray
    Cf: np.ndarray
    Df: np.ndarray
    Rf: np.ndarray
    nRHSf: int
    types: np.ndarray = field(default=None)      # per-line type map (1-based), 2-D
    blocks: np.ndarray = field(default=None)     # (nBlocks, 5) 1-based
    adj: list = field(default=None)              # transposed operators (adjoint_sets), or None

    def rounded(self):
        """Copy with every coefficient passed through the ``%.20f`` text format."""
        kw = dict(self.__dict__)
        for k in ("A", "B", "C", "D", "R", "Af", "Bf", "Cf", "Df", "Rf"):
            kw[k] = fortran_round(kw[k])
        return DirectionMatrices(**kw)


def _full_diag(M, k):
    """``fullDiag`` of ``prepareThomas.m:164-172``: element (r, r+k mod N) of each type."""
    N = M.shape[0]
    r = np.arange(N)
    return M[r, (r + k) % N, :]  # (N, nTypes)


def _rhs_diagonals(rhs_stack, filter_rule):
    N = rhs_stack.shape[0]
    diag = _full_diag(rhs_stack, 0)[:, None, :]
    nd = 1
    while True:
        nxt = _full_diag(rhs_stack, nd)
        prv = _full_diag(rhs_stack, -nd)
        if filter_rule:
            cont = (np.any(nxt) or np.any(prv)) and not (2 * nd - 1 > N)
        else:
            # prepareThomas.m:115 -- MATLAB precedence: any(next) || (any(prev) && ~(2n-1>N))
            cont = np.any(nxt) or (np.any(prv) and not (2 * nd - 1 > N))
            if nd > N:  # guard the wrap-around case the MATLAB loop never terminates on
                cont = False
        if cont:
            nd += 1
            diag = np.concatenate([prv[:, None, :], diag, nxt[:, None, :]], axis=1)
        else:
            break
    return diag, nd


def prepare_thomas(LHS, RHS, fLHS, fRHS, types):
    """Precompute the Thomas factors and RHS diagonals (``source/prepareThomas.m:1-162``).

    ``LHS``/``RHS``/``fLHS``/``fRHS`` are lists of dense N x N matrices (one per type).
    """
    is_periodic = LHS[0][-1, 0] != 0
    ntypes = int(np.max(types))
    N = LHS[0].shape[0]

    def diag(M, k):
        return np.diagonal(M, k).astype(np.float64).copy()

    A = np.zeros((max(N - 1, 0), ntypes)); B = np.zeros((N, ntypes)); C = np.zeros((max(N - 1, 0), ntypes))
    Af = np.zeros_like(A); Bf = np.zeros_like(B); Cf = np.zeros_like(C)
    D = np.zeros((N, ntypes)); Df = np.zeros((N, ntypes))
    for t in range(ntypes):
        A[:, t] = diag(LHS[t], -1); B[:, t] = diag(LHS[t], 0); C[:, t] = diag(LHS[t], 1)
        Af[:, t] = diag(fLHS[t], -1); Bf[:, t] = diag(fLHS[t], 0); Cf[:, t] = diag(fLHS[t], 1)

    if is_periodic:
        A1 = np.array([LHS[t][0, -1] for t in range(ntypes)])
        Cn = np.array([LHS[t][-1, 0] for t in range(ntypes)])
        A1f = np.array([fLHS[t][0, -1] for t in range(ntypes)])
        Cnf = np.array([fLHS[t][-1, 0] for t in range(ntypes)])
        A = A[1:]; B = B[1:]; C = C[1:]
        Af = Af[1:]; Bf = Bf[1:]; Cf = Cf[1:]
        for i in range(N - 2):
            C[i] = C[i] / B[i]
            B[i + 1] = B[i + 1] - A[i] * C[i]
            Cf[i] = Cf[i] / Bf[i]
            Bf[i + 1] = Bf[i + 1] - Af[i] * Cf[i]
        B = 1.0 / B
        Bf = 1.0 / Bf
        A = np.vstack([A1[None, :], A]); Af = np.vstack([A1f[None, :], Af])
        C = np.vstack([Cn[None, :], C]); Cf = np.vstack([Cnf[None, :], Cf])
        for t in range(ntypes):
            D[:, t] = np.linalg.inv(LHS[t])[0, :]
            Df[:, t] = np.linalg.inv(fLHS[t])[0, :]
    else:
        for i in range(N - 1):
            C[i] = C[i] / B[i]
            B[i + 1] = B[i + 1] - A[i] * C[i]
            Cf[i] = Cf[i] / Bf[i]
            Bf[i + 1] = Bf[i + 1] - Af[i] * Cf[i]
        B = 1.0 / B
        Bf = 1.0 / Bf

    rhs_stack = np.stack([np.asarray(RHS[t], dtype=np.float64) for t in range(ntypes)], axis=2)
    frhs_stack = np.stack([np.asarray(fRHS[t], dtype=np.float64) for t in range(ntypes)], axis=2)
    R, nR = _rhs_diagonals(rhs_stack, filter_rule=False)
    Rf, nRf = _rhs_diagonals(frhs_stack, filter_rule=True)
    return DirectionMatrices(periodic=int(bool(is_periodic)), nTypes=ntypes, A=A, B=B, C=C, D=D, R=R, nRHS=nR,
                             Af=Af, Bf=Bf, Cf=Cf, Df=Df, Rf=Rf, nRHSf=nRf,
                             types=np.asarray(types))


@dataclass
class OperatorSet:
    """One compact line operator x = LHS^-1 (R f) in the factored form the C-ABI takes
    (the arrays of one ``gatt_set_matrices`` call)."""
    periodic: int
    nTypes: int
    A: np.ndarray
    B: np.ndarray
    C: np.ndarray
    D: np.ndarray
    R: np.ndarray
    nRHS: int


def _identity_factors(N, ntypes, periodic):
    """Thomas factors of the identity LHS (cyclic form when periodic: D = e_1, no corners)."""
    if periodic:
        D = np.zeros((N, ntypes))
        D[0, :] = 1.0
        return np.zeros((N - 1, ntypes)), np.ones((N - 1, ntypes)), np.zeros((N - 1, ntypes)), D
    return np.zeros((N - 1, ntypes)), np.ones((N, ntypes)), np.zeros((N - 1, ntypes)), np.zeros((N, ntypes))


def _identity_band(N, ntypes):
    R = np.zeros((N, 3, ntypes))
    R[:, 1, :] = 1.0
    return R


def adjoint_sets(LHS, RHS, fLHS, fRHS, types):
    """Transposes of the derivative and filter line operators, each as two operators the
    forward kernels run: L^T = (LHS^-1 R)^T = R^T (LHS^T)^-1 is a solve with LHS^T and an
    identity band, then a band product with R^T and an identity LHS.  Returns
    [deriv LHS^T solve, deriv R^T band, filter LHS^T solve, filter R^T band]
    (``gatt_set_matrices`` kinds 2..5)."""
    ntypes = int(np.max(types))
    N = LHS[0].shape[0]
    eye = [np.eye(N) for _ in range(ntypes)]
    lt = prepare_thomas([m.T.copy() for m in LHS], eye, [m.T.copy() for m in fLHS], eye, types)
    per = lt.periodic
    out = []
    for A, B, C, D, Rt in ((lt.A, lt.B, lt.C, lt.D, RHS), (lt.Af, lt.Bf, lt.Cf, lt.Df, fRHS)):
        out.append(OperatorSet(per, ntypes, A, B, C, D if per else np.zeros((N, ntypes)), _identity_band(N, ntypes), 2))
        stack = np.stack([np.asarray(Rt[t], dtype=np.float64).T for t in range(ntypes)], axis=2)
        band, nd = _rhs_diagonals(stack, filter_rule=True)
        if nd < 2:
            band = np.concatenate([np.zeros((N, 1, ntypes)), band, np.zeros((N, 1, ntypes))], axis=1)
            nd = 2
        iA, iB, iC, iD = _identity_factors(N, ntypes, per)
        out.append(OperatorSet(per, ntypes, iA, iB, iC, iD, band, nd))
    return out


# ---------------------------------------------------------------------------
# Blocks and type maps
# ---------------------------------------------------------------------------

def get_domain_slices(n, p):
    """2DECOMP slice limits (1-based, shape (2, p)); ``source/getDomainSlices.m:1-24``."""
    if n == 1:
        return np.array([[1], [1]])
    base = n // p
    nceil = n - base * p
    npts = np.full(p, base)
    if nceil > 0:
        npts[p - nceil:] = base + 1
    ends = np.cumsum(npts)
    starts = np.concatenate([[1], ends[:-1] + 1])
    return np.vstack([starts, ends])


def get_matrix_type_blocks(type_map, p_row=1, p_col=1, max_block_size=128):
    """Block lists ``[type, j1, j2, k1, k2]`` per rank (``getMatrixTypeBlocks.m:1-102``)."""
    type_map = np.asarray(type_map)
    if type_map.ndim == 1:
        type_map = type_map[:, None]
    J, K = type_map.shape
    all_blocks = []
    for k in range(1, K + 1):
        col = type_map[:, k - 1]
        starts = np.concatenate([[1], np.nonzero(np.diff(col) != 0)[0] + 2])
        ends = np.concatenate([starts[1:] - 1, [J]])
        for s, e in zip(starts, ends):
            all_blocks.append([int(col[s - 1]), int(s), int(e), k, k])
    # merge along k
    i = 0
    while i < len(all_blocks) - 1:
        j = i + 1
        while j < len(all_blocks):
            bi, bj = all_blocks[i], all_blocks[j]
            if bi[0:3] == bj[0:3] and bi[4] + 1 == bj[3]:
                bi[4] = bj[4]
                del all_blocks[j]
            else:
                j += 1
        i += 1
    sy = get_domain_slices(J, p_row)
    sz = get_domain_slices(K, p_col)
    blocks = [None] * (p_row * p_col)
    for jr in range(p_row):
        for kc in range(p_col):
            nproc = kc + jr * p_col
            Ji, Jf = sy[0, jr], sy[1, jr]
            Ki, Kf = sz[0, kc], sz[1, kc]
            bl = [list(b) for b in all_blocks if not (b[1] > Jf or b[2] < Ji or b[3] > Kf or b[4] < Ki)]
            for b in bl:
                b[1] = max(b[1], Ji); b[2] = min(b[2], Jf); b[3] = max(b[3], Ki); b[4] = min(b[4], Kf)
            blocks[nproc] = bl
    if not math.isinf(max_block_size):
        for nproc in range(p_row * p_col):
            new = []
            for b in blocks[nproc]:
                isz = b[2] - b[1] + 1
                jsz = b[4] - b[3] + 1
                nsl = int(math.ceil(isz * jsz / max_block_size))
                if nsl == 1:
                    new.append(list(b))
                else:
                    isl = int(math.ceil(nsl / jsz))
                    jsl = int(math.floor(nsl / isl))
                    ii = get_domain_slices(isz, isl).T + b[1] - 1
                    jj = get_domain_slices(jsz, jsl).T + b[3] - 1
                    for a in range(isl):
                        for c in range(jsl):
                            new.append([b[0], int(ii[a, 0]), int(ii[a, 1]), int(jj[c, 0]), int(jj[c, 1])])
            blocks[nproc] = new
    return [np.array(b, dtype=np.int32).reshape(-1, 5) for b in blocks]


def _regions_one_direction(fr_lines, n_along, periodic):
    """Shared body of the three direction sections of ``findDerivativeRegions.m``.

    ``fr_lines`` has shape (L1, L2, n_along): the flow-region mask of every line.
    Returns (type_map (L1, L2) 1-based, starts list, ends list).
    """
    L1, L2, _ = fr_lines.shape
    rows = fr_lines.reshape(-1, n_along).astype(np.int8)
    C = np.unique(rows, axis=0)  # sorted unique rows, as MATLAB unique(...,'rows','sorted')
    lookup = {C[i].tobytes(): i + 1 for i in range(C.shape[0])}
    tmap = np.array([lookup[r.tobytes()] for r in rows], dtype=np.int64).reshape(L1, L2)
    starts, ends = [], []
    removed = 0
    for i in range(C.shape[0]):
        row = C[i].astype(np.int64)
        idx = i + 1 - removed
        if np.any(row != 0):
            d = np.diff(row)
            if periodic:
                starts.append(sorted(set((np.nonzero(d == 1)[0] + 1).tolist())))
                ends.append(sorted(set((np.nonzero(d == -1)[0] + 2).tolist())))
            else:
                starts.append(sorted(set([1] + (np.nonzero(d == 1)[0] + 1).tolist())))
                ends.append(sorted(set((np.nonzero(d == -1)[0] + 2).tolist() + [n_along])))
        else:
            tmap[tmap == idx] = 0
            tmap[tmap > idx] -= 1
            removed += 1
    if np.any(tmap > 0):
        tmap[tmap == 0] = tmap.max()
    return tmap, starts, ends


def _apply_break_points(tmap, starts, ends, break_points):
    """Cut lines at break points (``findDerivativeRegions.m:45-60``, same for y and z).

    Each break point row is ``[node, a_i, a_f, b_i, b_f]`` (1-based): the lines
    ``tmap[a_i-1:a_f, b_i-1:b_f]`` get, per matrix type present there, a new type whose
    boundary stencils are the old ones plus an end stencil at ``node`` and a start stencil
    at ``node + 1`` -- the derivative and filter stencils do not reach across the break.
    The new stencils are appended after the old ones, as the reference appends them.
    """
    for bp in np.atleast_2d(np.asarray(break_points, dtype=np.int64)):
        node, ai, af, bi, bf = (int(v) for v in bp)
        box = (slice(ai - 1, af), slice(bi - 1, bf))
        for t in np.unique(tmap[box]):
            t_new = int(tmap.max()) + 1
            starts.append(list(starts[t - 1]) + [node + 1])
            ends.append(list(ends[t - 1]) + [node])
            sub = tmap[box]
            sub[sub == t] = t_new
            tmap[box] = sub
    return tmap, starts, ends


def find_derivative_regions(flow_region, periodic=(False, False, False), break_points=(None, None, None)):
    """Per-line matrix types from the flow-region mask (``source/findDerivativeRegions.m``).

    ``flow_region`` is a boolean (nx, ny, nz) array.  Returns a dict with
    ``typeMapX (ny,nz)``, ``typeMapY (nx,nz)``, ``typeMapZ (nx,ny)`` and the
    start/end lists per type for each direction.  ``break_points[d]`` restates
    ``mesh.x/y/z.breakPoint`` (rows ``[node, line box]``, see :func:`_apply_break_points`).
    """
    fr = np.asarray(flow_region, dtype=bool)
    nx, ny, nz = fr.shape
    tx, sx, ex = _regions_one_direction(np.transpose(fr, (1, 2, 0)), nx, periodic[0])
    ty, sy, ey = _regions_one_direction(np.transpose(fr, (0, 2, 1)), ny, periodic[1])
    tz, sz, ez = _regions_one_direction(fr, nz, periodic[2])
    for bp, (tm, st, en) in zip(break_points, ((tx, sx, ex), (ty, sy, ey), (tz, sz, ez))):
        if bp is not None and len(bp):
            _apply_break_points(tm, st, en, bp)
    return dict(typeMapX=tx, typeMapY=ty, typeMapZ=tz,
                derivStartsX=sx, derivEndsX=ex, derivStartsY=sy, derivEndsY=ey,
                derivStartsZ=sz, derivEndsZ=ez)
