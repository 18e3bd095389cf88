"""Coefficient emitter (numpy restatement of the MATLAB preprocessing): known answers.

The reference ships no tests or golden vectors, so these pin the restatement with
closed-form properties of the schemes it emits:
* SL4 compact derivative: order conditions and the design point w = 1.8
  (finiteDifferenceCoefficients.m:95-112);
* Gaitonde 10th-order filter: T(0) = 1, T(pi) = 0 (spatialFilterCoefficients.m:5-7);
* prepareThomas.m: the precomputed Thomas factors and the cyclic D row reproduce the
  dense solve of the LHS matrix.
"""
import math

import numpy as np
import pytest

from gatt_dns_b200 import matrices as mx


def test_sl4_order_and_design_point():
    cl, cr, dl, dr = mx.finite_difference_coefficients("SL4")
    alpha, a, b = cl[1], cr[1], cr[2]
    # 2nd and 4th order Taylor conditions: 2a + 4b = 1 + 2 alpha ; 2a + 16b = 6 alpha  (times 1/3!)
    assert 2 * a + 4 * b == pytest.approx(1 + 2 * alpha, abs=1e-14)
    assert (2 * a + 16 * b) / 6 == pytest.approx(alpha, abs=1e-14)
    w = 1.8
    kp = (2 * a * math.sin(w) + 2 * b * math.sin(2 * w)) / (1 + 2 * alpha * math.cos(w))
    assert kp == pytest.approx(w, abs=1e-13)


def test_sl6_and_explicit_stencils_are_consistent():
    for m in ("SL6", "SL6O3", "EX2", "EX4"):
        cl, cr, dl, dr = mx.finite_difference_coefficients(m)
        # derivative of a linear function: sum of RHS weights * offset == LHS sum (interior)
        lhs_sum = cl[0] + 2 * sum(cl[1:])
        rhs_moment = 2 * sum(cr[i] * i for i in range(1, len(cr)))
        assert rhs_moment == pytest.approx(lhs_sum, rel=1e-12), m
        # boundary rows are exact for linear functions: sum(dr) == 0, sum(dr * offset) == sum(dl)
        for r in range(dl.shape[0]):
            assert np.sum(dr[r]) == pytest.approx(0.0, abs=1e-12)
            assert np.sum(dr[r] * np.arange(dr.shape[1])) == pytest.approx(np.sum(dl[r]), rel=1e-12)


@pytest.mark.parametrize("alpha", [0.0, 0.3, 0.49])
def test_filter_transfer_function(alpha):
    lhs, rhs, _, _ = mx.spatial_filter_coefficients(alpha, "decentered")

    def T(w):
        num = rhs[0] + 2 * sum(rhs[n] * math.cos(n * w) for n in range(1, 6))
        return num / (1 + 2 * alpha * math.cos(w))

    assert T(0.0) == pytest.approx(1.0, abs=1e-14)
    assert T(math.pi) == pytest.approx(0.0, abs=1e-14)
    # 10th order: T(w) = 1 - O(w^10)
    assert abs(T(0.1) - 1) < 1e-10


def test_filter_boundary_rows_preserve_constants():
    alpha = 0.4
    for borders in ("decentered", "reducedOrder", "off"):
        _, _, dl, dr = mx.spatial_filter_coefficients(alpha, borders)
        for r in range(dr.shape[0]):
            # rows below the decentered LHS rows keep the centered LHS [alpha 1 alpha]
            lhs_sum = np.sum(dl[r]) if dl.shape[0] > r else 1 + 2 * alpha
            assert np.sum(dr[r]) == pytest.approx(lhs_sum, abs=1e-13), borders


def _dense_solve(L, R, f):
    return np.linalg.solve(L, R @ f)


@pytest.mark.parametrize("periodic", [False, True])
def test_prepare_thomas_matches_dense_solve(periodic):
    n = 24
    cl, cr, dl, dr = mx.finite_difference_coefficients("SL4")
    starts, ends = ([[]], [[]]) if periodic else ([[1]], [[n]])
    L, R = mx.make_matrices_each_direction(cl, cr, dl, dr, starts, ends, n)
    fl, fr, fdl, fdr = mx.spatial_filter_coefficients(0.45, "decentered")
    fL, fR = mx.make_matrices_each_direction(fl, fr, fdl, fdr, starts, ends, n)
    m = mx.prepare_thomas(L, R, fL, fR, np.ones((3, 1), dtype=int))
    assert m.periodic == int(periodic)
    assert m.nRHS == (3 if periodic else 4)
    # the decentered filter's first boundary row reaches 10 nodes to the right
    assert m.nRHSf == (6 if periodic else 11)
    rng = np.random.default_rng(0)
    f = rng.standard_normal(n)
    for (A, B, C, D, Rd, nR, Lm, Rm) in ((m.A, m.B, m.C, m.D, m.R, m.nRHS, L[0], R[0]),
                                         (m.Af, m.Bf, m.Cf, m.Df, m.Rf, m.nRHSf, fL[0], fR[0])):
        rhs = np.array([sum(Rd[i, nR - 1 + l, 0] * f[(i + l) % n] for l in range(-(nR - 1), nR)) for i in range(n)])
        assert np.allclose(rhs, Rm @ f, rtol=0, atol=1e-13)
        x = rhs.copy()
        if not periodic:
            x[0] *= B[0, 0]
            for i in range(n - 1):
                x[i + 1] = (x[i + 1] - A[i, 0] * x[i]) * B[i + 1, 0]
            for i in range(n - 2, -1, -1):
                x[i] -= C[i, 0] * x[i + 1]
        else:
            x0 = np.dot(D[:, 0], x)
            x[0] = x0
            x[1] -= A[0, 0] * x0
            x[n - 1] -= C[0, 0] * x0
            x[1] *= B[0, 0]
            for i in range(1, n - 1):
                x[i + 1] = (x[i + 1] - A[i, 0] * x[i]) * B[i, 0]
            for i in range(n - 2, 0, -1):
                x[i] -= C[i, 0] * x[i + 1]
        ref = _dense_solve(Lm, Rm, f)
        assert np.max(np.abs(x - ref)) < 1e-12 * max(1.0, np.max(np.abs(ref)))


def test_fortran_round_is_idempotent_and_close():
    rng = np.random.default_rng(1)
    x = rng.standard_normal(1000) * 10.0 ** rng.integers(-6, 3, 1000)
    r = mx.fortran_round(x)
    assert np.array_equal(mx.fortran_round(r), r)
    assert np.all(np.abs(r - x) <= 1e-20 + 1e-15 * np.abs(x))


def test_matrix_type_blocks_cover_every_line_once():
    tmap = np.ones((300, 4), dtype=int)
    tmap[100:180, 1:3] = 2
    blocks = mx.get_matrix_type_blocks(tmap, 1, 1)[0]
    seen = np.zeros_like(tmap)
    for t, a1, a2, b1, b2 in blocks:
        assert (a2 - a1 + 1) * (b2 - b1 + 1) <= 128
        seen[a1 - 1:a2, b1 - 1:b2] += 1
        assert np.all(tmap[a1 - 1:a2, b1 - 1:b2] == t)
    assert np.all(seen == 1)


def test_domain_slices_match_2decomp_rule():
    s = mx.get_domain_slices(10, 3)
    assert s.tolist() == [[1, 4, 7], [3, 6, 10]]
    assert mx.get_domain_slices(1, 4).tolist() == [[1], [1]]


def test_derivative_regions_of_a_cavity():
    fr = np.ones((12, 10, 1), dtype=bool)
    fr[:, 0, :] = False
    fr[:, -1, :] = False
    fr[0:4, 0:4, :] = False
    reg = mx.find_derivative_regions(fr, (False, False, True))
    # y lines: two geometries (through the solid block, and clear) -> two types
    assert len(reg["derivStartsY"]) == 2
    assert set(np.unique(reg["typeMapY"])) == {1, 2}
    # x lines: the fully solid row j=1 maps to the largest type
    assert reg["typeMapX"][0, 0] == reg["typeMapX"].max()


def _apply_factored(A, B, C, D, R, nR, periodic, t, f):
    """One line through a factored operator, in the kernels' row semantics (numpy)."""
    N = f.size
    rhs = np.zeros(N)
    for i in range(N):
        for l in range(2 * nR - 1):
            rhs[i] += R[i, l, t] * f[(i + l - (nR - 1)) % N]
    x = np.zeros(N)
    if periodic:
        x1 = D[:, t] @ rhs
        rhs[1] -= A[0, t] * x1
        rhs[N - 1] -= C[0, t] * x1
        y = 0.0
        for r in range(1, N):
            y = (rhs[r] - (A[r - 1, t] if r >= 2 else 0.0) * y) * B[r - 1, t]
            x[r] = y
        xp = 0.0
        for r in range(N - 1, 0, -1):
            xp = x[r] - (C[r, t] if r <= N - 2 else 0.0) * xp
            x[r] = xp
        x[0] = x1
    else:
        y = 0.0
        for r in range(N):
            y = (rhs[r] - (A[r - 1, t] if r >= 1 else 0.0) * y) * B[r, t]
            x[r] = y
        xp = 0.0
        for r in range(N - 1, -1, -1):
            xp = x[r] - (C[r, t] if r <= N - 2 else 0.0) * xp
            x[r] = xp
    return x


@pytest.mark.parametrize("which", ["periodic", "walls"])
def test_adjoint_sets_are_transposes(which):
    """Kinds 2+3 (and 4+5) applied in turn are the transposes of the derivative (filter)."""
    from gatt_dns_b200 import case as cs
    c = cs.periodic_box(n=12) if which == "periodic" else cs.lid_driven(n=14)
    m = c.mats[0]
    N = c.nx
    fwd = [(m.A, m.B, m.C, m.D, m.R, m.nRHS), (m.Af, m.Bf, m.Cf, m.Df, m.Rf, m.nRHSf)]
    for kind in range(2):
        Lf = np.stack([_apply_factored(*fwd[kind], m.periodic, 0, e) for e in np.eye(N)], axis=1)
        s1, s2 = m.adj[2 * kind], m.adj[2 * kind + 1]
        Lt = np.stack([_apply_factored(s2.A, s2.B, s2.C, s2.D, s2.R, s2.nRHS, s2.periodic, 0,
                                       _apply_factored(s1.A, s1.B, s1.C, s1.D, s1.R, s1.nRHS, s1.periodic, 0, e))
                       for e in np.eye(N)], axis=1)
        assert np.max(np.abs(Lt - Lf.T)) < 1e-12 * np.max(np.abs(Lf)), (which, kind)
