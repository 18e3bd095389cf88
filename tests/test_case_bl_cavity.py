"""The boundary layer over a cavity (config 3) as the reference's preprocessing builds it.

Known answers for the pieces of ``boundaryLayerIsothermal.m`` / ``generateMesh.m`` /
``findDerivativeRegions.m`` / ``generateInitialFlow.m`` that this case restates, and a
bounded run on the CPU oracle that shows the restated case is stable from the Blasius start.
"""
import numpy as np
import pytest

from gatt_dns_b200 import case as cs
from gatt_dns_b200 import matrices as mx


def test_break_point_adds_a_type_cut_at_the_node():
    # 2 rows of 24 nodes, all fluid; break row 2 between nodes 10 and 11 (1-based)
    fr = np.ones((24, 2, 1), dtype=bool)
    reg = mx.find_derivative_regions(fr, (False, False, False), break_points=([[10, 2, 2, 1, 1]], None, None))
    assert reg["typeMapX"][:, 0].tolist() == [1, 2]
    assert reg["derivStartsX"][1] == [1, 11]
    assert reg["derivEndsX"][1] == [24, 10]
    # the cut operator: a derivative on each side uses only that side's values
    cl, cr, dl, dr = mx.finite_difference_coefficients("SL4")
    L, R = mx.make_matrices_each_direction(cl, cr, dl, dr, reg["derivStartsX"], reg["derivEndsX"], 24)
    D = np.linalg.solve(L[1], R[1])
    assert np.max(np.abs(D[:10, 10:])) < 1e-14 and np.max(np.abs(D[10:, :10])) < 1e-14
    x = np.arange(24.0)
    f = np.where(x < 10, 2.0 * x, 100.0 - 3.0 * x)  # a jump between the two sides
    assert np.allclose(D @ f, np.where(x < 10, 2.0, -3.0), atol=1e-12)
    # without the break the jump leaks into both sides
    D0 = np.linalg.solve(L[0], R[0])
    assert not np.allclose(D0 @ f, np.where(x < 10, 2.0, -3.0), atol=1e-3)


def test_attractor_mesh_and_fixed_points():
    Y = cs.generate_mesh(-1.0, 4.0, 120, mtype="attractors", attractor_regions=[(-2.0, -0.1, 0.1, 0.7, 12.0)],
                         fix_points=(-1.0, 0.0))
    assert Y[0] == -1.0 and Y[-1] == pytest.approx(4.0, abs=1e-12)
    assert np.any(Y == 0.0)
    d = np.diff(Y)
    assert np.all(d > 0)
    j = int(np.nonzero(Y == 0.0)[0][0])
    # refined inside the attractor region, smooth through the fixed point
    assert d[j] < 0.4 * d[-1]
    assert np.max(np.abs(d[j - 3:j + 3] / d[j - 4:j + 2] - 1)) < 0.05


def test_wall_move_free_slip_and_break_point():
    c = cs.boundary_layer_cavity(nx=120, ny=60, buffers=((6, 5), (0, 8)))
    X, Y = c.X, c.Y
    first_pos = int(np.nonzero(X >= 0)[0][0]) + 1
    last_neg = first_pos - 1
    j_plate = int(np.nonzero(Y == 0.0)[0][0]) + 1
    assert X[first_pos - 1] == 0.0
    # the free-slip wall: the last up wall; u (and w) Neumann on it, pressure Neumann too
    pn = c.bc.ind[("n", "P")].tolist()
    assert [1, last_neg, j_plate, j_plate, 1, 1] == pn[-1]
    assert c.bc.ind[("n", "U")].tolist() == [[1, last_neg, j_plate, j_plate, 1, 1]]
    assert c.bc.ind[("n", "W")].tolist() == [[1, last_neg, j_plate, j_plate, 1, 1]]
    # every other up wall starts at the leading edge or downstream of it
    for w in pn:
        assert w[0] >= first_pos or w == pn[-1] or w[2] != w[3] or c.bc.dirs[("n", "P")][pn.index(w)] != 3
    # the plate row's x lines carry their own matrix type
    m = c.mats[0]
    blk = np.asarray(m.blocks)
    plate = [b for b in blk if b[1] <= j_plate <= b[2]]
    assert len(plate) == 1 and plate[0][0] == m.nTypes


def test_blasius_start():
    c = cs.boundary_layer_cavity(nx=120, ny=60, buffers=((6, 5), (0, 8)))
    f = cs.blasius_flow(c)
    U = f["U"][:, :, 0]
    assert np.all(U[c.X <= 0] == 1.0)
    assert np.all(U[np.ix_(c.X > 0, c.Y < 0)] == 0.0)
    assert np.all(f["V"] == 0.0) and np.all(f["R"] == 1.0) and np.all(f["E"] == c.E0)
    i = int(np.argmin(np.abs(c.X - 3.0)))
    theta = 0.664 * np.sqrt(c.X[i] / c.Re)
    eta = c.Y * 0.664155332943009 / theta
    k = int(np.argmin(np.abs(eta - 2.0)))
    assert 0.5 < U[i, k] < 0.75  # u(eta = 2) ~ 0.63 for the Blasius profile
    assert np.all(U <= 1.0)


def test_bl_cavity_runs_stably_on_the_oracle(oracle_lib):
    """The restated case from the Blasius start: 150 steps at CFL 0.5 stay finite and the
    residual (max-change per step) decays."""
    import oracle
    c = cs.boundary_layer_cavity(nx=160, ny=80, buffers=((8, 6), (0, 10)))
    o = oracle.Oracle(c)
    f = o.apply_bound_cond(cs.blasius_flow(c), 0.0)
    st = o.new_state(f)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    hist = []
    for k in range(150):
        mc = np.asarray(o.step(st, k * dt, dt))
        assert np.all(np.isfinite(mc)), k
        hist.append(float(np.max(mc)))
    assert hist[-1] < 0.5 * max(hist[:20])
