"""Round trip through the generated-include text format (matrices.F90, boundaryInfo.F90,
parameters.F90, runDisturbances.F90) of the reference preprocessing."""
import numpy as np

from gatt_dns_b200 import case as cs
from gatt_dns_b200 import fortran_io as fio


def _same_mats(a, b):
    for k in ("A", "B", "C", "R", "Af", "Bf", "Cf", "Rf"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    if a.periodic:
        assert np.array_equal(a.D, b.D) and np.array_equal(a.Df, b.Df)
    assert (a.periodic, a.nRHS, a.nRHSf, a.nTypes) == (b.periodic, b.nRHS, b.nRHSf, b.nTypes)
    assert np.array_equal(np.asarray(a.blocks), np.asarray(b.blocks))


def test_case_round_trip(tmp_path):
    c = cs.lid_driven(n=20)
    fio.write_parameters_f90(c, tmp_path / "parameters.F90")
    fio.write_matrices_f90(c, tmp_path / "matrices.F90")
    fio.write_boundary_info_f90(c, tmp_path / "boundaryInfo.F90")
    fio.write_run_disturbances_f90(c, tmp_path / "runDisturbances.F90")
    r = fio.case_from_fortran_dir(str(tmp_path))
    assert (r.nx, r.ny, r.nz) == (c.nx, c.ny, c.nz)
    assert r.Re == c.Re and r.gamma == c.gamma
    for a, b in zip(c.mats, r.mats):
        if a is None:
            assert b is None
        else:
            _same_mats(a, b)
    for key, v in c.bc.ind.items():
        assert np.array_equal(r.bc.ind[key], v), key
    for key, v in c.bc.val.items():
        assert np.array_equal(r.bc.val[key], v)
    assert np.array_equal(r.bc.neumannCoeffs, c.bc.neumannCoeffs)
    d0, d1 = c.bc.disturbances[0], r.bc.disturbances[0]
    assert d1["type"] == "lidDrivenMovement" and d1["var"] == "U"
    assert np.array_equal(d0["ind"], d1["ind"]) and np.array_equal(d0["X"], d1["X"]) and d1["par"] == [1.0]


def test_periodic_and_corner_round_trip(tmp_path):
    c = cs.cavity_channel(nx=24, ny=20, nz=4, adiabatic_corners=True)
    fio.write_parameters_f90(c, tmp_path / "parameters.F90")
    fio.write_matrices_f90(c, tmp_path / "matrices.F90")
    fio.write_boundary_info_f90(c, tmp_path / "boundaryInfo.F90")
    r = fio.case_from_fortran_dir(str(tmp_path))
    for a, b in zip(c.mats, r.mats):
        _same_mats(a, b)
    assert np.array_equal(r.bc.cL, c.bc.cL) and np.array_equal(r.bc.cD, c.bc.cD)
    assert np.array_equal(r.bc.cAdiabatic, c.bc.cAdiabatic)


def test_forcings_and_time_stepping_round_trip(tmp_path):
    """runForcings3D.F90 (turbulenceGenerator, pressureGradient) and parameters.F90's
    timeStepping through the emitter and the reader; the golden vectors run the reference
    on these same emitted files (tests/golden/make_reference_golden.py)."""
    import dataclasses
    c = cs.turbulence_box(nxyz=(16, 12, 8))
    c.forcings.append({"type": "pressureGradient", "ind": [2, 11, 1, 10, 3, 6], "par": [0.125]})
    c = dataclasses.replace(c, time_stepping=3)
    fio.write_parameters_f90(c, tmp_path / "parameters.F90")
    fio.write_matrices_f90(c, tmp_path / "matrices.F90")
    fio.write_boundary_info_f90(c, tmp_path / "boundaryInfo.F90")
    fio.write_run_forcings_f90(c, tmp_path / "runForcings3D.F90")
    (tmp_path / "runForcings2D.F90").write_text("")
    r = fio.case_from_fortran_dir(str(tmp_path))
    assert r.time_stepping == 3
    assert len(r.forcings) == 2
    for a, b in zip(c.forcings, r.forcings):
        assert a["type"] == b["type"] and np.array_equal(np.asarray(a["ind"]), b["ind"])
        assert np.array_equal(np.asarray(a["par"], dtype=float), np.asarray(b["par"], dtype=float))
