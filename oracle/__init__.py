"""CPU oracle -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over ``oracle/liboracle.so``, the plain-C restatement of the reference
Fortran hot path (``source/Fortran/derivs.F90``, ``nseq.F90``, ``timeIntegration.F90``,
``main.F90:357-465``).  Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may use it, and only as the checker or the timed CPU baseline.

Parity status: pinned to the reference's own Fortran by golden vectors
(``tests/golden/reference_*.npz``, made by ``tests/golden/make_reference_golden.py``, which
runs the unmodified ``derivs.F90``, ``nseq.F90`` and ``timeIntegration.F90`` through a
Fortran-subset translator: the reference cannot be compiled here), and by known-answer tests
(spectral accuracy on trigonometric fields, filter transfer function, conservation).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "liboracle.so")

_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)


class _Dir(ctypes.Structure):
    _fields_ = [("periodic", ctypes.c_int), ("nR", ctypes.c_int), ("nTypes", ctypes.c_int), ("N", ctypes.c_int),
                ("A", _pd), ("B", _pd), ("C", _pd), ("D", _pd), ("R", _pd),
                ("nBlocks", ctypes.c_int), ("blocks", _pi)]


class _Case(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("Re", ctypes.c_double), ("Ma", ctypes.c_double), ("Pr", ctypes.c_double),
                ("gamma", ctypes.c_double), ("T0", ctypes.c_double),
                ("dmat", _Dir * 3), ("fmat", _Dir * 3),
                ("filterDir", ctypes.c_int * 3), ("filterCharTime", ctypes.c_double),
                ("neumannLength", ctypes.c_int), ("neumann2Length", ctypes.c_int),
                ("neumannCoeffs", _pd), ("neumann2Coeffs", _pd),
                ("nbc", (ctypes.c_int * 5) * 3), ("ibc", (_pi * 5) * 3), ("vbc", _pd * 5), ("dbc", (_pi * 5) * 3),
                ("cN", ctypes.c_int), ("cL", _pi), ("cD", _pi), ("cAdiabatic", _pi),
                ("nDist", ctypes.c_int), ("distType", _pi), ("distVar", _pi), ("distInd", _pi),
                ("distX", _pd), ("distXoff", _pi), ("distPar", _pd),
                ("sfdType", ctypes.c_int), ("sfdDelta", ctypes.c_double), ("sfdChi", _pd),
                ("timeStepping", ctypes.c_int),
                ("nForce", ctypes.c_int), ("forceType", _pi), ("forceInd", _pi), ("forcePar", _pd),
                ("distPar2", _pd), ("holdSave", _pd), ("holdOff", ctypes.POINTER(ctypes.c_long)),
                ("holdSaved", _pi)]


def build():
    """Compile liboracle.so with its Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = ctypes.CDLL(LIB)
        cp = ctypes.POINTER(_Case)
        lib.orc_solve.argtypes = [cp, ctypes.c_int, ctypes.c_int, _pd, _pd]
        lib.orc_nseq.argtypes = [cp] + [_pd] * 10
        lib.orc_apply_bc.argtypes = [cp] + [_pd] * 5 + [ctypes.c_double]
        lib.orc_rk4.argtypes = [cp] + [_pd] * 10 + [ctypes.c_double, ctypes.c_double]
        lib.orc_filters.argtypes = [cp] + [_pd] * 5 + [ctypes.c_double]
        lib.orc_step.argtypes = [cp] + [_pd] * 11 + [ctypes.c_double, ctypes.c_double, _pd]
        lib.orc_set_threads.argtypes = [ctypes.c_int]
        lib.orc_num_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def _f(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


class Oracle:
    """The reference hot path on the CPU for a :class:`gatt_dns_b200.case.Case`."""

    VARS = ("U", "V", "W", "P", "E")

    def __init__(self, case, threads=None):
        self.lib = load()
        if threads:
            self.lib.orc_set_threads(int(threads))
        self.case = case
        self._keep = []
        c = _Case()
        c.nx, c.ny, c.nz = case.nx, case.ny, case.nz
        c.Re, c.Ma, c.Pr, c.gamma, c.T0 = case.Re, case.Ma, case.Pr, case.gamma, case.T0
        for d, m in enumerate(case.mats):
            if m is None:
                continue
            for kind, tgt in ((0, c.dmat), (1, c.fmat)):
                A, B, C, D, R, nR = ((m.A, m.B, m.C, m.D, m.R, m.nRHS) if kind == 0
                                     else (m.Af, m.Bf, m.Cf, m.Df, m.Rf, m.nRHSf))
                A, B, C, D, R = (self._hold(_f(x)) for x in (A, B, C, D, R))
                blocks = self._hold(np.asfortranarray(np.asarray(m.blocks, dtype=np.int32)))
                tgt[d].periodic, tgt[d].nR, tgt[d].nTypes, tgt[d].N = m.periodic, nR, m.nTypes, (case.nx, case.ny, case.nz)[d]
                tgt[d].A, tgt[d].B, tgt[d].C, tgt[d].D, tgt[d].R = (x.ctypes.data_as(_pd) for x in (A, B, C, D, R))
                tgt[d].nBlocks, tgt[d].blocks = blocks.shape[0], blocks.ctypes.data_as(_pi)
        for d in range(3):
            c.filterDir[d] = int(case.filterDirections[d])
        c.filterCharTime = case.filterCharTime
        bc = case.bc
        n1, n2 = self._hold(_f(bc.neumannCoeffs)), self._hold(_f(bc.neumann2Coeffs))
        c.neumannLength, c.neumann2Length = n1.size, n2.size
        c.neumannCoeffs, c.neumann2Coeffs = n1.ctypes.data_as(_pd), n2.ctypes.data_as(_pd)
        vmap = {"U": 0, "V": 1, "W": 2, "P": 3, "E": 4}
        for ki, kind in enumerate("dns"):
            for V, vi in vmap.items():
                ind = bc.ind.get((kind, V))
                if ind is None or ind.shape[0] == 0:
                    continue
                ind = self._hold(np.asfortranarray(ind.astype(np.int32)))
                c.nbc[ki][vi] = ind.shape[0]
                c.ibc[ki][vi] = ind.ctypes.data_as(_pi)
                if kind == "d":
                    v = self._hold(_f(bc.val[V]))
                    c.vbc[vi] = v.ctypes.data_as(_pd)
                else:
                    dr = self._hold(np.asarray(bc.dirs[(kind, V)], dtype=np.int32))
                    c.dbc[ki][vi] = dr.ctypes.data_as(_pi)
        c.cN = bc.cL.shape[0]
        if c.cN:
            cL = self._hold(np.asfortranarray(bc.cL.astype(np.int32)))
            cD = self._hold(np.asfortranarray(bc.cD.astype(np.int32)))
            cA = self._hold(bc.cAdiabatic.astype(np.int32))
            c.cL, c.cD, c.cAdiabatic = cL.ctypes.data_as(_pi), cD.ctypes.data_as(_pi), cA.ctypes.data_as(_pi)
        nd = len(bc.disturbances)
        c.nDist = nd
        if nd:
            dcode = {"lidDrivenMovement": 1, "periodicSine": 2, "holdInlet": 3}
            typ = self._hold(np.array([dcode[d["type"]] for d in bc.disturbances], dtype=np.int32))
            var = self._hold(np.array([vmap["P" if d["var"][0] == "R" else d["var"][0]] for d in bc.disturbances],
                                      dtype=np.int32))
            ind = self._hold(np.asfortranarray(np.array([d["ind"] for d in bc.disturbances], dtype=np.int32)))
            xs, offs = [], []
            for d in bc.disturbances:
                offs.append(sum(len(x) for x in xs))
                xs.append(np.asarray(d["X"], dtype=np.float64))
            X = self._hold(np.concatenate(xs))
            off = self._hold(np.array(offs, dtype=np.int32))
            par = self._hold(np.array([d["par"][0] for d in bc.disturbances], dtype=np.float64))
            par2 = self._hold(np.array([d["par"][1] if len(d["par"]) > 1 else 0.0 for d in bc.disturbances],
                                       dtype=np.float64))
            c.distPar2 = par2.ctypes.data_as(_pd)
            # holdInlet: the first call's values, U V W E R per box (holdInlet.F90)
            sizes = [5 * int(np.prod([d["ind"][2 * a + 1] - d["ind"][2 * a] + 1 for a in range(3)]))
                     if d["type"] == "holdInlet" else 0 for d in bc.disturbances]
            hoff = self._hold(np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64))
            hsave = self._hold(np.zeros(max(1, int(np.sum(sizes)))))
            self.hold_saved = self._hold(np.zeros(nd, dtype=np.int32))
            c.holdSave, c.holdSaved = hsave.ctypes.data_as(_pd), self.hold_saved.ctypes.data_as(_pi)
            c.holdOff = hoff.ctypes.data_as(ctypes.POINTER(ctypes.c_long))
            c.distType, c.distVar, c.distInd = (a.ctypes.data_as(_pi) for a in (typ, var, ind))
            c.distX, c.distXoff, c.distPar = X.ctypes.data_as(_pd), off.ctypes.data_as(_pi), par.ctypes.data_as(_pd)
        c.timeStepping = int(getattr(case, "time_stepping", 1))
        fr = list(getattr(case, "forcings", None) or [])
        c.nForce = len(fr)
        if fr:
            code = {"pressureGradient": 1, "turbulenceGenerator": 2}
            ft = self._hold(np.array([code[f["type"]] for f in fr], dtype=np.int32))
            fi = self._hold(np.asfortranarray(np.array([f["ind"] for f in fr], dtype=np.int32)))
            fp = self._hold(np.array([list(f["par"]) + [0.0] * (2 - len(f["par"])) for f in fr], dtype=np.float64))
            c.forceType, c.forceInd, c.forcePar = ft.ctypes.data_as(_pi), fi.ctypes.data_as(_pi), fp.ctypes.data_as(_pd)
        c.sfdType = case.sfd_type
        c.sfdDelta = case.sfd_delta
        if case.sfd_type:
            chi = case.sfd_chi if case.sfd_type == 2 else np.full((case.nx, case.ny, case.nz), case.sfd_X)
            chi = self._hold(_f(chi))
            c.sfdChi = chi.ctypes.data_as(_pd)
        self.c = c
        self.cp = ctypes.pointer(c)

    def _hold(self, a):
        self._keep.append(a)
        return a

    @staticmethod
    def _ptrs(flow, keys=("U", "V", "W", "R", "E")):
        return [flow[k].ctypes.data_as(_pd) for k in keys]

    def calc_derivs(self, F, direction, kind="deriv"):
        F = _f(F)
        out = np.zeros_like(F, order="F")
        self.lib.orc_solve(self.cp, direction - 1, 0 if kind == "deriv" else 1, F.ctypes.data_as(_pd),
                           out.ctypes.data_as(_pd))
        return out

    def nseq(self, flow):
        f = {k: _f(flow[k]) for k in ("U", "V", "W", "R", "E")}
        out = {k: np.zeros_like(f["U"], order="F") for k in ("U", "V", "W", "R", "E")}
        self.lib.orc_nseq(self.cp, *self._ptrs(f), *self._ptrs(out))
        return out

    def apply_bound_cond(self, flow, t=0.0):
        f = {k: _f(flow[k]).copy(order="F") for k in ("U", "V", "W", "R", "E")}
        self.lib.orc_apply_bc(self.cp, *self._ptrs(f), t)
        return f

    def apply_filters(self, flow, blend=-1.0):
        f = {k: _f(flow[k]).copy(order="F") for k in ("U", "V", "W", "R", "E")}
        self.lib.orc_filters(self.cp, *self._ptrs(f), blend)
        return f

    def new_state(self, flow, mean=None):
        """Working state for :meth:`step`: copies of the flow, Wnew = 0, SFD mean."""
        st = {k: _f(flow[k]).copy(order="F") for k in ("U", "V", "W", "R", "E")}
        st["Wnew"] = np.zeros_like(st["U"], order="F")
        m = mean if mean is not None else flow
        for k in ("U", "V", "W", "R", "E"):
            st["m" + k] = _f(m[k]).copy(order="F")
        return st

    def step(self, st, t, dt):
        mc = np.zeros(5)
        self.lib.orc_step(self.cp, *self._ptrs(st), st["Wnew"].ctypes.data_as(_pd),
                          *self._ptrs(st, ("mU", "mV", "mW", "mR", "mE")), t, dt, mc.ctypes.data_as(_pd))
        return mc
