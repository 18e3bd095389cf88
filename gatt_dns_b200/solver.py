"""Host-side mirror of the reference solver interface over the C-ABI.

``GattDNS`` owns one ``gatt_ctx`` and exposes the reference's operations under its
own names: ``calc_derivs`` (solveSystem*), ``nseq`` (nseq2d/nseq3d),
``apply_bound_cond`` (applyBoundCond), ``apply_filters`` (applyFilters2D/3D) and
``step`` (one pass of the main.F90 time loop body).  Arrays are numpy FP64 in Fortran
order; every call goes through the CUDA library.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .case import Case, VAR_INDEX

_pd = ctypes.POINTER(ctypes.c_double)
_pi = ctypes.POINTER(ctypes.c_int)

KIND = {"d": 0, "n": 1, "s": 2}
DIST_TYPE = {"lidDrivenMovement": 1, "periodicSine": 2, "holdInlet": 3}
FORCE_TYPE = {"pressureGradient": 1, "turbulenceGenerator": 2}  # GATT_FORCE_*


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(_pd)


def _ip(a):
    if a is None:
        return None
    return a.ctypes.data_as(_pi)


def _f64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _i32(a):
    return np.asfortranarray(np.asarray(a, dtype=np.int32))


class GattDNS:
    """One solver context for a :class:`Case` with ``nbatch`` independent flow states."""

    def __init__(self, case: Case, nbatch: int = 1, stream=None):
        self.lib = _lib.load()
        self.case = case
        self.nbatch = nbatch
        h = ctypes.c_void_p()
        _lib.check(self.lib.gatt_create(ctypes.byref(h), case.nx, case.ny, case.nz, nbatch), "gatt_create")
        self.h = h
        if stream is not None:
            _lib.check(self.lib.gatt_set_stream(self.h, ctypes.c_void_p(int(stream))), "gatt_set_stream")
        self._configure()

    # -- setup -------------------------------------------------------------
    def _configure(self):
        c, L = self.case, self.lib
        _lib.check(L.gatt_set_physics(self.h, c.Re, c.Ma, c.Pr, c.gamma, c.T0), "gatt_set_physics")
        for d, m in enumerate(c.mats):
            if m is None:
                continue
            blocks = _i32(m.blocks)
            nb = blocks.shape[0]
            for kind, (A, B, C, D, R, nR) in enumerate(((m.A, m.B, m.C, m.D, m.R, m.nRHS),
                                                        (m.Af, m.Bf, m.Cf, m.Df, m.Rf, m.nRHSf))):
                A, B, C, D, R = _f64(A), _f64(B), _f64(C), _f64(D), _f64(R)
                _lib.check(L.gatt_set_matrices(self.h, d + 1, kind, m.periodic, nR, m.nTypes, _dp(A), _dp(B), _dp(C),
                                               _dp(D) if m.periodic else None, _dp(R), nb, _ip(blocks)),
                           "gatt_set_matrices")
            # transposed operators for the adjoint (kinds 2..5), when the emitter produced them
            for k, s in enumerate(m.adj or []):
                A, B, C, D, R = _f64(s.A), _f64(s.B), _f64(s.C), _f64(s.D), _f64(s.R)
                _lib.check(L.gatt_set_matrices(self.h, d + 1, 2 + k, s.periodic, s.nRHS, s.nTypes, _dp(A), _dp(B),
                                               _dp(C), _dp(D) if s.periodic else None, _dp(R), 0, None),
                           "gatt_set_matrices")
        fd = c.filterDirections
        _lib.check(L.gatt_set_filter(self.h, fd[0], fd[1], fd[2], c.filterCharTime), "gatt_set_filter")
        _lib.check(L.gatt_set_time_stepping(self.h, int(getattr(c, "time_stepping", 1))), "gatt_set_time_stepping")
        bc = c.bc
        n1, n2 = _f64(bc.neumannCoeffs), _f64(bc.neumann2Coeffs)
        _lib.check(L.gatt_set_neumann(self.h, n1.size, _dp(n1) if n1.size else None, n2.size,
                                      _dp(n2) if n2.size else None), "gatt_set_neumann")
        for kind in "dns":
            for V in ("U", "V", "W", "P", "E"):
                ind = bc.ind.get((kind, V))
                n = 0 if ind is None else ind.shape[0]
                if n == 0:
                    _lib.check(L.gatt_set_bc(self.h, VAR_INDEX[V], KIND[kind], 0, None, None, None), "gatt_set_bc")
                    continue
                ind = _i32(ind)
                if kind == "d":
                    val = _f64(bc.val[V])
                    _lib.check(L.gatt_set_bc(self.h, VAR_INDEX[V], 0, n, _ip(ind), _dp(val), None), "gatt_set_bc")
                else:
                    dr = _i32(bc.dirs[(kind, V)])
                    _lib.check(L.gatt_set_bc(self.h, VAR_INDEX[V], KIND[kind], n, _ip(ind), None, _ip(dr)),
                               "gatt_set_bc")
        cL, cD, cA = _i32(bc.cL), _i32(bc.cD), _i32(bc.cAdiabatic)
        nc = cL.shape[0]
        _lib.check(L.gatt_set_corners(self.h, nc, _ip(cL) if nc else None, _ip(cD) if nc else None,
                                      _ip(cA) if nc else None), "gatt_set_corners")
        _lib.check(L.gatt_clear_disturbances(self.h), "gatt_clear_disturbances")
        for d in bc.disturbances:
            ind = _i32(d["ind"])
            x = _f64(d["X"])
            par = _f64(d["par"])
            # holdInlet acts on all of U, V, R, W, E (its var is "UVRWE"); the others on one variable
            var = 0 if d["type"] == "holdInlet" else VAR_INDEX[d["var"]]
            _lib.check(L.gatt_add_disturbance(self.h, DIST_TYPE[d["type"]], var, _ip(ind), _dp(x),
                                              par.size, _dp(par)), "gatt_add_disturbance")
        for f in getattr(c, "forcings", None) or []:
            ind = np.ascontiguousarray(np.asarray(f["ind"], dtype=np.int32))
            par = _f64(f["par"])
            _lib.check(L.gatt_add_forcing(self.h, FORCE_TYPE[f["type"]], _ip(ind), par.size, _dp(par)),
                       "gatt_add_forcing")
        if c.sfd_type > 0:
            chi = _f64(c.sfd_chi) if c.sfd_chi is not None else None
            _lib.check(L.gatt_set_sfd(self.h, c.sfd_type, c.sfd_delta, c.sfd_X, _dp(chi)), "gatt_set_sfd")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.gatt_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ---------------------------------------------------------------
    def upload(self, flow, b=0):
        f = {k: _f64(flow[k]) for k in ("U", "V", "W", "R", "E")}
        _lib.check(self.lib.gatt_upload(self.h, b, *(_dp(f[k]) for k in ("U", "V", "W", "R", "E"))), "gatt_upload")

    def download(self, b=0, out=None):
        s = (self.case.nx, self.case.ny, self.case.nz)
        if out is None:
            out = {k: np.zeros(s, order="F") for k in ("U", "V", "W", "R", "E")}
        _lib.check(self.lib.gatt_download(self.h, b, *(_dp(out[k]) for k in ("U", "V", "W", "R", "E"))),
                   "gatt_download")
        return out

    def upload_mean(self, flow, b=0):
        f = {k: _f64(flow[k]) for k in ("U", "V", "W", "R", "E")}
        _lib.check(self.lib.gatt_upload_mean(self.h, b, *(_dp(f[k]) for k in ("U", "V", "W", "R", "E"))),
                   "gatt_upload_mean")

    def download_mean(self, b=0):
        s = (self.case.nx, self.case.ny, self.case.nz)
        out = {k: np.zeros(s, order="F") for k in ("U", "V", "W", "R", "E")}
        _lib.check(self.lib.gatt_download_mean(self.h, b, *(_dp(out[k]) for k in ("U", "V", "W", "R", "E"))),
                   "gatt_download_mean")
        return out

    def download_wnew(self, b=0):
        s = (self.case.nx, self.case.ny, self.case.nz)
        w = np.zeros(s, order="F")
        _lib.check(self.lib.gatt_download_wnew(self.h, b, _dp(w)), "gatt_download_wnew")
        return w

    def device_ptr(self, var, b=0):
        p = _pd()
        _lib.check(self.lib.gatt_state_device_ptr(self.h, b, VAR_INDEX[var], ctypes.byref(p)), "gatt_state_device_ptr")
        return ctypes.cast(p, ctypes.c_void_p).value

    # -- reference operations ----------------------------------------------
    KINDS = {"deriv": 0, "filter": 1, "deriv_lhsT": 2, "deriv_rT": 3, "filter_lhsT": 4, "filter_rT": 5}

    def calc_derivs(self, F, direction, kind="deriv"):
        """solveSystem{X,Y,Z}[per] of one field (derivs.F90:556-948); kind also names the
        transposed operators: "deriv_T" / "filter_T" apply both halves (L^T)."""
        F = _f64(F)
        if kind in ("deriv_T", "filter_T"):
            base = kind[:-2]
            return self.calc_derivs(self.calc_derivs(F, direction, base + "_lhsT"), direction, base + "_rT")
        out = np.zeros_like(F, order="F")
        _lib.check(self.lib.gatt_deriv_dir(self.h, direction, self.KINDS[kind], _dp(F), _dp(out)),
                   "gatt_deriv_dir")
        return out

    def nseq(self, flow):
        """nseq2d/nseq3d (nseq.F90:10-323); returns dict of dU, dV, dW, dR, dE."""
        f = {k: _f64(flow[k]) for k in ("U", "V", "W", "R", "E")}
        s = f["U"].shape
        out = {k: np.zeros(s, order="F") for k in ("U", "V", "W", "R", "E")}
        _lib.check(self.lib.gatt_rhs(self.h, *(_dp(f[k]) for k in ("U", "V", "W", "R", "E")),
                                     *(_dp(out[k]) for k in ("U", "V", "W", "R", "E"))), "gatt_rhs")
        return out

    def apply_bound_cond(self, t=0.0):
        _lib.check(self.lib.gatt_apply_bc(self.h, t), "gatt_apply_bc")

    def apply_filters(self, blend=-1.0):
        _lib.check(self.lib.gatt_filter(self.h, blend), "gatt_filter")

    def step(self, t, dt):
        """One time step (main.F90:255-465 minus time control); returns maxChange (nbatch, 5)."""
        mc = np.zeros(5 * self.nbatch)
        _lib.check(self.lib.gatt_step(self.h, t, dt, _dp(mc)), "gatt_step")
        return mc.reshape(self.nbatch, 5)

    def run(self, nsteps, t0, dt):
        mc = np.zeros(5 * self.nbatch)
        _lib.check(self.lib.gatt_run(self.h, nsteps, t0, dt, _dp(mc)), "gatt_run")
        return mc.reshape(self.nbatch, 5)

    def arnoldi(self, base, v0, m, nsteps, dt, eps=1e-7, t0=0.0, region=None):
        """Jacobian-free Arnoldi (calcInstability.m:304-400, first order) for every member.

        base: flow dict (the base flow, shared); v0: list of nbatch flow dicts (initial
        disturbances); region: boolean (nx, ny, nz) flow region or None.  Returns H of shape
        (nbatch, m+1, m); the Ritz values of member b are eig(H[b, :m, :m]) and the growth
        rates log(lambda)/T as calcInstability.m:411 computes them.
        """
        keys = ("U", "V", "W", "R", "E")
        if len(v0) != self.nbatch:
            raise ValueError("need one initial disturbance per member")
        bvec = np.concatenate([_f64(base[k]).ravel(order="F") for k in keys])
        v = np.concatenate([_f64(d[k]).ravel(order="F") for d in v0 for k in keys])
        reg = None
        if region is not None:
            reg = np.ascontiguousarray(np.asarray(region, dtype=bool).ravel(order="F").astype(np.uint8))
        H = np.zeros(self.nbatch * (m + 1) * m)
        _lib.check(self.lib.gatt_arnoldi(self.h, m, nsteps, t0, dt, eps, _dp(bvec), _dp(v),
                                         reg.ctypes.data_as(ctypes.c_void_p) if reg is not None else None,
                                         _dp(H)), "gatt_arnoldi")
        return H.reshape(self.nbatch, m, m + 1).transpose(0, 2, 1).copy()

    def arnoldi_vector(self, b, j):
        """Basis vector zeta_{j+1} of member b after arnoldi(), as a flow dict."""
        s = (self.case.nx, self.case.ny, self.case.nz)
        out = np.zeros(5 * self.case.nx * self.case.ny * self.case.nz)
        _lib.check(self.lib.gatt_arnoldi_vector(self.h, b, j, _dp(out)), "gatt_arnoldi_vector")
        n = out.size // 5
        return {k: out[i * n:(i + 1) * n].reshape(s, order="F") for i, k in enumerate(("U", "V", "W", "R", "E"))}

    # -- tangent-linear / adjoint (3-D, no boundary conditions, no SFD) ------------------
    def _pack(self, flows):
        """list (one per member) of flow dicts -> contiguous nbatch*5*npts vector"""
        if isinstance(flows, dict):
            flows = [flows]
        return np.concatenate([_f64(f[k]).ravel(order="F") for f in flows for k in ("U", "V", "W", "R", "E")])

    def _unpack(self, vec):
        s = (self.case.nx, self.case.ny, self.case.nz)
        n = self.case.nx * self.case.ny * self.case.nz
        out = []
        for b in range(self.nbatch):
            out.append({k: vec[(b * 5 + i) * n:(b * 5 + i + 1) * n].reshape(s, order="F")
                        for i, k in enumerate(("U", "V", "W", "R", "E"))})
        return out if self.nbatch > 1 else out[0]

    def rhs_jvp(self, q, dq):
        """F'(q) dq of the right-hand side (nseq3d linearised)."""
        qv, dv = self._pack(q), self._pack(dq)
        out = np.zeros_like(qv)
        _lib.check(self.lib.gatt_rhs_jvp(self.h, _dp(qv), _dp(dv), _dp(out)), "gatt_rhs_jvp")
        return self._unpack(out)

    def rhs_vjp(self, q, a):
        """F'(q)^T a."""
        qv, av = self._pack(q), self._pack(a)
        out = np.zeros_like(qv)
        _lib.check(self.lib.gatt_rhs_vjp(self.h, _dp(qv), _dp(av), _dp(out)), "gatt_rhs_vjp")
        return self._unpack(out)

    # step vectors of gatt_jvp / gatt_vjp: the five state fields, and with SFD the five mean
    # fields (keys "mU" ... "mE") after them
    _MEAN_KEYS = ("mU", "mV", "mW", "mR", "mE")

    def _pack_vec(self, flows):
        if not self.case.sfd_type:
            return self._pack(flows)
        if isinstance(flows, dict):
            flows = [flows]
        z = np.zeros(self.case.npts)
        return np.concatenate([_f64(f[k]).ravel(order="F") if k in f else z
                               for f in flows for k in ("U", "V", "W", "R", "E") + self._MEAN_KEYS])

    def _unpack_vec(self, vec):
        if not self.case.sfd_type:
            return self._unpack(vec)
        s = (self.case.nx, self.case.ny, self.case.nz)
        n = self.case.npts
        keys = ("U", "V", "W", "R", "E") + self._MEAN_KEYS
        out = [{k: vec[(b * 10 + i) * n:(b * 10 + i + 1) * n].reshape(s, order="F") for i, k in enumerate(keys)}
               for b in range(self.nbatch)]
        return out if self.nbatch > 1 else out[0]

    def jvp(self, dq0, nsteps, t0, dt):
        """Tangent over nsteps steps from the current state (which advances, as run()); with
        SFD the vectors carry the mean's tangent under the keys mU ... mE."""
        dv = self._pack_vec(dq0)
        out = np.zeros_like(dv)
        _lib.check(self.lib.gatt_jvp(self.h, nsteps, t0, dt, _dp(dv), _dp(out)), "gatt_jvp")
        return self._unpack_vec(out)

    def vjp(self, lamN, nsteps, t0, dt, checkpoint_every=20):
        """Adjoint over nsteps steps from the current state, checkpointed (mean keys as jvp)."""
        lv = self._pack_vec(lamN)
        out = np.zeros_like(lv)
        _lib.check(self.lib.gatt_vjp(self.h, nsteps, t0, dt, checkpoint_every, _dp(lv), _dp(out)), "gatt_vjp")
        return self._unpack_vec(out)

    def autotune(self, reps=3):
        """Pick the fastest line-solve configuration per matrix set (gatt_autotune).
        Returns {(dir, kind): (family, row blocks, us per launch)} for the sets present."""
        fam = np.zeros(18, dtype=np.int32)
        blk = np.zeros(18, dtype=np.int32)
        us = np.zeros(18)
        _lib.check(self.lib.gatt_autotune(self.h, reps, _ip(fam), _ip(blk), _dp(us)), "gatt_autotune")
        names = ("tile", "reg", "pipe")
        return {(i // 6 + 1, i % 6): (names[fam[i]], int(blk[i]), float(us[i])) for i in range(18) if fam[i] >= 0}

    def max_velocity(self):
        v = np.zeros(3 * self.nbatch)
        _lib.check(self.lib.gatt_max_velocity(self.h, _dp(v)), "gatt_max_velocity")
        return v.reshape(self.nbatch, 3)

    def synchronize(self):
        _lib.check(self.lib.gatt_synchronize(self.h), "gatt_synchronize")

    def kernel_launches(self):
        return int(self.lib.gatt_kernel_launches(self.h))

    def profile_kernels(self, t0, dt, nsteps=2):
        """Per kernel class: (mean ms per launch, launches per step), from CUDA events."""
        n = 17  # GATT_NPROF
        ms, la = np.zeros(n), np.zeros(n)
        _lib.check(self.lib.gatt_profile_kernels(self.h, t0, dt, nsteps, _dp(ms), _dp(la)), "gatt_profile_kernels")
        return {self.lib.gatt_profile_name(i).decode(): (float(ms[i]), float(la[i])) for i in range(n)}
