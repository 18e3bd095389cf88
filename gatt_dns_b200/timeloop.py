"""The reference's time loop around the step, on the host (source/Fortran/main.F90:192-533).

``run`` drives a :class:`~gatt_dns_b200.solver.GattDNS` context the way the Fortran main
program drives RK4: CFL time control (fixed dt, or the largest dt under maxCFL that lands
on the save times), one ``gatt_step`` per iteration, the divergence stop, ``log.txt`` lines,
and ``flow_%010d.mat`` exports.  Flow files are MAT-file level 5 (``scipy.io``), which the
reference's readFlow (readWriteMat.F90, ``matOpen`` / ``matGetVariable``) also opens; the
reference writes level 7.3 (HDF5), which this module cannot read (no HDF5 library here).
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import _lib

KEYS = ("U", "V", "W", "R", "E")


def flow_path(folder, n):
    """``flow_%010d.mat`` of save number n (readWriteMat.F90:173-179; -1 after divergence)."""
    return os.path.join(folder, "flow_%010d.mat" % n)


def write_flow(path, flow, t, inside_wall=None):
    """exportFlow.F90: the five fields and t, NaN inside walls."""
    import scipy.io
    out = {}
    for k in KEYS:
        a = np.array(flow[k], dtype=np.float64, order="F", copy=True)
        if inside_wall is not None:
            a[inside_wall] = np.nan
        out[k] = a
    out["t"] = np.array([[float(t)]])
    scipy.io.savemat(path, out, do_compression=False, oned_as="column")


def read_flow(path, shape=None):
    """importFlow.F90:26-40: the five fields and t; NaN (inside walls) becomes U = V = W = 0,
    R = E = 1.  A 2-D file gets a unit third dimension."""
    import scipy.io
    m = scipy.io.loadmat(path)
    flow = {}
    for k in KEYS:
        a = np.asarray(m[k], dtype=np.float64)
        if a.ndim == 2:
            a = a[:, :, None]
        if shape is not None:
            a = a.reshape(shape, order="F")
        flow[k] = np.asfortranarray(a)
    nan = np.isnan(flow["U"])
    for k in ("U", "V", "W"):
        flow[k][nan] = 0.0
    for k in ("R", "E"):
        flow[k][nan] = 1.0
    return flow, float(np.asarray(m["t"]).ravel()[0])


def cfl_rate(case, vmax):
    """CFLdt of main.F90:206-212: the CFL number per unit dt."""
    c = 1.0 / case.Ma
    r = (c + vmax[0]) * case.dxmin[0] + (c + vmax[1]) * case.dxmin[1]
    if case.is3d:
        r += (c + vmax[2]) * case.dxmin[2]
    return r


def log_line(nsave, tstep, t, dt, cfl, mc, tracked=()):
    """One log.txt line (main.F90:475-500): save number (0 between saves), step, t, dt, CFL,
    the five max changes, then the tracked nodes' values, tab separated."""
    cols = ["%10d" % nsave, "%10d" % tstep, "%13.8E" % t, "%10.5E" % dt, "%8.5f" % cfl]
    cols += ["%10.4E" % x for x in mc]
    for vals in tracked:
        cols += ["0" if v == 0 else "%15.8E" % v for v in vals]
    return "\t".join(cols)


def run(g, t0=0.0, tstep0=0, nsave0=0, time_control=2, dtmax=1.0, max_cfl=0.5, qtimes=1.0, tmax=1.0,
        folder=None, log_all=1, tracked=(), tracked_norm=0.0, inside_wall=None, on_step=None):
    """main.F90:192-533 on the context's member 0.

    time_control 1: fixed dt = dtmax, save every ``qtimes`` steps (an integer), stop after
    ``tmax`` steps; time_control 2: dt = min(max_cfl / CFLdt, dtmax) shrunk so that an integer
    number of steps reaches the next save time, save every ``qtimes`` time units, stop at
    ``tmax``.  With ``folder`` the flows are exported there and log.txt is appended to.
    ``tracked``: 1-based (i, j, k) nodes whose values go to the log (R - 1 and E/norm - 1
    when ``tracked_norm`` is non-zero, as main.F90:489-492).  Returns (t, tstep, nsave).
    """
    case = g.case
    t, tstep, nsave = float(t0), int(tstep0), int(nsave0)
    steps_until_saving = 0
    done = False
    qint, tmax_int = int(round(qtimes)), int(round(tmax))
    log = open(os.path.join(folder, "log.txt"), "a") if folder else None
    dt = dtmax
    try:
        while not done:
            vmax = g.max_velocity()[0]
            rate = cfl_rate(case, vmax)
            if time_control == 1:
                if (tstep + 1) % qint == 0:
                    steps_until_saving = 0
                    nsave = tstep + 1
                else:
                    steps_until_saving = 1
                dt = dtmax
                done = (tstep + 1) >= tmax_int
            else:
                if steps_until_saving == 0:
                    dt = min(max_cfl / rate, dtmax)
                    steps_until_saving = math.floor(qtimes / dt) + 1
                    dt = qtimes / steps_until_saving
                    nsave += 1
                steps_until_saving -= 1
                done = (t + dt) >= tmax
            cfl = dt * rate
            try:
                mc = g.step(t, dt)[0]
            except _lib.GattError as e:
                if e.code == 4 and folder:  # GATT_ERR_DIVERGED: export and stop (main.F90:440-448)
                    write_flow(flow_path(folder, -1), g.download(), t, inside_wall)
                raise
            tstep += 1
            t = t + dt
            if on_step:
                on_step(tstep, t, dt, cfl, mc)
            if log and (tstep % log_all == 0 or steps_until_saving == 0):
                vals = []
                if tracked:
                    f = g.download()
                    for (i, j, k) in tracked:
                        v = [float(f[key][i - 1, j - 1, k - 1]) for key in KEYS]
                        if tracked_norm != 0:
                            v[3] -= 1.0
                            v[4] = v[4] / tracked_norm - 1.0
                        vals.append(v)
                log.write(log_line(nsave if steps_until_saving == 0 else 0, tstep, t, dt, cfl, mc, vals) + "\n")
            if folder and steps_until_saving == 0:
                write_flow(flow_path(folder, nsave), g.download(), t, inside_wall)
    finally:
        if log:
            log.close()
    return t, tstep, nsave
