"""Jacobian-free Arnoldi on the CPU oracle -- TEST INFRASTRUCTURE ONLY.

numpy restatement of the Krylov loop of the reference's ``calcInstability.m:304-400``
(first-order variant, ``firstOrder = true``), with the DNS runs of the reference (one
``mpirun main`` per Krylov vector) replaced by the oracle's time step.  It is the checker of
``gatt_arnoldi``; nothing in the product imports it.

Follows the reference step by step:
* flow2vec / vec2flow (``:457-530``): a vector is [U; V; (W;) R; E] over the flow region;
* UM = Phi(base) once (``:327-340``);
* disturbance = vec2flow(zeta_k * epsilon * sqrt(N)) added to the base (``:353-362``);
* B = (UP - UM) / (epsilon * sqrt(N)) (``:390``);
* classical Gram-Schmidt with the original B (``:392-397``), H(k+1,k) = norm(uPrime),
  zeta_{k+1} = uPrime / H(k+1,k) (``:399-400``).
One deliberate difference, shared with ``gatt_arnoldi``: zeta_1 is the initial disturbance
normalised (the reference uses its Gaussian bump unnormalised, ``:309``).
"""
from __future__ import annotations

import numpy as np

KEYS3 = ("U", "V", "W", "R", "E")
KEYS2 = ("U", "V", "R", "E")


def _keys(case):
    return KEYS3 if case.is3d else KEYS2


def flow2vec(case, flow, region):
    return np.concatenate([np.asarray(flow[k], dtype=float)[region] for k in _keys(case)])


def vec2flow(case, vec, region):
    s = (case.nx, case.ny, case.nz)
    n = int(region.sum())
    out = {k: np.zeros(s, order="F") for k in KEYS3}
    for i, k in enumerate(_keys(case)):
        out[k][region] = vec[i * n:(i + 1) * n]
    return out


def run(oracle, flow, nsteps, t0, dt):
    """Phi: nsteps oracle steps from `flow` (SFD mean restarting from it, main.F90:158-163)."""
    st = oracle.new_state(flow)
    t = t0
    for _ in range(nsteps):
        oracle.step(st, t, dt)
        t = t + dt
    return {k: st[k] for k in KEYS3}


def arnoldi(oracle, case, base, v0, m, nsteps, dt, eps, t0=0.0, region=None):
    """H ((m+1) x m) of one problem, as gatt_arnoldi computes it for one member."""
    s = (case.nx, case.ny, case.nz)
    region = np.ones(s, dtype=bool) if region is None else np.asarray(region, dtype=bool).reshape(s, order="F")
    z1 = flow2vec(case, v0, region)
    N = z1.size
    zeta = np.zeros((N, m + 1))
    zeta[:, 0] = z1 / np.sqrt(np.sum(z1 * z1))
    H = np.zeros((m + 1, m))
    UM = flow2vec(case, run(oracle, base, nsteps, t0, dt), region)
    for k in range(m):
        d = vec2flow(case, zeta[:, k] * eps * np.sqrt(N), region)
        pert = {key: np.asarray(base[key], dtype=float) + d[key] for key in KEYS3}
        UP = flow2vec(case, run(oracle, pert, nsteps, t0, dt), region)
        B = (UP - UM) / (eps * np.sqrt(N))
        u = B.copy()
        for j in range(k + 1):
            H[j, k] = zeta[:, j] @ B
            u = u - H[j, k] * zeta[:, j]
        H[k + 1, k] = np.sqrt(np.sum(u * u))
        zeta[:, k + 1] = u / H[k + 1, k] if H[k + 1, k] != 0 else 0.0
    return H
