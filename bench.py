"""Benchmark: FP64 Mpoint-stages/s of the GATT_DNS RK4 time step on the 128^3 periodic box.

Workload (one "step"): one full time step of main.F90:255-465 -- four RK4 stages of the
compressible Navier-Stokes right-hand side with compact SL4 derivatives (cyclic line
solves in x, y, z), the 10th-order compact filter, boundary conditions (none on the
periodic box) and the max-change residual -- on a 128^3 grid, Re = 1600, Ma = 0.3, with a
seeded solenoidal initial field.  Throughput counts grid points x 4 stages per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): every rank advances its own box (batch
sharding of independent flows, no data-path collective: weak scaling); the timing is the
max over ranks.  --impl reference times the CPU restatement of the reference on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 128
STAGES = 4
# Sweep-model bytes per 3-D point-stage: 27 derivative sweeps x 16 B + 5 fields x 32 B of
# RK state traffic + 15 filter sweeps x 16 B / 4 stages.
BYTES_PER_POINT_STAGE = 27 * 16 + 5 * 32 + 15 * 16 / 4
# Fields the 3-D assembly + RK update moves per point, averaged over the four stages: stage
# input 5, gradients 15, second-sweep terms 12 and output 5 in every stage; step start 5
# (stages 2-4; in stage 1 it is the stage input), RK increment read 5 (stages 2-4) and
# written 5 (stages 1-3).  Stages 1..4: 42, 52, 52, 47 fields; mean 48.25.
ASSEMBLE_FIELDS = (5 + 15 + 12 + 5) + 3 * (3 * 5) / 4.0
# DRAM bytes per launch of each kernel function from an ncu capture of this workload
# (dram__bytes_read.sum + dram__bytes_write.sum), one "traffic <function> <bytes>" line per
# function; written by hand from the capture, with the capture's command in the file.
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_traffic_periodic_box_128.txt")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=N_GRID)
    p.add_argument("--no-clocks", action="store_true")
    p.add_argument("--no-arnoldi", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    # profiling runs: keep the default line-solve configuration (under a profiler the autotuner's
    # timings are distorted) and leave out the CPU, Arnoldi, adjoint and other-case samples
    p.add_argument("--no-autotune", action="store_true")
    p.add_argument("--kernels-only", action="store_true")
    return p.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1])); mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args, world, rank):
    """CPU restatement of the reference, all host threads, rank 0 only."""
    if rank != 0:
        return
    import oracle
    from gatt_dns_b200 import case as cs
    oracle.build()
    c = cs.periodic_box(n=args.n)
    o = oracle.Oracle(c)
    cores = o.lib.orc_num_threads()
    f = cs.solenoidal_turbulence(c, seed=1234)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    st = o.new_state(f)
    t = 0.0
    for _ in range(max(args.warmup, 1)):
        o.step(st, t, dt); t += dt
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(st, t, dt); t += dt
    el = time.perf_counter() - t0
    npts = c.npts
    value = npts * STAGES * args.steps / el / 1e6
    line = {"metric": "FP64 Mpoint-stages/s (RK4 step, 128^3 periodic box)", "value": value,
            "unit": "Mpoint-stages/s", "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded solenoidal field)",
            "config": {"workload": "periodic_box_%d^3_rk4_step" % args.n, "grid": [args.n] * 3, "Re": 1600,
                       "Ma": 0.3, "scheme": "SL4 compact + 10th-order filter (alpha 0.49)"},
            "cpu_baseline": {"value": value, "unit": "Mpoint-stages/s", "cores": cores, "kind": "port",
                             "sample": "%d full RK4 steps of the %d^3 box (C restatement of the reference "
                                       "Fortran, OpenMP over lines)" % (args.steps, args.n)},
            "e2e": {"value": value, "unit": "Mpoint-stages/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(c, seconds=10.0):
    """Oracle timed on a bounded sample (whole steps until ~`seconds` of CPU work)."""
    import oracle
    oracle.build()
    from gatt_dns_b200 import case as cs
    o = oracle.Oracle(c)
    f = cs.solenoidal_turbulence(c, seed=1234)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    st = o.new_state(f)
    o.step(st, 0.0, dt)  # warm
    n, t0 = 0, time.perf_counter()
    while True:
        o.step(st, n * dt, dt)
        n += 1
        el = time.perf_counter() - t0
        if el > seconds or n >= 20:
            break
    v = c.npts * STAGES * n / el / 1e6
    cores = o.lib.orc_num_threads()
    # one core: two steps (about 15 s on this grid)
    o.lib.orc_set_threads(1)
    t0 = time.perf_counter()
    for k in range(2):
        o.step(st, (n + k) * dt, dt)
    el1 = time.perf_counter() - t0
    o.lib.orc_set_threads(cores)
    v1 = c.npts * STAGES * 2 / el1 / 1e6
    return {"value": v, "unit": "Mpoint-stages/s", "cores": cores, "kind": "port",
            "sample": "%d full RK4 steps of the %d^3 box in %.1f s (C restatement of the reference Fortran, "
                      "OpenMP over lines; work arrays kept across calls like the Fortran's)" % (n, c.nx, el),
            "one_core": {"value": v1, "unit": "Mpoint-stages/s", "cores": 1,
                         "sample": "2 full RK4 steps of the %d^3 box in %.1f s" % (c.nx, el1)},
            "host": host_cpu()}


def arnoldi_sample(cs, GattDNS, case, base, members, m, nsteps, seed, label, dist=None):
    """Batched vs serial Jacobian-free Arnoldi (bounded sample).

    Batched: one context holding this rank's share of the `members` problems, one
    gatt_arnoldi call (every kernel launch covers all of them).  Serial: one single-member
    context reused for the same problems one after another.  Both include the host<->device
    transfers of the calls; each side's graphs are captured in an untimed warm-up call first.
    Times are CUDA events on the contexts' stream; with several ranks (torch.distributed
    initialised) the problems are sharded across ranks (shard.arnoldi_sharded, no data-path
    collective: the ranks gather H at the end) and each time is the max over ranks.
    """
    import torch
    from gatt_dns_b200.shard import arnoldi_sharded, max_over_ranks, member_range
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    rng = np.random.default_rng(seed)
    s = (case.nx, case.ny, case.nz)
    v0 = []
    for _ in range(members):
        d = {k: np.zeros(s, order="F") for k in "UVWRE"}
        d["U"][...] = 1e-6 * rng.standard_normal(s)
        d["V"][...] = 1e-6 * rng.standard_normal(s)
        v0.append(d)
    lo, hi = member_range(members, world, rank)
    mine = hi - lo
    dt = case.cfl_dt(base["U"], base["V"], base["W"], 0.5)
    stream = torch.cuda.Stream()

    def timed(fn):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, max_over_ranks(e0.elapsed_time(e1) / 1e3, dist, device="cuda")

    gb = GattDNS(case, nbatch=mine, stream=stream.cuda_stream)
    gb.arnoldi(base, v0[lo:hi], 1, 1, dt)               # warm-up: graph capture, buffers
    Hb, tb = timed(lambda: arnoldi_sharded(lambda v: gb.arnoldi(base, v, m, nsteps, dt), v0, dist, device="cuda"))
    step_b = time_steps(gb, dt, 10) / mine              # ms per member-step, batched
    gb.close()
    g1 = GattDNS(case, nbatch=1, stream=stream.cuda_stream)
    g1.arnoldi(base, v0[lo:lo + 1], 1, 1, dt)

    def serial():
        return [g1.arnoldi(base, [v0[b]], m, nsteps, dt)[0] for b in range(lo, hi)]

    Hs, ts = timed(serial)
    same = all(bool(np.array_equal(Hs[i], Hb[lo + i])) for i in range(mine))
    if dist is not None:
        flag = torch.tensor([1.0 if same else 0.0], device="cuda")
        dist.all_reduce(flag, op=dist.ReduceOp.MIN)
        same = bool(flag.item() == 1.0)
    step_1 = time_steps(g1, dt, 10)                    # ms per step, one member
    g1.close()
    return {"workload": label, "members": members, "ranks": world, "members_per_rank": mine, "krylov_steps": m,
            "rk4_steps_per_run": nsteps, "runs_per_member": m + 1, "batched_s": tb, "serial_s": ts,
            "serial_over_batched": ts / tb, "H_batched_equals_serial": same,
            "rk4_step_ms_per_member_batched": step_b, "rk4_step_ms_single": step_1,
            "full_config_serial_over_batched_est": step_1 / step_b,
            "sample": "%d Krylov steps of %d RK4 steps each (plus the base run) per problem; the full "
                      "config runs 32 Krylov steps of 500, where the RK4 steps dominate: its ratio is "
                      "estimated from the time per member-step (10 synchronised steps)%s" % (
                          m, nsteps, "; problems sharded over %d ranks, times max over ranks" % world
                          if world > 1 else "")}


def adjoint_sample(cs, GattDNS, nsteps=200, every=20, shape=(400, 150, 64)):
    """Config 5 on its full grid, bounded sample: gradient of the perturbation kinetic energy
    J = 1/2 sum |u - u_base|^2 after nsteps steps with respect to the initial perturbation
    (seed 99, amplitude 1e-6), by the checkpointed adjoint; checked by a central difference
    along a random direction and by a dot-product test against the tangent."""
    import torch
    c = cs.boundary_layer(nx=shape[0], ny=shape[1], nz=shape[2])
    base = cs.blasius_flow(c)
    s = (c.nx, c.ny, c.nz)
    rng = np.random.default_rng(99)
    pert = {k: 1e-6 * rng.standard_normal(s) for k in "UVWRE"}
    q0 = {k: base[k] + pert[k] for k in "UVWRE"}
    dt = c.cfl_dt(base["U"], base["V"], base["W"], 0.5)
    g = GattDNS(c)

    def run(q):
        g.upload(q)
        g.run(nsteps, 0.0, dt)
        return g.download()

    ub = run(base)  # also captures the step graphs
    t0 = time.perf_counter()
    uN = run(q0)
    t_fwd = time.perf_counter() - t0

    def J(u):
        return 0.5 * float(sum(np.sum((u[k] - ub[k]) ** 2) for k in "UVW"))

    lam = {k: (uN[k] - ub[k]) if k in "UVW" else np.zeros(s) for k in "UVWRE"}
    g.upload(q0)
    grad = g.vjp(lam, nsteps, 0.0, dt, checkpoint_every=every)  # first call: allocates the adjoint buffers
    v = {k: 1e-6 * rng.standard_normal(s) for k in "UVWRE"}
    h = 0.1
    jp = J(run({k: q0[k] + h * v[k] for k in "UVWRE"}))
    jm = J(run({k: q0[k] - h * v[k] for k in "UVWRE"}))
    fd = (jp - jm) / (2 * h)
    ad = float(sum(np.sum(grad[k] * v[k]) for k in "UVWRE"))
    g.upload(q0)
    g.jvp(v, nsteps, 0.0, dt)  # first call: allocates the tangent buffers
    g.upload(q0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    jv = g.jvp(v, nsteps, 0.0, dt)
    t_tl = time.perf_counter() - t0
    w = {k: rng.standard_normal(s) for k in "UVWRE"}
    g.upload(q0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    jtw = g.vjp(w, nsteps, 0.0, dt, checkpoint_every=every)
    t_adj = time.perf_counter() - t0
    a = float(sum(np.sum(jv[k] * w[k]) for k in "UVWRE"))
    b = float(sum(np.sum(v[k] * jtw[k]) for k in "UVWRE"))
    g.close()
    return {"workload": "boundary layer %dx%dx%d, Blasius base, Re 1000, Ma 0.5" % shape, "steps": nsteps,
            "checkpoint_every": every, "forward_s": t_fwd, "tangent_s": t_tl, "adjoint_s": t_adj,
            "adjoint_over_forward": t_adj / t_fwd, "gradient_vs_central_difference_rel": abs(ad - fd) / abs(fd),
            "dot_product_test_rel": abs(a - b) / abs(a),
            "sample": "%d of the config's 200 steps (checkpoint every %d); times are wall clock of the "
                      "synchronous C-ABI calls, host transfers included, each after an untimed first call "
                      "(graph capture, buffer allocation)" % (nsteps, every)}


def kernel_functions(case, tuned):
    """Map each profiled launch class to the kernel function it launches (the line-solve
    family the context uses for that matrix set: the autotuner's choice, else the pipelined
    solver) and to its algorithmic bytes per point (16 B per field for a line solve: read and
    write once)."""
    fam_name = {"pipe": "k_psweep", "reg": "k_rsweep", "tile": "k_sweep"}

    def uniform_band(m, kind):
        # cyclic, one matrix type, every row the same band: the uniform-band instantiation
        R = np.asarray(m.R if kind == 0 else m.Rf)
        return bool(m.periodic) and m.nTypes == 1 and bool(np.all(R[:, :, 0] == R[0:1, :, 0]))

    def solver(d, kind):
        m = case.mats[d - 1]
        fam = tuned.get((d, kind), ("pipe",))[0]
        nR = m.nRHS if kind == 0 else m.nRHSf
        ub = ", uniform band" if fam == "pipe" and uniform_band(m, kind) else ""
        return "%s<%s, %s, nR=%d%s>" % (fam_name[fam], "x" if d == 1 else "y/z",
                                        "cyclic" if m.periodic else "banded", nR, ub)

    return {"sweep_d1_x": (solver(1, 0), 5 * 16), "sweep_d1_y": (solver(2, 0), 5 * 16),
            "sweep_d1_z": (solver(3, 0), 5 * 16), "sweep_d1_yz": (solver(2, 0), 10 * 16),
            "sweep_d2_x": (solver(1, 0), 4 * 16), "sweep_d2_y": (solver(2, 0), 4 * 16),
            "sweep_d2_z": (solver(3, 0), 4 * 16), "sweep_d2_yz": (solver(2, 0), 8 * 16),
            "filter_x": (solver(1, 1), 5 * 16), "filter_y": (solver(2, 1), 5 * 16),
            "filter_z": (solver(3, 1), 5 * 16),
            "visc": ("k_visc3d", (13 + 9) * 8), "assemble_rk": ("k_assemble3d_pipe", ASSEMBLE_FIELDS * 8),
            "maxchange": ("k_maxchange", 10 * 8)}


def dominant_kernel(prof, funcs, npts):
    """The kernel function with the largest device time per step (summed over all of its
    launch classes), with its algorithmic bytes and time per step."""
    per = {}
    for cls, (ms, nl) in prof.items():
        if nl <= 0 or cls not in funcs:
            continue
        fn, bpp = funcs[cls]
        t, b, n = per.get(fn, (0.0, 0.0, 0.0))
        per[fn] = (t + ms * nl, b + bpp * npts * nl, n + nl)
    fn = max(per, key=lambda k: per[k][0])
    return fn, per[fn], {k: round(v[0] / sum(x[0] for x in per.values()), 4) for k, v in per.items()}


def captured_traffic(fn):
    """DRAM bytes per launch of kernel function `fn` from the capture file, or None."""
    if not os.path.exists(TRAFFIC_FILE):
        return None
    with open(TRAFFIC_FILE) as f:
        for line in f:
            if line.startswith("traffic "):
                name, val = line[len("traffic "):].rsplit(" ", 1)
                if name.strip() == fn:
                    return float(val)
    return None


def host_cpu():
    """CPU model and logical core count of this host."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


def lid_sample(cs, GattDNS, nsteps=1000, cpu_steps=200):
    """Config 1: the 128^2 lid-driven cavity from rest, nsteps RK4 steps at CFL 0.5 on the GPU
    (wall clock of one gatt_run), and the CPU oracle on a bounded sample of the same steps."""
    import oracle
    c = cs.lid_driven(n=128)
    f = cs.uniform_flow(c)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    g = GattDNS(c)
    g.upload(f)
    g.apply_bound_cond(0.0)
    g.run(5, 0.0, dt)
    g.upload(f)
    g.apply_bound_cond(0.0)
    t0 = time.perf_counter()
    g.run(nsteps, 0.0, dt)
    el = time.perf_counter() - t0
    g.close()
    o = oracle.Oracle(c)
    st = o.new_state(o.apply_bound_cond(f, 0.0))
    t0 = time.perf_counter()
    for k in range(cpu_steps):
        o.step(st, k * dt, dt)
    cel = (time.perf_counter() - t0) / cpu_steps * nsteps
    npts = c.nx * c.ny
    return {"workload": "lid-driven cavity 128^2 from rest, CFL 0.5, %d RK4 steps" % nsteps, "gpu_s": el,
            "gpu_mpoint_stages_s": npts * STAGES * nsteps / el / 1e6, "cpu_s_est": cel,
            "cpu_cores": o.lib.orc_num_threads(), "gpu_over_cpu": cel / el,
            "sample": "GPU: all %d steps in one gatt_run (launch-bound at this size); CPU oracle: %d steps "
                      "timed, scaled to %d" % (nsteps, cpu_steps, nsteps)}


def cavity_sample(cs, GattDNS, nsteps=20000, chunk=1000, cpu_steps=10):
    """Config 3 on its full grid: the 800x300 boundary layer over a cavity with buffer zones
    and SFD, from the Blasius start at CFL 0.5, nsteps RK4 steps in chunks of `chunk` (one
    gatt_run each), with the residual (max-change of the last step of each chunk, the
    log.txt residual of main.F90:414-420); and the CPU oracle on a bounded sample of steps."""
    import oracle
    c = cs.boundary_layer_cavity()
    f = cs.blasius_flow(c)
    o = oracle.Oracle(c)
    f = o.apply_bound_cond(f, 0.0)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    g = GattDNS(c)
    g.upload(f)
    g.run(2, 0.0, dt)  # graph capture
    g.upload(f)
    hist = []
    el, done = 0.0, 0
    while done < nsteps:
        k = min(chunk, nsteps - done)
        t0 = time.perf_counter()
        mc = g.run(k, done * dt, dt)
        el += time.perf_counter() - t0
        done += k
        hist.append([done, float(np.max(mc[0]))])
        if not np.all(np.isfinite(mc)):
            break
    g.close()
    st = o.new_state(f)
    t0 = time.perf_counter()
    for k in range(cpu_steps):
        o.step(st, k * dt, dt)
    cel = (time.perf_counter() - t0) / cpu_steps * done
    npts = c.nx * c.ny
    return {"workload": "boundary layer over a cavity 800x300, buffers 40/30/40, SFD (X 0.02, Delta 15)",
            "dt": dt, "steps": done, "gpu_s": el, "gpu_ms_per_step": el / done * 1e3,
            "gpu_mpoint_stages_s": npts * STAGES * done / el / 1e6, "cpu_s_est": cel,
            "cpu_cores": o.lib.orc_num_threads(), "gpu_over_cpu": cel / el,
            "residual_history": hist, "max_change_last": [float(x) for x in mc[0]],
            "sample": "%d steps from the Blasius start (t = %.3f); residual = max over variables of the last "
                      "step's max-change per chunk; CPU oracle: %d steps timed, scaled" % (done, done * dt, cpu_steps)}


def time_steps(g, dt, k):
    """ms per step of k back-to-back gatt_run steps (gatt_run returns after synchronising the
    context's own stream, so the wall time brackets the device work)."""
    g.run(2, 0.0, dt)
    t0 = time.perf_counter()
    g.run(k, 0.0, dt)
    return (time.perf_counter() - t0) * 1e3 / k


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from gatt_dns_b200 import build as bld
    if rank == 0:
        bld.build()
    if world > 1:
        dist.barrier()
    from gatt_dns_b200 import case as cs
    from gatt_dns_b200.solver import GattDNS
    from gatt_dns_b200.shard import max_over_ranks

    c = cs.periodic_box(n=args.n)
    f = cs.solenoidal_turbulence(c, seed=1234 + rank)
    dt = c.cfl_dt(f["U"], f["V"], f["W"], 0.5)
    stream = torch.cuda.Stream()
    g = GattDNS(c, stream=stream.cuda_stream)
    tuned = {} if args.no_autotune else g.autotune(reps=3)  # line-solve family and row blocks per set
    npts = c.npts

    # pinned host buffers for the end-to-end leg
    pinned = {k: torch.from_numpy(np.ascontiguousarray(f[k].ravel(order="F"))).pin_memory() for k in "UVWRE"}
    host = {k: pinned[k].numpy().reshape((c.nx, c.ny, c.nz), order="F") for k in "UVWRE"}
    pinned_out = {k: torch.empty(npts, dtype=torch.float64).pin_memory() for k in "UVWRE"}
    host_out = {k: pinned_out[k].numpy().reshape((c.nx, c.ny, c.nz), order="F") for k in "UVWRE"}
    g.upload(host)

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up (also captures the step graphs)
    g.run(max(args.warmup, 3), 0.0, dt)
    t = max(args.warmup, 3) * dt

    # ---- device-resident timed region -------------------------------------------
    sampler = ClockSampler(local)
    if not args.no_clocks:
        sampler.start()
        time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    l0 = g.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    mc = g.run(args.steps, t, dt)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop() if not args.no_clocks else None
    launches = g.kernel_launches() - l0
    ms = ev0.elapsed_time(ev1)
    t += args.steps * dt
    ms_max = max_over_ranks(ms, dist if world > 1 else None, device="cuda")
    value = world * npts * STAGES * args.steps / (ms_max / 1e3) / 1e6

    # ---- end-to-end through the C-ABI with host buffers ------------------------------
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    g.upload(host)                       # H2D of the flow from pinned memory
    for s in range(args.steps):
        g.step(t + s * dt, dt)           # per step: params H2D, graph, maxChange D2H + sync
    g.download(out=host_out)             # D2H of the flow into pinned memory
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    e_ms = max(e0.elapsed_time(e1), wall * 1e3)
    e2e_value = world * npts * STAGES * args.steps / (max_over_ranks(e_ms, dist if world > 1 else None,
                                                                     device="cuda") / 1e3) / 1e6
    field_bytes = 5 * npts * 8
    h2d = (field_bytes + args.steps * 24) / args.steps
    d2h = (field_bytes + args.steps * 5 * 8) / args.steps

    # ---- per-kernel timing for the roofline (CUDA events around each launch) ------------
    prof = g.profile_kernels(t, dt, nsteps=2)
    funcs = kernel_functions(c, tuned)
    dom, (dom_ms_step, dom_bytes_step, dom_launches), shares = dominant_kernel(prof, funcs, npts)
    peak, peak_kind = measured_peaks()
    achieved = dom_bytes_step / (dom_ms_step / 1e3) / 1e9
    step_ms = ms_max / args.steps
    stage_model = BYTES_PER_POINT_STAGE * npts * STAGES / (step_ms / 1e3) / 1e9
    traffic = captured_traffic(dom) if args.n == 128 else None

    line = {"metric": "FP64 Mpoint-stages/s (RK4 step, 128^3 periodic box)", "value": value,
            "unit": "Mpoint-stages/s", "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded solenoidal field, E(k)~k^4 exp(-2(k/4)^2), u_rms=1)",
            "config": {"workload": "periodic_box_%d^3_rk4_step" % args.n, "grid": [args.n] * 3, "Re": 1600,
                       "Ma": 0.3, "scheme": "SL4 compact + 10th-order filter (alpha 0.49)",
                       "per_gpu": "one independent box per GPU",
                       "parallelism": "batch-sharded replicas x%d" % world,
                       "l2": "inputs larger than L2 (working set %.2f GB per GPU > 126 MB)" % (
                           (5 * 5 + 15 + 9 + 12 + 2) * npts * 8 / 1e9)},
            "e2e": {"value": e2e_value, "unit": "Mpoint-stages/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "path": "gatt_upload from pinned host, K x gatt_step (host maxChange each step), gatt_download"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": traffic,
                         "traffic_source": ("ncu capture of this workload (dram__bytes_read.sum + "
                                            "dram__bytes_write.sum per launch), profiles/"
                                            + os.path.basename(TRAFFIC_FILE)) if traffic else None,
                         "bytes_algorithmic": dom_bytes_step / dom_launches, "launches_per_step": dom_launches,
                         "ms_per_launch": dom_ms_step / dom_launches, "peak_source": peak_kind,
                         "step_sweep_model_gbs": stage_model, "step_sweep_model_frac": stage_model / peak},
            "kernel_time_shares": shares,
            "kernels_ms_per_launch": {k: round(v[0], 5) for k, v in prof.items() if v[1] > 0},
            "autotuned": {"%s/%s" % ("xyz"[d - 1], ("deriv", "filter", "derivT_lhs", "derivT_band", "filterT_lhs",
                                                   "filterT_band")[k]): [fam, P, round(us, 1)]
                          for (d, k), (fam, P, us) in tuned.items()},
            "max_change_last": [float(x) for x in mc[0]]}
    if clocks:
        line["clocks"] = clocks
    if not args.kernels_only and not args.no_arnoldi:
        # config 4: the batched Arnoldi problems on the box after 200 steps, sharded across ranks
        g.upload(host)
        g.run(200, 0.0, dt)
        base200 = g.download()
        g.close()
        line["arnoldi"] = [arnoldi_sample(cs, GattDNS, c, base200, 32, 2, 10, 4321,
                                          "32 problems on the %d^3 periodic box after 200 steps" % args.n,
                                          dist if world > 1 else None)]
        if world == 1:
            lid = cs.lid_driven(n=128)
            line["arnoldi"].append(arnoldi_sample(cs, GattDNS, lid, cs.uniform_flow(lid), 32, 2, 100, 4321,
                                                  "32 problems on the 128^2 lid-driven cavity (rest state base)"))
    if rank == 0 and world == 1 and not args.kernels_only:
        line["cpu_baseline"] = cpu_baseline_sample(c)
        if not args.no_adjoint:
            g.close()
            line["adjoint"] = adjoint_sample(cs, GattDNS)
        line["lid_driven"] = lid_sample(cs, GattDNS)
        line["cavity"] = cavity_sample(cs, GattDNS)
    if rank == 0:
        print(json.dumps(line), flush=True)
    g.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
