"""Benchmark: explicit DG time stepping on one B200 (and N replicas on N GPUs).

Workload (the largest single-GPU configuration): 3D linear advection,
a = (1, 0.7, 0.3), 64^3 periodic hexahedra on [0,1]^3, hpGEM's default basis
of order p = 3 (64 DoF per element, 16,777,216 DoF), classical RK4,
dt = 2e-4, FP64; initial condition the Gaussian bump exp(-|x-0.5|^2/0.01),
L2-projected.  Synthetic mesh from the structured description, so no data
files.

A "step" is one RK4 time step of the whole mesh (4 stage kernels).
  value   DoF-updates/s = elements * basis functions * steps / device time,
          state resident in HBM, CUDA events on the launching stream, max
          over ranks; each rank advances its own copy of the mesh
          (independent replicas, weak scaling).
  e2e     the same metric through the C ABI with host buffers: per e2e step,
          one full 200-step solve including the host->device copy of the
          initial coefficients (pinned) and the device->host copy of the result.
The five state vectors (134 MB each) exceed the 126 MB L2, so no flush is
needed between steps.

`forms` repeats the measurement in the FP32-mixed form (stage vectors and
contractions in FP32; solution, geometry and the Runge-Kutta accumulation in
FP64) and states for both forms the L2 error of the 200-step solution against
the exact translated bump u0(x - a t) (periodic wrap; rule of order 2p+2), and
for the mixed form its L2 distance and largest relative coefficient difference
to the FP64 solution.

Secondary legs in the same line (rank 0, one GPU): `tet_wave` (32^3 x 5
periodic tetrahedra, p = 2, acoustic wave with the upwind flux in both forms
and the central flux in FP64), `linear` (HpgemAPILinear's stored matrices on
the benchmark mesh, FP64 tensor-core tiles, roofline against cuBLAS DGEMM
measured in the same run), `batched` (512 seeded 2D problems in one batch) and
`served` (the seeded 2000-request Poisson stream through the serving loop at
200 requests/s in both forms, then at a sustainable load; p50/p99 latency).
`--only linear|tet_wave|served` runs one of them alone for profiling.

--impl reference times the CPU oracle (the restated hpGEM loop: quadrature
loops, per-element mass matrix rebuilt and LU-solved every stage) on all host
cores as independent replica processes, each on a 2^3 sample of the same mesh
family (same order, same per-element work), one RK4 step per bench step.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "DG DoF-updates/s FP64 vs FP32-mixed at stated error; served p50/p99 latency"
UNIT = "DoF-updates/s"
N_CELLS = 64
ORDER = 3
ADV = [1.0, 0.7, 0.3]
DT = 2e-4
SOLVE_STEPS = 200
# algorithmic bytes per DoF-update of one RK4 step (FP64), per stage launch:
# stage 1 reads u, writes k1 (16 B); stages 2-3 read u, k_{i-1}, write k_i
# (24 B each); stage 4 reads u, k3, k1, k2 and writes u^{n+1} (40 B; the k4
# store is switched off here, with it the stage moves 48 B).  State: 104 B.
# Plus per-stage geometry 4 * (G_e + (F/E) G_f) / nB = 4 * (80 + 3 * 48) / 64 = 14 B
B_STATE = 16.0 + 24.0 + 24.0 + 40.0
B_GEO = 4.0 * (8 * (3 * 3 + 1) + 3 * (8 * (3 + 1) + 16)) / 64.0
B_ALG = B_STATE + B_GEO
# FP32-mixed form: stage vectors stored in FP32 (u and u^{n+1} stay FP64):
# 12 + 16 + 16 + 28 = 72 B of state
B_ALG_MIXED = (8.0 + 4) + (8 + 4 + 4) + (8 + 4 + 4) + (8 + 3 * 4 + 8) + B_GEO


def description(n):
    return "structured 1 3\n%d %d %d\n0 0 0\n1 1 1\nrectangular\ntrue true true\n" % (n, n, n)


def bump(x):
    return np.exp(-((x - 0.5) ** 2).sum(axis=1) / 0.01)


def config():
    return {"workload": "advection3d_hex64_p3_rk4", "mesh": "64^3 periodic hexahedra",
            "order": ORDER, "dof": N_CELLS ** 3 * (ORDER + 1) ** 3, "velocity": ADV, "dt": DT,
            "tableau": "RK4_4", "form": "fp64", "flush": "none: 5 state vectors of 134 MB exceed L2"}


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def traffic_per_dof_step():
    """DRAM bytes (read + write) per DoF of one RK4 step of the stage kernel, summed over
    its 4 launches, from the committed ncu summary of the same workload, if any."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get("tensor_slice_hex64_p3_rk4_dram_bytes_per_dof_step")
    except (OSError, ValueError):
        return None


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def cpu_sample_rate(budget_s=12.0):
    """The oracle on one core: 4^3 hexahedra, p = 3, RK4 steps until the budget is used."""
    from oracle.dg import ADVECTION, Problem
    from oracle.mesh import mesh_from_description

    n = 4
    prob = Problem(mesh_from_description(description(n)), ORDER, ADVECTION, a=ADV)
    u = prob.project(lambda x: bump(x)[:, None])
    steps, t0 = 0, time.perf_counter()
    while True:
        u = prob.step(u, DT, 1, "RK4_4")
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s or steps >= 1000:
            break
    return prob.n_dof * steps / el, "%d^3 hexahedra p=3 (%d DoF), %d RK4 steps, %.1f s" % (
        n, prob.n_dof, steps, el)


def _replica(args):
    n_steps, n_warm, barrier_time = args
    from oracle.dg import ADVECTION, Problem
    from oracle.mesh import mesh_from_description

    prob = Problem(mesh_from_description(description(2)), ORDER, ADVECTION, a=ADV)
    u = prob.project(lambda x: bump(x)[:, None])
    u = prob.step(u, DT, n_warm, "RK4_4") if n_warm else u
    while time.time() < barrier_time:
        time.sleep(0.001)
    t0 = time.perf_counter()
    u = prob.step(u, DT, n_steps, "RK4_4")
    return time.perf_counter() - t0, prob.n_dof


def run_reference(args):
    import multiprocessing as mp

    from oracle.build import build as build_oracle

    build_oracle()
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    start_at = time.time() + 5.0 + 0.5 * cores
    with ctx.Pool(cores) as pool:
        res = pool.map(_replica, [(args.steps, args.warmup, start_at)] * cores)
    wall = max(r[0] for r in res)
    dof = res[0][1]
    value = dof * cores * args.steps / wall
    sample = ("%d replica processes, each 2^3 periodic hexahedra p=3 (%d DoF), %d timed RK4 "
              "steps after %d warm-up" % (cores, dof, args.steps, args.warmup))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config(),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def exact_translated(x, t):
    """u0(x - a t) with the periodic wrap of the unit cube."""
    return bump(np.mod(x - t * np.asarray(ADV), 1.0))


def run_ours(args):
    import torch

    import hpgem_b200
    from hpgem_b200 import _native

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    def barrier():
        if dist is not None:
            dist.barrier()

    from hpgem_b200 import replicas

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, "cuda")

    # a dedicated (non-default) stream: the library launches on it, the events are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    def measure(precision, sample_clocks):
        """K timed steps with the state resident, then the end-to-end solve (host in, host out)."""
        solver = hpgem_b200.Advection(3, ORDER, ADV, tableau="RK4_4", precision=precision)
        solver.readMesh(description(N_CELLS))
        h = solver.handle
        ndof = h.vector_length
        solver.setInitialSolution(bump)
        u0 = solver.getTimeIntegrationVector(0).reshape(-1).copy()
        h.set_stream(stream.cuda_stream)
        h.set_store_last_stage(False)
        assert h.kernel_kind == "tensor"
        t = h.step(0.0, DT, max(args.warmup, 3))
        torch.cuda.synchronize()
        sampler = ClockSampler(dev) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.2)
        launches0 = h.launch_count
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        t = h.step(t, DT, args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
        clocks = sampler.stop() if sampler else None
        launches = h.launch_count - launches0
        ms = max_over_ranks(ev0.elapsed_time(ev1))
        # end to end: host initial coefficients in, host solution out, one 200-step solve each
        host_in = torch.from_numpy(u0).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        reps = 2
        h.step(0.0, DT, 1)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            h.set_state_ptr(0, host_in.data_ptr())
            h.step(0.0, DT, SOLVE_STEPS)
            h.get_state_ptr(0, host_out.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1) / reps)
        u_end = host_out.numpy().copy()
        return dict(solver=solver, ndof=ndof, ms=ms, launches=launches, clocks=clocks,
                    e2e_ms=e2e_ms, u_end=u_end)

    f64 = measure(_native.PRECISION_FP64, True)
    ndof = f64["ndof"]
    value = ndof * args.steps * world / (f64["ms"] / 1e3)
    e2e_value = ndof * SOLVE_STEPS * world / (f64["e2e_ms"] / 1e3)
    f32 = measure(_native.PRECISION_FP32, False)

    # errors of the 200-step solutions (rank 0; every rank runs the same replica)
    forms = {}
    if rank == 0:
        s64 = f64["solver"]
        T = SOLVE_STEPS * DT
        err64 = s64.computeTotalError(exact_translated, T)
        s64.setTimeIntegrationVector(0, f32["u_end"])
        err32 = s64.computeTotalError(exact_translated, T)
        d = s64.l2Distance(f32["u_end"], f64["u_end"])
        rel = float(np.abs(f32["u_end"] - f64["u_end"]).max() / np.abs(f64["u_end"]).max())
        for name, r, extra in (("fp64", f64, {"l2_error_vs_exact": err64}),
                               ("fp32_mixed", f32, {"l2_error_vs_exact": err32, "l2_distance_to_fp64": d,
                                                    "max_rel_coef_diff_vs_fp64": rel})):
            forms[name] = dict({"value": ndof * args.steps * world / (r["ms"] / 1e3),
                                "ms_per_step": r["ms"] / args.steps,
                                "e2e_value": ndof * SOLVE_STEPS * world / (r["e2e_ms"] / 1e3),
                                "solve_steps": SOLVE_STEPS}, **extra)
        forms["fp32_mixed"]["stage_vector_bytes"] = 4
        forms["fp32_mixed"]["algorithmic_bytes_per_dof_update"] = B_ALG_MIXED
        forms["fp32_mixed"]["roofline_frac"] = (B_ALG_MIXED * forms["fp32_mixed"]["value"] / world / 1e9
                                                / measured_peak_hbm()[0])
        forms["note"] = ("errors of the 200-step solve; the FP64 GPU form equals the oracle to 1e-12 on "
                         "every parity case, so it is the reference at this size")

    peak, peak_kind = measured_peak_hbm()
    step_s = (f64["ms"] / 1e3) / args.steps
    achieved = B_ALG * ndof / step_s / 1e9
    tr = traffic_per_dof_step()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": f64["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(config(), parallelism="replicas%d" % world),
            "clocks": f64["clocks"],
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": ndof * 8,
                    "d2h_bytes_per_step": ndof * 8, "step": "one %d-step solve" % SOLVE_STEPS,
                    "ms_per_step": f64["e2e_ms"], "finite": bool(np.isfinite(f64["u_end"]).all())},
            "gpu_launches": int(f64["launches"]),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "kernel": "tensor_slice (4 launches per step, back to back in one graph)",
                         "algorithmic_bytes_per_dof_update": B_ALG,
                         "traffic": (tr * ndof if tr else None),
                         "traffic_unit": "bytes per RK4 step (4 launches)"},
            "forms": forms}
    if rank == 0 and world == 1 and not args.no_batched:
        line["tet_wave"] = run_tet_wave(args, stream)
        line["linear"] = run_linear(args, stream)
        # split-BF16 of this mesh: the matrix-free handle with HGG_PRECISION_BF16X3 folds its
        # operator into the per-element matrices the stored-matrix leg runs on tcgen05
        bf = dict(line["linear"]["forms"]["split_bf16"])
        bf["measured_as"] = ("the linear leg's split-BF16 form (the same operator, folded; same mesh, "
                             "bump and dt)")
        line["forms"]["split_bf16"] = bf
        line["batched"] = run_batched_forms(args, stream)
        line["batched"]["forms"]["split_bf16"] = {
            "unavailable": "split-BF16 runs only on tiles of 128 elements with equal matrices; most of the "
                           "512 meshes (8^2..128^2 cells) do not form them"}
    if rank == 0 and world == 1 and not args.no_served:
        line["served"] = run_served_legs(args)
        line["served"]["forms"]["split_bf16"] = {
            "unavailable": "split-BF16 needs tiles of 128 elements with equal matrices; the stream's "
                           "small meshes (from 1e3 DoF) do not form them"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample = cpu_sample_rate()
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": sample}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batched(args, stream, precision=0):
    """512 independent 2D advection problems (quads/triangles, p 1..5, 8^2..128^2, per-problem
    velocity and CFL dt), RK4, 100 steps each, advanced together by one batch."""
    import torch

    import hpgem_b200
    from hpgem_b200 import workloads

    specs = workloads.batched_problems()
    # host set-up of the 512 handles on a pool of threads (the library's set-up is
    # thread-safe per handle; the ctypes calls release the interpreter lock)
    from concurrent.futures import ThreadPoolExecutor
    setup_threads = max(1, min(16, os.cpu_count() or 4))
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=setup_threads) as pool:
        solvers = list(pool.map(lambda sp: workloads.make_solver(sp, precision=precision), specs))
    setup_s = time.perf_counter() - t0
    total_dof = sum(workloads.dof(sp) for sp in specs)
    warm = 3
    steps = specs[0]["steps"]
    batch = hpgem_b200.Batch(len(specs))
    u0 = [s.getTimeIntegrationVector(0).reshape(-1).copy() for s in solvers]
    for s, sp in zip(solvers, specs):
        batch.add(s, sp["dt"], steps + warm + 1)
    batch.step(warm)  # first steps: tables, autotuning, graph capture
    batch.synchronize()
    # one step class after class, each timed with CUDA events: the per-class breakdown
    info, class_ms = batch.class_info(), batch.profile_step()
    per_class = [dict(c, ms_per_step=float(ms), dof_updates_per_s=c["coefficients"] / (ms / 1e3))
                 for c, ms in zip(info, class_ms)]
    launches0 = batch.launch_count
    torch.cuda.synchronize()
    bstream = torch.cuda.ExternalStream(batch.cuda_stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    ev0.record(bstream)
    batch.step(steps)
    ev1.record(bstream)
    batch.synchronize()
    wall = time.perf_counter() - t0
    dev_s = ev0.elapsed_time(ev1) / 1e3
    launches = batch.launch_count - launches0
    # end to end through the public API: initial coefficients from the host into every
    # problem, the 100 steps, every solution back to the host
    for i, s in enumerate(solvers):
        batch.remove(i)
    t0 = time.perf_counter()
    for i, (s, sp) in enumerate(zip(solvers, specs)):
        s.setTimeIntegrationVector(0, u0[i])
        batch.add(s, sp["dt"], steps)
    batch.step(steps)
    batch.synchronize()
    outs = [s.getTimeIntegrationVector(0) for s in solvers]
    e2e = time.perf_counter() - t0
    finite = all(np.isfinite(o).all() for o in outs)
    classes = batch.num_classes
    batch.close()
    value = total_dof * steps / dev_s
    state_bytes = 72 if precision else 104  # RK4 state per DoF-update (geometry not counted)
    peak, peak_kind = measured_peak_hbm()
    res = {"workload": "512 2D advection problems, quads/triangles, p 1..5, 8^2..128^2 cells, "
                       "RK4, 100 steps each, seed 4",
           "value": value, "unit": UNIT, "dtype": "f32-mixed" if precision else "f64",
           "problems": len(specs), "dof": total_dof, "steps": steps, "device_s": dev_s, "wall_s": wall,
           "kernel_classes": classes, "gpu_launches": int(launches), "host_setup_s": setup_s,
           "host_setup_threads": setup_threads,
           "timing": "CUDA events on the batch's stream around the 100 steps (wall clock beside it)",
           "roofline": {"bound": "hbm", "achieved": state_bytes * value / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": state_bytes * value / 1e9 / peak, "peak_kind": peak_kind,
                        "algorithmic_bytes_per_dof_update": state_bytes,
                        "note": "RK4 state bytes only (the per-element geometry is not counted)"},
           "per_class": per_class,
           "e2e": {"value": total_dof * steps / e2e, "unit": UNIT, "wall_s": e2e,
                   "h2d_bytes": 8 * total_dof, "d2h_bytes": 8 * total_dof, "finite": bool(finite)}}
    return res, outs, solvers


def run_batched_forms(args, stream):
    """The batched set in both forms; the mixed form's error against the FP64 result."""
    r64, o64, s64 = run_batched(args, stream, 0)
    r32, o32, _ = run_batched(args, stream, 1)
    r32["max_rel_coef_diff_vs_fp64"] = max(float(np.abs(a - b).max() / np.abs(b).max()) for a, b in zip(o32, o64))
    r32["max_l2_distance_to_fp64"] = max(s.l2Distance(a, b) for s, a, b in zip(s64, o32, o64))
    return dict(r64, forms={"fp32_mixed": r32})


def run_tet_wave(args, stream):
    """3D acoustic wave on 32^3 x 5 periodic tetrahedra, p = 2 (6.55 M DoF), RK4, dt = 5e-4,
    seeded 3-mode Fourier pressure, zero velocity, upwind flux: DoF-updates/s over 20 steps in
    both forms, and the reference's central flux in FP64 beside it."""
    import torch

    import hpgem_b200

    rng = np.random.default_rng(20261203)
    ks, amps, phases = [], [], []
    while len(ks) < 3:
        k = rng.integers(-4, 5, size=3)
        if np.abs(k).max() >= 1:
            ks.append(k)
            amps.append(rng.uniform(0.5, 1.0))
            phases.append(rng.uniform(0, 2 * math.pi))
    ks, amps, phases = np.array(ks, float), np.array(amps), np.array(phases)

    def p0(x):
        q = (amps[None] * np.sin(2 * math.pi * x @ ks.T + phases[None])).sum(1)
        return np.concatenate([q[:, None], np.zeros((len(x), 3))], axis=1)

    d = hpgem_b200.structured_description([32, 32, 32], [0, 0, 0], [1, 1, 1], True, True)
    out = {}
    sols = {}
    for name, prec, flux in (("fp64", 0, "upwind"), ("fp32_mixed", 1, "upwind"), ("split_bf16", 2, "upwind"),
                             ("fp64_central", 0, "central")):
        s = hpgem_b200.AcousticWave(3, 2, c_inv=1.0, tableau="RK4_4", precision=prec, flux=flux).readMesh(d)
        h = s.handle
        h.set_stream(stream.cuda_stream)
        h.set_store_last_stage(False)
        s.setInitialSolution(p0)
        t = h.step(0.0, 5e-4, 3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        steps = 20
        launches0 = h.launch_count
        e0.record(stream)
        h.step(t, 5e-4, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        n = h.vector_length
        sols[name] = (s, s.getTimeIntegrationVector(0))
        out[name] = {"value": n / (ms / 1e3), "unit": UNIT, "dof": n, "ms_per_step": ms, "steps": steps,
                     "gpu_launches": int(h.launch_count - launches0), "kernel": h.kernel_kind,
                     "finite": bool(np.isfinite(sols[name][1]).all())}
    s64, u64 = sols["fp64"]
    for name in ("fp32_mixed", "split_bf16"):
        u = sols[name][1]
        out[name]["l2_distance_to_fp64"] = s64.l2Distance(u, u64)
        out[name]["max_rel_coef_diff_vs_fp64"] = float(np.abs(u - u64).max() / np.abs(u64).max())
    res = {"workload": "3D acoustic wave, 32^3 x 5 periodic tetrahedra, p = 2, upwind flux, RK4, "
                       "dt = 5e-4, seeded 3-mode pressure, 23 steps", "dtype": "f64",
           "kernel": "dense_group_stage<double,3,4,10> (FP64: 32-element tiles of equal operators, "
                     "lane = element); dense_stage<float,3,4,1,10> (FP32-mixed: one thread per element row); "
                     "linear_umma_stage (split-BF16: the operator folded into per-element matrices, "
                     "128-element tiles on tcgen05, FP32 accumulation in tensor memory)"}
    res.update(out["fp64"])
    # roofline of the FP64 kernel: the state an RK4 step must move (stage inputs u and the
    # previous stage vector, neighbour traces from L2, the stage output; the final update
    # reads k1..k3 and writes u): 130 bytes per DoF-update, against the measured HBM copy
    peak, peak_kind = measured_peak_hbm()
    achieved = 130.0 * res["value"] / 1e9
    res["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "peak_kind": peak_kind, "algorithmic_bytes_per_dof_update": 130}
    res["forms"] = {"fp32_mixed": out["fp32_mixed"], "split_bf16": out["split_bf16"]}
    res["central_flux_fp64"] = out["fp64_central"]
    return res


def measured_fp64_gemm_tflops():
    """Dense FP64 peak measured here: cuBLAS DGEMM (torch.matmul, float64) at 8192^3."""
    import torch

    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record()
    for _ in range(reps):
        torch.matmul(a, b)
    e1.record()
    torch.cuda.synchronize()
    tflops = 2.0 * n ** 3 * reps / (e0.elapsed_time(e1) / 1e3) / 1e12
    del a, b
    torch.cuda.empty_cache()
    return tflops


def run_linear(args, stream):
    """HpgemAPILinear (stored element and face matrices) on the benchmark mesh: 64^3 periodic
    hexahedra, p = 3, the Gaussian bump, RK4, dt = 2e-4, 20 timed steps in both forms; the
    FP64 solution is compared with the matrix-free solver's after the same steps."""
    import torch

    import hpgem_b200

    nc = args.linear_cells
    d = hpgem_b200.structured_description([nc, nc, nc], [0, 0, 0], [1, 1, 1])
    a = [1.0, 0.7, 0.3]
    warm, steps = (args.warmup, args.steps) if args.only else (3, 20)
    out, sols = {}, {}
    for name, prec in (("fp64", 0), ("fp32_mixed", 1), ("split_bf16", 2)):
        t0 = time.time()
        s = hpgem_b200.HpgemAPILinear(3, 3, "advection", advection=a, tableau="RK4_4", precision=prec).readMesh(d)
        setup = time.time() - t0
        h = s.handle
        h.set_stream(stream.cuda_stream)
        h.set_store_last_stage(False)
        s.setInitialSolution(lambda x: np.exp(-((x - 0.5) ** 2).sum(axis=1) / 0.01))
        t = h.step(0.0, DT, warm)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = h.launch_count
        e0.record(stream)
        h.step(t, DT, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        n = h.vector_length
        sols[name] = (s, s.getTimeIntegrationVector(0))
        out[name] = {"value": n / (ms / 1e3), "unit": UNIT, "dof": n, "ms_per_step": ms, "steps": steps,
                     "setup_s": setup, "gpu_launches": int(h.launch_count - launches0),
                     "kernel": h.kernel_kind, "finite": bool(np.isfinite(sols[name][1]).all())}
        del h
    # the matrix-free solver after the same warm-up + timed steps
    free = hpgem_b200.Advection(3, 3, a, tableau="RK4_4").readMesh(d)
    free.setInitialSolution(lambda x: np.exp(-((x - 0.5) ** 2).sum(axis=1) / 0.01))
    free.handle.step(0.0, DT, warm + steps)
    u_free = free.getTimeIntegrationVector(0)
    s64, u64 = sols["fp64"]
    rows, slots = 64, 6
    flop = 2.0 * rows * (1 + slots) * 4  # per DoF-update: 1 + 6 matrices of 64 x 64, 4 stages
    peak = measured_fp64_gemm_tflops()
    achieved = out["fp64"]["value"] * flop / 1e12
    res = {"workload": "HpgemAPILinear advection, %d^3 periodic hexahedra, p = 3, RK4, dt = 2e-4, "
                       "Gaussian bump, %d timed steps after %d" % (nc, steps, warm),
           "dtype": "f64", "kernel": "linear_tile_stage (FP64 DMMA m8n8k4, 64-element tiles)"}
    res.update(out["fp64"])
    res["l2_distance_to_matrix_free"] = s64.l2Distance(u64, u_free)
    res["max_rel_coef_diff_vs_matrix_free"] = float(np.abs(u64 - u_free).max() / np.abs(u_free).max())
    res["roofline"] = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                       "frac": achieved / peak, "peak_kind": "cuBLAS DGEMM 8192^3 measured in this run",
                       "algorithmic_flop_per_dof_update": flop}
    for name in ("fp32_mixed", "split_bf16"):
        u = sols[name][1]
        out[name]["l2_distance_to_fp64"] = s64.l2Distance(u, u64)
        out[name]["max_rel_coef_diff_vs_fp64"] = float(np.abs(u - u64).max() / np.abs(u64).max())
    res["forms"] = {"fp32_mixed": out["fp32_mixed"], "split_bf16": out["split_bf16"]}
    return res


def run_served(args, precision=0, n=None, rate=200.0):
    """Poisson stream (seed 5) of 2D/3D advection and acoustic-wave solves, 1e3..2e6 DoF,
    p 1..4, 50..2000 steps, replayed in real time into the server; at 200 requests/s, or
    the same requests with their arrival times stretched to a lower rate."""
    import hpgem_b200
    from hpgem_b200 import workloads

    specs = workloads.served_requests(n=n or args.served_requests, rate=rate)
    setup_threads = max(2, min(16, (os.cpu_count() or 4) // 2))
    server = hpgem_b200.Server(budget_bytes=48 << 30, max_chunk=args.served_chunk, setup_threads=setup_threads)

    def desc(sp):
        d = len(sp["cells"])
        return hpgem_b200.structured_description(sp["cells"], [0.0] * d, [1.0] * d, sp["triangular"], True)

    ids = []
    t_start = time.perf_counter()
    for sp in specs:
        delay = sp["arrival"] - (time.perf_counter() - t_start)
        if delay > 0:
            time.sleep(delay)
        d = len(sp["cells"])
        u0 = sp["u0"]
        if sp["physics"] == "advection":
            fn, nv = u0, 1
        else:
            fn, nv = (lambda x, u0=u0, d=d: np.concatenate([u0(x)[:, None], np.zeros((len(x), d))], axis=1)), d + 1
        ids.append(server.submit(desc(sp), sp["order"], sp["physics"], sp["params"], sp["dt"], sp["steps"],
                                 initial=fn, n_vars=nv, precision=precision))
    lat, done_t, sub_t = [], [], []
    for rid in ids:
        ok, _, l = server.poll(rid, wait=True, result=False)
        t = server.times(rid)
        lat.append(l)
        sub_t.append(t[0])
        done_t.append(t[3])
        server.release(rid)
    stats = server.stats()
    server.stop()
    span = max(done_t) - min(sub_t)
    lat = np.array(lat)
    return {"workload": "Poisson stream, %g requests/s, %d requests, seed 5: 2D/3D advection and "
                        "acoustic wave, 1e3..2e6 DoF, p 1..4, 50..2000 steps" % (rate, len(specs)),
            "value": stats["dof_updates"] / span, "unit": UNIT, "dtype": "f32-mixed" if precision else "f64",
            "requests": len(specs), "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
            "span_s": span, "dof_updates": stats["dof_updates"], "chunks": stats["chunks"],
            "gpu_thread_s": {"stepping": stats["gpu_thread_step_s"], "joining_retiring": stats["gpu_thread_members_s"],
                             "idle": stats["gpu_thread_idle_s"]},
            "joining_retiring_parts_s": {"joins": stats["gpu_thread_join_s"],
                                         "tables_and_captures": stats["gpu_thread_tables_s"]},
            "retire_thread_s": stats["retire_thread_s"], "retire_copyback_s": stats["retire_copyback_s"],
            "device_chunk_s": stats["device_chunk_s"],
            "device_busy_frac": stats["device_chunk_s"] / span,
            "setup_threads": setup_threads, "budget_bytes": 48 << 30, "steps_per_chunk": args.served_chunk,
            "offered_dof_updates_per_s": sum(workloads.dof(sp) * sp["steps"] for sp in specs)
            / max(specs[-1]["arrival"], 1e-9),
            "timing": "host steady clock, latency = done - submit (set-up, queueing, steps, copy back)"}


def run_served_legs(args):
    """The overloaded stream (200 requests/s) in FP64 and FP32-mixed, then the better form
    at a sustainable load: the same requests arriving at a rate whose offered DoF-updates/s
    is 60 % of what the overloaded run served, so the latency is service time, not queue."""
    served = run_served(args, 0)
    print("served f64: " + json.dumps(served), file=sys.stderr, flush=True)
    mixed = run_served(args, 1)
    print("served f32-mixed: " + json.dumps(mixed), file=sys.stderr, flush=True)
    served["forms"] = {"fp32_mixed": mixed}
    if args.sustained_requests > 0:
        best, prec = (mixed, 1) if mixed["value"] > served["value"] else (served, 0)
        rate = 200.0 * 0.6 * best["value"] / best["offered_dof_updates_per_s"]
        sus = run_served(args, prec, n=args.sustained_requests, rate=rate)
        sus["load"] = "offered 60 %% of the overloaded run's served DoF-updates/s (%s form)" % best["dtype"]
        served["sustained"] = sus
    return served


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 512-problem batched leg")
    ap.add_argument("--no-served", action="store_true", help="skip the served request-stream leg")
    ap.add_argument("--served-requests", type=int, default=2000,
                    help="requests of the seeded stream to serve at 200 requests/s (the stream has 2000)")
    ap.add_argument("--served-chunk", type=int, default=6, help="the server's steps per chunk")
    ap.add_argument("--sustained-requests", type=int, default=500,
                    help="requests of the same stream served at a sustainable load (0: skip)")
    ap.add_argument("--only", choices=["linear", "tet_wave", "served"],
                    help="run one secondary leg alone (profiling): --steps / --warmup set its timed loop")
    ap.add_argument("--linear-cells", type=int, default=64,
                    help="cells per direction of the stored-matrix leg's hexahedral mesh")
    args = ap.parse_args()
    if args.only:
        import torch

        stream = torch.cuda.Stream()
        if args.only == "served":
            leg = run_served_legs(args)
        else:
            leg = run_linear(args, stream) if args.only == "linear" else run_tet_wave(args, stream)
        print(json.dumps(leg), flush=True)
        return
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        run_reference(args)
        return
    run_ours(args)


if __name__ == "__main__":
    main()
