"""Throughput benchmark of the IF-RK4 pseudo-spectral step (w, r1, r2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl qaf|reference] [--dtype f32|f64]
                    [--workload plain|ensemble|adjoint|control]

Workload: the "plain throughput" configuration — 1024 x 1024 periodic grid,
L = 16 pi, friction solver parameters Re = 1 (nu = 1), Rf = 0.1 (mu = 0.1),
Er = 1, lambda = 0.1, activity Ra = 1, IF-RK4 with dt = 5e-4, seeded random Q
~ U(-0.01, 0.01) (seed 1), w = 0; FP32 by default (--dtype f64 for FP64).
A bench step is one solver time step; the metric is grid-point steps per
second of the whole job.

Arms:
  qaf (default)   this library. `value`: the device-resident state advanced one
                  step at a time with CUDA events around each step and the L2
                  flushed (a 256 MiB write) between timed steps. `e2e`: the same
                  through the public API with host I/O every step — the activity
                  field uploaded from pinned memory (the control input of a
                  closed-loop run; on a copy stream, double-buffered, so that
                  step k+1's upload overlaps step k) and the step's
                  energy/enstrophy read back; one event pair around all steps,
                  uploads, read-backs and L2 flushes.
  reference       the reference's own CUDA build (oracle/_ref, built from its
                  unmodified headers; FP32 through the macro shim, FP64 as
                  shipped) timed on the same GPU with CUDA events. The reference
                  has no CPU implementation of the path.

Multi-GPU: the path does not shard (one grid per GPU); N GPUs run N
independent replicas under torchrun, value = total over ranks / max time.

--workload ensemble: 256 instances (seeded draw: N ~ U{64,128,256},
activity ~ U(0.5,2), friction ~ U(0.01,0.5)), FP32, IF-RK4 dt = 1e-3, the
other parameters as above; metric sum_i N_i^2 * steps / s. `value` is the
batched stepper (one CUDA graph per step); `looped` is the plain solver
looped over the same instances. Under torchrun the instances are sharded
over ranks (strong scaling, no exchange while stepping).

--workload adjoint: 256 x 256, FP32, 2000 IF-RK4 steps dt = 1e-3, activity
Ra(x) = 1 + 0.1 * (unit-variance Gaussian-smoothed N(0,1) noise, width 4
cells, seed 2), loss = mean enstrophy of the states after the last 100 steps,
checkpoints every 64 steps. A bench step is one forward + backward pass of
the whole horizon (--steps is capped at 5, 3 warm-up passes). `value` is
(adjoint + recompute time) / (plain forward time); also reported: the
directional derivatives of the FP32 and FP64 adjoint gradients against
central differences of the FP64 forward on 16 random directions.

--workload control: the batched forward + adjoint control loop — 64
instances of 256 x 256 FP32, each with its own activity field Ra_k(x) as
above (seeds 100..163) and its own seeded initial Q, 1000-step horizon,
gradient descent on each instance's terminal enstrophy. A bench step is one
gradient-descent iteration of all 64 instances (forward, recompute + adjoint,
update). `value`: instance-iterations per second; `looped`: one instance's
iteration through the single-instance adjoint, times 64.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nature-control_b200"))

METRIC = "grid-pt*steps/s at 1024^2, IF-RK4 (w, r1, r2)"
UNIT = "grid-pt*steps/s"
N_GRID = 1024
L = 16 * 3.141592653589793
DT = 5e-4
SEED = 1
FALLBACK_HBM_GBS = 6650.0
ENS_COUNT = 256
ENS_SEED = 3
ENS_DT = 1e-3
ENS_METRIC = "sum_i N_i^2*steps/s, 256-instance mixed-size ensemble, IF-RK4"
ADJ_N, ADJ_STEPS, ADJ_DT, ADJ_K, ADJ_WINDOW, ADJ_SEED = 256, 2000, 1e-3, 64, 100, 2
ADJ_METRIC = "(adjoint + recompute) time / forward time, 256^2 FP32, 2000 IF-RK4 steps, K=64"
CTL_N, CTL_INST, CTL_STEPS, CTL_K, CTL_LR = 256, 64, 1000, 50, 0.05
CTL_METRIC = "gradient-descent instance-iterations/s, 64 x 256^2 FP32, 1000-step horizon, terminal enstrophy"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["qaf", "reference"], default="qaf")
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32")
    ap.add_argument("--n", type=int, default=N_GRID)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=2)
    ap.add_argument("--workload", choices=["plain", "ensemble", "adjoint", "control"], default="plain")
    ap.add_argument("--horizon", type=int, default=CTL_STEPS, help="control workload: steps per rollout")
    ap.add_argument("--adj-steps", type=int, default=ADJ_STEPS, help="adjoint workload: steps per rollout")
    ap.add_argument("--no-fd", action="store_true", help="adjoint workload: skip the finite-difference check")
    ap.add_argument("--no-tune", action="store_true",
                    help="ensemble, adjoint and control workloads: keep the built-in launch shapes")
    ap.add_argument("--shapes", default=None,
                    help="adjoint workload: launch shapes to use instead of tuning, e.g. col:e8m4,row:e8r2 "
                         "(to profile the shapes a tuned run reported)")
    ap.add_argument("--instances", type=int, default=ENS_COUNT)
    ap.add_argument("--no-extras", action="store_true",
                    help="plain workload: skip the shortened FP64, adjoint and ensemble measurements")
    return ap.parse_args()


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap,utilization.gpu"

    def __init__(self, local_rank):
        import torch
        self.uuid = None
        try:
            self.uuid = str(torch.cuda.get_device_properties(local_rank).uuid)
            if not self.uuid.startswith("GPU-"):
                self.uuid = "GPU-" + self.uuid
        except Exception:
            pass
        self.proc = None

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd.insert(1, f"--id={self.uuid}")
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[2:7], float(parts[7]) if parts[7] not in ("[N/A]", "") else 0.0))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        loaded = [r for r in rows if r[3] > 0] or rows
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in loaded:
            for nm, v in zip(names[1:], r[2][1:]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(loaded)}


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def plain_config(n, world):
    """The plain workload's config, the same dict in both arms."""
    return {"workload": f"plain throughput {n}x{n}, L=16pi, IF-RK4 dt={DT}, Re=1 Rf=0.1 Er=1 lambda=0.1 Ra=1",
            "grid": n, "integrator": "IF-RK4", "dt": DT, "seed": SEED, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 between timed steps (qaf: a 256 MiB write flushes it; the reference's "
                  "22-field working set, ~185 MB in FP32, exceeds it)"}


def traffic_of(kernel):
    """Per-launch DRAM bytes (read + write) of `kernel` from profiles/traffic.txt
    (ncu captures of the current kernels) and the commit they were captured at."""
    tpath = os.path.join(ROOT, "profiles", "traffic.txt")
    traffic, commit = None, None
    if os.path.exists(tpath):
        for line in open(tpath):
            f = line.split()
            if line.startswith("# captured at"):
                commit = f[-1]
            elif len(f) == 2 and not line.startswith("#") and f[0] == kernel:
                traffic = float(f[1])
    return traffic, commit


def cpu_baseline(n, steps, dtype_name):
    """The FP64 host oracle (a restatement of the reference's scheme) on the
    host cores, on a bounded sample of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    p = O.params(n=n, L=L, dt=DT)
    s0 = O.initial_spectra(SEED, n)
    O.step(p, *s0, 1)          # warm the FFT plans
    t0 = time.perf_counter()
    final = O.step(p, *s0, steps)
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("QAF_ORACLE_THREADS", os.cpu_count() or 1))
    line = {"value": n * n * steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} IF-RK4 steps of the {n}^2 workload in FP64 ({dt:.1f} s) with the host oracle, "
                      f"which follows the reference's operation sequence (~120 2D FFTs per step)"}
    return line, (O, p, final)


def spectrum_vs_oracle(mesh, qaf, oracle_run, steps, nshells=64):
    """Energy spectrum, energy and enstrophy of the GPU state after `steps` steps of the
    workload against the oracle's (the state the CPU-baseline leg computed)."""
    import numpy as np
    O, p, final = oracle_run
    pq = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=DT, q_lin=1.0, advect_omega=1)
    mesh.load(*mesh.random_q(SEED))
    mesh.advance(pq, steps)
    w, _, _ = mesh.store()
    e, z, spec = mesh.diagnostics(w, nshells)
    eo, zo, speco = O.diagnostics(p, final[0], nshells)
    big = speco > 1e-6 * speco.max()
    return {"steps": steps, "shells": nshells,
            "max_rel_err_shells": float(np.max(np.abs(spec[big] - speco[big]) / speco[big])),
            "energy_rel_err": abs(e - eo) / abs(eo), "enstrophy_rel_err": abs(z - zo) / abs(zo),
            "reference": "FP64 host oracle, same seeded initial state"}


def run_qaf(a, world, rank, local):
    import torch

    import qaf

    dtype = qaf.F32 if a.dtype == "f32" else qaf.F64
    n = a.n
    mesh = qaf.Mesh(n, lx=L, dtype=dtype)
    p = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=DT, q_lin=1.0, advect_omega=1)
    state = mesh.random_q(SEED)
    mesh.load(*state)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    # ---- device-resident throughput -------------------------------------
    for _ in range(a.warmup):
        mesh.advance(p, 1)
    barrier(world)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    l0 = mesh.launch_count()
    with ClockSampler(local) as clk:
        barrier(world)
        for e0, e1 in ev:
            flush.zero_()
            e0.record()
            mesh.advance(p, 1)
            e1.record()
        barrier(world)
    launches = mesh.launch_count() - l0
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    ms = max_over_ranks(ms, world)
    mesh.check_finite()
    value = world * n * n * a.steps / (ms * 1e-3)

    # ---- per-kernel timing for the roofline (CUDA events on the launching stream)
    row_ms, col_ms, _ = mesh.advance_timed(p, max(4, min(a.steps, 50)))
    real_b = 4 if dtype == qaf.F32 else 8
    ca = (n // 2 + 1) * n * 2 * real_b                 # one complex spectral array
    # algorithmic bytes per launch (three-pass model): row pass reads 9 and writes 11
    # arrays; the column pass (combine + stage update + next stage's inverse) moves 35
    kern = {"row": (row_ms, 20 * ca), "column": (col_ms, 35 * ca)}
    dom = max(kern, key=lambda k: kern[k][0])
    k_ms, k_bytes = kern[dom]
    peak, peak_kind = peaks()
    achieved = k_bytes / (k_ms * 1e-3) / 1e9
    traffic, traffic_commit = traffic_of(f"{dom}_{a.dtype}_{n}")

    # ---- end to end through the public API, host I/O every step ----------
    # Step k's activity field is uploaded from pinned host memory on a copy
    # stream into device buffer k % 2 while step k - 1 runs; step k waits for
    # its upload, and its energy/enstrophy come back asynchronously. One event
    # pair brackets every step, upload and read-back, and the L2 flushes
    # between the steps.
    alpha_host = torch.ones((n, n), dtype=mesh.real_dtype).pin_memory()
    alpha_dev = [torch.empty((n, n), dtype=mesh.real_dtype, device="cuda") for _ in range(2)]
    pe = [qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=DT, alpha_field=alpha_dev[b]) for b in range(2)]
    main = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    ready = [torch.cuda.Event() for _ in range(2)]
    free = [torch.cuda.Event() for _ in range(2)]

    def upload(k):
        b = k % 2
        with torch.cuda.stream(copy):
            if k >= 2:
                copy.wait_event(free[b])           # the step that read this buffer is done
            alpha_dev[b].copy_(alpha_host, non_blocking=True)
            ready[b].record(copy)

    def e2e_steps_run(steps, diag_host):
        upload(0)
        for k in range(steps):
            if k + 1 < steps:
                upload(k + 1)                      # overlaps step k
            main.wait_event(ready[k % 2])
            mesh.advance(pe[k % 2], 1)
            free[k % 2].record(main)
            mesh.last_diagnostics_async(diag_host[k])
            if k + 1 < steps:
                flush.zero_()

    e2e_steps = max(50, a.steps)
    diag_host = torch.empty((e2e_steps, 2), dtype=torch.float64).pin_memory()
    e2e_steps_run(2, diag_host)                    # warm-up of the same pipeline
    torch.cuda.synchronize()
    barrier(world)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(main)
    copy.wait_event(t0)                            # the first upload starts inside the timed region
    e2e_steps_run(e2e_steps, diag_host)
    t1.record(main)
    torch.cuda.synchronize()
    barrier(world)
    mesh.check_finite()
    assert bool(torch.isfinite(diag_host).all()) and bool((diag_host[:, 1] > 0).all())
    ms2 = max_over_ranks(t0.elapsed_time(t1), world)
    e2e = {"value": world * n * n * e2e_steps / (ms2 * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": n * n * real_b, "d2h_bytes_per_step": 2 * 8, "steps": e2e_steps,
           "what": "closed loop through the public API: the state stays resident; every step uploads the "
                   "activity field from pinned host memory and reads back energy and enstrophy"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": a.dtype, "data": "synthetic (seeded random Q ~ U(-0.01,0.01), w = 0)",
        "config": plain_config(n, world),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                                        f"captured at commit {traffic_commit}" if traffic is not None else None),
                     "algorithmic_bytes_per_launch": k_bytes, "ms_per_launch": k_ms,
                     "row_ms": row_ms, "col_ms": col_ms},
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"], oracle_run = cpu_baseline(n, a.cpu_sample_steps, a.dtype)
        line["spectrum_vs_oracle"] = spectrum_vs_oracle(mesh, qaf, oracle_run, a.cpu_sample_steps)
    if world == 1 and not a.no_extras:
        del mesh
        line["targets"] = target_extras(a, qaf, torch, flush)
    return line


def target_extras(a, qaf, torch, flush):
    """Shortened measurements of the other stated targets, beside the headline:
    the same workload in FP64, the adjoint's cost against a forward step (with
    a finite-difference check of its gradient), and the batched ensemble
    against the plain solver looped over the same instances."""
    out = {}
    # ---- the plain workload in FP64 (the reference's own precision) -------
    if a.dtype != "f64":
        m = qaf.Mesh(a.n, lx=L, dtype=qaf.F64)
        p = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=DT)
        m.load(*m.random_q(SEED))
        for _ in range(3):
            m.advance(p, 1)
        steps = 50
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for e0, e1 in ev:
            flush.zero_()
            e0.record()
            m.advance(p, 1)
            e1.record()
        torch.cuda.synchronize()
        m.check_finite()
        ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
        out["fp64"] = {"value": a.n * a.n * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps,
                       "steps": steps, "what": "the same workload in FP64, device resident, L2 flushed between steps"}
        del m
    # ---- adjoint cost (target: at most 3x a forward) ----------------------
    T = 320
    r = adjoint_ratio(qaf, torch, T, fd_dirs=4)
    out["adjoint_cost_ratio"] = r
    # ---- batched ensemble against the looped plain solver (target: >= 2x) -
    out["ensemble_vs_looped"] = ensemble_ratio(qaf, torch, flush, steps=5)
    return out


def adjoint_ratio(qaf, torch, T, fd_dirs):
    """The adjoint workload shortened to T steps: (recompute + adjoint) time
    over the plain forward's, built-in launch shapes, plus the FD check."""
    import numpy as np
    n, dt = ADJ_N, ADJ_DT
    K, Wn = min(ADJ_K, T), min(ADJ_WINDOW, T)
    alpha_np = smoothed_alpha(n, ADJ_SEED)
    base = dict(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=dt, q_lin=1.0, advect_omega=1)
    mesh = qaf.Mesh(n, lx=L, dtype=qaf.F32)
    p = qaf.Params(**base)
    p.alpha_field = torch.as_tensor(alpha_np).to(device="cuda", dtype=mesh.real_dtype)
    s0 = mesh.random_q(SEED)
    adj = qaf.Adjoint(mesh, T, K, Wn)
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    for _ in range(2):
        mesh.load(*s0); mesh.advance(p, T)
        adj.forward(p, *s0, final_state=False); adj.backward(None, 1.0)
    tp, tb = [], []
    for _ in range(3):
        e0, e1 = ev()
        mesh.load(*s0)
        e0.record(); mesh.advance(p, T); e1.record()
        torch.cuda.synchronize()
        tp.append(e0.elapsed_time(e1))
        adj.forward(p, *s0, final_state=False)
        e0, e1 = ev()
        e0.record(); adj.backward(None, 1.0); e1.record()
        torch.cuda.synchronize()
        tb.append(e0.elapsed_time(e1))
    fwd, bwd = statistics.median(tp), statistics.median(tb)
    fd = adjoint_fd_check(qaf, torch, np, n, T, K, Wn, dt, base, alpha_np, adj, p, s0, dirs=fd_dirs)
    return {"value": bwd / fwd, "unit": "x", "forward_ms": fwd, "backward_ms": bwd, "fd_check": fd,
            "what": f"{n}^2 FP32, {T} IF-RK4 steps dt={dt}, checkpoints every {K}, loss = mean enstrophy of the "
                    f"last {Wn} states; (recompute + adjoint) / plain forward, medians of 3; built-in launch shapes"}


def ensemble_ratio(qaf, torch, flush, steps):
    """The 256-instance ensemble shortened to a few steps: the batched stepper
    against the plain solver looped over the same instances (built-in shapes)."""
    n_all, al, rf, seeds = ensemble_table(ENS_COUNT)
    p = qaf.Params(re=1.0, er=1.0, rf=0.0, lam=0.1, alpha=1.0, dt=ENS_DT, q_lin=1.0, advect_omega=1)
    ens = qaf.Ensemble(n_all, p, al, rf, lx=L, dtype=qaf.F32, tune=False)
    ens.init_random(seeds)
    for _ in range(2):
        ens.advance(1)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for e0, e1 in ev:
        flush.zero_()
        e0.record(); ens.advance(1); e1.record()
    torch.cuda.synchronize()
    ens.diagnostics()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / steps
    del ens
    states = []
    for k in range(len(n_all)):
        m = qaf.Mesh(n_all[k], lx=L, dtype=qaf.F32)
        m.load(*m.random_q(seeds[k]))
        states.append((m, qaf.Params(re=1.0, er=1.0, rf=rf[k], lam=0.1, alpha=al[k], dt=ENS_DT)))
    for m, pk in states:
        m.advance(pk, 1)
    loop_steps = 3
    flush.zero_()
    l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0.record()
    for m, pk in states:
        m.advance(pk, loop_steps)
    l1.record()
    torch.cuda.synchronize()
    ms_loop = l0.elapsed_time(l1) / loop_steps
    work = sum(n * n for n in n_all)
    return {"value": ms_loop / ms, "unit": "x", "batched_ms_per_step": ms, "looped_ms_per_step": ms_loop,
            "batched": work / (ms * 1e-3), "looped": work / (ms_loop * 1e-3), "metric_unit": UNIT,
            "what": f"{ens_workload_desc(ENS_COUNT)}; {steps} batched steps (one CUDA graph each) against "
                    f"{loop_steps} steps of each instance through the plain solver; built-in launch shapes"}


def run_reference(a, world, rank, local):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness_f32" if a.dtype == "f32" else "ref_harness")
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": "the reference's CUDA build (oracle/_ref) was not built: "
                                                    "its sources were not present when build() ran"}
    def timed(path):
        cmd = [path, "time", "--n", str(a.n), "--L", repr(L), "--dt", repr(DT), "--seed", str(SEED),
               "--re", "1", "--er", "1", "--rf", "0.1", "--lambda", "0.1", "--alpha", "1",
               "--warmup", str(a.warmup), "--timed", str(a.steps)]
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local)))
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if r.returncode != 0:
            return None, f"reference build exited {r.returncode}: {r.stderr.strip()[-200:]}"
        return json.loads(r.stdout.strip().splitlines()[-1])["ms_per_step"], None

    with ClockSampler(local) as clk:
        ms, err = timed(exe)
    if err:
        return {"impl": "reference", "unavailable": err}
    value = a.n * a.n / (ms * 1e-3)
    targets = {}
    exe64 = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if a.dtype == "f32" and os.path.exists(exe64):
        ms64, err64 = timed(exe64)
        targets["fp64"] = ({"value": a.n * a.n / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64,
                            "steps": a.steps, "what": "the reference's build as shipped (FP64), same workload"}
                           if err64 is None else {"unavailable": err64})
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": a.dtype, "data": "synthetic (seeded random Q ~ U(-0.01,0.01), w = 0)",
        "config": plain_config(a.n, world),
        "targets": targets,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"{a.steps} steps of the reference's own CUDA build (friction.cu step sequence, "
                                   f"unmodified headers{', FP32 macro shim' if a.dtype == 'f32' else ''}) on the B200; "
                                   "the reference has no CPU implementation of the path"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    }


def ensemble_table(count):
    from qaf.shard import draw_ensemble
    return draw_ensemble(count, ENS_SEED)


def ens_workload_desc(count):
    return (f"ensemble of {count} instances, N ~ U{{64,128,256}}, Ra ~ U(0.5,2), Rf ~ U(0.01,0.5), FP32, "
            f"IF-RK4 dt={ENS_DT}, L=16pi, Re=1 Er=1 lambda=0.1, draw seed {ENS_SEED}")


def ens_cpu_baseline(sizes, steps):
    """The FP64 host oracle on one instance of each grid size, extrapolated to the ensemble's mix."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    per = {}
    total = 0.0
    for n in sorted(set(sizes)):
        p = O.params(n=n, L=L, dt=ENS_DT)
        s0 = O.initial_spectra(SEED, n)
        O.step(p, *s0, 1)
        t0 = time.perf_counter()
        O.step(p, *s0, steps)
        per[n] = (time.perf_counter() - t0) / steps
        total += per[n] * steps
    work = sum(n * n for n in sizes)
    t_step = sum(per[n] for n in sizes)
    cores = int(os.environ.get("QAF_ORACLE_THREADS", os.cpu_count() or 1))
    return {"value": work / t_step, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} FP64 IF-RK4 steps of one instance of each size "
                      f"({', '.join(f'{n}^2: {per[n]*1e3:.1f} ms/step' for n in sorted(per))}; {total:.1f} s), "
                      f"extrapolated to the ensemble's size mix with the host oracle"}


def run_ensemble(a, world, rank, local):
    import torch

    import qaf
    from qaf.shard import shard_instances

    n_all, al_all, rf_all, seed_all = ensemble_table(a.instances)
    mine = shard_instances(n_all, world)[rank]
    sizes = [n_all[k] for k in mine]
    alpha = [al_all[k] for k in mine]
    rf = [rf_all[k] for k in mine]
    seeds = [seed_all[k] for k in mine]
    p = qaf.Params(re=1.0, er=1.0, rf=0.0, lam=0.1, alpha=1.0, dt=ENS_DT, q_lin=1.0, advect_omega=1)
    import tempfile
    tune_cache = os.path.join(tempfile.mkdtemp(prefix="qaf_tune_"), "autotune.jsonl")
    ens = qaf.Ensemble(sizes, p, alpha, rf, lx=L, dtype=qaf.F32, tune=not a.no_tune, tune_cache=tune_cache)
    ens.init_random(seeds)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    work_mine = sum(n * n for n in sizes)
    work_all = sum(n * n for n in n_all)
    ngroups = len(set(sizes))

    # ---- batched, device resident --------------------------------------
    for _ in range(a.warmup):
        ens.advance(1)
    barrier(world)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    with ClockSampler(local) as clk:
        barrier(world)
        for e0, e1 in ev:
            flush.zero_()
            e0.record()
            ens.advance(1)
            e1.record()
        barrier(world)
    ms = max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in ev), world)
    ens.diagnostics()       # raises on a non-finite instance
    value = work_all * a.steps / (ms * 1e-3)

    # ---- the plain solver looped over the same instances ---------------
    loop_steps = max(4, min(a.steps, 20))
    states = []
    for k in range(len(sizes)):
        m = qaf.Mesh(sizes[k], lx=L, dtype=qaf.F32)
        m.load(*m.random_q(seeds[k]))
        states.append((m, qaf.Params(re=1.0, er=1.0, rf=rf[k], lam=0.1, alpha=alpha[k], dt=ENS_DT)))
    for m, pk in states:
        m.advance(pk, 2)
    barrier(world)
    flush.zero_()
    l0 = torch.cuda.Event(enable_timing=True)
    l1 = torch.cuda.Event(enable_timing=True)
    l0.record()
    for m, pk in states:
        m.advance(pk, loop_steps)
    l1.record()
    barrier(world)
    ms_loop = max_over_ranks(l0.elapsed_time(l1), world)
    looped = work_all * loop_steps / (ms_loop * 1e-3)
    del states

    # ---- model bytes of one step over all instances (three-pass model) --
    ca = lambda n: (n // 2 + 1) * n * 2 * 4
    step_bytes = sum(4 * 55 * ca(n) for n in sizes)
    peak, peak_kind = peaks()
    achieved = step_bytes / (ms / a.steps * 1e-3) / 1e9

    # ---- end to end: controls in, diagnostics out, every step ----------
    for _ in range(2):
        ens.set_controls(alpha, rf)
        ens.advance(1)
        ens.diagnostics()
    barrier(world)
    e2e_steps = max(10, a.steps // 2)
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(e2e_steps)]
    for e0, e1 in ev2:
        flush.zero_()
        e0.record()
        ens.set_controls(alpha, rf)         # H2D: activity and friction factors per instance
        ens.advance(1)
        ens.diagnostics()                   # D2H: energy, enstrophy per instance (+ status word per size)
        e1.record()
    barrier(world)
    ms2 = max_over_ranks(sum(e0.elapsed_time(e1) for e0, e1 in ev2), world)
    e2e = {"value": work_all * e2e_steps / (ms2 * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": 5 * 4 * len(sizes), "d2h_bytes_per_step": 16 * len(sizes) + 4 * ngroups}

    line = {
        "metric": ENS_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded instance table; seeded random Q ~ U(-0.01,0.01), w = 0 per instance)",
        "config": {"workload": ens_workload_desc(a.instances), "instances": a.instances,
                   "sizes": {str(n): n_all.count(n) for n in sorted(set(n_all))},
                   "launch_shapes": ens.tuned,
                   "parallelism": f"instances sharded over {world} rank(s)",
                   "l2": "flushed (256 MiB write) between timed steps"},
        "looped": {"value": looped, "unit": UNIT, "steps": loop_steps, "ms_per_step": ms_loop / loop_steps,
                   "what": "the plain single-grid solver looped over this rank's instances (qaf_state_advance each)"},
        "roofline": {"bound": "hbm", "kernel": "ensemble step (all row and column launches of every size group)",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "algorithmic_bytes_per_step": step_bytes},
        "e2e": e2e,
        "gpu_launches": a.steps * ngroups * 8,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = ens_cpu_baseline(n_all, a.cpu_sample_steps)
    return line


def run_reference_ensemble(a):
    """The reference's CUDA build looped over the instances: one timed run per grid size, summed per instance."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness_f32")
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": "the reference's CUDA build (oracle/_ref) was not built: "
                                                    "its sources were not present when build() ran"}
    n_all, _, _, _ = ensemble_table(a.instances)
    per = {}
    for n in sorted(set(n_all)):
        cmd = [exe, "time", "--n", str(n), "--L", repr(L), "--dt", repr(ENS_DT), "--seed", str(SEED),
               "--re", "1", "--er", "1", "--rf", "0.1", "--lambda", "0.1", "--alpha", "1",
               "--warmup", str(a.warmup), "--timed", str(a.steps)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            return {"impl": "reference", "unavailable": f"reference build exited {r.returncode}: {r.stderr.strip()[-200:]}"}
        per[n] = json.loads(r.stdout.strip().splitlines()[-1])["ms_per_step"]
    ms = sum(per[n] for n in n_all)
    work = sum(n * n for n in n_all)
    value = work / (ms * 1e-3)
    return {
        "impl": "reference", "metric": ENS_METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded instance table)",
        "config": {"workload": ens_workload_desc(a.instances), "instances": a.instances,
                   "per_size_ms_per_step": {str(n): per[n] for n in per}},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "the reference's own CUDA build (FP32 macro shim), one timed run per grid size, "
                                   "summed over the instances as a loop of single-grid runs"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def smoothed_alpha(n, seed, width=4.0):
    """1 + 0.1 * (N(0,1) noise smoothed by a periodic Gaussian of `width` cells, rescaled to unit variance)."""
    import numpy as np
    g = np.random.default_rng(seed).standard_normal((n, n))
    k = np.fft.fftfreq(n) * n
    kk = k[:, None] ** 2 + k[None, :] ** 2
    s = np.real(np.fft.ifft2(np.fft.fft2(g) * np.exp(-0.5 * (2 * np.pi * width / n) ** 2 * kk)))
    return 1.0 + 0.1 * s / s.std()


def run_adjoint(a, world, rank, local):
    import numpy as np
    import torch

    import qaf
    import qaf.autograd as QA

    n, T, dt = ADJ_N, a.adj_steps, ADJ_DT
    K, Wn = min(ADJ_K, T), min(ADJ_WINDOW, T)
    reps, warm = max(1, min(a.steps, 5)), 3
    alpha_np = smoothed_alpha(n, ADJ_SEED)
    base = dict(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=dt, q_lin=1.0, advect_omega=1)

    def setup(dtype):
        mesh = qaf.Mesh(n, lx=L, dtype=dtype)
        p = qaf.Params(**base)
        p.alpha_field = torch.as_tensor(alpha_np).to(device="cuda", dtype=mesh.real_dtype)
        return mesh, p, mesh.random_q(SEED)

    shapes = "col:default row:default"
    if a.shapes:                              # given shapes, e.g. those a tuned run reported
        col, row = (s.strip() for s in a.shapes.split(","))
        qaf.set_variant(n, qaf.F32, False, col, row)
        shapes = f"{col} {row}"
    elif not a.no_tune:                       # launch shapes for this grid (untimed)
        shapes, _ = qaf.autotune(n, qaf.F32, 1, None)
    mesh, p, s0 = setup(qaf.F32)
    adj = qaf.Adjoint(mesh, T, K, Wn)
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))

    def plain_forward():
        mesh.load(*s0)
        mesh.advance(p, T)

    def fwd_bwd():
        adj.forward(p, *s0, final_state=False)
        adj.backward(None, 1.0)

    for _ in range(warm):
        plain_forward()
        fwd_bwd()
    barrier(world)
    t_plain, t_af, t_bw = [], [], []
    with ClockSampler(local) as clk:
        for _ in range(reps):
            e0, e1 = ev()
            e0.record(); plain_forward(); e1.record()
            torch.cuda.synchronize()
            t_plain.append(e0.elapsed_time(e1))
            e0, e1 = ev()
            e0.record(); adj.forward(p, *s0, final_state=False); e1.record()
            torch.cuda.synchronize()
            t_af.append(e0.elapsed_time(e1))
            l0 = mesh.launch_count()
            e0, e1 = ev()
            e0.record(); adj.backward(None, 1.0); e1.record()
            torch.cuda.synchronize()
            t_bw.append(e0.elapsed_time(e1))
            launches = mesh.launch_count() - l0
    barrier(world)
    tp = max_over_ranks(statistics.median(t_plain), world)
    taf = max_over_ranks(statistics.median(t_af), world)
    tbw = max_over_ranks(statistics.median(t_bw), world)
    ratio = tbw / tp

    # end to end through the autograd wrapper: host activity and initial state in, gradients out
    host_alpha = torch.as_tensor(alpha_np, dtype=mesh.real_dtype).pin_memory()
    host_s0 = [x.cpu().pin_memory() for x in s0]
    host_ga = torch.empty((n, n), dtype=mesh.real_dtype).pin_memory()

    def e2e_pass():
        al = host_alpha.to("cuda", non_blocking=True).requires_grad_()
        st = [h.to("cuda", non_blocking=True).requires_grad_() for h in host_s0]
        loss, _, _, _ = QA.rollout(mesh, p, *st, al, nsteps=T, checkpoint_every=K, loss_window=Wn)
        loss.backward()
        host_ga.copy_(al.grad, non_blocking=True)
        return float(loss.item())

    e2e_pass()
    e0, e1 = ev()
    e0.record(); e2e_pass(); e1.record()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1), world)

    # model bytes of one backward step: the recompute (4 stages x 55 arrays + 9 recorded real fields
    # per stage) and the adjoint (column: 9 in + 11 out + 9 RK arrays; row: 11 in + 9 real fields +
    # 9 out + the activity gradient read and written)
    ca = (n // 2 + 1) * n * 2 * 4
    pr = n * n * 4
    bytes_step = 4 * (55 * ca + 9 * pr) + 4 * ((9 + 11 + 9) * ca + (11 + 9) * ca + (9 + 2) * pr)
    peak, peak_kind = peaks()
    achieved = bytes_step * T / (tbw * 1e-3) / 1e9

    fd = None
    if not a.no_fd and rank == 0:
        fd = adjoint_fd_check(qaf, torch, np, n, T, K, Wn, dt, base, alpha_np, adj, p, s0)

    line = {
        "metric": ADJ_METRIC, "value": ratio, "unit": "x", "n_gpus": world, "steps": reps, "warmup": warm,
        "ms_per_step": tbw, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random Q ~ U(-0.01,0.01), w = 0; seeded smoothed activity field)",
        "config": {"workload": f"adjoint {n}x{n} FP32, {T} IF-RK4 steps dt={dt}, Ra(x) = 1 + 0.1 smoothed N(0,1) "
                               f"(width 4 cells, seed {ADJ_SEED}), loss = mean enstrophy of the last {Wn} states, "
                               f"checkpoints every {K} steps", "grid": n, "horizon": T,
                   "launch_shapes": shapes, "parallelism": f"replicas x{world}",
                   "l2": "working set of a segment's recording (~600 MB) larger than L2"},
        "forward_ms": tp, "adjoint_forward_ms": taf, "backward_ms": tbw,
        "ratio_forward_with_checkpoints_plus_backward": (taf + tbw) / tp,
        "fd_check": fd,
        "roofline": {"bound": "hbm", "kernel": "backward step (recompute + adjoint kernels)",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "algorithmic_bytes_per_step": bytes_step},
        "e2e": {"value": t_e2e / tp, "unit": "x", "ms": t_e2e,
                "h2d_bytes_per_step": n * n * 4 + 3 * ca, "d2h_bytes_per_step": n * n * 4 + 8},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = adjoint_cpu_baseline(n, dt, alpha_np)
    return line


def adjoint_fd_check(qaf, torch, np, n, T, K, Wn, dt, base, alpha_np, adj32, p32, s0_32, dirs=16):
    """Directional derivatives of the FP32 and FP64 adjoint gradients against central
    differences of the FP64 forward, along `dirs` random directions of (Ra(x), initial spectra)."""
    mesh = qaf.Mesh(n, lx=L, dtype=qaf.F64)
    p = qaf.Params(**base)
    alpha = torch.as_tensor(alpha_np, dtype=torch.float64, device="cuda")
    p.alpha_field = alpha
    s0 = [x.to(torch.complex128) for x in s0_32]
    adj = qaf.Adjoint(mesh, T, K, Wn)
    loss0, _ = adj.forward(p, *s0, final_state=False)
    g64 = adj.backward(None, 1.0)
    adj32.forward(p32, *s0_32, final_state=False)
    g32 = adj32.backward(None, 1.0)
    rng = np.random.default_rng(7)
    scale = float(max(x.abs().max().item() for x in s0[1:]))
    err32, err64 = [], []
    for _ in range(dirs):
        da = torch.as_tensor(smoothed_alpha(n, int(rng.integers(1 << 30))) - 1.0, device="cuda") * 10.0
        ds = [torch.complex(torch.as_tensor(rng.standard_normal(x.shape)), torch.as_tensor(rng.standard_normal(x.shape)))
              .to("cuda") * scale for x in s0]
        eps = 1e-5

        def loss_at(sign):
            q = qaf.Params(**base)
            q.alpha_field = (alpha + sign * eps * da).contiguous()
            return adj.forward(q, *[(x + sign * eps * d).contiguous() for x, d in zip(s0, ds)], final_state=False)[0]

        fdv = (loss_at(1) - loss_at(-1)) / (2 * eps)

        def dot(g):
            v = float((g[3].double() * da).sum())
            for gi, d in zip(g[:3], ds):
                gi = gi.to(torch.complex128)
                v += float((gi.real * d.real + gi.imag * d.imag).sum())
            return v
        err64.append(abs(dot(g64) - fdv) / abs(fdv))
        err32.append(abs(dot(g32) - fdv) / abs(fdv))
    return {"directions": dirs, "eps": 1e-5, "loss": loss0,
            "max_rel_err_fp64_adjoint": max(err64), "max_rel_err_fp32_adjoint": max(err32),
            "median_rel_err_fp32_adjoint": statistics.median(err32),
            "reference": "central differences of the FP64 forward on the GPU"}


def adjoint_cpu_baseline(n, dt, alpha_np):
    """The FP64 host oracle's tangent-linear step on a bounded sample, per forward step (the oracle has
    no adjoint: one TLM pass gives one directional derivative)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    p = O.params(n=n, L=L, dt=dt)
    s0 = O.initial_spectra(SEED, n)
    z = [np.zeros_like(s0[0])] * 3
    steps = 2
    O.step(p, *s0, 1, alpha_field=alpha_np)
    t0 = time.perf_counter()
    O.step(p, *s0, steps, alpha_field=alpha_np)
    tf = (time.perf_counter() - t0) / steps
    t0 = time.perf_counter()
    O.step_tlm(p, *s0, *z, steps, 0, alpha_field=alpha_np, dalpha_field=alpha_np)
    tt = (time.perf_counter() - t0) / steps
    cores = int(os.environ.get("QAF_ORACLE_THREADS", os.cpu_count() or 1))
    return {"value": tt / tf, "unit": "x", "cores": cores, "kind": "port",
            "sample": f"{steps} FP64 steps at {n}^2 with the host oracle: forward {tf*1e3:.1f} ms/step, forward + "
                      f"tangent-linear {tt*1e3:.1f} ms/step (one directional derivative per pass)"}


def run_control(a, world, rank, local):
    import numpy as np
    import torch

    import qaf

    n, ni, T, K, lr = CTL_N, CTL_INST, a.horizon, min(CTL_K, a.horizon), CTL_LR
    iters, warm = max(1, min(a.steps, 5)), 1
    p = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=ADJ_DT, q_lin=1.0, advect_omega=1)
    shapes = {"batched": "col:default row:default", "single": "col:default row:default"}
    if not a.no_tune:                         # launch shapes for the batch and the looped single grid (untimed)
        shapes = {"batched": qaf.autotune(n, qaf.F32, ni, None)[0], "single": qaf.autotune(n, qaf.F32, 1, None)[0]}
    batch = qaf.AdjointBatch(ni, n, p, T, K, 1, lx=L, dtype=qaf.F32)
    mesh = batch.mesh
    alpha = torch.stack([torch.as_tensor(smoothed_alpha(n, 100 + k), dtype=torch.float32) for k in range(ni)]).cuda()
    st = [mesh.random_q(100 + k) for k in range(ni)]
    s0 = [torch.stack([st[k][f] for k in range(ni)]).contiguous() for f in range(3)]
    history = []

    def iteration():
        nonlocal alpha
        losses, _ = batch.forward(*s0, alpha=alpha, final_state=False)
        _, _, _, ga = batch.backward(None, [1.0] * ni)
        scale = ga.abs().amax(dim=(1, 2), keepdim=True).clamp_min(1e-30)
        alpha = (alpha - lr * ga / scale).contiguous()       # normalised descent step per instance
        return losses

    for _ in range(warm):
        history.append(iteration())
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record()
        for _ in range(iters):
            history.append(iteration())
        e1.record()
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world) / iters
    final, _ = batch.forward(*s0, alpha=alpha, final_state=False)
    history.append(final)
    value = world * ni / (ms * 1e-3)

    # looped: the same iteration for one instance through the single-instance adjoint, times 64
    single = qaf.Adjoint(qaf.Mesh(n, lx=L, dtype=qaf.F32), T, K, 1)
    ps = qaf.Params(re=1.0, er=1.0, rf=0.1, lam=0.1, alpha=1.0, dt=ADJ_DT, q_lin=1.0, advect_omega=1)
    ps.alpha_field = alpha[0].contiguous()
    for _ in range(2):
        single.forward(ps, *st[0], final_state=False)
        single.backward(None, 1.0)
    e0.record()
    single.forward(ps, *st[0], final_state=False)
    single.backward(None, 1.0)
    e1.record()
    torch.cuda.synchronize()
    ms_single = e0.elapsed_time(e1)
    looped = 1.0 / (ms_single * 1e-3)

    ca = (n // 2 + 1) * n * 2 * 4
    pr = n * n * 4
    bytes_iter = ni * T * (4 * 55 * ca + 4 * (55 * ca + 9 * pr) + 4 * ((9 + 11 + 9) * ca + (11 + 9) * ca + (9 + 2) * pr))
    peak, peak_kind = peaks()
    achieved = bytes_iter / (ms * 1e-3) / 1e9
    l0 = np.mean(history[0])
    lN = np.mean(history[-1])
    return {
        "metric": CTL_METRIC, "value": value, "unit": "instance-iterations/s", "n_gpus": world, "steps": iters,
        "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded random Q per instance; seeded smoothed activity fields)",
        "config": {"workload": f"control loop: {ni} x {n}^2 FP32, horizon {T} IF-RK4 steps dt={ADJ_DT}, Ra_k(x) = "
                               f"1 + 0.1 smoothed N(0,1) (seeds 100..{100 + ni - 1}), loss = terminal enstrophy, "
                               f"checkpoints every {K} steps, normalised descent step {lr}",
                   "instances": ni, "grid": n, "horizon": T, "launch_shapes": shapes,
                   "parallelism": f"replicas x{world}",
                   "l2": f"recording of a segment ({ni * K * 4 * 9 * pr / 1e9:.0f} GB) larger than L2"},
        "loss_mean_first": l0, "loss_mean_last": lN, "loss_history_mean": [float(np.mean(h)) for h in history],
        "looped": {"value": looped, "unit": "instance-iterations/s", "ms_per_instance_iteration": ms_single,
                   "what": "one instance's iteration through the single-instance adjoint (qaf_adjoint_*); 64 such run one after another"},
        "roofline": {"bound": "hbm", "kernel": "one iteration (forward, recompute, adjoint) of the batch",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "algorithmic_bytes_per_step": bytes_iter},
        "e2e": {"value": value, "unit": "instance-iterations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": ni * 8},
        "gpu_launches": None,
        "clocks": clk.summary(),
    }


def main():
    a = parse()
    if a.impl == "reference":
        # one rank runs the reference; under torchrun the others exit without work
        rank, local = int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))
        if rank == 0:
            if a.workload == "ensemble":
                line = run_reference_ensemble(a)
            elif a.workload in ("adjoint", "control"):
                line = {"impl": "reference", "unavailable": "the reference computes no gradients (no adjoint or "
                                                            "tangent model anywhere in it)"}
            else:
                line = run_reference(a, 1, rank, local)
            print(json.dumps(line), flush=True)
        return
    world, rank, local = dist_init()
    import torch
    torch.cuda.set_device(local)
    if a.workload == "ensemble":
        line = run_ensemble(a, world, rank, local)
    elif a.workload == "adjoint":
        line = run_adjoint(a, world, rank, local)
    elif a.workload == "control":
        line = run_control(a, world, rank, local)
    else:
        line = run_qaf(a, world, rank, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
