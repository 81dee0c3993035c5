"""Benchmark: DG residual + VJP DOF-updates/s on the 3D compressible-Euler workload.

Workload (one "step"): the HLLC Euler operator on a periodic 32^3 hex grid,
DG degree k=3 (Np=20 per variable, 5 variables, 3,276,800 DOFs), quadrature
order 7 (4^3 volume / 4^2 face nodes), seeded synthetic state (see
bosss_b200/problems.py). A step evaluates the residual R(U) and the adjoint
product J(U)^T W at the same state; DOF-updates per step = 2 x 3,276,800.

* ``value``: device-resident throughput (inputs in HBM), CUDA events on the
  launching stream around each step; L2 (126 MB) is flushed between steps by
  writing a 512 MB buffer outside the timed events (the working set, 105 MB,
  would otherwise stay L2-resident).
* ``e2e``: the same steps through the host-buffer C-ABI entry point
  bosss_b200_residual_vjp from pinned host memory: every step copies U and W host->device
  and R and J^T W device->host inside the timed region (streamed by chunks of x-planes,
  overlapped with the evaluation).
* ``roofline``: the VJP kernel (the dominant launch) -- algorithmic bytes
  (8 B x (inputs + outputs)) over its CUDA-event duration, against the measured HBM
  copy bandwidth; the FP64 pipe figure is reported beside it (nominal peak).
* ``cpu_baseline``: the CPU FP64 oracle (a C++/OpenMP restatement of the reference
  evaluator; the reference's .NET code cannot run here): residual + exact VJP per step on a
  bounded 16^3 sample of the same operator (median of >= 5 steps on all host cores, plus a
  single-core figure).
* ``split_fp32``: the same step with the residual's volume contractions on the tensor cores
  (BOSSS_PRECISION_SPLIT_FP32: exact 8-bit slices, int32 accumulation, FP64 recombination;
  faces and VJP in FP64), with its difference from the FP64 results.

N > 1 GPUs (or ``--partitioned``): weak scaling with a real exchange step -- the periodic
Euler box grows to (N*32) x 32 x 32 and every rank owns an x-slab of 32 planes plus ghost
planes; each step exchanges the ghost planes of U and W by NCCL point-to-point (overlapped
with the interior cells) and evaluates residual and VJP of the owned cells; time = max over
ranks.

``--impl reference`` times the CPU oracle alone on the host cores (rank 0).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DOF_PER_STEP_FACTOR = 2   # residual + VJP


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--k", type=int, default=3)
    ap.add_argument("--workload", default="euler3d", choices=["euler3d", "batched", "batched-solve", "newton", "xdg", "rk", "spmv"],
                    help="euler3d: the headline (residual + VJP, Euler/HLLC 32^3 k=3); batched: 256 "
                         "independent advection-diffusion instances (16..48^3, k=1..4) in one captured "
                         "graph; newton: matrix-free Newton-GMRES on -div((1+u^2) grad u) = 1, 48^3; rk: "
                         "classical RK4 time steps of the Euler workload, one step captured in a CUDA graph")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--precond", default=None, choices=["multigrid", "block-jacobi", "none"],
                    help="preconditioner of the newton (default multigrid) and batched-solve (default "
                         "block-jacobi) workloads")
    ap.add_argument("--precond-update", type=int, default=1,
                    help="newton workload: rebuild the preconditioner every this many Newton steps")
    ap.add_argument("--xdg-rule", default="moment-fitting", choices=["moment-fitting", "saye"],
                    help="xdg workload: cut-cell rule family")
    ap.add_argument("--kernel", default="auto", choices=["auto", "generic", "slab", "faces"],
                    help="kernel path of the euler3d workload (auto: the library's choice)")
    ap.add_argument("--partitioned", action="store_true",
                    help="euler3d through the partitioned (x-slab, ghost-plane) evaluator even on one GPU; "
                         "always used for --gpus > 1")
    return ap.parse_args()


def out_dir():
    """Directory for the bench's side files (clock samples, autotuner table): $BOSSS_BENCH_DIR,
    else a per-user temporary directory."""
    import tempfile
    d = os.environ.get("BOSSS_BENCH_DIR") or os.path.join(tempfile.gettempdir(), "bosss_b200_bench")
    os.makedirs(d, exist_ok=True)
    return d


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_json(path):
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(out_dir(), "bench_clocks_%d.csv" % os.getpid())

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler is running (its first line is written)
            t0 = time.time()
            while time.time() - t0 < 5.0 and self.proc.poll() is None:
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _oracle_step_times(pr, W, reps, budget_s):
    """Wall times of `reps` (residual + exact VJP) oracle steps of problem pr (at most
    budget_s seconds in total, at least one step)."""
    from oracle import oracle as orc
    opd, gd = pr.descs()
    ts = []
    t_all = time.perf_counter()
    while len(ts) < reps and (not ts or time.perf_counter() - t_all < budget_s):
        t0 = time.perf_counter()
        orc.evaluate(opd, gd, pr.U)
        orc.vjp(opd, gd, pr.U, W)
        ts.append(time.perf_counter() - t0)
    return ts


def cpu_sample_problem(args):
    """Bounded CPU sample of the euler3d workload: the same operator, degree and rule on a
    16^3 periodic box (1/8 of the 32^3 cells, same per-cell work), so that >= 5 timed
    oracle steps stay within seconds."""
    from bosss_b200 import problems as P
    n = min(args.n, 16)
    return P.euler3d(n=n, k=args.k, seed=2000)


def run_reference(args):
    """The reference's evaluator restated on the CPU (the C++ FP64 oracle; the .NET
    reference cannot run here) on the host cores, rank 0 only: residual + exact VJP per
    step on a bounded sample of the workload (16^3 cells of the same operator)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as orc
    pr = cpu_sample_problem(args)
    cores = orc.threads(os.cpu_count() or 1)
    W = np.random.default_rng(9).uniform(-1, 1, pr.n_dofs)
    for _ in range(max(args.warmup, 1) if args.warmup else 0):
        _oracle_step_times(pr, W, 1, 0.0)
    t = _oracle_step_times(pr, W, args.steps, 120.0)
    med = float(np.median(t))
    v = DOF_PER_STEP_FACTOR * pr.n_dofs / med
    line = {
        "impl": "reference", "metric": "dg_residual_vjp_dof_updates_per_s", "value": v, "unit": "DOF/s",
        "n_gpus": args.gpus, "steps": len(t), "warmup": args.warmup, "ms_per_step": 1e3 * med,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "euler3d_hllc_%d^3_k%d_residual+vjp" % (args.n, args.k), "dofs": pr.n_dofs,
                   "sample": pr.config["workload"]},
        "cpu_baseline": {"value": v, "unit": "DOF/s", "cores": cores, "kind": "port",
                         "sample": "median of %d steps (residual + exact VJP) of %s (same operator and rule as "
                                   "the 32^3 workload, 1/8 of its cells), C++ FP64 oracle, OpenMP over %d host "
                                   "threads" % (len(t), pr.config["workload"], cores)},
        "e2e": {"value": v, "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(args):
    """CPU baseline beside the GPU line: median of >= 5 oracle steps (residual + exact VJP)
    on all host cores, and the median of 3 on one core, of the bounded 16^3 sample."""
    from oracle import oracle as orc
    pr = cpu_sample_problem(args)
    W = np.random.default_rng(9).uniform(-1, 1, pr.n_dofs)
    cores = orc.threads(os.cpu_count() or 1)
    _oracle_step_times(pr, W, 1, 0.0)
    t_all = _oracle_step_times(pr, W, 5, 60.0)
    orc.threads(1)
    t_one = _oracle_step_times(pr, W, 3, 30.0)
    orc.threads(cores)
    per = DOF_PER_STEP_FACTOR * pr.n_dofs
    return {"value": per / float(np.median(t_all)), "unit": "DOF/s", "cores": cores, "kind": "port",
            "single_core_value": per / float(np.median(t_one)),
            "sample": "median of %d steps (residual + exact VJP) of %s (same operator and rule, 1/8 of the 32^3 "
                      "cells), C++ FP64 oracle, OpenMP %d threads; single_core_value: median of %d steps on 1 thread"
                      % (len(t_all), pr.config["workload"], cores, len(t_one))}


def run_batched_solve(args):
    """Per-instance implicit-step solves over the batched mix (``bosss_b200_batch_solve``):
    (I/dt_i + A_i) x_i = b_i for every instance, dt_i = h_i / |a_i| (one cell per time step
    at the instance's transport speed), FP32 GMRES(30) with the multigrid V-cycle (or block-Jacobi) inside FP64
    refinement to 1e-10; then the adjoint systems on the VJP. value = DOFs solved per second
    (forward + adjoint); the oracle checks the true residuals of a sample of instances."""
    import torch
    from bosss_b200 import operator as O
    from bosss_b200 import problems as P
    from oracle import oracle as orc
    # SIPLaplace discretises +nu Laplace(u) (ipLaplace.cs:183-186): nu = -0.01 makes the operator
    # dissipative (du/dt = -Op(u)), so that I/dt + J is the implicit Euler matrix of the mix
    probs = P.batched_advection_diffusion(n_instances=args.instances, seed=5000, nu=-0.01)
    # block-Jacobi by default: measured on B200 over the first 32 instances, the V-cycle cuts the
    # Krylov iterations 4.7x but costs 1.7x the time (per-instance assembly by 7 Np probes + setup)
    precond = {"multigrid": 2, "block-jacobi": 1, "none": 0}[args.precond or "block-jacobi"]
    n = sum(p.n_dofs for p in probs)
    dev = torch.device("cuda", 0)
    b = np.random.default_rng(8).uniform(-1, 1, n)
    dts = np.array([(1.0 / p.grid.n[0]) / np.linalg.norm(p.config["velocity"]) for p in probs])
    with O.BatchEvaluator(probs) as B:
        off = B.dom_offsets
        bt = torch.from_numpy(b).to(dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x, reps = B.solve(dts, bt, restart=30, precond=precond)
        torch.cuda.synchronize()
        t_fwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        xa, repa = B.solve(dts, bt, transpose=True, restart=30, precond=precond)
        torch.cuda.synchronize()
        t_adj = time.perf_counter() - t0
        x, xa = x.cpu().numpy(), xa.cpu().numpy()
    worst = 0.0
    for i in range(0, len(probs), max(1, len(probs) // 8)):   # oracle check of a sample
        p = probs[i]
        if p.n_dofs > 400000:
            continue
        sl = slice(off[i], off[i + 1])
        z = np.zeros(p.n_dofs)
        r1 = x[sl] / dts[i] + orc.jvp(*p.descs(), z, x[sl]) - b[sl]
        r2 = xa[sl] / dts[i] + orc.vjp(*p.descs(), z, xa[sl]) - b[sl]
        worst = max(worst, np.linalg.norm(r1) / np.linalg.norm(b[sl]), np.linalg.norm(r2) / np.linalg.norm(b[sl]))
    line = {"metric": "batched_implicit_solve_dofs_per_s", "value": 2 * n / (t_fwd + t_adj), "unit": "DOF/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "f64 (FP32 inner GMRES)", "data": "synthetic",
            "config": {"workload": "batched_advdiff_%d_instances_implicit_step_solves" % len(probs), "dofs": n,
                       "dt": "h / |a| per instance", "restart": 30,
                       "precond": {2: "multigrid V-cycle on the assembled I/dt + J (transposed for the adjoint)",
                                   1: "block-Jacobi (probed)", 0: "none"}[precond],
                       "rtol": 1e-10},
            "s_forward": t_fwd, "s_adjoint": t_adj,
            "converged": int(sum(r["converged"] for r in reps + repa)), "systems": 2 * len(probs),
            "krylov_iters_forward": int(sum(r["krylov_iters"] for r in reps)),
            "krylov_iters_adjoint": int(sum(r["krylov_iters"] for r in repa)),
            "max_outer_iters": int(max(r["outer_iters"] for r in reps + repa)),
            "oracle_max_rel_residual_sample": worst}
    print(json.dumps(line), flush=True)


def run_batched(args):
    """Batched mixed workload: residual + VJP of every instance, captured in one CUDA graph
    (two persistent launches); value = DOF-updates/s over all instances."""
    import torch
    from bosss_b200 import operator as O
    from bosss_b200 import problems as P
    probs = P.batched_advection_diffusion(n_instances=args.instances, seed=5000)
    n = sum(p.n_dofs for p in probs)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    U = torch.from_numpy(np.concatenate([p.U for p in probs])).to(dev)
    W = torch.from_numpy(np.random.default_rng(7).uniform(-1, 1, n)).to(dev)
    R = torch.zeros_like(U)
    G = torch.zeros_like(U)
    b = O.BatchEvaluator(probs)
    table = os.path.join(out_dir(), "batch_tiles.txt")
    t0 = time.perf_counter()
    b.autotune(U, W, R, G, table)
    tune_s = time.perf_counter() - t0
    b.capture(U, W, R, G)
    for _ in range(max(args.warmup, 3)):
        b.replay(stream)
    torch.cuda.synchronize()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    clocks = ClockSampler(0)
    clocks.start()
    ts = []
    for i in range(args.steps):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.replay(stream)
        e1.record(stream)
        ts.append((e0, e1))
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = [a.elapsed_time(c) for a, c in ts]
    total_ms = float(np.sum(ms))
    value = 2 * n * args.steps / (total_ms * 1e-3)

    # plain FP64 path: every instance through its own evaluator on the generic kernel, one
    # residual and one VJP launch per instance (what a caller does without the batched path)
    from bosss_b200 import _capi as C
    import ctypes
    L = C.lib()
    sp = ctypes.c_void_p(stream.cuda_stream)
    evs = [p.evaluator(kernel=C.KERNEL_GENERIC) for p in probs]
    off = b.dom_offsets
    Rp, Gp = torch.zeros_like(R), torch.zeros_like(G)

    def plain_step():
        for i, e in enumerate(evs):
            a0, a1 = int(off[i]), int(off[i + 1])
            C.check(L.bosss_b200_evaluate_device(e.handle, 1.0, 0.0, C.ptr(U[a0:a1]), C.ptr(Rp[a0:a1]), 0.0, sp))
            C.check(L.bosss_b200_vjp_device(e.handle, C.ptr(U[a0:a1]), C.ptr(W[a0:a1]), C.ptr(Gp[a0:a1]), 0.0, sp))

    plain_step()
    torch.cuda.synchronize()
    plain_ms = []
    for i in range(min(args.steps, 5)):
        flush.fill_(float(i))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plain_step()
        e1.record(stream)
        plain_ms.append((e0, e1))
    torch.cuda.synchronize()
    plain_step_ms = float(np.mean([a.elapsed_time(c) for a, c in plain_ms]))
    plain_value = 2 * n / (plain_step_ms * 1e-3)
    plain_diff = max(float((Rp - R).abs().max() / R.abs().max()), float((Gp - G).abs().max() / G.abs().max()))
    for e in evs:
        e.Dispose()
    hbm = (load_json(os.path.join(ROOT, "MEASURED_PEAKS.json")) or {}).get("hbm_gbs", 6650.0)
    bytes_step = 8.0 * (2 * n + 3 * n)   # residual: U in, R out; VJP: U, W in, G out
    achieved = bytes_step / (np.mean(ms) * 1e-3) / 1e9
    ks = [p.config["k"] for p in probs]
    line = {"metric": "dg_residual_vjp_dof_updates_per_s", "value": value, "unit": "DOF/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batched_advdiff_%d_instances_residual+vjp" % len(probs), "dofs": n,
                       "instances": len(probs), "k_hist": {str(k): ks.count(k) for k in sorted(set(ks))},
                       "launch": "one CUDA graph per step: residual then VJP, schedule chosen by the autotuner "
                                 "(persistent queue lpt/fifo, or one launch per (k, Q) class)",
                       "schedule": b.tiles(1, 2)[1],
                       "l2": "flushed between steps", "autotune_s": tune_s},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None, "kernel": "batch_kernel<PhysScalar<3,true>> (RES + VJP)"},
            "plain_fp64": {"kernel": "dg_cell_kernel per instance (generic fused FP64, 2 launches per instance)",
                           "value": plain_value, "ms_per_step": plain_step_ms, "chosen_over_plain": value / plain_value,
                           "max_rel_diff": plain_diff},
            "gpu_launches": (2 * len({p.config["k"] for p in probs}) if b.tiles(1, 2)[1] == "classes" else 2) * args.steps,
            "clocks": clk}
    print(json.dumps(line), flush=True)
    b.Dispose()


def run_spmv(args):
    """BlockMsrMatrix.SpMV on the C3 Jacobian's block pattern (48^3 hexes, k = 2: 110,592 block
    rows, 7 blocks of 10 x 10 inside, Dirichlet boundary), seeded values; a step = one
    y = A x (alpha 1, beta 0) on device-resident data; e2e through the host-buffer entry point
    (x in, y out per step, the matrix resident)."""
    import torch
    import ctypes
    from bosss_b200 import _capi as C
    from bosss_b200 import problems as P
    from oracle import oracle as orc
    n, npc = 48, 10
    rp, ci, vals = P.hex_block_pattern(n, npc)
    nbr = len(rp) - 1
    rows = nbr * npc
    A = ctypes.c_void_p()
    C.check(C.lib().bosss_b200_bsr_create(nbr, nbr, npc, npc, C.ptr(rp), C.ptr(ci), C.ptr(vals), 0, ctypes.byref(A)))
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sp = ctypes.c_void_p(stream.cuda_stream)
    xh = np.random.default_rng(11).uniform(-1, 1, rows)
    x = torch.from_numpy(xh).to(dev)
    y = torch.zeros(rows, dtype=torch.float64, device=dev)
    L = C.lib()
    for _ in range(max(args.warmup, 3)):
        C.check(L.bosss_b200_bsr_spmv_device(A, 1.0, C.ptr(x), 0.0, C.ptr(y), sp))
    torch.cuda.synchronize()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    clocks = ClockSampler(0)
    clocks.start()
    ev = []
    for i in range(args.steps):
        flush.fill_(float(i))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        C.check(L.bosss_b200_bsr_spmv_device(A, 1.0, C.ptr(x), 0.0, C.ptr(y), sp))
        b.record(stream)
        ev.append((a, b))
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    ref = orc.bsr_spmv(rp, ci, vals, 1.0, xh, 0.0, np.zeros(rows))
    err = float(np.linalg.norm(y.cpu().numpy() - ref) / np.linalg.norm(ref))
    # algorithmic bytes: values, column indices, row pointers, x once, y written
    bytes_ = vals.nbytes + ci.nbytes + rp.nbytes + 8 * rows + 8 * rows
    peaks = load_json(os.path.join(ROOT, "MEASURED_PEAKS.json"))
    hbm_peak = peaks["hbm_gbs"] if peaks else 6650.0
    achieved = bytes_ / (ms * 1e-3) / 1e9
    # host buffers: x in, y out per step
    xp = torch.from_numpy(xh.copy()).pin_memory()
    yp = torch.zeros(rows, dtype=torch.float64).pin_memory()
    C.check(L.bosss_b200_bsr_spmv(A, 1.0, C.ptr(xp), 0.0, C.ptr(yp)))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        C.check(L.bosss_b200_bsr_spmv(A, 1.0, C.ptr(xp), 0.0, C.ptr(yp)))
    e2e_s = (time.perf_counter() - t0) / args.steps
    assert np.array_equal(yp.numpy(), y.cpu().numpy())
    # CPU restatement, median of 5 on all host threads
    cores = orc.threads(os.cpu_count() or 1)
    orc.bsr_spmv(rp, ci, vals, 1.0, xh, 0.0, np.zeros(rows))
    tc = []
    for _ in range(5):
        t0 = time.perf_counter()
        orc.bsr_spmv(rp, ci, vals, 1.0, xh, 0.0, np.zeros(rows))
        tc.append(time.perf_counter() - t0)
    C.lib().bosss_b200_bsr_destroy(A)
    line = {
        "metric": "bsr_spmv_row_updates_per_s", "value": rows / (ms * 1e-3), "unit": "rows/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "bsr_spmv_hex48_k2", "block_rows": nbr, "blocks": int(rp[-1]), "block": [npc, npc],
                   "l2": "flushed between steps (512 MB write outside the timed events)"},
        "rel_err_vs_oracle": err,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak,
                     "traffic": (load_json(os.path.join(ROOT, "profiles", "traffic.json")) or {}).get(
                         "bsr_spmv_hex48_k2_bytes_per_launch"),
                     "kernel": "k_ell_spmv (sliced ELL copy of the block-sparse matrix, 32-row slices)",
                     "algorithmic_bytes": bytes_},
        "e2e": {"value": rows / e2e_s, "unit": "rows/s", "h2d_bytes_per_step": 8 * rows,
                "d2h_bytes_per_step": 8 * rows},
        "cpu_baseline": {"value": rows / float(np.median(tc)), "unit": "rows/s", "cores": cores, "kind": "port",
                         "sample": "median of 5 full SpMVs, C++ restatement of BlockMsrMatrix.SpMV (OpenMP)"},
        "gpu_launches": args.steps, "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_newton(args):
    """Matrix-free Newton-GMRES (exact JVP; multigrid V-cycle or block-Jacobi preconditioner) on
    the nonlinear diffusion problem, to a 1e-10 relative residual, confirmed by the oracle.
    Beside the solve time: the device time of one JVP, one V-cycle and one Jacobian assembly
    at the solution, the per-iteration budget the solver's iteration rate is compared with."""
    import torch
    from bosss_b200 import _capi as C
    from bosss_b200 import problems as P
    from oracle import oracle as orc
    pr = P.nonlinear_diffusion3d(n=args.n, k=args.k, seed=3000, source=1.0)
    precond = {"multigrid": 2, "block-jacobi": 1, "none": 0}[args.precond or "multigrid"]
    with pr.evaluator() as ev:
        t0 = time.perf_counter()
        U, rep = ev.NewtonSolve(np.zeros(pr.n_dofs), rtol=1e-10, restart=60, max_krylov=3000, inner_rtol=1e-6,
                                precond=precond, precond_update=args.precond_update)
        dt = time.perf_counter() - t0
        # component times at the solution (device events, legacy stream)
        dev = torch.device("cuda", 0)
        Ud = torch.from_numpy(U).to(dev)
        V = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, pr.n_dofs)).to(dev)
        Y = torch.zeros_like(V)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def timed(fn, reps=20):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps

        legacy = ctypes.c_void_p(C.CUDA_STREAM_LEGACY)
        ms_jvp = timed(lambda: C.check(C.lib().bosss_b200_jvp_device(ev.handle, C.ptr(Ud), C.ptr(V), C.ptr(Y), 0.0,
                                                                     legacy)))
        t0a = time.perf_counter()
        A = ev.ComputeJacobian(U)
        s_assembly = time.perf_counter() - t0a
        ms_vcycle = None
        if precond == 2:
            M = ev.Multigrid(A)
            ms_vcycle = timed(lambda: M.apply_device(V, Y, legacy))
            M.Dispose()
        A.Dispose()
    R = orc.evaluate(*pr.descs(), U)
    R0 = orc.evaluate(*pr.descs(), np.zeros(pr.n_dofs))
    line = {"metric": "newton_gmres_solve_time", "value": dt, "unit": "s", "n_gpus": 1, "higher_is_better": False,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": pr.config["workload"] + "_newton_gmres", "dofs": pr.n_dofs,
                       "preconditioner": args.precond or "multigrid", "precond_update": args.precond_update, "restart": 60,
                       "inner_rtol": 1e-6},
            "report": rep, "oracle_relative_residual": float(np.linalg.norm(R) / np.linalg.norm(R0)),
            "ms_jvp": ms_jvp, "ms_vcycle": ms_vcycle, "s_jacobian_assembly": s_assembly,
            "krylov_iters_per_s": rep["krylov_iters"] / dt}
    print(json.dumps(line), flush=True)


def run_xdg(args):
    """XDG two-phase Poisson, 128^3, k=2: rule construction (moments + weights on the device,
    surface rules on the host) and one step = the per-species bulk evaluation of both species
    followed by the level-set interface term (XLaplace_Interface, SIP, mu 1 / 10)."""
    import torch
    from bosss_b200 import _capi as C
    from bosss_b200 import operator as O
    from bosss_b200 import problems as P
    opA, opB, g, c, UA, UB = P.xdg_poisson3d(n=128, k=2, seed=4000)
    t0 = time.perf_counter()
    rule = C.XDG_RULE_SAYE if args.xdg_rule == "saye" else C.XDG_RULE_MOMENT_FITTING
    X = O.XdgEvaluator(opA, opB, g, 2, c, 0.4, rule=rule)
    torch.cuda.synchronize()
    t_rules = time.perf_counter() - t0
    t0 = time.perf_counter()
    X.SetInterface(1.0, 10.0, 4.0, X.SIP, 6)
    t_surface = time.perf_counter() - t0
    if_rules = X.interface_rules()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    U = [torch.from_numpy(UA).to(dev), torch.from_numpy(UB).to(dev)]
    out = [torch.zeros_like(U[0]), torch.zeros_like(U[1])]
    for _ in range(max(args.warmup, 3)):
        for s in (0, 1):
            X.Evaluate(s, 1.0, 0.0, out[s], U[s])
        X.EvaluateInterface(1.0, U[0], U[1], out[0], out[1])
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    t_bulk, t_if = 0.0, 0.0
    for _ in range(args.steps):
        e0.record(stream)
        for s in (0, 1):
            X.Evaluate(s, 1.0, 0.0, out[s], U[s])
        e1.record(stream)
        X.EvaluateInterface(1.0, U[0], U[1], out[0], out[1])
        e2.record(stream)
        torch.cuda.synchronize()
        t_bulk += e0.elapsed_time(e1)
        t_if += e1.elapsed_time(e2)
    ms = (t_bulk + t_if) / args.steps
    infos = [X.info(0), X.info(1)]
    dofs = sum(i["cells"] for i in infos) * 10
    line = {"metric": "xdg_dof_updates_per_s", "value": dofs / (ms * 1e-3), "unit": "DOF/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "xdg_poisson_128^3_k2_both_species_bulk+interface",
                                            "rule_family": args.xdg_rule,
                                            "species_dofs": dofs, "rule_construction_s": t_rules,
                                            "surface_rule_construction_s": t_surface,
                                            "surface_cells": int(len(if_rules["cells"])),
                                            "surface_nodes": int(if_rules["weights"].size),
                                            "species_A": infos[0], "species_B": infos[1]},
            "ms_bulk": t_bulk / args.steps, "ms_interface": t_if / args.steps}
    print(json.dumps(line), flush=True)
    X.Dispose()


def run_rk(args):
    """Classical RK4 time steps (RungeKutta.Perform) of the Euler 32^3 k=3 workload: each step
    is four residual launches and four fused stage-combination launches, captured once into a
    CUDA graph; value = DOF stage-updates/s (DOFs x 4 per step). Beside it: the same steps as
    an uncaptured host loop of residual launches and torch vector updates."""
    import torch
    from bosss_b200 import problems as P
    from bosss_b200 import timestepping as T
    pr = P.euler3d(n=args.n, k=args.k, seed=2000)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ev = pr.evaluator()
    scheme = T.RungeKuttaScheme.RungeKutta1901()
    rk = T.RungeKutta(scheme, ev, None)
    dt = 1e-4
    U = torch.from_numpy(pr.U).to(dev)
    nsteps = max(args.steps // 10, 5)
    rk.PerformDevice(U, dt, nsteps=max(args.warmup, 3))
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rk.PerformDevice(U, dt, nsteps=nsteps)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / nsteps

    # uncaptured host loop: k_s = Op(u_s) with evaluate_device, stage sums with torch
    a, b = scheme.a, scheme.b
    K = [torch.empty_like(U) for _ in range(4)]
    us = torch.empty_like(U)

    def host_step():
        for s_ in range(4):
            us.copy_(U)
            for r in range(s_):
                if a[s_, r] != 0.0:
                    us.add_(K[r], alpha=-dt * a[s_, r])
            ev.Evaluate(1.0, 0.0, K[s_], us)
        for s_ in range(4):
            U.add_(K[s_], alpha=-dt * b[s_])

    for _ in range(3):
        host_step()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(nsteps):
        host_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_host = e0.elapsed_time(e1) / nsteps
    ev.Dispose()
    value = 4 * pr.n_dofs / (ms * 1e-3)
    line = {"metric": "rk4_dof_stage_updates_per_s", "value": value, "unit": "DOF/s", "n_gpus": 1,
            "steps": nsteps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": pr.config["workload"] + "_rk4", "dofs": pr.n_dofs, "dt": dt,
                       "launch": "one step captured in a CUDA graph: 4 residual + 4 stage-combination launches",
                       "l2": "not flushed (working set of U, k_0..k_3 and u_s: 6 x %.0f MB)" % (pr.n_dofs * 8 / 1e6)},
            "host_loop": {"ms_per_step": ms_host, "value": 4 * pr.n_dofs / (ms_host * 1e-3),
                          "graph_speedup": ms_host / ms},
            "gpu_launches": 8 * nsteps, "clocks": clk}
    print(json.dumps(line), flush=True)


def run_partitioned(args, rank, world, local):
    """Weak scaling over N GPUs: the Euler workload on a periodic (N*n) x n x n grid, each rank
    owning an x-slab of n planes (n^3 cells, as on one GPU) plus one ghost plane per side. A
    step posts the exchange of the ghost planes of U and W (NCCL point-to-point over NVLink),
    evaluates the residual and the VJP of the interior cells while it is in flight, then the
    planes next to the ghosts. value = DOF-updates of all ranks / max-over-ranks time."""
    import ctypes  # noqa: F401
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from bosss_b200 import _capi as C
    from bosss_b200 import distributed as Dd
    from bosss_b200 import problems as P
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    pr = P.euler3d(n=args.n, k=args.k, seed=2000, nx=args.n * world)
    npc = pr.n_dofs // pr.grid.NoOfCells
    part = Dd.SlabPartition(pr.grid, world, rank, npc)
    pe = Dd.PartEvaluator(pr.op, pr.grid, [args.k] * 5, [args.k] * 5, part, device=local)
    halo = Dd.HaloExchange(part)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    Wg = np.random.default_rng(77).uniform(-1, 1, pr.n_dofs)
    U = torch.from_numpy(part.from_global(pr.U)).to(dev)
    W = torch.from_numpy(part.from_global(Wg)).to(dev)
    R = torch.zeros_like(U)
    G = torch.zeros_like(U)
    interior, rims = part.interior_cells(), part.rim_cells()
    ranges = ([interior] if interior[1] > interior[0] else []) + rims
    n_own = part.count * part.plane_dofs

    def step():
        reqs = halo.start(U, W)
        if interior[1] > interior[0]:
            pe.apply(C.MODE_RESIDUAL, U, None, R, interior)
            pe.apply(C.MODE_VJP, U, W, G, interior)
        Dd.HaloExchange.wait(reqs)
        for cells in rims:
            pe.apply(C.MODE_RESIDUAL, U, None, R, cells)
            pe.apply(C.MODE_VJP, U, W, G, cells)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world == 1:
        # one part: the owned cells must equal the whole-grid evaluator's results
        with pr.evaluator(device=local) as ev:
            Rw = torch.zeros_like(R)
            ev.Evaluate(1.0, 0.0, Rw, U)
            Gw = ev.vjp(U, W)
            torch.cuda.synchronize()
            assert torch.equal(Rw, R) and torch.equal(Gw, G)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_(float(i))           # evict L2 outside the timed events
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = float(sum(a.elapsed_time(b) for a, b in evs))
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * 2 * n_own * args.steps / (total_ms * 1e-3)

    # end to end: owned U and W from pinned host memory, owned R and G back, every step
    Uh = part.own(U).cpu().pin_memory()
    Wh = part.own(W).cpu().pin_memory()
    Rh = torch.empty(n_own, dtype=torch.float64).pin_memory()
    Gh = torch.empty(n_own, dtype=torch.float64).pin_memory()

    def e2e_step():
        part.own(U).copy_(Uh, non_blocking=True)
        part.own(W).copy_(Wh, non_blocking=True)
        step()
        Rh.copy_(part.own(R), non_blocking=True)
        Gh.copy_(part.own(G), non_blocking=True)
        stream.synchronize()

    for _ in range(2):
        e2e_step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * 2 * n_own * args.steps / e2e_s
    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": "dg_residual_vjp_dof_updates_per_s", "value": value, "unit": "DOF/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": pr.config["workload"] + "_residual+vjp", "dofs": pr.n_dofs,
                       "dofs_per_rank": n_own, "cells_per_rank": part.count * part.plane_cells, "k": args.k,
                       "precision": "fp64", "l2": "flushed between steps (512 MB write outside the timed events)",
                       "parallelism": "x-slab domain decomposition over %d GPUs, ghost planes of U and W "
                                      "exchanged by NCCL point-to-point each step, overlapped with the "
                                      "interior cells" % world},
            "e2e": {"value": e2e, "unit": "DOF/s", "h2d_bytes_per_step": 16 * n_own, "d2h_bytes_per_step": 16 * n_own},
            "gpu_launches": 2 * len(ranges) * args.steps,
            "halo_bytes_per_step": 2 * 8 * part.plane_dofs * (part.ghost_lo + part.ghost_hi),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    pe.Dispose()
    if world > 1:
        dist.destroy_process_group()


# kernels of one call per kernel path (bosss_b200_kernel_info)
PATH_KERNELS = {1: "dg_cell_kernel<PhysEuler<3>,K,Q,%s>",
                2: "dg_slab_kernel<PhysEuler<3>,K,Q,%s>",
                3: "dg_slab_kernel<PhysEuler<3>,K,Q,%s> volume pass + k_euler_faces + k_euler_face_project",
                4: "tc_volume_kernel + %s face terms"}


def main():
    args = parse()
    if args.workload == "rk" and args.impl != "reference":
        return run_rk(args)
    if args.workload == "xdg" and args.impl != "reference":
        return run_xdg(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "batched-solve":
        return run_batched_solve(args)
    if args.workload == "spmv":
        return run_spmv(args)
    if args.workload == "newton":
        if args.n == 32 and args.k == 3:
            args.n, args.k = 48, 2
        return run_newton(args)
    rank, world, local = dist_env()
    if world > 1 or args.partitioned:
        return run_partitioned(args, rank, world, local)
    import torch
    import torch.distributed as dist
    import ctypes
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from bosss_b200 import _capi as C
    from bosss_b200 import problems as P

    pr = P.euler3d(n=args.n, k=args.k, seed=2000 + rank)
    kern = {"auto": C.KERNEL_AUTO, "generic": C.KERNEL_GENERIC, "slab": C.KERNEL_SLAB,
            "faces": C.KERNEL_FACES}[args.kernel]
    ev = pr.evaluator(device=local, kernel=kern)
    path_res, launch_res = ev.kernel_info(C.MODE_RESIDUAL)
    path_vjp, launch_vjp = ev.kernel_info(C.MODE_VJP)
    L = C.lib()
    dev = torch.device("cuda", local)
    n = pr.n_dofs
    U = torch.from_numpy(pr.U).to(dev)
    W = torch.from_numpy(np.random.default_rng(77 + rank).uniform(-1, 1, n)).to(dev)
    R = torch.zeros(n, dtype=torch.float64, device=dev)
    G = torch.zeros(n, dtype=torch.float64, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(dev)          # all timed work and the events on one stream
    torch.cuda.set_stream(stream)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    h = ev.handle

    def step():
        C.check(L.bosss_b200_evaluate_device(h, 1.0, 0.0, C.ptr(U), C.ptr(R), 0.0, sptr))
        C.check(L.bosss_b200_vjp_device(h, C.ptr(U), C.ptr(W), C.ptr(G), 0.0, sptr))

    launches_per_step = launch_res + launch_vjp
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev_s = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev_m = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev_e = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_(float(i))           # evict L2 outside the timed events
        ev_s[i].record(stream)
        C.check(L.bosss_b200_evaluate_device(h, 1.0, 0.0, C.ptr(U), C.ptr(R), 0.0, sptr))
        ev_m[i].record(stream)
        C.check(L.bosss_b200_vjp_device(h, C.ptr(U), C.ptr(W), C.ptr(G), 0.0, sptr))
        ev_e[i].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_res = [ev_s[i].elapsed_time(ev_m[i]) for i in range(args.steps)]
    t_vjp = [ev_m[i].elapsed_time(ev_e[i]) for i in range(args.steps)]
    total_ms = float(np.sum(t_res) + np.sum(t_vjp))
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * DOF_PER_STEP_FACTOR * n * args.steps / (total_ms * 1e-3)

    # ---- the plain fused FP64 kernel (generic, one CTA per tile) on the same state, for
    # the chosen-vs-plain ratio
    ev_plain = pr.evaluator(device=local, kernel=C.KERNEL_GENERIC)
    hp = ev_plain.handle
    Rp, Gp = torch.empty_like(R), torch.empty_like(G)   # R, G keep the chosen kernel's results
    for _ in range(3):
        C.check(L.bosss_b200_evaluate_device(hp, 1.0, 0.0, C.ptr(U), C.ptr(Rp), 0.0, sptr))
        C.check(L.bosss_b200_vjp_device(hp, C.ptr(U), C.ptr(W), C.ptr(Gp), 0.0, sptr))
    torch.cuda.synchronize()
    plain_ms = []
    for i in range(min(args.steps, 50)):
        flush.fill_(float(i))
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        C.check(L.bosss_b200_evaluate_device(hp, 1.0, 0.0, C.ptr(U), C.ptr(Rp), 0.0, sptr))
        C.check(L.bosss_b200_vjp_device(hp, C.ptr(U), C.ptr(W), C.ptr(Gp), 0.0, sptr))
        a1.record(stream)
        plain_ms.append((a0, a1))
    torch.cuda.synchronize()
    plain_step_ms = float(np.mean([a.elapsed_time(b) for a, b in plain_ms]))
    plain_value = world * DOF_PER_STEP_FACTOR * n / (plain_step_ms * 1e-3)
    plain_diff = max(float((Rp - R).abs().max() / R.abs().max()), float((Gp - G).abs().max() / G.abs().max()))
    ev_plain.Dispose()

    # ---- split precision: the residual's volume contractions on the tensor cores (exact
    # 8-bit slices, int32 accumulation, FP64 recombination), faces and VJP in FP64
    split = None
    try:
        ev_split = pr.evaluator(device=local, precision=C.PRECISION_SPLIT_FP32)
    except C.BosssError as ex:
        split = {"unavailable": str(ex)}
    if split is None:
        hs = ev_split.handle
        Rs, Gs = torch.empty_like(R), torch.empty_like(G)
        for _ in range(max(args.warmup, 3)):
            C.check(L.bosss_b200_evaluate_device(hs, 1.0, 0.0, C.ptr(U), C.ptr(Rs), 0.0, sptr))
            C.check(L.bosss_b200_vjp_device(hs, C.ptr(U), C.ptr(W), C.ptr(Gs), 0.0, sptr))
        torch.cuda.synchronize()
        sp = []
        for i in range(args.steps):
            flush.fill_(float(i))
            a0, a1, a2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a0.record(stream)
            C.check(L.bosss_b200_evaluate_device(hs, 1.0, 0.0, C.ptr(U), C.ptr(Rs), 0.0, sptr))
            a1.record(stream)
            C.check(L.bosss_b200_vjp_device(hs, C.ptr(U), C.ptr(W), C.ptr(Gs), 0.0, sptr))
            a2.record(stream)
            sp.append((a0, a1, a2))
        torch.cuda.synchronize()
        C.check(L.bosss_b200_synchronize(hs))   # reports an expired tensor-core wait
        s_res = [a.elapsed_time(b) for a, b, _ in sp]
        s_vjp = [b.elapsed_time(c) for _, b, c in sp]
        s_total = float(np.sum(s_res) + np.sum(s_vjp))
        split = {"value": DOF_PER_STEP_FACTOR * n * args.steps / (s_total * 1e-3), "unit": "DOF/s",
                 "ms_per_step": s_total / args.steps, "ms_residual": float(np.mean(s_res)),
                 "ms_vjp": float(np.mean(s_vjp)), "launches_per_step": 3,
                 "residual_rel_l2_vs_fp64": float(torch.linalg.norm(Rs - R) / torch.linalg.norm(R)),
                 "residual_over_fp64_residual_time": float(np.mean(s_res)) / float(np.mean(t_res)),
                 "kernels": "tc_volume_kernel (tcgen05 kind::i8, volume terms) + dg_slab_kernel faces-only pass; "
                            "VJP: dg_slab_kernel FP64"}
        ev_split.Dispose()

    # ---- end to end through the host-buffer C-ABI (pinned host memory)
    Uh = torch.from_numpy(pr.U.copy()).pin_memory()
    Wh = torch.from_numpy(W.cpu().numpy()).pin_memory()
    Rh = torch.zeros(n, dtype=torch.float64).pin_memory()
    Gh = torch.zeros(n, dtype=torch.float64).pin_memory()
    # one host call per step: residual and VJP at the same state, U and W uploaded once,
    # transfers streamed by chunks of x-planes and overlapped with the evaluation
    for _ in range(2):
        C.check(L.bosss_b200_residual_vjp(h, 1.0, 0.0, C.ptr(Uh), C.ptr(Rh), C.ptr(Wh), C.ptr(Gh), 0.0))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        C.check(L.bosss_b200_residual_vjp(h, 1.0, 0.0, C.ptr(Uh), C.ptr(Rh), C.ptr(Wh), C.ptr(Gh), 0.0))
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * DOF_PER_STEP_FACTOR * n * args.steps / e2e_s
    # U and W in, R and J^T W out
    h2d = 8 * (n + n)
    d2h = 8 * (n + n)
    # the host-buffer path must agree with the device-resident one (both outputs)
    assert np.array_equal(Rh.numpy(), R.cpu().numpy())
    assert np.array_equal(Gh.numpy(), G.cpu().numpy())

    # ---- roofline: the VJP launch dominates the step (ncu launch list in profiles/)
    peaks = load_json(os.path.join(ROOT, "MEASURED_PEAKS.json"))
    hbm_peak = peaks["hbm_gbs"] if peaks else 6650.0
    prof = load_json(os.path.join(ROOT, "profiles", "traffic.json")) or {}
    flops = load_json(os.path.join(ROOT, "profiles", "flops.json")) or {}
    t_r = float(np.mean(t_res)) * 1e-3
    t_v = float(np.mean(t_vjp)) * 1e-3
    bytes_res = 8.0 * (n + n)          # U in, R out
    bytes_vjp = 8.0 * (n + n + n)      # U, W in, J^T W out
    # ncu figures per call (summed over the call's launches) exist for the 32^3 k=3 workload
    # on the slab path ("euler3d_*") and on the face-once path ("euler3d_faces_*")
    def _prof(table, path, what):
        if (args.n, args.k) != (32, 3) or path not in (2, 3):
            return None
        return table.get(("euler3d_" if path == 2 else "euler3d_faces_") + what)
    per_kernel = {
        "residual": {"ms": t_r * 1e3, "algorithmic_bytes": bytes_res, "hbm_gbs": bytes_res / t_r / 1e9,
                     "launches": launch_res, "kernels": PATH_KERNELS[path_res] % "RESIDUAL",
                     "traffic": _prof(prof, path_res, "residual_bytes_per_launch"),
                     "fp64_flops": _prof(flops, path_res, "residual_fp64_flops_per_launch")},
        "vjp": {"ms": t_v * 1e3, "algorithmic_bytes": bytes_vjp, "hbm_gbs": bytes_vjp / t_v / 1e9,
                "launches": launch_vjp, "kernels": PATH_KERNELS[path_vjp] % "VJP",
                "traffic": _prof(prof, path_vjp, "vjp_bytes_per_launch"),
                "fp64_flops": _prof(flops, path_vjp, "vjp_fp64_flops_per_launch")},
    }
    for kk, t in (("residual", t_r), ("vjp", t_v)):
        f = per_kernel[kk]["fp64_flops"]
        per_kernel[kk]["fp64_tflops"] = (f / t / 1e12) if f else None
    achieved = per_kernel["vjp"]["hbm_gbs"]
    traffic = per_kernel["vjp"]["traffic"]
    fp64_flops = per_kernel["vjp"]["fp64_flops"]
    t_r = t_v   # the fp64 figure below refers to the dominant kernel

    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": "dg_residual_vjp_dof_updates_per_s", "value": value, "unit": "DOF/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": pr.config["workload"] + "_residual+vjp", "dofs": n, "cells": pr.grid.NoOfCells,
                       "k": args.k, "quad_nodes_1d": ev.quad_nodes_1d, "precision": "fp64",
                       "l2": "flushed between steps (512 MB write outside the timed events)",
                       "parallelism": "independent instance per rank" if world > 1 else "single GPU"},
            "ms_residual": float(np.mean(t_res)), "ms_vjp": float(np.mean(t_vjp)),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic,
                         "kernel": "VJP call (dominant): " + PATH_KERNELS[path_vjp] % "VJP",
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650"},
            "fp64": {"kernel": "VJP", "flops_per_launch": fp64_flops,
                     "achieved_tflops": (fp64_flops / t_r / 1e12) if fp64_flops else None,
                     "nominal_peak_tflops": 37.0,
                     "note": "FP64 pipe bound; flops per launch from the ncu capture in profiles/"},
            "per_kernel": per_kernel,
            "plain_fp64": {"kernel": "dg_cell_kernel (generic fused FP64, one CTA per tile of cells)",
                           "value": plain_value, "ms_per_step": plain_step_ms,
                           "chosen_over_plain": value / plain_value,
                           "max_rel_diff": plain_diff},
            "split_fp32": split,
            "e2e": {"value": e2e, "unit": "DOF/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk,
        }
        if world == 1:
            line["cpu_baseline"] = cpu_baseline_sample(args)
        print(json.dumps(line), flush=True)
    ev.Dispose()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
