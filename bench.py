"""Benchmark of the Biot LBM hot path on B200.

Default workload (one line of JSON on rank 0): D2Q9 Darcy flow on a 1024 x 1024
grid with log-normal permeability (GRF, correlation length 16 cells, sigma 1,
seed 0), per-cell omega, Dirichlet pressure left/right, no flux top/bottom,
FP32 populations with an FP64 residual norm.  One step = 200 fused sweeps
(one CUDA-graph replay) plus the FP64 residual reduction.  ``value`` is GLUPS
(10^9 lattice-cell updates per second) with the populations resident in HBM;
``e2e`` adds, per step, the host->device copy of the populations from pinned
host memory and the device->host read of the residual.  L2 is flushed (a
256 MiB write) between timed steps.

``--impl reference`` times the CPU restatement of the reference's JAX solver
(the oracle, NumPy) on the host on a bounded sample of the same workload.

Multi-GPU (``torchrun --nproc-per-node N``): the Darcy path of the reference
runs one domain per device, and a second GPU holds an independent replica
(replicas only, weak scaling); timing is the max over ranks.
"""
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

SWEEPS_PER_STEP = 200
N = 1024
BYTES_PER_LU_F32 = (9 + 9 + 1) * 4     # read f, write f, read per-cell omega
METRIC = "GLUPS"
SPEC_HBM_GBS = 8000.0                  # B200 HBM3e specification (the roofline's second denominator)
WORKLOAD = "darcy_d2q9_1024x1024_lognormal_k"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled every ~10 ms during
    the timed region, read through NVML (read-only queries; nvidia-smi as the
    fallback).  The GPU is identified by the CUDA device's UUID."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.stop_flag = threading.Event()
        self.thread = None
        self.source = None

    def _handle(self, nv):
        import torch
        nv.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            import pynvml as nv
            h = self._handle(nv)
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            masks = [(name, getattr(nv, attr, 0)) for name, attr in self.REASONS]
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def run():
                while not self.stop_flag.is_set():
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        r = get_reasons(h)
                        self.samples.append((float(sm), float(mx), [n for n, m in masks if m and (r & m)]))
                    except Exception:
                        pass
                    time.sleep(0.01)
            self.source = "nvml"
            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
        except Exception:
            self._start_smi()

    def _start_smi(self):
        fields = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={fields}",
                                     "--format=csv,noheader,nounits", "-lms", "50"],
                                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return
        self.source = "nvidia-smi"
        self.proc = proc

        def run():
            for line in proc.stdout:
                p = [x.strip() for x in line.split(",")]
                try:
                    self.samples.append((float(p[0]), float(p[1]),
                                         [n for (n, _), v in zip(self.REASONS, p[2:6]) if v.lower() == "active"]))
                except (ValueError, IndexError):
                    continue
        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        self.stop_flag.set()
        if getattr(self, "proc", None) is not None:
            self.proc.terminate()
        if self.thread is not None:
            self.thread.join(timeout=5)
        if not self.samples:
            return None
        sm = [s[0] for s in self.samples]
        reasons = sorted({r for s in self.samples for r in s[2]})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(s[1] for s in self.samples)),
                "reasons": reasons, "samples": len(sm), "source": self.source}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, cold caches, read from "
                  "profiles/darcy_sweep_1024x1024_lognormal.md (not measured in this run)")


def ncu_traffic_per_launch():
    """DRAM bytes per launch of the Darcy sweep from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "darcy_sweep_1024x1024_lognormal.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def cpu_oracle_glups(seconds=12.0, n=N):
    """The oracle (NumPy, one host thread) on the same workload: full-size
    sweeps until ``seconds`` of CPU work are done."""
    import oracle.api as O
    from xlb_biot_b200.workloads import darcy_lognormal
    solver, _ = darcy_lognormal(O, n=n)
    f = solver.assign_fields_sharded()
    f, _ = solver.step(f, 0)             # warm-up
    t0 = time.perf_counter()
    sweeps = 0
    while time.perf_counter() - t0 < seconds:
        f, _ = solver.step(f, sweeps)
        sweeps += 1
    dt = time.perf_counter() - t0
    return n * n * sweeps / dt / 1e9, sweeps


def _reference_worker(steps, warmup, sweeps_per_step, barrier, queue):
    """One host process: the oracle's Darcy solver on the full workload, timed
    after a barrier shared with the other processes."""
    import oracle.api as O
    from xlb_biot_b200.workloads import darcy_lognormal
    solver, _ = darcy_lognormal(O, n=N)
    f = solver.assign_fields_sharded()
    for w in range(warmup):
        f, _ = solver.step(f, w)
    barrier.wait()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        for k in range(sweeps_per_step):
            f, _ = solver.step(f, k)
        times.append(time.perf_counter() - t0)
    queue.put(times)


def run_reference(args):
    """The reference's CPU path (its NumPy restatement: JAX is not installable
    offline) on every usable host core: one independent replica of the 1024^2
    workload per process (the path has no cross-core exchange), started
    together; GLUPS = all replicas' lattice updates / the slowest replica's time."""
    import multiprocessing as mproc
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sweeps_per_step = 3                      # bounded sample of the 200-sweep step
    cores = len(os.sched_getaffinity(0))
    mem_gb = os.sysconf("SC_PHYS_PAGES") * os.sysconf("SC_PAGE_SIZE") / 2 ** 30
    nproc = max(1, min(cores, 32, int(mem_gb // 2)))       # about 1 GB per replica, with margin
    ctx = mproc.get_context("spawn")
    barrier, queue = ctx.Barrier(nproc), ctx.Queue()
    procs = [ctx.Process(target=_reference_worker, args=(args.steps, args.warmup, sweeps_per_step, barrier, queue))
             for _ in range(nproc)]
    for p in procs:
        p.start()
    results = [queue.get() for _ in range(nproc)]
    for p in procs:
        p.join()
    totals = [float(np.sum(t)) for t in results]
    total = max(totals)
    glups = nproc * N * N * sweeps_per_step * args.steps / total / 1e9
    sample = (f"{nproc} concurrent processes (one per host core, capped at 32 and by memory), each "
              f"{sweeps_per_step} full 1024x1024 sweeps per step of the NumPy restatement of the reference's JAX "
              "Darcy solver (JAX is not installable offline)")
    line = {"impl": "reference", "metric": METRIC, "value": glups, "unit": "GLUPS", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nx": N, "ny": N, "sweeps_per_step": sweeps_per_step},
            "cpu_baseline": {"value": glups, "unit": "GLUPS", "cores": nproc, "kind": "port", "sample": sample},
            "e2e": {"value": glups, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def replica_totals(dev_ms, e2e_ms, ws, device):
    """Max over ranks of the device-timed totals.  Every rank runs one
    independent replica of the workload (the path has no data exchange on one
    node: replicas only, weak scaling), so the job's time is the slowest rank's."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([dev_ms, e2e_ms], dtype=torch.float64, device=device)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    return float(t[0]), float(t[1])


def replica_glups(lu_per_rank, ws, ms):
    """Whole-job GLUPS: the lattice updates of all ranks over the max time."""
    return ws * lu_per_rank / (ms * 1e-3) / 1e9


def run_ours(args):
    import torch
    import torch.distributed as dist
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import darcy_lognormal

    from xlb_biot_b200 import autotune
    solver, _ = darcy_lognormal(G, n=N)
    f0 = solver.assign_fields_sharded()
    # launch-shape autotuning on the production grid (outside every timed region)
    L = solver._layout
    bufs = [L.empty(9), L.empty(9)]
    bufs[0].copy_(f0)

    def tune_run():
        x, y = bufs
        for _ in range(10):
            solver._sweep(x, None, out=y)
            x, y = y, x
    if args.launch_shape:
        tx, depth, cps, mrows, pipe = (int(v) for v in args.launch_shape.split(","))
        autotune.set_config(autotune.DARCY, tx, depth, cps, mrows, pipe)
        tuned, table = autotune.get_config(autotune.DARCY), []
    else:
        tuned, tuned_ms, table = autotune.tune(autotune.DARCY, tune_run, key=f"f32|{N}x{N}|omega_field",
                                               use_cache=False)
    if os.environ.get("XLBB_TUNE_VERBOSE"):
        for ms, cfg in table[:20]:
            print(f"tune {ms / 10 * 1e3:8.2f} us/sweep {cfg}", file=sys.stderr)
    del bufs
    loop = solver.sweep_graph(SWEEPS_PER_STEP)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")     # 256 MiB > L2
    stream = torch.cuda.current_stream()

    # host buffers of the end-to-end variant (pinned)
    host_f = torch.empty(loop.state.shape[2] * loop.state.stride(2), dtype=loop.state.dtype).pin_memory()
    state_flat = loop.state.as_strided((host_f.numel(),), (1,))
    state_flat.copy_(f0.as_strided((host_f.numel(),), (1,)))
    host_f.copy_(state_flat)
    host_res = torch.empty(1, dtype=torch.float64).pin_memory()

    def device_step():
        loop.replay()

    for _ in range(max(3, args.warmup)):
        device_step()
    torch.cuda.synchronize()

    # -- device-resident timing (value) --------------------------------------
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for s in range(args.steps):
        flush.fill_(float(s))
        ev[s][0].record(stream)
        device_step()
        ev[s][1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    dev_ms = sum(a.elapsed_time(b) for a, b in ev)

    # -- end-to-end through the public loop with host buffers ------------------
    # Every step uploads its populations from pinned host memory and reads its
    # residual back.  The upload of step s + 1 runs on a copy stream into one of
    # two device staging buffers while step s sweeps; step s waits for its own
    # upload, copies it into the loop's state (device to device), flushes L2 and
    # sweeps.  Timed on the compute stream from before the first upload to after
    # the last read-back (everything inside the region, the first upload exposed).
    copy_stream = torch.cuda.Stream()
    staging = [torch.empty_like(state_flat), torch.empty_like(state_flat)]
    uploaded = [torch.cuda.Event(), torch.cuda.Event()]
    consumed = [torch.cuda.Event(), torch.cuda.Event()]

    def e2e_loop(steps):
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0.record(stream)
        copy_stream.wait_event(t0)

        def upload(k):
            b = k % 2
            with torch.cuda.stream(copy_stream):
                if k >= 2:
                    copy_stream.wait_event(consumed[b])     # step k - 2 has copied it out
                staging[b].copy_(host_f, non_blocking=True)
                uploaded[b].record(copy_stream)
        upload(0)
        for s in range(steps):
            if s + 1 < steps:
                upload(s + 1)
            b = s % 2
            stream.wait_event(uploaded[b])
            state_flat.copy_(staging[b])
            consumed[b].record(stream)
            flush.fill_(float(s))
            device_step()
            host_res.copy_(loop.sumsq, non_blocking=True)
        t1.record(stream)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1)
    e2e_loop(2)                                     # warm-up of the copy path
    e2e_ms = e2e_loop(args.steps)

    # -- per-launch kernel time for the roofline (same stream, no flush) --------
    kev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    reps = 5
    kev[0].record(stream)
    for _ in range(reps):
        device_step()
    kev[1].record(stream)
    torch.cuda.synchronize()
    per_sweep_ms = kev[0].elapsed_time(kev[1]) / (reps * SWEEPS_PER_STEP)

    pipeline = solver.sweep_pipeline()          # the launch the library resolved for this sweep
    out_of_l2 = None if args.no_out_of_l2 else darcy_out_of_l2(measured_peak_hbm()[0])
    dev_ms, e2e_ms = replica_totals(dev_ms, e2e_ms, ws, "cuda")
    value = replica_glups(N * N * SWEEPS_PER_STEP * args.steps, ws, dev_ms)
    e2e = replica_glups(N * N * SWEEPS_PER_STEP * args.steps, ws, e2e_ms)
    peak, peak_kind = measured_peak_hbm()
    achieved = N * N * BYTES_PER_LU_F32 / (per_sweep_ms * 1e-3) / 1e9
    traffic = ncu_traffic_per_launch()
    res = float(host_res[0])
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            g, sweeps = cpu_oracle_glups()
            cpu = {"value": g, "unit": "GLUPS", "cores": 1, "kind": "port",
                   "sample": f"{sweeps} full 1024x1024 sweeps of the NumPy restatement of the reference's Darcy "
                             "solver on one host thread"}
        line = {
            "metric": METRIC, "value": value, "unit": "GLUPS", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nx": N, "ny": N, "sweeps_per_step": SWEEPS_PER_STEP,
                       "permeability": "exp(GRF), SE covariance, ell=16 cells, sigma=1, seed 0",
                       "bcs": "ADR anti-bounce-back p=1 left, p=0 right; ADR bounce-back top/bottom",
                       "residual": "FP64 sum (f_new - f_old)^2 fused into the last sweep",
                       "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas{ws}",
                       "launch_shape": tuned},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "frac_of_spec": achieved / SPEC_HBM_GBS, "spec_gbs": SPEC_HBM_GBS,
                         "traffic": traffic, "traffic_source": TRAFFIC_SOURCE,
                         "algorithmic_bytes_per_launch": N * N * BYTES_PER_LU_F32,
                         "kernel": PIPELINE_KERNELS[pipeline], "kernel_ms": per_sweep_ms,
                         "out_of_l2": out_of_l2},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "GLUPS", "h2d_bytes_per_step": host_f.numel() * host_f.element_size(),
                    "copies": "every step uploads its populations from pinned host memory (the next step's on a "
                              "copy stream while this one sweeps) and reads its FP64 residual back; one timed "
                              "region on the compute stream, L2 flushed between steps inside it",
                    "d2h_bytes_per_step": 8},
            "gpu_launches": args.steps * loop.launches_per_replay,
            "clocks": clk,
            "residual_sumsq_last_sweep": res,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()
    return 0


def _timed(fn):
    import torch
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    out = fn()
    b.record()
    torch.cuda.synchronize()
    return out, a.elapsed_time(b) * 1e-3


def run_c1(args):
    """Plain elasticity, 128^2 periodic, lam = mu = 1, manufactured force, zero
    start, pseudo-time to a relative residual of 1e-8 (graph-captured sweeps,
    FP64 residual every 200 sweeps); FP32 and FP64 runs."""
    import numpy as np
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import plain_elasticity_128
    res = {}
    for prec in ("f32/f32", "f64/f64"):
        s, u = plain_elasticity_128(G, precision=prec)
        s.solve(tol=1e-8, check_every=200)                 # warm-up: module load, graph capture, clocks
        (f, it, rel), t = _timed(lambda: s.solve(tol=1e-8, check_every=200))
        eta, _ = s.update_macroscopic(f)
        res[prec] = (eta.double().cpu().numpy(), it, rel, t, s.stalled)
    e32, it, rel, t, stalled = res["f32/f32"]
    e64, it64, rel64, t64, _ = res["f64/f64"]
    # FP32 bulk sweeps to the FP64 tolerance: mixed-precision iterative refinement
    s, u = plain_elasticity_128(G, precision="f32/f32")
    s.solve_refined(tol=1e-8, check_every=200)           # warm-up: FP64 twin, graph capture
    (fr, itr, relr), tr = _timed(lambda: s.solve_refined(tol=1e-8, check_every=200))
    er, _ = s._twin.update_macroscopic(fr)
    er = er.double().cpu().numpy()
    st = s.refine_stats
    line = {"workload": "c1_plain_elasticity_128x128_periodic", "metric": "GLUPS",
            "value": 128 * 128 * itr / tr / 1e9, "unit": "GLUPS",
            "dtype": "f32 sweeps with f64 defects and master state (iterative refinement; reaches 1e-8)",
            "time_to_solution_s": tr, "sweeps": itr, "sweeps_f32": st["sweeps_f32"], "sweeps_f64": st["sweeps_f64"],
            "outer_steps": st["outer"], "relative_residual": relr,
            "rel_err_vs_exact": float(np.linalg.norm(er - u) / np.linalg.norm(u)),
            "rel_err_vs_fp64": float(np.linalg.norm(er - e64) / np.linalg.norm(e64)),
            "fp64": {"glups": 128 * 128 * it64 / t64 / 1e9, "seconds": t64, "sweeps": it64,
                     "relative_residual": rel64,
                     "rel_err_vs_exact": float(np.linalg.norm(e64 - u) / np.linalg.norm(u))},
            "fp32_plain": {"glups": 128 * 128 * it / t / 1e9, "seconds": t, "sweeps": it, "relative_residual": rel,
                           "stalled_at_rounding_floor": bool(stalled),
                           "rel_err_vs_exact": float(np.linalg.norm(e32 - u) / np.linalg.norm(u)),
                           "rel_err_vs_fp64": float(np.linalg.norm(e32 - e64) / np.linalg.norm(e64))},
            "note": "L2-resident 0.5 MB problem: launch/latency bound, sweeps replayed as CUDA graphs; "
                    "plain FP32 residuals cannot fall below ~1e-5 of the first update"}
    print(json.dumps(line), flush=True)
    return 0


def run_c3(args):
    """Periodic Biot 1024^2, 5-level V-cycle elasticity (FP32, FP64 coarsest
    level, 8 V-cycles per step as the reference's fixed N_E), FP64 pressure;
    compared with the all-FP64 run."""
    import numpy as np
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import periodic_biot_1024
    steps = args.biot_steps

    def run(prec, dprec, coarse):
        sim = periodic_biot_1024(G, precision=prec, darcy_precision=dprec, coarsest_precision=coarse)
        graph = sim.capture_step(*sim.init_state())          # the coupled step as one CUDA graph
        graph.replay()                                       # warm-up step
        graph.load(*sim.init_state())

        def body():
            out = None
            for _ in range(steps):
                out = graph.replay()
            return out
        out, secs = _timed(body)
        return sim, out, steps * sim.elasticitySteps, secs, graph

    sim, out, cycles, secs, _g = run("f32/f32", "f64/f64", "f64")
    n, L, k = 1024, 5, sim.elasticity.k_smooth
    sizes = [(n // 2 ** l) ** 2 for l in range(L)]
    lu_cycle = sum((2 * k + 1) * s for s in sizes[:-1]) + 2 * k * sizes[-1]
    lus = cycles * lu_cycle + steps * n * n
    ref = run("f64/f64", "f64/f64", None)
    eta = sim.elasticity.update_macroscopic(out[0])[0].double().cpu().numpy()
    eta_r = ref[0].elasticity.update_macroscopic(ref[1][0])[0].cpu().numpy()
    p, p_r = out[5].double().cpu().numpy(), ref[1][5].cpu().numpy()
    # roofline of the dominant kernel, the level-0 FP32 damped smoothing sweep
    # (collide and push): 8 populations read and written plus the coupling
    # force's 2 planes (and 2 for a static body force), 4 B each.  Its operands
    # (~75 MB) fit in L2, so L2 is flushed before each timed sweep by reading a
    # 256 MB buffer (clean lines: no write-back inside the timed sweep) and
    # each sweep is timed alone: the HBM-bound figure
    el = sim.elasticity
    L0 = el._L(0)
    f0, ext, buf = out[0], L0.zeros(2), L0.empty(8)
    planes = 8 + 8 + 2 + (2 if el.force is not None else 0)
    flush = torch.ones(64 << 20, dtype=torch.float32, device=f0.device)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(23)]
    for e0, e1 in evs:
        flush.sum()
        e0.record()
        el._sweep(f0, 0, 1.0 - el.gamma, el.gamma, fext=ext, out=buf)
        e1.record()
    torch.cuda.synchronize()
    t_sw = sum(e0.elapsed_time(e1) for e0, e1 in evs[3:]) * 1e-3      # 3 warm-up sweeps
    del flush
    (_, t_warm) = _timed(lambda: [el._sweep(f0, 0, 1.0 - el.gamma, el.gamma, fext=ext, out=buf) for _ in range(20)])
    peak, peak_kind = measured_peak_hbm()
    sweep_gbs = n * n * planes * 4 / (t_sw / 20) / 1e9
    line = {"workload": "c3_periodic_biot_1024x1024_mg5", "metric": "GLUPS", "value": lus / secs / 1e9,
            "unit": "GLUPS", "biot_steps": steps, "vcycles": cycles, "lattice_updates": lus,
            "seconds": secs, "dtype": "f32 elasticity, f64 coarsest level, f64 pressure",
            "material": "E=0.11, nu=0.8 (reference periodic examples); lam=2, mu=1 diverges in the reference's V-cycle",
            "inner_solve": f"{sim.elasticitySteps} V-cycles per step (the reference's fixed N_E)",
            "launch": "one CUDA graph replay per coupled step",
            "rel_err_u_vs_fp64": float(np.linalg.norm(eta - eta_r) / np.linalg.norm(eta_r)),
            "rel_err_p_vs_fp64": float(np.linalg.norm(p - p_r) / np.linalg.norm(p_r)),
            "fp64": {"seconds": ref[3], "vcycles": ref[2]},
            "roofline": {"kernel": "level-0 FP32 smoothing sweep (collide and push)", "bound": "hbm",
                         "achieved": sweep_gbs, "peak": peak, "unit": "GB/s", "frac": sweep_gbs / peak,
                         "frac_of_spec": sweep_gbs / SPEC_HBM_GBS, "spec_gbs": SPEC_HBM_GBS,
                         "peak_kind": peak_kind, "bytes_per_cell": planes * 4, "ms_per_sweep": t_sw / 20 * 1e3,
                         "l2": "flushed (read) before each timed sweep",
                         "ms_per_sweep_back_to_back": t_warm / 20 * 1e3}}
    print(json.dumps(line), flush=True)
    return 0


def run_c3inner(args):
    """The periodic Biot configuration with each step's inner elasticity solve
    run to a relative level-0 residual of 1e-8 (``elasticity_tol``; at most 200
    V-cycles per step) instead of a fixed cycle count: V-cycles per step and
    time, for FP64 and for FP32 smoothing with FP64 coarsest level and FP64
    level-0 residual arithmetic, on the first ``--biot-steps`` steps."""
    import numpy as np
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import periodic_biot_1024
    steps = args.biot_steps
    out = {}
    for name, kw in (("f64", dict(precision="f64/f64")),
                     ("f32", dict(precision="f32/f32", darcy_precision="f64/f64", coarsest_precision="f64",
                                  residual_precision="f64"))):
        sim = periodic_biot_1024(G, tol=1e-8, max_cycles=200, **kw)
        state = sim.init_state()
        cyc, rel = [], []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for t in range(steps):
            f_el, f_d, _, _, dt, _, _ = sim.step(*state, t)
            state = (f_el, f_d, dt)
            cyc.append(sim.last_inner_cycles)
            rel.append(sim.last_inner_rel)
        torch.cuda.synchronize()
        out[name] = {"vcycles_per_step": cyc, "final_relative_residual_per_step": rel,
                     "mean_contraction_per_cycle": float(np.mean([r ** (1.0 / max(1, c - 1)) for r, c in zip(rel, cyc)])),
                     "seconds": time.perf_counter() - t0, "capped_steps": int(sum(c >= 200 for c in cyc))}
    print(json.dumps({"workload": "c3_periodic_biot_1024x1024_inner_tol_1e-8", "metric": "V-cycles per step",
                      "unit": "cycles", "value": float(np.mean(out["f32"]["vcycles_per_step"])),
                      "higher_is_better": False, "biot_steps": steps, "runs": out,
                      "material": "E=0.11, nu=0.8 (reference periodic examples)"}), flush=True)
    return 0


def run_c4(args):
    """Batched multigrid elasticity: 512 heterogeneous periodic instances, each
    with its own level count (coarsest side 3-4 cells); FP32 storage and
    smoothing, FP64 arithmetic in the level-0 residual sweep, an FP64 coarsest
    level and FP64 norms; one launch per sweep for the whole batch, the V-cycle
    as one CUDA graph.  Each instance runs until its estimated relative error
    (coarse-correction norm x rho / (1 - rho)) is below 1e-6, and the solve
    ends by resetting the rigid-displacement mode that FP32 rounding lets drift
    (``remove_mean_moment``, inside the timed solve); the error is then
    measured against an all-FP64 batched solve to 1e-11 (the FP64 GPU oracle).
    Compared with looping the single-instance multigrid solver (same algorithm,
    levels and precisions, each instance run for the cycles it needed in the
    batch) over a sample."""
    import numpy as np
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    target, max_cycles = 1e-6, 200
    tol = target
    sizes, lams, mus, forces = batch_instances(count=args.instances)
    b = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision="f32/f32", coarsest_precision="f64",
                          residual_precision="f64", persistent_tail=args.tail_smem > 0,
                          tail_smem=max(args.tail_smem, 1))
    b.solve(tol=1e-2, max_cycles=3)                                   # warm-up + graph capture
    (cycles, est), secs = _timed(lambda: b.solve(tol=tol, max_cycles=max_cycles, criterion="error"))
    lu = b.lattice_updates_per_cycle() * cycles
    # roofline of the batched kernel: level-0 smoothing sweeps of the whole batch
    # (72 B per cell: 8 populations read and written, 2 force planes, FP32)
    lns = b.smooth_xy[0]
    (_, t_sw) = _timed(lambda: [b._sweep(0, ln, 1.0 - b.gamma, b.gamma) for _ in range(20) for ln in lns])
    cells0 = sum(nx * ny for nx, ny in sizes)
    peak, peak_kind = measured_peak_hbm()
    sweep_gbs = cells0 * 72 / (t_sw / 20) / 1e9

    # FP64 GPU oracle: the same batch in FP64 to a relative residual of 1e-11
    b64 = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision="f64/f64")
    cyc64, rel64 = b64.solve(tol=1e-11, max_cycles=400)
    err = np.array([float(torch.linalg.vector_norm(b.displacement(i) - b64.displacement(i))
                          / torch.linalg.vector_norm(b64.displacement(i))) for i in range(b.n)])
    del b64

    # looping the single-instance solver over a sample, each for its own cycle count
    sample = list(range(0, args.instances, max(1, args.instances // 24)))[:24]
    t_single, cyc_single = 0.0, 0
    for i in sample:
        n = sizes[i][0]

        class E(G.LBMElasticity):
            def get_force(self, _f=forces[i], _n=n):
                return self.distributed_array_init((_n, _n, 2), self.precisionPolicy.compute_dtype, init_val=_f)
        s = E(lattice=G.LatticeD2Q8("f32/f32"), **{"lambda": float(lams[i])}, mu=float(mus[i]), nx=n, ny=n, nz=0,
              precision="f32/f32", MG_levels=b.instance_levels[i], coarsest_precision="f64",
              residual_precision="f64", print_info_rate=0)
        s.step(s.assign_fields_sharded(), 0)                          # warm-up
        k = int(b.converged_at[i])

        def single(s=s, k=k):
            f = s.assign_fields_sharded()
            for t in range(k):
                f, _ = s.step(f, t)
            return f
        _, t1 = _timed(single)
        t_single += t1
        cyc_single += k
    single_sps = len(sample) / t_single
    line = {"workload": "c4_batched_mg_512_instances", "metric": "solves/s", "value": args.instances / secs,
            "unit": "solves/s", "instances": args.instances, "vcycles": cycles, "seconds": secs,
            "criterion": "estimated relative error < 1e-6 (coarse-correction norm x rho / (1 - rho)), or the "
                         "estimate stops falling (rounding floor of FP32 storage); then the drifted mean first "
                         "moment (rigid displacement, zero in exact arithmetic) is removed",
            "persistent_tail": {"tail_smem_bytes": args.tail_smem, "batched_levels": b.batched_depth,
                                "tail_start_level_counts": {str(k): int(v) for k, v in
                                                            zip(*np.unique(b.tail_start, return_counts=True))}},
            "instances_at_rounding_floor": int(b.stalled.sum()),
            "vcycles_per_instance": {"min": int(b.converged_at.min()), "median": float(np.median(b.converged_at)),
                                     "max": int(b.converged_at.max())},
            "displacement_rel_err_vs_fp64": {"max": float(err.max()), "median": float(np.median(err)),
                                             "count_above_1e-6": int((err > target).sum()),
                                             "count_above_1e-6_at_rounding_floor":
                                                 int(((err > target) & b.stalled).sum())},
            "fp64_oracle_vcycles": cyc64, "glups": lu / secs / 1e9,
            "single_instance_loop": {"solves_per_s": single_sps, "sample": len(sample),
                                     "mean_vcycles": cyc_single / len(sample)},
            "speedup_vs_single_loop": (args.instances / secs) / single_sps,
            "launches_per_vcycle": b.launches_per_cycle,
            "batched_sweep_roofline": {"bound": "hbm", "achieved": sweep_gbs, "peak": peak, "unit": "GB/s",
                                       "frac": sweep_gbs / peak, "peak_kind": peak_kind,
                                       "frac_of_spec": sweep_gbs / SPEC_HBM_GBS, "spec_gbs": SPEC_HBM_GBS,
                                       "kernel": batched_kernel_name(lns) + " (level-0 smoothing sweep, "
                                                 "all instances, 72 B/LU)", "sweep_ms": t_sw / 20 * 1e3},
            "dtype": "f32 storage and smoothing, f64 level-0 residual arithmetic, f64 coarsest level and norms",
            "levels": "per instance: coarsest side 3-4 cells (5 to 8 levels)",
            "material": "mu in [0.5, 2] / 16, nu in [0.1, 0.4] (lattice lambda + mu <= 0.29: the D2Q8 "
                        "model is singular at 1/3 and the reference's V-cycle diverges for moduli of order 1)"}
    print(json.dumps(line), flush=True)
    return 0


def batched_kernel_name(launches):
    """Kernel(s) of a list of FP32 batched sweep launches."""
    names = sorted({"xlbb::batched_push4_kernel<float>" if ln.vec else "xlbb::batched_push_kernel<float>"
                    for ln in launches})
    return " + ".join(names)


def run_c4sweep(args):
    """The batched kernel alone: level-0 damped smoothing sweeps (a = 1/4,
    b = 3/4) of the 512-instance batch, timed with CUDA events; prints the
    sweep's roofline (72 B per cell: 8 populations read and written, 2 force
    planes, FP32)."""
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=args.instances)
    b = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision="f32/f32", coarsest_precision="f64",
                          residual_precision="f64")
    lns = b.smooth_xy[0]
    for _ in range(max(3, args.warmup)):
        for ln in lns:
            b._sweep(0, ln, 0.25, 0.75)
    (_, t) = _timed(lambda: [b._sweep(0, ln, 0.25, 0.75) for _ in range(args.steps) for ln in lns])
    cells = sum(nx * ny for nx, ny in sizes)
    peak, peak_kind = measured_peak_hbm()
    gbs = cells * 72 / (t / args.steps) / 1e9
    print(json.dumps({"workload": "c4_batched_level0_sweep", "metric": "GB/s", "value": gbs, "unit": "GB/s",
                      "kernel": batched_kernel_name(lns), "launches_per_sweep": len(lns),
                      "cells": cells, "sweeps": args.steps, "ms_per_sweep": t / args.steps * 1e3,
                      "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                   "frac": gbs / peak, "peak_kind": peak_kind,
                                   "frac_of_spec": gbs / SPEC_HBM_GBS, "spec_gbs": SPEC_HBM_GBS}}), flush=True)
    return 0


def run_c4vcycle(args):
    """Whole batched V-cycles of the 512-instance batch (one CUDA-graph replay
    each, every level and transfer): ``--steps`` timed after ``--warmup``
    (the first captures the graph); the workload of the per-kernel launch
    list of a V-cycle."""
    import torch
    from xlb_biot_b200.batched import BatchedElasticity
    from xlb_biot_b200.workloads import batch_instances
    sizes, lams, mus, forces = batch_instances(count=args.instances)
    b = BatchedElasticity(sizes, lams, mus, forces, levels="auto", precision="f32/f32", coarsest_precision="f64",
                          residual_precision="f64", persistent_tail=args.tail_smem > 0,
                          tail_smem=max(args.tail_smem, 1))
    b.reset()
    for _ in range(max(3, args.warmup)):
        b.vcycle()
    (_, t) = _timed(lambda: [b.vcycle() for _ in range(args.steps)])
    lu = b.lattice_updates_per_cycle()
    print(json.dumps({"workload": "c4_batched_vcycle", "metric": "ms per V-cycle", "value": t / args.steps * 1e3,
                      "unit": "ms", "higher_is_better": False, "vcycles": args.steps,
                      "launches_per_vcycle": b.launches_per_cycle, "levels": b.levels,
                      "tail_smem_bytes": args.tail_smem, "batched_levels": b.batched_depth,
                      "glups": lu * args.steps / t / 1e9}), flush=True)
    return 0


def run_mlups2d(args):
    """The fluid path of ``examples/performance/MLUPS2d.py``: lid-driven cavity
    (Re = 100, u_wall = 0.1, full-way bounce-back walls, equilibrium lid),
    D2Q9, FP32, ``--cavity-n`` squared cells (4096^2: 1.2 GB of populations,
    far above L2), BGK and KBC collisions, ``--steps`` calls of the public
    ``step`` timed with CUDA events; roofline at 72 B per cell (9 populations
    read and written, FP32).  CPU baseline: the oracle's BGK step (vectorised
    NumPy, one process) on a 512^2 cavity."""
    import time
    import numpy as np
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import lid_driven_cavity as make_cavity
    n = args.cavity_n
    peak, peak_kind = measured_peak_hbm()
    out = {}
    for model in ("bgk", "kbc"):
        C, om = make_cavity(G, model)
        s = C(lattice=G.LatticeD2Q9("f32/f32"), omega=om(n), nx=n, ny=n, nz=0, precision="f32/f32")
        f = s.assign_fields_sharded()
        for t in range(args.warmup):
            f, _ = s.step(f, t)
        # the loop holds only its current state: the ping-pong pair of population
        # sets stays in the allocator's pool (no allocation inside the timed steps)
        state = [f]
        del f

        def loop():
            g = state.pop()
            for t in range(args.steps):
                g, _ = s.step(g, t)
            return g
        f, t = _timed(loop)
        mlups = n * n * args.steps / t / 1e6
        gbs = n * n * 72 * args.steps / t / 1e9
        out[model] = {"mlups": mlups, "ms_per_step": t / args.steps * 1e3,
                      "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                                   "peak_kind": peak_kind, "frac_of_spec": gbs / SPEC_HBM_GBS,
                                   "spec_gbs": SPEC_HBM_GBS},
                      "finite": bool(torch.isfinite(f).all())}
        del s, f
        torch.cuda.empty_cache()
    cpu = None
    if not args.no_cpu_baseline:
        import oracle.api as O
        Co, omo = make_cavity(O, "bgk")
        so = Co(lattice=O.LatticeD2Q9("f32/f32"), omega=omo(512), nx=512, ny=512, nz=0, precision="f32/f32")
        fo = so.assign_fields_sharded()
        fo, _ = so.step(fo, 0)
        t0, k = time.time(), 0
        while time.time() - t0 < 10.0:
            fo, _ = so.step(fo, k)
            k += 1
        cpu = {"value": 512 * 512 * k / (time.time() - t0) / 1e6, "unit": "MLUPS", "cores": 1, "kind": "port",
               "sample": f"oracle BGK cavity step (NumPy, FP32), 512^2 cells, {k} steps"}
    print(json.dumps({"workload": f"mlups2d_cavity_{n}x{n}", "metric": "MLUPS", "value": out["bgk"]["mlups"],
                      "unit": "MLUPS", "dtype": "f32", "steps": args.steps, "warmup": args.warmup,
                      "bgk": out["bgk"], "kbc": out["kbc"], "cpu_baseline": cpu,
                      "data": "synthetic (cavity from rest, as the example)"}), flush=True)
    return 0


def run_mlups3d(args):
    """The fluid path of ``examples/performance/MLUPS3d.py``: lid-driven cavity
    (Re = 100, u_wall = 0.1, full-way bounce-back on five faces, equilibrium
    lid), FP32, ``--cavity3d-n`` cubed cells (256^3: 1.3 GB of D3Q19
    populations, far above L2), BGK on D3Q19 (the example's lattice; the
    headline of this line) and D3Q27, and KBC on D3Q27, ``--steps`` calls of
    the public ``step`` timed with CUDA events; roofline at 8 q B per cell (q
    populations read and written, FP32).  CPU baseline: the oracle's D3Q19 BGK step (vectorised
    NumPy, one process) on a 64^3 cavity."""
    import time
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import lid_driven_cavity_3d as make_cavity
    n = args.cavity3d_n
    peak, peak_kind = measured_peak_hbm()
    out = {}
    for name, model in (("D3Q19", "bgk"), ("D3Q27", "bgk"), ("D3Q27", "kbc")):
        C, om = make_cavity(G, model=model)
        s = C(lattice=getattr(G, "Lattice" + name)("f32/f32"), omega=om(n), nx=n, ny=n, nz=n, precision="f32/f32",
              print_info_rate=0)
        q = s.q
        f = s.assign_fields_sharded()
        for t in range(args.warmup):
            f, _ = s.step(f, t)
        # the loop holds only its current state: the ping-pong pair of population
        # sets stays in the allocator's pool (no allocation inside the timed steps)
        state = [f]
        del f

        def loop():
            g = state.pop()
            for t in range(args.steps):
                g, _ = s.step(g, t)
            return g
        f, t = _timed(loop)
        cells = n ** 3
        gbs = cells * 8 * q * args.steps / t / 1e9
        out[name.lower() + ("" if model == "bgk" else "_kbc")] = {
                             "mlups": cells * args.steps / t / 1e6, "ms_per_step": t / args.steps * 1e3,
                             "bytes_per_lu": 8 * q,
                             "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                          "frac": gbs / peak, "peak_kind": peak_kind},
                             "finite": bool(torch.isfinite(f).all())}
        del s, f
        torch.cuda.empty_cache()
    cpu = None
    if not args.no_cpu_baseline:
        import oracle.api as O
        m = 64
        Co, omo = make_cavity(O)
        so = Co(lattice=O.LatticeD3Q19("f32/f32"), omega=omo(m), nx=m, ny=m, nz=m, precision="f32/f32")
        fo = so.assign_fields_sharded()
        fo, _ = so.step(fo, 0)
        t0, k = time.time(), 0
        while time.time() - t0 < 10.0:
            fo, _ = so.step(fo, k)
            k += 1
        cpu = {"value": m ** 3 * k / (time.time() - t0) / 1e6, "unit": "MLUPS", "cores": 1, "kind": "port",
               "sample": f"oracle D3Q19 BGK cavity step (NumPy, FP32), {m}^3 cells, {k} steps"}
    print(json.dumps({"workload": f"mlups3d_cavity_{n}^3", "metric": "MLUPS", "value": out["d3q19"]["mlups"],
                      "unit": "MLUPS", "dtype": "f32", "steps": args.steps, "warmup": args.warmup,
                      "d3q19": out["d3q19"], "d3q27": out["d3q27"], "d3q27_kbc": out["d3q27_kbc"],
                      "cpu_baseline": cpu,
                      "data": "synthetic (cavity from rest, as the example)"}), flush=True)
    return 0


def run_c2solve(args):
    """The Darcy configuration as stated: 1024^2, log-normal k, run to steady
    state at a relative residual ||f^{n+1} - f^n|| / ||f^1 - f^0|| < 1e-8
    (FP64 norms reduced on the device every ``check`` sweeps; the sweeps of one
    check interval are one CUDA-graph replay).  Three runs from the same start:
    all FP64; FP32 populations until the residual stops falling (the FP32
    rounding floor); FP32 correction sweeps under FP64 defects and master
    state (mixed-precision iterative refinement) to 1e-8.  Reports sweeps and
    time to solution and the relative L2 pressure error of each run against
    the FP64 run."""
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200 import autotune
    from xlb_biot_b200.workloads import darcy_lognormal
    autotune.set_config(autotune.DARCY, 128, 1, 1, 8, 3)
    check, tol = 2000, 1e-8
    out = {}

    def run(prec, f=None, r0=None, max_sweeps=10 ** 8):
        solver, _ = darcy_lognormal(G, n=N, precision=prec)
        solver.solve(solver.assign_fields_sharded(), tol=1.0, check_every=check)     # capture + warm-up
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        (fs, sweeps, rel), t = _timed(lambda: solver.solve(f, tol=tol, check_every=check, r0=r0,
                                                           max_sweeps=max_sweeps))
        clk = clocks.stop()
        p = solver.update_macroscopic(fs).double()
        return solver, fs, p, {"sweeps": int(sweeps), "seconds": t, "relative_residual": rel,
                               "stalled": bool(solver.stalled), "glups": N * N * sweeps / t / 1e9, "clocks": clk}
    s64, f64, p64, out["f64"] = run("f64/f64")
    # the error reference: the FP64 run continued to 1e-11 (a residual of 1e-8
    # still leaves the slow diffusion mode ~1e-8 / (1 - rho) away from the steady state)
    r0 = s64._sweep_loop(check, None).first(s64.assign_fields_sharded())
    fref, sref, relref = s64.solve(f64.clone(), tol=1e-11, check_every=check, r0=r0)
    pref = s64.update_macroscopic(fref).double()
    out["f64_reference_1e-11"] = {"extra_sweeps": int(sref), "relative_residual": relref}
    s32, f32, p32, out["f32"] = run("f32/f32")
    # FP32 bulk sweeps to the FP64 tolerance: mixed-precision iterative refinement
    s32.solve_refined(tol=1e-3, check_every=check)        # warm-up: FP64 twin, graph capture
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    (fr, sweeps, rel), t = _timed(lambda: s32.solve_refined(tol=tol, check_every=check))
    st = s32.refine_stats
    out["f32_refined"] = {"seconds": t, "sweeps_f32": st["sweeps_f32"], "sweeps_f64": st["sweeps_f64"],
                          "outer_steps": st["outer"], "relative_residual": rel,
                          "inner": [{k: v for k, v in d.items()} for d in st["inner"]],
                          "glups": N * N * sweeps / t / 1e9, "clocks": clocks.stop()}
    pr = s64.update_macroscopic(fr).double()

    def err(p, ref):
        return float(torch.linalg.vector_norm(p - ref) / torch.linalg.vector_norm(ref))
    out["f64"]["pressure_rel_err_vs_f64_1e-11"] = err(p64, pref)
    for k, p in (("f32", p32), ("f32_refined", pr)):
        out[k]["pressure_rel_err_vs_f64"] = err(p, p64)
        out[k]["pressure_rel_err_vs_f64_1e-11"] = err(p, pref)
    print(json.dumps({"workload": "c2_darcy_1024x1024_lognormal_steady_state", "metric": "time_to_solution",
                      "unit": "s", "higher_is_better": False, "value": out["f32_refined"]["seconds"],
                      "tolerance": tol, "check_every": check, "runs": out, "data": "synthetic"}), flush=True)
    return 0


PIPELINE_KERNELS = {0: "xlbb::sweep_kernel<DarcyPhys<float>>", 1: "xlbb::sweep_bulk_kernel<DarcyPhys<float>>",
                    2: "xlbb::sweep_warp_kernel<DarcyPhys<float>>", 3: "xlbb::push_kernel<DarcyPhys<float>>",
                    4: "xlbb::darcy_push4_kernel"}


def darcy_out_of_l2(peak, replays=5):
    """The headline Darcy sweep (same kernel, launch shape and 76 B per lattice
    update) measured out of L2: (a) 4096^2 cells (1.27 GB of populations and
    omega, ten times L2) in CUDA-graph replays of 20 sweeps; (b) 1024^2 with a
    256 MiB L2 flush before every single sweep, each sweep timed alone with
    CUDA events (median of 50)."""
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200.workloads import darcy_lognormal
    stream = torch.cuda.current_stream()
    out = {}
    n = 4096
    solver, _ = darcy_lognormal(G, n=n)
    loop = solver.sweep_graph(20)
    loop.state.copy_(solver.assign_fields_sharded())
    for _ in range(3):
        loop.replay()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(replays):
        loop.replay()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / (replays * 20)
    gbs = n * n * BYTES_PER_LU_F32 / (ms * 1e-3) / 1e9
    out["4096x4096_graph"] = {"us_per_sweep": ms * 1e3, "glups": n * n / (ms * 1e-3) / 1e9, "achieved_gbs": gbs,
                              "frac": gbs / peak, "kernel": PIPELINE_KERNELS[solver.sweep_pipeline()]}
    del solver, loop
    torch.cuda.empty_cache()
    solver, _ = darcy_lognormal(G, n=N)
    L = solver._layout
    x, y = L.empty(9), L.empty(9)
    x.copy_(solver.assign_fields_sharded())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    reps = 50
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for i in range(reps + 5):
        flush.fill_(float(i))
        if i >= 5:
            ev[i - 5][0].record(stream)
        solver._sweep(x, None, out=y)
        if i >= 5:
            ev[i - 5][1].record(stream)
        x, y = y, x
    torch.cuda.synchronize()
    ts = sorted(e0.elapsed_time(e1) for e0, e1 in ev)
    ms = float(np.median(ts))
    gbs = N * N * BYTES_PER_LU_F32 / (ms * 1e-3) / 1e9
    out["1024x1024_l2_flushed_each_sweep"] = {"us_per_sweep_median": ms * 1e3, "us_min": ts[0] * 1e3,
                                              "achieved_gbs": gbs, "frac": gbs / peak,
                                              "kernel": PIPELINE_KERNELS[solver.sweep_pipeline()]}
    del solver, x, y, flush
    torch.cuda.empty_cache()
    return out


def run_darcy_hbm(args):
    """The out-of-L2 measurements of the headline sweep alone (one JSON line)."""
    import torch
    from xlb_biot_b200 import autotune
    peak, peak_kind = measured_peak_hbm()
    shape = [int(v) for v in args.launch_shape.split(",")] if args.launch_shape else [128, 1, 1, 8, 3]
    autotune.set_config(autotune.DARCY, *shape)
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    out = darcy_out_of_l2(peak, replays=args.steps)
    clk = clocks.stop()
    print(json.dumps({"workload": "darcy_sweep_out_of_l2", "metric": "GB/s", "unit": "GB/s",
                      "value": out["4096x4096_graph"]["achieved_gbs"], "peak": peak, "peak_kind": peak_kind,
                      "bytes_per_lu": BYTES_PER_LU_F32, "launch_shape": shape, "runs": out, "clocks": clk}),
          flush=True)
    return 0


def run_c5(args):
    """Adjoint of heterogeneous Terzaghi-type consolidation: 512 x 256 cells
    (arrays 512 x 258 with the boundary rows), 200 Biot steps, each with 4
    five-level V-cycles (4 smoothing sweeps per level), checkpoints every 16
    steps; per-cell log-shear-modulus and log-permeability fields (seeded
    Gaussian random fields, correlation length 24 cells, sigma 0.5); misfit of
    the last step's displacement and pressure against a forward run with
    perturbed fields.  Gradients through ``ConsolidationMisfit`` (hand-written
    adjoint kernels, CUDA graphs for the forward step, the taping step and
    the adjoint step).  Reports backward / forward time, central finite
    differences along random directions (FP64), FP32 vs FP64 gradients."""
    import numpy as np
    import torch
    import xlb_biot_b200.api as G
    from xlb_biot_b200.biot_adjoint import BiotAdjointModel, ConsolidationMisfit, consolidation_parameters
    from xlb_biot_b200.workloads import gaussian_random_field, terzaghi_heterogeneous
    steps, ndir = args.adjoint_steps, args.fd_directions
    dev = torch.device("cuda")
    nx, ny = 512, 258

    def build(prec, log_mu=None, log_k=None):
        sim, mat = terzaghi_heterogeneous(G, precision=prec, log_mu=log_mu, log_k=log_k)
        return BiotAdjointModel(sim, steps, checkpoint_every=16, graphs=True), mat

    # observations: the same problem with perturbed material fields
    base_mu = gaussian_random_field(nx, ny, 24.0, 0.5, 0)
    base_k = gaussian_random_field(nx, ny, 24.0, 0.5, 1)
    pert_mu = base_mu + gaussian_random_field(nx, ny, 24.0, 0.1, 11)
    pert_k = base_k + gaussian_random_field(nx, ny, 24.0, 0.1, 12)
    mobs, _ = build("f64/f64", pert_mu, pert_k)
    mobs.forward()
    obs = (mobs.eta.double().clone(), mobs.p.double().clone())
    del mobs

    def grad(model):
        model.set_observations(*obs)
        lm = torch.as_tensor(base_mu, dtype=torch.float64, device=dev).requires_grad_()
        lk = torch.as_tensor(base_k, dtype=torch.float64, device=dev).requires_grad_()
        (J, t_f) = _timed(lambda: ConsolidationMisfit.apply(*consolidation_parameters(lm, lk), model))
        (_, t_b) = _timed(lambda: J.backward())
        return float(J.detach()), lm.grad.double(), lk.grad.double(), t_f, t_b

    out = {}
    for prec in ("f64/f64", "f32/f32"):
        model, _ = build(prec)
        grad(model)                                   # graph capture + warm-up
        J, gm, gk, t_f, t_b = grad(model)
        out[prec] = dict(J=J, gm=gm, gk=gk, forward_s=t_f, backward_s=t_b, model=model)
    # central differences along random directions (FP64, the same graphs)
    m64 = out["f64/f64"]["model"]
    rng = np.random.default_rng(3)
    errs = []
    lm0 = torch.as_tensor(base_mu, dtype=torch.float64, device=dev)
    lk0 = torch.as_tensor(base_k, dtype=torch.float64, device=dev)
    t0 = time.time()
    for _ in range(ndir):
        dm = torch.as_tensor(rng.standard_normal((nx, ny)), device=dev)
        dk = torch.as_tensor(rng.standard_normal((nx, ny)), device=dev)
        eps = 1e-5
        vals = []
        for sgn in (1.0, -1.0):
            m64.set_parameters(*consolidation_parameters(lm0 + sgn * eps * dm, lk0 + sgn * eps * dk))
            vals.append(m64.forward())
        fd = (vals[0] - vals[1]) / (2 * eps)
        ad = float((out["f64/f64"]["gm"] * dm).sum() + (out["f64/f64"]["gk"] * dk).sum())
        errs.append(abs(fd - ad) / abs(fd))
    t_fd = time.time() - t0
    errs = np.asarray(errs)

    def rel(a, b):
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    r32, r64 = out["f32/f32"], out["f64/f64"]
    levels, k, cyc = 5, 4, 4
    lus = steps * cyc * sum((2 * k + (1 if l < levels - 1 else 0)) * (nx >> l) * ((ny - 2) // 2 ** l + 2)
                            for l in range(levels))
    line = {"workload": "c5_adjoint_consolidation_512x256_200steps", "metric": "adjoint/forward time",
            "value": r32["backward_s"] / r32["forward_s"], "unit": "x", "higher_is_better": False,
            "fp32": {"forward_s": r32["forward_s"], "backward_s": r32["backward_s"],
                     "forward_glups": lus / r32["forward_s"] / 1e9},
            "fp64": {"forward_s": r64["forward_s"], "backward_s": r64["backward_s"],
                     "ratio": r64["backward_s"] / r64["forward_s"]},
            "backward_includes": "recomputation of every 16-step segment with tapes (checkpoints every 16 steps)",
            "fd_check_fp64": {"directions": ndir, "eps": 1e-5, "max_rel_err": float(errs.max()),
                              "median_rel_err": float(np.median(errs)), "seconds": t_fd},
            "fp32_vs_fp64_gradient_rel_err": {"log_mu": rel(r32["gm"], r64["gm"]),
                                              "log_k": rel(r32["gk"], r64["gk"])},
            "J": {"fp64": r64["J"], "fp32": r32["J"]},
            "steps": steps, "cycles_per_step": cyc, "levels": levels, "k_smooth": k,
            "peak_memory_gb": torch.cuda.max_memory_allocated() / 1e9}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-out-of-l2", action="store_true",
                    help="skip the out-of-L2 measurements of the headline sweep (4096^2; 1024^2 L2-flushed)")
    ap.add_argument("--launch-shape", default="",
                    help="tx,depth,ctas_per_sm,min_rows,pipeline of the Darcy sweep (skips the autotuner)")
    ap.add_argument("--elast-shape", default="",
                    help="tx,depth,ctas_per_sm,min_rows,pipeline of the elasticity sweeps (all workloads)")
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--fd-directions", type=int, default=32)
    ap.add_argument("--cavity-n", type=int, default=4096)
    ap.add_argument("--cavity3d-n", type=int, default=256)
    ap.add_argument("--workload", choices=["darcy", "c1", "c2solve", "c3", "c3inner", "c4", "c4sweep", "c4vcycle",
                                           "c5", "mlups2d", "mlups3d", "darcy_hbm"],
                    default="darcy",
                    help="darcy: the headline line; c1/c3/c4/c5: the other configurations (one JSON line each)")
    ap.add_argument("--biot-steps", type=int, default=100)
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--tail-smem", type=int, default=100 * 1024,
                    help="shared-memory budget (bytes) of the batched persistent multigrid tail; 0: no tail")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.elast_shape:
        from xlb_biot_b200 import autotune
        autotune.set_config(autotune.ELASTICITY, *[int(v) for v in args.elast_shape.split(",")])
    if args.workload == "c1":
        return run_c1(args)
    if args.workload == "c3":
        return run_c3(args)
    if args.workload == "c4":
        return run_c4(args)
    if args.workload == "c5":
        return run_c5(args)
    if args.workload == "c4sweep":
        return run_c4sweep(args)
    if args.workload == "c4vcycle":
        return run_c4vcycle(args)
    if args.workload == "mlups2d":
        return run_mlups2d(args)
    if args.workload == "mlups3d":
        return run_mlups3d(args)
    if args.workload == "c2solve":
        return run_c2solve(args)
    if args.workload == "c3inner":
        return run_c3inner(args)
    if args.workload == "darcy_hbm":
        return run_darcy_hbm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
