"""Benchmark of the B200 FDTD time-stepping path.

Workload (one bench "step"): the batched forward -- 256 seeded tubes of
uneven length (12-20 cm) and width (2-4 cm), 3:1 elliptical sections,
Gaussian source, 6-cell PML, FP32 fields, 50 ms simulated (33 075 time
steps) -- run through the C ABI.  Metric: Gcell-updates/s, one cell-update =
one interior cell advanced one full step (P and V).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the reference's CPU engine on the host cores over a
bounded sample of the same workload: its own FDTDEngineCPU compiled from the
reference sources (oracle/_ref/ref_engine; the grid setup runs on the GPU,
only the time loop is timed), or the oracle's FP32 restatement of it where
that binary is not built.
--profile-steps S builds the batch and runs S time steps, untimed, for ncu.
Under torchrun every rank runs its own 256-tube batch (weak scaling; no
collective on the data path) and rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "vocalsim-2p5d-fdtd_b200" / "python"))

N_TUBES = 256
SIM_STEPS = 33075                      # 50 ms at 44.1 kHz x 15
BYTES_PER_CELL_UPDATE = 37             # P,Vx,Vy read+write (24) + dP,dX,dY (12) + code (1)
METRIC = "Gcell-updates/s"
PEAKS = REPO / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def workload_config(n_tubes: int = N_TUBES, sim_steps: int = SIM_STEPS) -> dict:
    """The workload both arms measure: the 256-tube batch, 50 ms at fs = 44100 x 15."""
    return {"workload": f"batched forward, {n_tubes} seeded tubes 12-20 cm x 2-4 cm, 3:1 elliptical, Gaussian, PML 6, "
                        f"{sim_steps} steps (50 ms) at fs 661.5 kHz; one step = one full forward",
            "tubes": n_tubes, "sim_steps": sim_steps}


def rank_tube_seeds(rank: int, n_tubes: int) -> list[int]:
    """Seeds of the tubes rank `rank` owns: every rank runs its own disjoint batch (weak scaling)."""
    return [rank * n_tubes + i for i in range(n_tubes)]


def max_over_ranks(ms: float, world: int, device=None) -> float:
    """Slowest rank's time; the aggregate throughput divides all ranks' work by it."""
    if world <= 1:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def strong_seeds(rank: int, world: int, n_tubes: int) -> list[int]:
    """Strong scaling: the fixed batch of seeds 0..n_tubes-1 split across the
    ranks by LPT on each tube's interior cell count."""
    from vocalsim_b200 import synthetic as S
    import vocalsim_b200 as V
    from vocalsim_b200.sharding import shard_batch
    costs = [V.build_maps(V.params(cross_sectional_shape=2), V.Geometry(*S.batch_tube(sd)[:2]))["dims"]["interior_cells"]
             for sd in range(n_tubes)]
    return shard_batch(costs, rank, world)


def sum_over_ranks(x: int, world: int, device=None) -> int:
    if world <= 1:
        return int(x)
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
    return int(t.item())


def workload_params(rank: int, n_tubes: int, fast_math: int = 1, seeds=None):
    from vocalsim_b200 import synthetic as S
    import vocalsim_b200 as V
    ps, gs = [], []
    for seed in (rank_tube_seeds(rank, n_tubes) if seeds is None else seeds):
        L, A, _, _ = S.batch_tube(seed)
        ps.append(V.params(cross_sectional_shape=2, num_steps=SIM_STEPS, fast_math=fast_math))
        gs.append(V.Geometry(L, A))
    return ps, gs


def hbm_peak():
    if PEAKS.exists():
        d = json.loads(PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profiled_kernel(cells: int, shape: int, fast: int) -> dict:
    """DRAM bytes (read + write) per step-kernel launch and the issue-active
    percentage from the committed ncu summary of the same kernel (launch shape
    and arithmetic) on this same workload (same interior cell count); None
    where no summary matches."""
    out = {"traffic": None, "issue_active_pct": None}
    for name in ("quad2_kernel_fast_batch256.json", "quad_kernel_fast_batch256.json", "quad2_kernel_exact_batch256.json",
                 "strip_kernel_batch256.json"):
        f = REPO / "profiles" / name
        if not f.exists():
            continue
        d = json.loads(f.read_text())
        if int(d.get("interior_cells", -1)) != int(cells) or int(d.get("fast_math", 0)) != int(fast):
            continue
        by_shape = d.get("traffic_by_shape", {})
        if str(shape) in by_shape:
            out["traffic"] = int(by_shape[str(shape)]["dram_bytes_per_launch"])
        elif int(d.get("shape", -1)) == int(shape):
            out["traffic"] = int(d["dram_bytes_per_launch"])
        else:
            continue
        if str(shape) in by_shape and "smsp_issue_active_pct" in by_shape[str(shape)]:
            out["issue_active_pct"] = float(by_shape[str(shape)]["smsp_issue_active_pct"])
        elif int(d.get("shape", -1)) == int(shape) and "smsp_issue_active_pct" in d:
            out["issue_active_pct"] = float(d["smsp_issue_active_pct"])
        return out
    return out


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- CPU reference
def _cpu_worker(args):
    seed, steps = args
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    from vocalsim_b200 import synthetic as S
    L, A, _, _ = S.batch_tube(seed)
    p = O.params(cross_sectional_shape=2, num_steps=SIM_STEPS)
    g = O.Geometry(L, A)
    cells = O.maps(p, g)["dims"]["interior_cells"]
    t0 = time.perf_counter()
    O.run(p, g, steps, "f32")
    return cells * steps, time.perf_counter() - t0


def cpu_reference(n_tubes: int, steps_per_tube: int, procs: int):
    """Throughput of the FP32 CPU engine over `n_tubes` tubes x `steps_per_tube` steps, one process per core."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    work = [(i, steps_per_tube) for i in range(n_tubes)]
    with ctx.Pool(procs) as pool:
        pool.map(_cpu_worker, [(0, 10)] * procs)          # import + build cost outside the clock
        t0 = time.perf_counter()
        res = pool.map(_cpu_worker, work, chunksize=1)
        wall = time.perf_counter() - t0
    cell_updates = sum(r[0] for r in res)
    return cell_updates / wall / 1e9, wall, cell_updates


def ref_engine_available() -> bool:
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    return O.REF_ENGINE.exists()


def ref_engine_throughput(n_sample: int, steps: int, procs: int):
    """Throughput of the reference's own FDTDEngineCPU (oracle/_ref/ref_engine:
    its SimulationParams -> FDTDSolver::setupWaveSolver -> startSolverEngine
    compiled from the reference sources) on batch tubes 0..n_sample-1, `procs`
    processes at a time, one tube each.  Work = interior cells x steps; time =
    from the first loop's start to the last loop's end (monotonic clock), so
    set-up and process start-up are outside it."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    from concurrent.futures import ThreadPoolExecutor
    from vocalsim_b200 import synthetic as S

    def one(seed):
        L, A = S.batch_tube(seed)[:2]
        r = O.reference_engine(O.params(cross_sectional_shape=2), O.Geometry(L, A), steps, with_maps=False)
        m = r["meta"]
        return (m["frame_h"] - 2) * (m["frame_w"] - 2) * steps, m["loop_t0"], m["loop_t1"]

    with ThreadPoolExecutor(procs) as ex:
        res = list(ex.map(one, range(n_sample)))
    work = sum(x[0] for x in res)
    span = max(x[2] for x in res) - min(x[1] for x in res)
    return work / span / 1e9, span, work


REF_ENGINE_STEPS = 1500


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample_steps(n_sample: int) -> int:
    """Time steps per sampled tube so one sample is ~20 core-seconds of the CPU engine (~60 Mcell/s/core)."""
    return int(min(5000, max(200, 20 * 6e7 / (n_sample * 13000))))


def run_reference(args, rank):
    if rank != 0:
        return None
    procs = host_cores()
    per_step = []
    if ref_engine_available():
        # the reference's own engine, compiled from its sources
        kind = "reference"
        n_sample = min(N_TUBES, procs)
        steps = REF_ENGINE_STEPS
        for _ in range(min(args.warmup, 1)):
            ref_engine_throughput(min(procs, 4), 50, procs)
        for _ in range(args.steps):
            g, wall, _ = ref_engine_throughput(n_sample, steps, procs)
            per_step.append((g, wall))
        sample = (f"{n_sample} of the {N_TUBES} batch tubes x {steps} of {SIM_STEPS} time steps per bench step: the "
                  f"reference's FDTDEngineCPU built from its sources (setup on the GPU, loop timed), one process "
                  f"per host core")
    else:
        kind = "port"
        n_sample = min(N_TUBES, max(procs, 16))
        steps = cpu_sample_steps(n_sample)
        for _ in range(args.warmup):
            cpu_reference(procs, 50, procs)
        for _ in range(args.steps):
            g, wall, cu = cpu_reference(n_sample, steps, procs)
            per_step.append((g, wall))
        sample = (f"{n_sample} of the {N_TUBES} batch tubes x {steps} of {SIM_STEPS} time steps per bench step, "
                  f"FP32 restatement of FDTDEngineCPU, one spawn process per host core")
    value = statistics.median(g for g, _ in per_step)
    return {
        "metric": METRIC, "value": round(value, 4), "unit": "Gcell-updates/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * statistics.median(w for _, w in per_step), 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded area functions)",
        "config": workload_config(N_TUBES),
        "run": {"engine": "the reference's FDTDEngineCPU" if kind == "reference" else "FP32 port of FDTDEngineCPU",
                "arithmetic": "reference rounding (FP32, host)"},
        "cpu_baseline": {"value": round(value, 4), "unit": "Gcell-updates/s", "cores": procs, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# --------------------------------------------------------------------------- GPU arm
GRAD_STEPS = 13230                     # 20 ms at 44.1 kHz x 15
GRAD_CKPT = 512


def gradient_cost(V, stream, reps: int = 3) -> dict:
    """Cost of one gradient against one forward on the same tube: a seeded
    vowel tube (44 sections, 3:1 elliptical, two-mass source at 800 Pa in
    double), 20 ms simulated.  forward = the plain graph-replayed run (device trace);
    gradient = vs_batch_adjoint after vs_batch_forward_ckpt (checkpoints every
    512 steps, segment recomputation, reverse-time adjoint).  Both include
    their host synchronisation; medians of `reps` runs after one warm-up."""
    import torch
    from vocalsim_b200 import synthetic as S

    L, A = S.vowel_tube(0)
    p = V.params(cross_sectional_shape=2, source_type=V.SRC_TMM, tmm_ps_pa=800.0, tmm_f64=1, num_steps=GRAD_STEPS)
    g = V.Geometry(L, A)
    b = V.Batch([p], [g])
    b.set_stream(stream.cuda_stream)
    b.autotune(128)
    fwd, ck, adj = [], [], []
    rng = np.random.default_rng(0)
    gt = rng.standard_normal((1, GRAD_STEPS)).astype(np.float32) * 1e-3
    for i in range(reps + 1):
        b.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run_device(GRAD_STEPS)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        b.forward_ckpt(GRAD_STEPS, GRAD_CKPT)
        t2 = time.perf_counter()
        b.adjoint(gt)
        t3 = time.perf_counter()
        if i:
            fwd.append((t1 - t0) * 1e3)
            ck.append((t2 - t1) * 1e3)
            adj.append((t3 - t2) * 1e3)
    cells = b.interior_cells
    b.close()
    f, c, a = statistics.median(fwd), statistics.median(ck), statistics.median(adj)
    return {"workload": f"vowel tube (seed 0), two-mass source 800 Pa, {GRAD_STEPS} steps, checkpoints every "
                        f"{GRAD_CKPT}, {cells} interior cells",
            "forward_ms": round(f, 2), "forward_ckpt_ms": round(c, 2), "adjoint_ms": round(a, 2),
            "ratio": round(a / f, 3), "ratio_with_ckpt_forward": round((c + a) / f, 3)}


INV_TUBES = 64
INV_SRATE_MUL = 30
INV_STEPS = 26460                      # 20 ms at 44.1 kHz x 30


def inversion_cost(iters: int) -> dict:
    """Batched inversion: 64 tubes at fs = 44100 x 30 (ds 0.374 mm), 20 ms per
    forward, Adam over 44 widths + 44 depths + z_inv per tube against the
    spectra of other seeded tubes, reciprocal-form arithmetic; each iteration
    = depth maps from the sections on the device + one batched checkpointed
    forward + one batched adjoint + the section reverse pass (+ Adam and the
    FFT loss in torch).
    Seconds per iteration (median) and the mean spectral error."""
    from vocalsim_b200.inversion import BatchInversion, synthetic_problem

    ps, gs, targets, seeds = synthetic_problem(INV_TUBES, INV_SRATE_MUL, INV_STEPS, fast_math=1)
    inv = BatchInversion(ps, gs, targets, INV_STEPS, ckpt_every=512, lr=0.02)
    cells = inv.batch.interior_cells
    secs, losses, parts = [], [], []
    for _ in range(iters):
        t0 = time.perf_counter()
        losses.append(inv.step())
        secs.append(time.perf_counter() - t0)
        parts.append(inv.timings)
    # the plain batched forward of the same tubes (graph-replayed steps, device trace)
    import torch
    fwd = inv.batch
    fwd.reset()
    torch.cuda.synchronize()
    from vocalsim_b200.abi import VS_ERR_NONFINITE, VsError
    t0 = time.perf_counter()
    try:
        fwd.run_device(INV_STEPS)
    except VsError as e:                # a tube near the stability limit: the time still counts
        if e.status != VS_ERR_NONFINITE:
            raise
    torch.cuda.synchronize()
    fwd_s = time.perf_counter() - t0
    fwd.reset()
    split = {k: round(statistics.median(p[k] for p in parts), 3) for k in parts[0]}
    best = float(inv.best.mean())
    inv.close()
    return {"workload": f"{INV_TUBES} tubes (stable seeds {seeds[0]}..{seeds[-1]}), fs 44100 x {INV_SRATE_MUL}, "
                        f"{INV_STEPS} steps, {cells} interior cells, checkpoints every 512, fast_math=1",
            "iterations": iters, "s_per_iteration": round(statistics.median(secs), 3),
            "split_s": split, "plain_forward_s": round(fwd_s, 3),
            # gradient (recomputation + reverse steps) against one plain forward, at batch scale
            "grad_fwd_ratio_batch": round((split["recompute_s"] + split["reverse_s"]) / fwd_s, 3),
            "spectral_error_initial": round(float(np.nanmean(losses[0])), 4),
            "spectral_error_best": round(best, 4),
            "diverged_steps": int(sum(np.isnan(x).sum() for x in losses))}


def run_b200(args, rank, world):
    import torch
    import vocalsim_b200 as V

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    fast = 1 if args.arith == "fast" else 0
    seeds = strong_seeds(rank, world, args.tubes) if args.strong else None
    ps, gs = workload_params(rank, args.tubes, fast, seeds)
    batch = V.Batch(ps, gs)
    batch.set_stream(stream.cuda_stream)
    cells = batch.interior_cells
    sim_steps = args.sim_steps
    if args.profile_adjoint:
        # profiling workload of the reverse sweep: 16 stable fs x 30 tubes in
        # the bench's arithmetic, checkpointed forward + adjoint over
        # `profile_adjoint` steps
        from vocalsim_b200 import synthetic as S
        seeds = [1, 2, 3, 5, 6, 8, 9, 11, 14, 16, 17, 18, 19, 20, 21, 22]
        k = args.profile_adjoint
        pa = [V.params(cross_sectional_shape=2, srate_mul=30, num_steps=k, fast_math=fast) for _ in seeds]
        ga = [V.Geometry(*S.batch_tube(sd)[:2]) for sd in seeds]
        ba = V.Batch(pa, ga)
        tr = ba.forward_ckpt(k, 512)
        ba.adjoint((tr * 1e-3).astype(np.float32))
        ba.close()
        return None
    if args.profile_single:
        # profiling workload of the cluster kernel: the uniform 17.5 x 3 cm tube,
        # `profile_single` steps in one launch after a 256-step warm-up launch
        from vocalsim_b200 import synthetic as S
        s1 = V.Solver(V.params(mu3d=0.005, uniform_depth_m=0.02, fast_math=fast), V.Geometry(*S.uniform_tube()))
        s1.set_stream(stream.cuda_stream)
        buf = torch.empty(args.profile_single, dtype=torch.float32, device=dev)
        s1.run_device(256, buf.data_ptr())
        s1.reset()
        s1.run_device(args.profile_single, buf.data_ptr())
        torch.cuda.synchronize()
        s1.close()
        return None
    if args.profile_steps:
        if args.tile >= 0:
            batch.set_tile(args.tile)
        batch.run_device(args.profile_steps)
        torch.cuda.synchronize()
        return None
    tile, tune_ms = batch.autotune(128)

    def forward():
        batch.reset()
        batch.run_device(sim_steps)

    for _ in range(args.warmup):
        forward()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clocks:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            forward()
        e1.record(stream)
        torch.cuda.synchronize()
    ms_total = e0.elapsed_time(e1)
    if world > 1:
        torch.distributed.barrier()
    ms_total = max_over_ranks(ms_total, world, dev)
    ms_step = ms_total / args.steps
    cell_updates_rank = cells * sim_steps
    # whole-job cell-updates: every rank's own tubes (equal per rank under weak
    # scaling; the LPT shares of the one batch under --strong)
    job_cells = sum_over_ranks(cells, world, dev)
    value = job_cells * sim_steps / (ms_step / 1e3) / 1e9
    # a two-step shape advances two time steps per launch and moves the state
    # planes once per launch: algorithmic bytes per launch = 37 B x cells
    per_launch = V.tile_shape_steps(tile)
    step_launches = sim_steps // per_launch + sim_steps % per_launch
    launches_per_forward = step_launches + math.ceil(sim_steps / 128)
    launch_ms = ms_step / step_launches        # average per step-kernel launch incl. graph gaps
    # algorithmic bytes per launch = 37 B per cell-update x the cell-updates one
    # launch performs (cells x time steps per launch)
    achieved_gbs = BYTES_PER_CELL_UPDATE * cells * per_launch / (launch_ms / 1e3) / 1e9
    peak, peak_kind = hbm_peak()
    prof = profiled_kernel(cells, tile, fast)

    # ---- e2e: public API with host buffers: build + upload maps, run, download traces
    e2e = None
    if not args.no_e2e:
        trace_host = torch.empty((args.tubes, sim_steps), dtype=torch.float32, pin_memory=True)
        trace_np = trace_host.numpy()
        e2e_ms = []
        for i in range(max(args.steps, 5) + 1):     # at least 5 timed runs: the host side is noisy
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b2 = V.Batch(ps, gs)
            b2.set_tile(tile)
            b2.run(sim_steps, out=trace_np)
            b2.close()
            dt = (time.perf_counter() - t0) * 1e3
            if i > 0:
                e2e_ms.append(dt)
        e2e_step = statistics.median(e2e_ms)
        # bytes that cross per step: the maps are painted on the device from
        # per-column data (wall rows, gap-fill extents, segment ids: 20 B per
        # tube column, 4 B per section's minor axis); the descriptor plane
        # (1 B per padded cell) and tables (8 KiB) go up (every batch without
        # the coupled wall has them, in either arithmetic); each distinct
        # source table (4 B per step; the tubes here share one) goes up once;
        # the code plane (1 B per padded cell) and the traces come back
        padded = [d["frame_h"] * ((d["frame_w"] + 31) // 32 * 32) for d in batch.dims]
        sources = {(p.source_type, p.srate_mul, p.gauss_peak_s, p.gauss_width_s, p.gauss_amp, p.sine_freq_hz,
                    p.sine_amp) for p in ps}
        h2d = 4 * sim_steps * len(sources) + sum(20 * d["tube_length_cells"] + 4 * g.struct.n_sections + pc + 8192
                                                 for d, g, pc in zip(batch.dims, gs, padded))
        d2h = 4 * sim_steps * args.tubes + sum(padded)
        e2e = {"value": round(job_cells * sim_steps / (e2e_step / 1e3) / 1e9, 3), "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_step, 2)}

    # ---- plain single-tube GPU path (the uniform 17.5 x 3 cm tube) for the batched-vs-single ratio
    single = None
    if not args.no_single:
        from vocalsim_b200 import synthetic as S
        L, A = S.uniform_tube()
        s = V.Solver(V.params(mu3d=0.005, uniform_depth_m=0.02, num_steps=SIM_STEPS, fast_math=fast),
                     V.Geometry(L, A))
        s.set_stream(stream.cuda_stream)
        dtr = torch.empty(SIM_STEPS, dtype=torch.float32, device=dev)
        s.run_device(SIM_STEPS, dtr.data_ptr())
        torch.cuda.synchronize()
        s.reset()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.run_device(SIM_STEPS, dtr.data_ptr())
        b.record(stream)
        torch.cuda.synchronize()
        sms = a.elapsed_time(b)
        single = {"workload": "uniform tube 17.5 x 3 cm, 57x253 frame, 33075 steps (cluster kernel: one launch)",
                  "value": round(s.dims["interior_cells"] * SIM_STEPS / (sms / 1e3) / 1e9, 3),
                  "unit": "Gcell-updates/s", "ms": round(sms, 2)}
        s.close()
        # the same tube on the graph-replayed step kernels (its best step shape)
        bs = V.Batch([V.params(mu3d=0.005, uniform_depth_m=0.02, num_steps=SIM_STEPS, fast_math=fast)],
                     [V.Geometry(L, A)])
        bs.set_stream(stream.cuda_stream)
        best_ms, best_k = None, None
        for k in range(len(V.tile_shapes()) - 1):
            try:
                bs.set_tile(k)
            except V.VsError:
                continue
            bs.reset()
            bs.run_device(2048)
            bs.reset()
            a.record(stream)
            bs.run_device(SIM_STEPS)
            b.record(stream)
            torch.cuda.synchronize()
            t = a.elapsed_time(b)
            if best_ms is None or t < best_ms:
                best_ms, best_k = t, k
        bs.close()
        single["step_kernels_value"] = round(s.dims["interior_cells"] * SIM_STEPS / (best_ms / 1e3) / 1e9, 3)
        single["step_kernels_ms"] = round(best_ms, 2)
        single["step_kernels_shape"] = best_k
        single["cluster_speedup"] = round(best_ms / sms, 2)

    # ---- a 1 s vowel tube with the two-mass source (800 Pa)
    vowel_1s = None
    if not args.no_single:
        from vocalsim_b200 import synthetic as S
        n2 = 661500
        s2 = V.Solver(V.params(cross_sectional_shape=2, source_type=V.SRC_TMM, tmm_ps_pa=800.0, tmm_f64=1,
                               num_steps=n2, fast_math=fast), V.Geometry(*S.vowel_tube(0)))
        s2.set_stream(stream.cuda_stream)
        d2 = torch.empty(n2, dtype=torch.float32, device=dev)
        s2.run_device(2000, d2.data_ptr())
        s2.reset()
        a.record(stream)
        s2.run_device(n2, d2.data_ptr())
        b.record(stream)
        torch.cuda.synchronize()
        ms2 = a.elapsed_time(b)
        vowel_1s = {"workload": "vowel tube (seed 0, 44 sections, 3:1 elliptical), two-mass source 800 Pa in double, "
                               f"1 s simulated ({n2} steps), one cluster-kernel launch",
                   "interior_cells": s2.dims["interior_cells"],
                   "value": round(s2.dims["interior_cells"] * n2 / (ms2 / 1e3) / 1e9, 3), "unit": "Gcell-updates/s",
                   "ms": round(ms2, 2), "s_per_simulated_s": round(ms2 / 1e3, 4)}
        s2.close()

    grad = None
    if not args.no_grad:
        grad = gradient_cost(V, stream)
    inversion = None
    if args.inversion_iters > 0 and rank == 0:
        inversion = inversion_cost(args.inversion_iters)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        procs = host_cores()
        if ref_engine_available():
            n_sample = min(args.tubes, procs)
            g, wall, _ = ref_engine_throughput(n_sample, REF_ENGINE_STEPS, procs)
            cpu = {"value": round(g, 4), "unit": "Gcell-updates/s", "cores": procs, "kind": "reference",
                   "sample": f"{n_sample} batch tubes x {REF_ENGINE_STEPS} of {SIM_STEPS} steps, the reference's "
                             f"FDTDEngineCPU built from its sources, one process per core (loops {wall:.1f} s)"}
        else:
            n_sample = min(args.tubes, max(procs, 16))
            csteps = cpu_sample_steps(n_sample)
            g, wall, _ = cpu_reference(n_sample, csteps, procs)
            cpu = {"value": round(g, 4), "unit": "Gcell-updates/s", "cores": procs, "kind": "port",
                   "sample": f"{n_sample} batch tubes x {csteps} of {SIM_STEPS} steps, FP32 restatement of "
                             f"FDTDEngineCPU, one process per core ({wall:.1f} s)"}

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Gcell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
        "higher_is_better": True, "scaling": "strong" if args.strong else "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded area functions, no dataset)",
        "config": workload_config(args.tubes, sim_steps),
        "run": {"tubes_per_gpu": len(ps), "interior_cells_per_gpu": cells, "tile": list(V.tile_shapes()[tile]),
                "parallelism": (f"LPT tube sharding of one {args.tubes}-tube batch x{world} (no collective)"
                                if args.strong else f"tube sharding x{world} (no collective)"),
                "arithmetic": "reciprocal form (fast_math=1)" if fast else "reference rounding (fast_math=0)",
                "l2": "state + maps per GPU > 126 MB L2 and 33075 launches per timed step; no flush"},
        "roofline": {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved_gbs / peak, 4), "traffic": prof["traffic"],
                     # DRAM bytes the launch really moves (ncu, same kernel and workload) per
                     # launch time: the two-step kernel moves the planes once per two steps
                     "dram_frac": (round(prof["traffic"] / (launch_ms / 1e3) / 1e9 / peak, 4)
                                   if prof["traffic"] else None),
                     "issue_active_pct": prof["issue_active_pct"],
                     # the metric's own form: Gcell-updates/s per GPU against the one-step
                     # roofline (37 B per cell-update moved once per step at the peak)
                     "gcell_roofline": round(peak / BYTES_PER_CELL_UPDATE, 1),
                     "gcell_frac": round(value / world / (peak / BYTES_PER_CELL_UPDATE), 4),
                     "note": f"{BYTES_PER_CELL_UPDATE} B algorithmic per cell-update x {cells} cells x {per_launch} "
                             f"time step(s) per launch / mean launch time {launch_ms * 1e3:.2f} us; peak {peak_kind}; "
                             f"dram_frac and issue_active_pct from the committed ncu summary of the same kernel"},
        "gpu_launches": args.steps * launches_per_forward,
        "clocks": clocks.summary(),
        "e2e": e2e,
        "cpu_baseline": cpu,
        "single_tube": single,
        "vowel_1s": vowel_1s,
        # against the library's default single-tube path (the cluster kernel), and
        # against the same step kernels the batch uses, run on the one tube
        "batched_vs_single": round(value / world / single["value"], 2) if single else None,
        "batched_vs_single_step_kernels": round(value / world / single["step_kernels_value"], 2) if single else None,
        "grad_fwd_ratio": grad["ratio"] if grad else None,
        "gradient": grad,
        "inversion": inversion,
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--tubes", type=int, default=N_TUBES)
    ap.add_argument("--strong", action="store_true",
                    help="split one batch of --tubes tubes across the ranks (LPT by cells) instead of one batch per rank")
    ap.add_argument("--sim-steps", type=int, default=SIM_STEPS)
    ap.add_argument("--profile-steps", type=int, default=0)
    ap.add_argument("--profile-adjoint", type=int, default=0,
                    help="run a 16-tube checkpointed forward + adjoint of this many steps, untimed, for ncu")
    ap.add_argument("--profile-single", type=int, default=0,
                    help="run the uniform tube for this many steps on the cluster kernel, untimed, for ncu")
    ap.add_argument("--tile", type=int, default=-1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-single", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-grad", action="store_true")
    ap.add_argument("--inversion-iters", type=int, default=2,
                    help="Adam iterations of the 64-tube inversion to time (0 = skip)")
    ap.add_argument("--arith", choices=["fast", "exact"], default="fast",
                    help="fast: reciprocal-form arithmetic (fast_math = 1); exact: the reference's rounding")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        line = run_b200(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
