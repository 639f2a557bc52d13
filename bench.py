"""bench.py — throughput of the all-atom search hot path on B200.

One "step" = one phase-1 block of the search (diffusion.rs:1018-1057 with
scoring every 10 steps): 10 gradient-only allatom_diffusion_steps of every
candidate (coarse-grained grid force, restraint, 2 A clamp, rigid residue
translation), one all-atom LJ + Coulomb + hydrophobic score of every candidate,
and the top-64 survivor selection.  Workload: 1024 antibodies x 20 residues
against a 300-residue (2505-atom) compact globule, seeded synthetic inputs.
Steps walk through phase-1 passes: blocks 0..19 (gradient steps 0..199) from
the initial population, then the population is reset (outside the timed
events) and the next pass starts, so every timed block is a block of the
200-step phase the workload defines.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line.  value = candidate-steps/s over all ranks (device time
with CUDA events on the library's stream, max over ranks); e2e = the same
metric through the C ABI with host buffers (state upload, block, state +
energies + survivors download every step).  The reference arm times the CPU
restatement of the reference's algorithm (the Rust crate cannot be built on
this image) with every host thread.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_STEPS_PER_BLOCK = 10
TOP_K = 64
PHASE1_STEPS = 200   # GPU_STEPS (diffusion.rs:1018)
PHASE1_BLOCKS = PHASE1_STEPS // N_STEPS_PER_BLOCK
PHASE2_STEPS = 600   # Langevin + Metropolis steps on the survivors
# Algorithmic flops per in-cutoff pair (FADD/FMUL = 1, FFMA = 2, rsqrt/sqrt/div
# MUFU sequences not counted):
#  all-atom score pair: dx,dy,dz 3 + r^2 5 + 1/r^2 1 + R 1 + R^2 1 + s2 1 + s6 2 +
#    eps 1 + LJ 3 + Coulomb 2 + hydrophobic 1 + accumulate 2 = 23 -> 24 with the cutoff select
SCORE_FLOPS_PER_PAIR = 24
#  coarse-grained force pair (energy.rs:362-391): dx,dy,dz 3 + r^2 5 + eps 1 + sigma 2 +
#    sigma^2 1 + s2 1 + s6 2 + s12 1 + f_lj 5 + f_total 2 + 3 x (mul + add) 6 = 29
CG_FLOPS_PER_PAIR = 29
FALLBACK_HBM_GBS = 6650.0


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": FALLBACK_HBM_GBS, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        self.t_start = time.time()

    def mark(self, which):
        setattr(self, which, time.time())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        rows = []
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9], float(parts[3])))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        # samples with the GPU busy (the timed loop keeps it busy; idle samples read ~120 MHz)
        busy = [r for r in rows if r[0] > 0.5 * r[1]] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in busy for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in busy), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows), "samples_busy": len(busy),
                "power_w_max": max(r[3] for r in rows)}


def dist_init(world):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        dist.init_process_group(backend="cpu:gloo,cuda:nccl", timeout=timedelta(seconds=120))
    return torch, dist


def max_over_ranks(torch, dist, world, value, device):
    if world == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(torch, dist, world, value, device):
    if world == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def merge_survivors(torch, dist, world, energies, idx, rank, n_cand, k=TOP_K):
    """Global top-k of every rank's local survivors: one all-gather of k (E, index) pairs."""
    local = np.stack([energies[idx], (idx + rank * n_cand).astype(np.float64)], axis=1)
    if world == 1:
        allv = local
    else:
        t = torch.from_numpy(np.ascontiguousarray(local))
        out = [torch.zeros_like(t) for _ in range(world)]
        dist.all_gather(out, t)
        allv = torch.cat(out).numpy()
    order = np.lexsort((allv[:, 1], np.where(np.isnan(allv[:, 0]), np.inf, allv[:, 0])))
    return allv[order[:k], 1].astype(np.int64), allv[order[:k], 0]


def build_workload(pkg, ctx, rank):
    wl = pkg.workloads
    cfg = wl.config1(salt=rank)
    ag_aa, ag_ca = cfg["antigens"][0]
    ag_pos, _ = ctx.build_residues(ag_ca, ag_aa)
    ctx.clear_antigens()
    p = ctx.params
    p.shell_radius = float(cfg["shell"][0])
    ctx.set_params(p)
    ctx.add_antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    pos, chi = ctx.build_residues(pop.ca, pop.aa)
    return cfg, ag_aa, ag_pos, pop, pos, chi


def cpu_reference_block(orc, A, prm, aa, chi, pos, n_res, ag_atoms, threads, step0):
    """The reference algorithm on the host: 10 gradient steps (grid CG force),
    brute-force f32 all-atom score (energy.rs:261-301 order), stable top-64."""
    n_cand = len(aa) // n_res
    ids = np.arange(n_cand, dtype=np.uint32)
    for s in range(N_STEPS_PER_BLOCK):
        A.step(prm, aa, chi, pos, n_res, ids, step0 + s, 3.0, False, False, threads=threads)
    cands, off = [], [0]
    for c in range(n_cand):
        g = orc.gpu_atoms(orc.flatten(aa[c * n_res:(c + 1) * n_res], pos[c * n_res:(c + 1) * n_res]))
        cands.append(g)
        off.append(off[-1] + len(g))
    e = orc.score_batch32(ag_atoms, np.concatenate(cands), np.asarray(off, np.int64), threads=threads)
    return orc.topk(e.astype(np.float64), min(TOP_K, n_cand))


def cpu_sample(orc, cfg, ag_aa, ag_pos, pop, target_s, threads, n_max=None):
    """Time the reference algorithm on a bounded sample: candidates are doubled
    until one block takes a quarter of target_s (or all are in), then blocks of a
    phase-1 pass are run until target_s is spent.  Returns (candidates, blocks,
    seconds, ...)."""
    n_res = int(pop.n_res[0])
    A = orc.Antigen(ag_aa, ag_pos)
    prm = orc.OrcParams.defaults(shell_radius=float(cfg["shell"][0]))
    ag_atoms = orc.gpu_atoms(orc.flatten(ag_aa, ag_pos))
    n_total = pop.n_cand if n_max is None else min(n_max, pop.n_cand)
    n = min(threads * 2, n_total)
    while True:
        aa = pop.aa[: n * n_res].copy()
        pos, chi = orc.build_residues(pop.ca[: n * n_res], aa)
        t0 = time.perf_counter()
        cpu_reference_block(orc, A, prm, aa, chi, pos, n_res, ag_atoms, threads, 0)
        dt = time.perf_counter() - t0
        if dt > 0.25 * target_s or n >= n_total:
            break
        n = min(n_total, max(n * 2, int(n * 0.5 * target_s / max(dt, 1e-6))))
    blocks = 1
    while dt < target_s and blocks < PHASE1_BLOCKS:
        t0 = time.perf_counter()
        cpu_reference_block(orc, A, prm, aa, chi, pos, n_res, ag_atoms, threads, blocks * N_STEPS_PER_BLOCK)
        dt += time.perf_counter() - t0
        blocks += 1
    return n, blocks, dt, A, prm, ag_atoms, n_res


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ctypes as orc
    from __graft_entry__ import load_package
    pkg = load_package()
    cfg = pkg.workloads.config1()
    ag_aa, ag_ca = cfg["antigens"][0]
    ag_pos, _ = orc.build_residues(ag_ca, ag_aa)
    pop = cfg["pop"]
    threads = os.cpu_count() or 1
    # each step: one block over a sample sized so the whole K+W run stays within minutes
    budget = max(0.5, min(4.0, 150.0 / max(1, args.steps + args.warmup)))
    n, _, _, A, prm, ag_atoms, n_res = cpu_sample(orc, cfg, ag_aa, ag_pos, pop, budget, threads)
    aa0 = pop.aa[: n * n_res].copy()
    pos0, chi0 = orc.build_residues(pop.ca[: n * n_res], aa0)
    aa, chi, pos = aa0.copy(), chi0.copy(), pos0.copy()
    times = []
    for k in range(args.warmup + args.steps):
        b = k % PHASE1_BLOCKS  # phase-1 passes, as in the GPU arm
        if b == 0:
            aa[:], chi[:], pos[:] = aa0, chi0, pos0
        t0 = time.perf_counter()
        cpu_reference_block(orc, A, prm, aa, chi, pos, n_res, ag_atoms, threads, b * N_STEPS_PER_BLOCK)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    value = n * N_STEPS_PER_BLOCK / (ms / 1e3)
    sample = (f"{n} of 1024 candidates per step (10 gradient steps + brute-force f32 score + top-64), "
              f"phase-1 passes of 20 blocks, CPU restatement of the reference")
    line = {"impl": "reference", "metric": "candidate-steps/s", "value": value, "unit": "candidate-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": workload_config(),
            "cpu_baseline": {"value": value, "unit": "candidate-steps/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "candidate-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_mc_sample(orc, cfg, ag_aa, ag_pos, aa, chi, pos, n_res, target_s, threads):
    """Phase-2 steps (Langevin + Metropolis, diffusion.rs:290-463) of the oracle on
    the survivors, as many as fit in about target_s seconds."""
    A = orc.Antigen(ag_aa, ag_pos)
    prm = orc.OrcParams.defaults(shell_radius=float(cfg["shell"][0]))
    n_cand = len(aa) // n_res
    ids = np.arange(n_cand, dtype=np.uint32)
    aa, chi, pos = aa.copy(), chi.copy(), pos.copy()
    steps, t0 = 0, time.perf_counter()
    while steps < PHASE2_STEPS and time.perf_counter() - t0 < target_s:
        A.step(prm, aa, chi, pos, n_res, ids, steps, orc.temperature(steps, PHASE2_STEPS), True, True,
               threads=threads)
        steps += 1
    return steps, time.perf_counter() - t0


def measure_phase2(torch, ctx, ext, survivors, n_res, reps=3):
    """Phase 2 of run_allatom on the survivors: PHASE2_STEPS Langevin + Metropolis
    steps (noise on, annealed), one launch, device time on the library stream."""
    ctx.state_select(np.asarray(survivors, np.int32))
    aa, chi, pos = ctx.state_download()
    temps = np.array([np.float32(3.0) * np.power(np.float32(0.02 / 3.0), np.float32(i) / np.float32(PHASE2_STEPS))
                      for i in range(PHASE2_STEPS)], np.float32)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    for rep in range(reps + 1):
        ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
        torch.cuda.synchronize()
        a.record(ext)
        ctx.diffuse(PHASE2_STEPS, PHASE1_STEPS, with_noise=True, with_mc=True, temps=temps)
        b.record(ext)
        b.synchronize()
        if rep:
            ms.append(a.elapsed_time(b))
    st = ctx.mc_stats().sum(0)
    n = len(survivors)
    t = statistics.mean(ms)
    return {"candidates": n, "steps": PHASE2_STEPS, "ms": t, "candidate_steps_per_s": n * PHASE2_STEPS / (t * 1e-3),
            "moves_per_candidate_step": {"mutation_rotamer": float(st[0]) / (n * PHASE2_STEPS),
                                         "backbone": float(st[2]) / (n * PHASE2_STEPS)},
            "acceptance": {"mutation_rotamer": float(st[1]) / max(1, st[0]), "backbone": float(st[3]) / max(1, st[2])},
            "accumulate": "f32 pair terms summed in FP64, FP64 Metropolis test"}, (aa, chi, pos)


def run_post_search(pkg, ctx, cfg, ag_aa, ag_pos, n_res, cpu, reps=3):
    """The post-search refinement of run_allatom's 64 ranked results (main.rs:336-346):
    minimize (60 steps), affinity maturation over the interface residues, structure
    validation -- wall time of each batched call (median of reps after one untimed),
    and the CPU restatement of the same calls on the same results (every host thread)."""
    aa0, chi0, pos0 = ctx.state_download()
    n = len(aa0) // n_res

    def timed(fn):
        ms = []
        for rep in range(reps + 1):
            ctx.state_upload(aa0, chi0, pos0, uniform_n_res=n_res)
            t0 = time.perf_counter()
            out = fn()
            if rep:
                ms.append(1e3 * (time.perf_counter() - t0))
        return statistics.median(ms), out

    t_min, e_min = timed(lambda: ctx.minimize(60))
    t_mat, (e_mat, kept) = timed(lambda: ctx.affinity_maturation())
    t_val, (cl, ra) = timed(lambda: ctx.validate())
    out = {"candidates": n, "minimize_steps": 60,
           "minimize_ms": t_min, "affinity_maturation_ms": t_mat, "validate_ms": t_val,
           "mutations_kept": int(kept.sum()), "clashes": int(cl.sum()), "rama_outliers": int(ra.sum()),
           "api": "binder_minimize / binder_affinity_maturation / binder_validate, wall clock per batched call"}
    if cpu:
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_ctypes as orc
        threads = os.cpu_count() or 1
        A = orc.Antigen(ag_aa, np.ascontiguousarray(ag_pos))
        a, c, p = aa0.copy(), chi0.copy(), pos0.copy()
        t0 = time.perf_counter()
        A.minimize(a, c, p, n_res, 60, acc64=False, threads=threads)
        t1 = time.perf_counter()
        a, c, p = aa0.copy(), chi0.copy(), pos0.copy()
        A.affinity_maturation(a, c, p, n_res, acc64=False, threads=threads)
        t2 = time.perf_counter()
        for k in range(n):
            orc.validate(aa0[k * n_res:(k + 1) * n_res], pos0[k * n_res:(k + 1) * n_res])
        t3 = time.perf_counter()
        out["cpu_baseline"] = {"minimize_ms": 1e3 * (t1 - t0), "affinity_maturation_ms": 1e3 * (t2 - t1),
                               "validate_ms": 1e3 * (t3 - t2), "cores": threads, "kind": "port",
                               "sample": f"the same {n} results, f32 energies as the reference computes them"}
    return out


def workload_config():
    return {"workload": "search block: 1024 antibodies x 20 residues vs 300-residue globule (2505 atoms); "
                        "10 gradient steps + all-atom score + top-64 per step",
            "n_candidates": 1024, "residues_per_candidate": 20, "antigen_residues": 300,
            "gradient_steps_per_block": N_STEPS_PER_BLOCK, "top_k": TOP_K, "score_cell_A": 8.0,
            "cutoff_A": 10.0, "ca_cell_A": 10.0,
            "l2": "256 MiB buffer written between timed steps (flush); working set 5 MiB",
            "steps": "blocks 0..19 of 200-step phase-1 passes from the initial population, repeated",
            "precision": "f32 pair terms, Kahan lane sums, FP64 reductions"}


def run_ours(args, rank, world, local_rank):
    torch, dist = dist_init(world)
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    from __graft_entry__ import load_package
    pkg = load_package()
    ctx = pkg.GpuContext.create(local_rank)
    cfg, ag_aa, ag_pos, pop, pos, chi = build_workload(pkg, ctx, rank)
    n_cand, n_res = pop.n_cand, int(pop.n_res[0])
    ctx.state_upload(pop.aa, chi, pos, uniform_n_res=n_res)
    ext = torch.cuda.ExternalStream(ctx.stream, device=device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    # launch shapes for this state (autotuner; results do not depend on them), then
    # warm-up (untimed; the first block captures the CUDA graph of a block)
    tuned = ctx.autotune(reps=5).as_dict()

    def reset():  # start of a phase-1 pass: the initial population (same buffers, same graph)
        ctx.state_upload(pop.aa, chi, pos, uniform_n_res=n_res)

    for w in range(args.warmup):
        if w % PHASE1_BLOCKS == 0:
            reset()
        ctx.block_async(N_STEPS_PER_BLOCK, (w % PHASE1_BLOCKS) * N_STEPS_PER_BLOCK, TOP_K)
    ctx.block_fetch(TOP_K)

    sampler = ClockSampler(local_rank)
    sampler.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches = 0
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        b = (args.warmup + k) % PHASE1_BLOCKS
        if b == 0:
            reset()  # host upload, before the start event
        with torch.cuda.stream(ext):
            flush.zero_()  # L2 flush between timed steps, outside the timed events
            starts[k].record(ext)
        l0 = ctx.launch_count
        ctx.block_async(N_STEPS_PER_BLOCK, b * N_STEPS_PER_BLOCK, TOP_K)
        launches += ctx.launch_count - l0
        with torch.cuda.stream(ext):
            stops[k].record(ext)
    e_last, top_last = ctx.block_fetch(TOP_K)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    # per-phase device times and in-cutoff pair counts over one phase-1 pass: eagerly
    # issued blocks with events between the phases (the graph replay above has none);
    # pairs counted before each block on the same state (untimed, state unchanged)
    reset()
    cg_pairs = score_pairs = 0
    ctx.set_timing(True)
    for b in range(PHASE1_BLOCKS):
        cg, sc = ctx.state_pair_counts(N_STEPS_PER_BLOCK)
        cg_pairs += cg
        score_pairs += sc
        ctx.block_async(N_STEPS_PER_BLOCK, b * N_STEPS_PER_BLOCK, TOP_K)
    ctx.block_fetch(TOP_K)
    phase_ms, n_blocks = ctx.timing_summary()
    ctx.set_timing(False)
    cg_pairs /= PHASE1_BLOCKS
    score_pairs /= PHASE1_BLOCKS
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    ms_local = statistics.mean(step_ms)
    ms = max_over_ranks(torch, dist, world, ms_local, device)
    total_cand = sum_over_ranks(torch, dist, world, float(n_cand), device)
    value = total_cand * N_STEPS_PER_BLOCK / (ms / 1e3)
    ph = phase_ms / max(1, n_blocks)  # mean ms per launch: [gradient, score, top-k]
    survivors, surv_e = merge_survivors(torch, dist, world, e_last, top_last[0].astype(np.int64), rank, n_cand)

    # e2e through the C ABI with pinned host buffers, copies in the timed region
    h_aa = torch.empty(n_cand * n_res, dtype=torch.uint8, pin_memory=True).numpy()
    h_chi = torch.empty((n_cand * n_res, 4), dtype=torch.float32, pin_memory=True).numpy()
    h_pos = torch.empty((n_cand * n_res, 14, 3), dtype=torch.float32, pin_memory=True).numpy()
    h_e = torch.empty(n_cand, dtype=torch.float64, pin_memory=True).numpy()
    h_top = torch.empty(TOP_K, dtype=torch.int32, pin_memory=True).numpy()
    e2e_steps = max(1, min(args.steps, 200))
    t_e2e = []
    for k in range(e2e_steps + 1):
        b = k % PHASE1_BLOCKS
        if b == 0:  # phase-1 pass from the initial population
            h_aa[:], h_chi[:], h_pos[:] = pop.aa, chi, pos
        t0 = time.perf_counter()
        # upload, block, write-back of the moved residues (copied beside the score)
        ctx.block_io(h_aa, h_chi, h_pos, N_STEPS_PER_BLOCK, TOP_K, uniform_n_res=n_res, out_e=h_e, out_top=h_top)
        if k:  # first iteration warms the pinned paths
            t_e2e.append(time.perf_counter() - t0)
    e2e_ms = max_over_ranks(torch, dist, world, 1e3 * statistics.mean(t_e2e), device)
    h2d = h_aa.nbytes + h_chi.nbytes + h_pos.nbytes
    d2h = h_e.nbytes + h_top.nbytes + h_aa.nbytes + h_chi.nbytes + h_pos.nbytes

    # phase 2 on this rank's survivors, then the whole run_allatom pipeline
    phase2, surv_state = measure_phase2(torch, ctx, ext, top_last[0], n_res)
    run_cfg = pkg.RunCfg.defaults(phase1_steps=PHASE1_STEPS, score_every=N_STEPS_PER_BLOCK, survivors=TOP_K,
                                  phase2_steps=PHASE2_STEPS, top_n=TOP_K)
    run_times = []
    for rep in range(8):  # the first call (untimed) pays the one-time kernel loading and buffer growth
        ctx.state_upload(pop.aa, chi, pos, uniform_n_res=n_res)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run_cand, run_e = ctx.run_allatom(run_cfg)
        if rep:
            run_times.append(1e3 * (time.perf_counter() - t0))
    run_ms = statistics.median(run_times)
    run_allatom = {"ms": run_ms, "ms_all": [round(t, 3) for t in run_times], "phase1_steps": PHASE1_STEPS,
                   "phase2_steps": PHASE2_STEPS, "candidates": n_cand, "survivors": TOP_K,
                   "best_energy": float(run_e[0][0]), "best_index": int(run_cand[0][0]),
                   "api": "binder_run_allatom (wall clock, host call to results; median of 7 calls after one untimed)"}

    peaks, peaks_kind = load_peaks()
    fp32_scalar, fp32_packed = ctx.fp32_peak()
    fp32_peak = max(fp32_scalar, fp32_packed)
    kern = {
        "langevin_cg": {"ms": float(ph[0]), "pairs": int(cg_pairs),
                        "tflops": CG_FLOPS_PER_PAIR * cg_pairs / (ph[0] * 1e-3) / 1e12},
        "score_allatom": {"ms": float(ph[1]), "pairs": int(score_pairs),
                          "tflops": SCORE_FLOPS_PER_PAIR * score_pairs / (ph[1] * 1e-3) / 1e12},
        "sum_select": {"ms": float(ph[2]),
                       "what": "candidate sums (FP64, residue order) + stable top-64, one launch"},
    }
    dom = max(("langevin_cg", "score_allatom"), key=lambda k: kern[k]["ms"])
    achieved = kern[dom]["tflops"]
    line = {
        "metric": "candidate-steps/s", "value": value, "unit": "candidate-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": dict(workload_config(), launch=tuned, cuda_graph=True),
        "pair_evals_per_s": total_cand / n_cand * score_pairs / (ph[1] * 1e-3),
        "roofline": {"kernel": dom, "bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak, "traffic": NCU_DRAM_BYTES.get(dom),
                     "traffic_unit": "bytes per launch", "traffic_source": NCU_DRAM_SOURCE,
                     "peak_source": "FP32 FMA microbenchmark on this GPU (max of scalar/f32x2), "
                                    f"scalar {fp32_scalar:.1f}, packed {fp32_packed:.1f}; "
                                    f"nominal {148 * 128 * 2 * 1.965e-3:.1f} at 1965 MHz",
                     "flops_per_pair": SCORE_FLOPS_PER_PAIR if dom == "score_allatom" else CG_FLOPS_PER_PAIR},
        "kernels": kern,
        "e2e": {"value": total_cand * N_STEPS_PER_BLOCK / (e2e_ms / 1e3), "unit": "candidate-steps/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "api": "binder_block_io (state upload, block, state write-back), pinned host buffers"},
        "clocks": clocks, "gpu_launches": int(launches),
        "survivors": {"best_energy": float(surv_e[0]), "best_index": int(survivors[0])},
        "hbm_peak_gbs": peaks.get("hbm_gbs"), "peaks_file": peaks_kind,
        "phase2": phase2, "run_allatom": run_allatom,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_ctypes as orc
        threads = os.cpu_count() or 1
        n, nb, dt, *_ = cpu_sample(orc, cfg, ag_aa, np.ascontiguousarray(ag_pos), pop, args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": n * nb * N_STEPS_PER_BLOCK / dt, "unit": "candidate-steps/s",
                                "cores": threads, "kind": "port",
                                "sample": f"blocks 0..{nb - 1} of a phase-1 pass (10 gradient steps + brute-force "
                                          f"f32 score + top-64 each) over {n} of 1024 candidates, {dt:.1f} s"}
        ms_steps, mdt = cpu_mc_sample(orc, cfg, ag_aa, np.ascontiguousarray(ag_pos), *surv_state, n_res,
                                      args.cpu_seconds / 3, threads)
        cpu_p2 = len(surv_state[0]) // n_res * ms_steps / mdt
        line["phase2"]["cpu_baseline"] = {
            "value": cpu_p2, "unit": "candidate-steps/s", "cores": threads, "kind": "port",
            "sample": f"{ms_steps} of {PHASE2_STEPS} phase-2 steps on the 64 survivors, {mdt:.1f} s"}
        cpu_run_s = n_cand * PHASE1_STEPS / (n * nb * N_STEPS_PER_BLOCK / dt) + TOP_K * PHASE2_STEPS / cpu_p2
        line["run_allatom"]["cpu_estimate_ms"] = 1e3 * cpu_run_s
    if rank == 0 and world == 1:
        line["post_search"] = run_post_search(pkg, ctx, cfg, ag_aa, ag_pos, n_res, not args.no_cpu_baseline)
    if rank == 0 and world == 1 and not args.no_learned:
        line["batched_uneven"] = run_batched(pkg, ctx, torch, ext)
        line["learned_proposal"] = run_learned(pkg, ctx)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_batched(pkg, ctx, torch, ext):
    """The batched uneven workload: 8 antigens of 50..800 residues resident
    together, 4096 antibodies of 10..30 residues assigned round-robin, one phase-1
    pass (20 blocks of 10 gradient steps + score + per-antigen top-64, CUDA graph,
    autotuned launch shapes), device time per block."""
    cfg = pkg.workloads.config2()
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=26.0))
    pop = cfg["pop"]
    # the restraint radius is per context: the antigens' shells differ, so each
    # candidate keeps the radius of the config-1 globule (26 A); the grid, scoring
    # and top-k are per antigen
    for ag_aa, ag_ca in cfg["antigens"]:
        pos_a, _ = ctx.build_residues(ag_ca, ag_aa)
        ctx.add_antigen(ag_aa, pos_a)
    pos, chi = ctx.build_residues(pop.ca, pop.aa)
    ctx.state_upload(pop.aa, chi, pos, n_res=pop.n_res, antigen_id=pop.antigen_id)
    tuned = ctx.autotune(reps=3).as_dict()
    n_seg = len(cfg["antigens"])
    times = []
    for p in range(2):  # pass 0 warms up (graph capture), pass 1 is timed
        ctx.state_upload(pop.aa, chi, pos, n_res=pop.n_res, antigen_id=pop.antigen_id)
        for b in range(PHASE1_BLOCKS):
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(ext)
            ctx.block_async(N_STEPS_PER_BLOCK, b * N_STEPS_PER_BLOCK, TOP_K)
            e.record(ext)
            if p:
                times.append((a, e))
        e_last, top = ctx.block_fetch(TOP_K, n_segments=n_seg)
    ms = [a.elapsed_time(e) for a, e in times]
    mean_ms = float(np.mean(ms))
    return {"workload": "8 globules of 50..800 residues resident together, 4096 antibodies of 10..30 residues "
                        "(round-robin), one phase-1 pass: 20 x (10 gradient steps + all-atom score + top-64 per "
                        "antigen), CUDA graph", "candidates": int(pop.n_cand), "residues": int(pop.n_res.sum()),
            "ms_per_block": mean_ms, "candidate_steps_per_s": pop.n_cand * N_STEPS_PER_BLOCK / (mean_ms * 1e-3),
            "launch": tuned, "survivors_per_antigen": [int((t >= 0).sum()) for t in top],
            "best_energy_per_antigen": [float(e_last[t[0]]) for t in top]}


# DRAM bytes (read + write) of one launch of each block kernel, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of `bench.py --block-only 8,8,3,0,8`,
# the same per-launch work and launch shape as the timed blocks
NCU_DRAM_BYTES = {"langevin_cg": 7_249_152, "score_allatom": 3_888_384}
NCU_DRAM_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch of "
                   "bench.py --block-only 8,8,3,0,8 (cold cache, serialised)")

SCHEDULES = (150, 200, 250, 300, 375, 450, 600)  # annealed schedule lengths of the learned-proposal study
LEARNED_SEEDS = tuple(range(21, 33))
# Proposal temperature floor Tp = max(T, T_PROP_MIN), chosen on the validation antigen
# (held-out antigen 2 of the learned-proposal workload; `--learned-validation`), never
# on the antigen the study reports.
T_PROP_MIN = 0.5
LEARNED_METHODS = (("uniform", {}),
                   ("learned", {"learned": True, "t_prop_min": T_PROP_MIN}),
                   ("learned_below_T1", {"learned": True, "t_prop_min": T_PROP_MIN, "t_max": 1.0}))


def _finite(x):
    """x, or None (JSON null) when it is not finite: a run that never reaches the target."""
    return float(x) if np.isfinite(x) else None


def run_learned(pkg, ctx, seeds=LEARNED_SEEDS, n_res=20, eval_index=0, methods=LEARNED_METHODS,
                schedules=SCHEDULES):
    """The learned proposal (configs of the learned-proposal workload): plain-MC
    tuples on 4 training antigens, GPU training, then annealed runs on a held-out
    antigen (eval_index 0: the reported one; 1: the validation one), uniform vs
    learned proposal.  Time to target = first wall time at which a run's champion is
    within 0.5 kcal/mol of the uniform proposal's median final champion on the
    600-step schedule; reported per schedule length (the same grid for every method)
    and for each method at its best length (median over the seeds)."""
    L = pkg.learned
    cfg = pkg.workloads.config4(n_train=4, n_eval=eval_index + 1)
    shell = float(cfg["train"][0][1])
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=shell, seed=11))
    train_ids = L.add_antigens(ctx, [t[0] for t in cfg["train"]])
    eval_ag, _, eval_pop = cfg["eval"][eval_index]
    (eval_id,) = L.add_antigens(ctx, [eval_ag])
    t0 = time.perf_counter()
    n_tuples = L.generate_tuples(ctx, [t[2] for t in cfg["train"]], train_ids, n_res, gen_steps=300)
    gen_s = time.perf_counter() - t0
    train_steps = 1500
    losses, train_s = L.train(ctx, train_steps, batch=8192, lr=1e-3)
    agid = L.upload_populations(ctx, [eval_pop], [eval_id], n_res)
    ctx.diffuse(PHASE1_STEPS, 0)  # phase-1 gradient steps bring the population into contact
    s0 = ctx.state_download()
    # every method on every schedule length; the 600-step schedule is the reference's
    runs = {(name, n): [] for name, _ in methods for n in schedules}
    acc = {k: [] for k in runs}
    for n_steps in schedules:
        for seed in seeds:
            ctx.set_params(pkg.Params.defaults(shell_radius=shell, seed=seed))
            for name, kw in methods:
                traj, st = L.anneal_champions(ctx, s0, agid, n_res, n_steps=n_steps, **kw)
                runs[(name, n_steps)].append(traj)
                acc[(name, n_steps)].append(st["mutation_rotamer_acceptance"])
    out = {"workload": "4 training antigens x 1024 antibodies (plain-MC tuples, 300 annealed steps), held-out "
                       "300-residue antigen %d x 1024 antibodies x 20 residues, annealed Langevin + Metropolis "
                       "runs of %s steps, %d seeds" % (eval_index + 1, "/".join(map(str, schedules)), len(seeds)),
           "methods": {name: {k: _finite(v) if isinstance(v, float) else v for k, v in kw.items()}
                       for name, kw in methods},
           "tuples": int(n_tuples), "tuple_gen_s": gen_s, "train_steps": train_steps,
           "train_batch": 8192, "train_s": train_s, "loss_first": float(np.mean(losses[:10])),
           "loss_last": float(np.mean(losses[-50:])), "time_unit": "ms of Metropolis steps (wall clock)"}
    # target: the uniform proposal's median final champion on the 600-step schedule
    target, _, _ = L.time_to_target(runs[("uniform", PHASE2_STEPS)], [])
    out["target_champion"] = target
    med = {}
    for (name, n), rs in runs.items():
        _, _, tt = L.time_to_target(runs[("uniform", PHASE2_STEPS)], rs)
        med[(name, n)] = float(np.median(tt))
        out.setdefault(name, {})["steps_%d" % n] = {
            "time_to_target_ms": [_finite(x) for x in tt], "median_ms": _finite(med[(name, n)]),
            "final_champions": [r[-1][1] for r in rs],
            "ms_per_run": float(np.mean([r[-1][0] for r in rs])), "acceptance": float(np.mean(acc[(name, n)]))}
    best = {name: min((med[(name, n)], n) for n in schedules) for name, _ in methods}
    for name, _ in methods:
        out[name]["best"] = {"median_ms": _finite(best[name][0]), "schedule_steps": best[name][1]}
        if name != "uniform":
            out[name]["speedup_vs_uniform_600"] = _finite(med[("uniform", PHASE2_STEPS)] / med[(name, PHASE2_STEPS)])
            out[name]["speedup_vs_uniform_best_schedules"] = _finite(best["uniform"][0] / best[name][0])
    return out


def run_learned_validation(args):
    """The proposal temperature floor and the learned-below-T cutoff on the
    validation antigen: the study's time to target for t_prop_min 0.1 / 0.3 / 0.5 /
    1.0 x learned on every step / below T = 1 / below T = 0.5.  Prints one JSON line
    of speedups (best schedules) per setting."""
    from __graft_entry__ import load_package
    pkg = load_package()
    ctx = pkg.GpuContext.create(0)
    methods = (("uniform", {}),) + tuple(
        ("tp%g_%s" % (tp, "every_step" if tm == float("inf") else "below_T%g" % tm),
         {"learned": True, "t_prop_min": tp, "t_max": tm})
        for tp in (0.1, 0.3, 0.5, 1.0) for tm in (float("inf"), 1.0, 0.5))
    out = run_learned(pkg, ctx, eval_index=1, methods=methods)
    print(json.dumps({"learned_validation": {
        name: {"speedup_vs_uniform_best_schedules": out[name].get("speedup_vs_uniform_best_schedules", 1.0),
               "best": out[name]["best"]} for name, _ in methods},
        "target_champion": out["target_champion"], "workload": out["workload"]}), flush=True)
    ctx.close()
    return 0


def run_learned_anneal_only(args):
    """Small profiling case for the Metropolis kernel with the learned proposal: on
    the held-out antigen of the learned-proposal workload (1024 x 20 residues), one
    25-step launch with the uniform proposal and one with a network of zero weights
    (constant outputs: the same trajectory, every network call made)."""
    from __graft_entry__ import load_package
    pkg = load_package()
    ctx = pkg.GpuContext.create(0)
    L = pkg.learned
    cfg = pkg.workloads.config4(n_train=1, n_eval=1)
    shell = float(cfg["train"][0][1])
    ctx.set_params(pkg.Params.defaults(shell_radius=shell, seed=11))
    eval_ag, _, eval_pop = cfg["eval"][0]
    (eval_id,) = L.add_antigens(ctx, [eval_ag])
    agid = L.upload_populations(ctx, [eval_pop], [eval_id], 20)
    ctx.diffuse(PHASE1_STEPS, 0)
    s0 = ctx.state_download()
    ctx.mlp_set_params(np.zeros(pkg.MLP_N_PARAMS, np.float32))
    ms = {}
    for learned in (False, True):
        traj, _ = L.anneal_champions(ctx, s0, agid, 20, n_steps=25, chunk=25, learned=learned)
        ms["learned" if learned else "uniform"] = traj[-1][0]
    print(json.dumps({"learned_anneal_only": {"steps": 25, "candidates": 1024, "ms": ms}}), flush=True)
    ctx.close()
    return 0


def run_block_only(args):
    """Small profiling case for the search block: 3 enqueued blocks (CUDA graph, the
    selection of each block beside the next block's steps) of the bench workload at
    launch shape (cg_warps, cg_lanes[, cg_order[, cg_queue[, cg_flat]]])."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    ctx = pkg.GpuContext.create(0)
    ctx.set_params(pkg.Params.defaults(flags=pkg.FLAG_GRAPH))
    cfg, ag_aa, ag_pos, pop, pos, chi = build_workload(pkg, ctx, 0)
    shape = [int(x) for x in args.block_only.split(",")]
    w, lanes, order, queue, flat = (shape + [1, 1, 0][len(shape) - 2:])[:5]  # defaults: order 1, queue 1, flat 0
    # scoring: 16 warps x 4 CTAs per SM, residue-index queue order (the shape the
    # autotuner keeps for this workload)
    ctx.set_launch_cfg(16, 4, w, lanes, order, 1, queue, flat)
    ctx.state_upload(pop.aa, chi, pos, uniform_n_res=int(pop.n_res[0]))
    for k in range(3):  # enqueued blocks, as the bench issues them (graph replays)
        ctx.block_async(N_STEPS_PER_BLOCK, k * N_STEPS_PER_BLOCK, TOP_K)
    ctx.block_fetch(TOP_K)
    torch.cuda.synchronize()
    print(json.dumps({"block_only": {"cg_warps": w, "cg_lanes": lanes, "cg_order": order, "cg_queue": queue,
                                     "cg_flat": flat, "blocks": 3}}), flush=True)
    ctx.close()
    return 0


def run_mlp_only(args):
    """Small profiling case for the proposal network's tensor-core GEMMs: 3 loss +
    gradient passes on `rows` random feature rows."""
    from __graft_entry__ import load_package
    pkg = load_package()
    ctx = pkg.GpuContext.create(0)
    rng = np.random.default_rng(0)
    n = args.mlp_only
    f = np.zeros((n, pkg.MLP_IN), np.float32)
    f[np.arange(n), rng.integers(0, 20, n)] = 1.0
    f[:, 20:] = np.log1p(rng.poisson(0.6, (n, pkg.MLP_IN - 20))).astype(np.float32)
    ctx.mlp_set_params(pkg.mlp_init_params(0))
    for _ in range(3):
        loss, _ = ctx.mlp_loss_grad(f, rng.integers(0, 25, n).astype(np.int32), rng.normal(size=n).astype(np.float32))
    print(json.dumps({"mlp_only": {"rows": n, "loss": loss}}), flush=True)
    ctx.close()
    return 0


def run_phase2_only(args):
    """Small profiling case for the Metropolis kernel (one GPU, one launch timed)."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    ctx = pkg.GpuContext.create(0)
    cfg, ag_aa, ag_pos, pop, pos, chi = build_workload(pkg, ctx, 0)
    n_res = int(pop.n_res[0])
    ctx.state_upload(pop.aa, chi, pos, uniform_n_res=n_res)
    ext = torch.cuda.ExternalStream(ctx.stream)
    global PHASE2_STEPS
    PHASE2_STEPS = args.phase2_only
    out, _ = measure_phase2(torch, ctx, ext, np.arange(TOP_K), n_res, reps=1)
    print(json.dumps({"phase2_only": out}), flush=True)
    ctx.close()
    return 0


def launch_ranks(n, argv, timeout_s=3600):
    """`bench.py --gpus N` started as one process (no WORLD_SIZE in the environment):
    start N ranks, one per GPU, under torch.distributed.run on 127.0.0.1 and return
    its exit status.  Rank 0 prints the one JSON line; the others print nothing."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve())] + list(argv)
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "1"))
    try:
        return subprocess.run(cmd, env=env, timeout=timeout_s).returncode
    except subprocess.TimeoutExpired:
        sys.stderr.write(f"bench.py: {n} ranks did not finish within {timeout_s} s\n")
        return 124


def run_rank_check(args, rank, world):
    """The multi-rank plumbing of the timed run without a GPU (CPU `gloo`): every rank
    holds a seeded local population's energies and times, the ranks meet at the
    barrier, the timed region is the max over ranks, the candidate total the sum, and
    the survivors are merged by the one all-gather -- the calls run_ours makes on N
    GPUs.  Rank 0 prints one JSON line."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        dist.init_process_group(backend="gloo", timeout=timedelta(seconds=60))
    cpu = torch.device("cpu")
    rng = np.random.default_rng(1000 + rank)
    n_cand = 1024
    e = rng.normal(-20.0, 5.0, size=n_cand)
    local = np.lexsort((np.arange(n_cand), e))[:TOP_K]
    if world > 1:
        dist.barrier()
    ms = max_over_ranks(torch, dist, world, 0.2 + 0.01 * rank, cpu)
    total = sum_over_ranks(torch, dist, world, float(n_cand), cpu)
    idx, ev = merge_survivors(torch, dist, world, e, local, rank, n_cand)
    if rank == 0:
        print(json.dumps({"rank_check": True, "n_gpus": world, "ms_per_step": ms, "candidates": int(total),
                          "survivors": idx.tolist(), "survivor_energies": ev.tolist()}), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-proposal time-to-target runs")
    ap.add_argument("--phase2-only", type=int, default=0, metavar="STEPS",
                    help="profiling case: one launch of STEPS Langevin + Metropolis steps on 64 candidates")
    ap.add_argument("--block-only", default="", metavar="WARPS,LANES[,ORDER[,QUEUE[,FLAT]]]",
                    help="profiling case: 3 search blocks at this gradient-step launch shape")
    ap.add_argument("--mlp-only", type=int, default=0, metavar="ROWS",
                    help="profiling case: 3 loss + gradient passes of the proposal network on ROWS rows")
    ap.add_argument("--learned-anneal-only", action="store_true",
                    help="profiling case: one uniform and one learned-proposal Metropolis launch of 25 steps")
    ap.add_argument("--learned-validation", action="store_true",
                    help="proposal temperature settings of the learned proposal on the validation antigen")
    ap.add_argument("--rank-check", action="store_true",
                    help="the multi-rank plumbing (barrier, max/sum over ranks, survivor all-gather) on CPU gloo")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args.gpus, sys.argv[1:])
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.rank_check:
        return run_rank_check(args, rank, world)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.phase2_only:
        return run_phase2_only(args)
    if args.block_only:
        return run_block_only(args)
    if args.mlp_only:
        return run_mlp_only(args)
    if args.learned_validation:
        return run_learned_validation(args)
    if args.learned_anneal_only:
        return run_learned_anneal_only(args)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
