"""The learned mutation / rotamer proposal workflow on one GPU context.

1. generate_tuples: plain Metropolis runs (the reference's uniform proposal,
   diffusion.rs:354-399) on training antigens log every mutation / rotamer
   decision (environment + exact energy change) into the training set.
2. train: Adam on the GPU (tcgen05 forward / backward GEMMs) on minibatches of it.
3. anneal_champions: annealed Langevin + Metropolis runs on a held-out antigen
   with the uniform or the learned Metropolis-Hastings proposal; after every chunk
   of steps the champion (lowest Metropolis energy of the population) and the wall
   time spent in the Metropolis steps.
4. time_to_target: the plain method's median final champion is the target; the
   wall time each run needs to come within `tol` kcal/mol of it.

Every number is computed by the library's kernels through the C ABI; this module
only sequences the calls.
"""
from __future__ import annotations

import time

import numpy as np


def add_antigens(ctx, antigens):
    """Build and add (aa, Calpha trace) antigens; returns their resident ids."""
    ids = []
    for ag_aa, ag_ca in antigens:
        pos, _ = ctx.build_residues(ag_ca, ag_aa)
        ids.append(ctx.add_antigen(ag_aa, pos))
    return ids


def upload_populations(ctx, pops, ids, n_res):
    aa = np.concatenate([p.aa for p in pops])
    ca = np.concatenate([p.ca for p in pops])
    agid = np.concatenate([np.full(p.n_cand, i, np.int32) for p, i in zip(pops, ids)])
    pos, chi = ctx.build_residues(ca, aa)
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res, antigen_id=agid)
    return agid


def annealing(n_steps, total, t_hot=3.0, t_cold=0.02, start=0):
    """temperature() of steps start..start+n_steps-1 of a `total`-step schedule (diffusion.rs:102-104)."""
    t_hot, t_cold = np.float32(t_hot), np.float32(t_cold)
    i = np.arange(start, start + n_steps, dtype=np.float32)
    return (t_hot * np.power(np.float32(t_cold / t_hot), i / np.float32(total))).astype(np.float32)


def generate_tuples(ctx, pops, ids, n_res, gen_steps=300, contact_steps=100, capacity=8_000_000):
    """Plain Metropolis steps over a full annealing schedule compressed into
    gen_steps, every decision logged; the log becomes the training set."""
    upload_populations(ctx, pops, ids, n_res)
    ctx.diffuse(contact_steps, 0, with_noise=False, with_mc=False)  # gradient steps: into contact
    ctx.set_proposal(False)
    ctx.mc_log(capacity)
    temps = np.array([annealing(1, 600, start=min(599, i * 600 // gen_steps))[0] for i in range(gen_steps)],
                     np.float32)
    ctx.diffuse(gen_steps, 100000, with_noise=True, with_mc=True, temps=temps)
    n = ctx.mlp_take_log()
    ctx.mc_log(0)
    return n


def train(ctx, n_steps=1500, batch=8192, lr=1e-3, huber_delta=1.0, seed=3, init_seed=0, init=None):
    from . import mlp_init_params
    ctx.mlp_set_params(mlp_init_params(init_seed) if init is None else init)
    t0 = time.perf_counter()
    losses = ctx.mlp_train(n_steps, batch=batch, lr=lr, huber_delta=huber_delta, seed=seed)
    return losses, time.perf_counter() - t0


def anneal_champions(ctx, state, agid, n_res, n_steps=600, chunk=25, learned=False, t_prop_min=0.5,
                     t_max=float("inf"), step0=200000):
    """One annealed run from `state`; [(cumulative Metropolis wall ms, champion,
    median energy)] after each chunk, and the run's move statistics."""
    ctx.state_upload(*state, uniform_n_res=n_res, antigen_id=agid)
    ctx.set_proposal(learned, t_prop_min=t_prop_min, t_max=t_max)
    traj, cum = [], 0.0
    for c in range(n_steps // chunk):
        temps = annealing(chunk, n_steps, start=c * chunk)
        t0 = time.perf_counter()
        ctx.diffuse(chunk, step0 + c * chunk, with_noise=True, with_mc=True, temps=temps)  # synchronous
        cum += 1e3 * (time.perf_counter() - t0)
        e = ctx.mc_energy()
        traj.append((cum, float(e.min()), float(np.median(e))))
    st = ctx.mc_stats().sum(0)
    ctx.set_proposal(False)
    return traj, {"mutation_rotamer_acceptance": float(st[1] / max(1, st[0]))}


def time_to_target(plain_runs, other_runs, tol=0.5):
    """Target = median final champion of the plain runs; per run the first wall
    time at which its champion is <= target + tol (inf when never)."""
    target = float(np.median([r[-1][1] for r in plain_runs]))

    def tt(run):
        for ms, champ, _ in run:
            if champ <= target + tol:
                return ms
        return float("inf")

    return target, [tt(r) for r in plain_runs], [tt(r) for r in other_runs]
