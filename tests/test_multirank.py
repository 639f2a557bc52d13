"""The multi-GPU host logic of bench.py, on CPU: world-size-2 `gloo` process groups
(one process per rank, as torchrun starts them) merge their local top-k survivors
into the global top-k with one all-gather, and reduce the timed region with MAX and
the candidate totals with SUM -- the calls bench.py makes on N GPUs.  Energies
include ties across ranks and NaNs (which sort after every number)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
WORLD = 2
N_CAND = 96
K = 16


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _energies():
    rng = np.random.default_rng(5)
    e = rng.normal(size=(WORLD, N_CAND)).round(1)  # rounding makes ties, also across ranks
    e[0, [3, 40]] = np.nan
    e[1, 7] = np.nan
    e[1, 11] = e[0, 5]
    return e


def _order(e, gidx):
    """Ascending energy, NaN last, ties by global index."""
    return np.lexsort((gidx, np.where(np.isnan(e), np.inf, e)))


def _rank_main(rank, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=timedelta(seconds=60))
    try:
        e = _energies()[rank]
        local_top = _order(e, np.arange(N_CAND))[:K]
        idx, ev = bench.merge_survivors(torch, dist, WORLD, e, local_top, rank, N_CAND, k=K)
        cpu = torch.device("cpu")
        ms = bench.max_over_ranks(torch, dist, WORLD, 1.5 * (rank + 1), cpu)
        total = bench.sum_over_ranks(torch, dist, WORLD, float(N_CAND), cpu)
        q.put((rank, idx.tolist(), ev.tolist(), ms, total))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_survivor_merge_and_reductions():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    try:
        got = {}
        for _ in range(WORLD):
            rank, idx, ev, ms, total = q.get(timeout=180)
            got[rank] = (np.array(idx), np.array(ev), ms, total)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    e = _energies().reshape(-1)
    gidx = np.arange(WORLD * N_CAND)
    exp = _order(e, gidx)[:K]
    for rank in range(WORLD):
        idx, ev, ms, total = got[rank]
        assert np.array_equal(idx, gidx[exp])  # every rank holds the same global survivors
        assert np.array_equal(ev, e[exp], equal_nan=True)
        assert ms == pytest.approx(1.5 * WORLD)
        assert total == WORLD * N_CAND


def test_merge_single_rank_is_local_top_k():
    sys.path.insert(0, str(ROOT))
    import bench
    e = _energies()[0]
    local = _order(e, np.arange(N_CAND))[:K]
    idx, ev = bench.merge_survivors(None, None, 1, e, local, 0, N_CAND, k=K)
    assert np.array_equal(idx, local) and np.array_equal(ev, e[local], equal_nan=True)


def test_bench_gpus_2_starts_two_ranks():
    """`bench.py --gpus 2` run as one process starts two ranks (torch.distributed.run
    on 127.0.0.1) that meet in a world-size-2 group; with --rank-check they run the
    timed run's collective calls on CPU gloo and rank 0 alone prints one line."""
    import json
    import subprocess
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--rank-check"], capture_output=True,
                       text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    out = json.loads(lines[0])
    assert out["n_gpus"] == 2 and out["candidates"] == 2048
    # the merged survivors = the global top-64 of both ranks' seeded energies
    e = np.concatenate([np.random.default_rng(1000 + rank).normal(-20.0, 5.0, size=1024) for rank in range(2)])
    exp = _order(e, np.arange(2048))[:64]
    assert out["survivors"] == exp.tolist()
    assert out["ms_per_step"] == pytest.approx(0.21)
