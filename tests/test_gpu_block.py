"""The search block through its CUDA graph, every launch shape and the autotuner:
results are bit-identical to the eagerly launched block (launch shapes only change
which warp takes which residue, never the arithmetic)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(ctx, oracle, pkg, n_cand=256, flags=None):
    cfg = pkg.workloads.config1(n_cand=n_cand)
    ag_aa, ag_ca = cfg["antigens"][0]
    ag_pos, _ = oracle.build_residues(ag_ca, ag_aa)
    ctx.clear_antigens()
    kw = {} if flags is None else {"flags": flags}
    ctx.set_params(pkg.Params.defaults(shell_radius=cfg["shell"][0], seed=5, **kw))
    ctx.add_antigen(ag_aa, ag_pos)
    pop = cfg["pop"]
    n_res = int(pop.n_res[0])
    aa = pop.aa[: n_cand * n_res].copy()
    pos, chi = oracle.build_residues(pop.ca[: n_cand * n_res], aa)
    return aa, chi, pos, n_res


def _run_blocks(ctx, aa, chi, pos, n_res, n_blocks=3):
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    outs = [ctx.block(10, 10 * b, k=64) for b in range(n_blocks)]
    return outs, ctx.state_download()


def _same(a, b):
    (oa, sa), (ob, sb) = a, b
    for (ea, ta), (eb, tb) in zip(oa, ob):
        assert np.array_equal(ea, eb) and np.array_equal(ta, tb)
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)


def test_graph_block_matches_eager(ctx, oracle, pkg):
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg, flags=0)
    eager = _run_blocks(ctx, aa, chi, pos, n_res)
    ctx.set_params(pkg.Params.defaults(shell_radius=ctx.params.shell_radius, seed=5, flags=pkg.FLAG_GRAPH))
    n0 = ctx.launch_count
    graph = _run_blocks(ctx, aa, chi, pos, n_res)
    assert ctx.launch_count > n0
    _same(eager, graph)
    # a new upload (new buffers) re-captures the graph
    again = _run_blocks(ctx, aa, chi, pos, n_res)
    _same(eager, again)


@pytest.mark.parametrize("shape", [(4, 1, 2, 4, 0, 1, 0), (16, 8, 4, 8, 1, 0, 1), (8, 2, 4, 4, 2, 1, 1),
                                   (8, 4, 2, 8, 0, 0, 0), (8, 4, 8, 8, 2, 1, 0), (8, 4, 8, 8, 1, 1, 1),
                                   (8, 4, 2, 4, 0, 0, 1), (8, 4, 4, 8, 1, 0, 1, 32), (8, 4, 8, 8, 0, 1, 1, 16),
                                   (8, 4, 8, 8, 3, 1, 0, 8), (8, 4, 8, 8, 3, 1, 1, 8), (8, 4, 4, 8, 3, 0, 1, 16),
                                   (8, 4, 8, 8, 3, 1, 0), (8, 4, 2, 4, 3, 0, 1),
                                   (8, 4, 8, 8, 2, 0, 0, 8), (8, 4, 4, 8, 1, 1, 0, 16), (8, 4, 8, 8, 1, 1, 1, 4),
                                   (8, 4, 4, 8, 2, 0, 1, 4)])
def test_launch_shapes_bit_identical(ctx, oracle, pkg, shape):
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg)
    ctx.set_launch_cfg(8, 4, 8, 8, 0, 0, 0)
    ref = _run_blocks(ctx, aa, chi, pos, n_res)
    ctx.set_launch_cfg(*shape)
    got = _run_blocks(ctx, aa, chi, pos, n_res)
    ctx.set_launch_cfg(8, 4, 8, 8, 0, 0, 0)
    _same(ref, got)


def test_autotune_restores_state_and_caches(ctx, oracle, pkg, tmp_path, monkeypatch):
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg)
    ref = _run_blocks(ctx, aa, chi, pos, n_res)
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    cfg = ctx.autotune(reps=2)
    assert cfg.score_warps in (4, 8, 16) and cfg.cg_warps in (2, 4, 8) and 1 <= cfg.score_ctas_per_sm <= 8
    assert cfg.cg_lanes in (4, 8) and cfg.cg_order in (0, 1, 2, 3) and cfg.score_order in (0, 1) and cfg.cg_queue in (0, 1)
    assert cfg.cg_flat in (0, 4, 8, 16, 32)
    _, _, p_after = ctx.state_download()
    assert np.array_equal(p_after, pos)  # the timing runs worked on a copy
    got = [ctx.block(10, 10 * b, k=64) for b in range(3)], ctx.state_download()
    _same(ref, got)
    # a fresh context finds the choice in the cache file and does not re-tune
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("BINDER_TUNE_CACHE", str(cache))
    c2 = pkg.GpuContext.create(0)
    try:
        _setup(c2, oracle, pkg)
        c2.state_upload(aa, chi, pos, uniform_n_res=n_res)
        first = c2.autotune(reps=2)
        lines = cache.read_text().splitlines()
        assert len(lines) == 1
        c3 = pkg.GpuContext.create(0)
        try:
            _setup(c3, oracle, pkg)
            c3.state_upload(aa, chi, pos, uniform_n_res=n_res)
            again = c3.autotune(reps=2)
            assert again.as_dict() == first.as_dict()
            assert len(cache.read_text().splitlines()) == 1
        finally:
            c3.close()
    finally:
        c2.close()


def test_autotune_flag_in_block(ctx, oracle, pkg):
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg, n_cand=128, flags=pkg.FLAG_GRAPH | pkg.FLAG_AUTOTUNE)
    ref_ctx = pkg.GpuContext.create(0)
    try:
        _setup(ref_ctx, oracle, pkg, n_cand=128, flags=0)
        ref = _run_blocks(ref_ctx, aa, chi, pos, n_res)
    finally:
        ref_ctx.close()
    got = _run_blocks(ctx, aa, chi, pos, n_res)
    _same(ref, got)
    ctx.set_params(pkg.Params.defaults(shell_radius=ctx.params.shell_radius, seed=5))


def test_block_io_matches_upload_block_download(ctx, oracle, pkg):
    """binder_block_io (upload, block, write-back with the copy beside the score) gives
    the results of binder_state_upload + binder_block + binder_state_download, block
    after block on the written-back population, and leaves the same resident state."""
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg)
    ref = []
    a, c, p = aa.copy(), np.ascontiguousarray(chi, np.float32), np.ascontiguousarray(pos, np.float32)
    for b in range(3):
        ctx.state_upload(a, c, p, uniform_n_res=n_res)
        e, t = ctx.block(10, 0, k=64)
        a, c, p = ctx.state_download()
        ref.append((e, t, a.copy(), c.copy(), p.copy()))
    a, c, p = aa.copy(), np.array(chi, np.float32), np.array(pos, np.float32)
    for b in range(3):
        e, t = ctx.block_io(a, c, p, 10, k=64, uniform_n_res=n_res)
        re, rt, ra, rc, rp = ref[b]
        assert np.array_equal(e, re) and np.array_equal(t, rt)
        assert np.array_equal(a, ra) and np.array_equal(c, rc) and np.array_equal(p, rp)
    # the resident state is the written-back one
    da, dc, dp = ctx.state_download()
    assert np.array_equal(da, a) and np.array_equal(dc, c) and np.array_equal(dp, p)


def test_block_io_ragged_antigens(ctx, pkg):
    """Ragged candidates over several resident antigens: binder_block_io's energies,
    per-antigen top-k and written-back residues equal those of the three separate
    calls."""
    cfg = pkg.workloads.config2(n_cand=256)
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=26.0, seed=6))
    for ag_aa, ag_ca in cfg["antigens"]:
        p_a, _ = ctx.build_residues(ag_ca, ag_aa)
        ctx.add_antigen(ag_aa, p_a)
    pop = cfg["pop"]
    pos, chi = ctx.build_residues(pop.ca, pop.aa)
    n_seg = len(cfg["antigens"])
    ctx.state_upload(pop.aa, chi, pos, n_res=pop.n_res, antigen_id=pop.antigen_id)
    e0, t0 = ctx.block(10, 0, k=16, n_segments=n_seg)
    a0, c0, p0 = ctx.state_download()
    a = pop.aa.copy()
    c = np.array(chi, np.float32)
    p = np.array(pos, np.float32)
    e1, t1 = ctx.block_io(a, c, p, 10, k=16, n_res=pop.n_res, antigen_id=pop.antigen_id, n_segments=n_seg)
    assert np.array_equal(e0, e1) and np.array_equal(t0, t1)
    assert np.array_equal(a0, a) and np.array_equal(c0, c) and np.array_equal(p0, p)


def test_block_io_edge_cases(ctx, oracle, pkg):
    """binder_block_io without gradient steps scores the uploaded population as
    binder_score_state does and writes it back unchanged; without top-k it returns
    the energies only; bad step counts, k and amino acids are rejected."""
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg, n_cand=64)
    chi, pos = np.array(chi, np.float32), np.array(pos, np.float32)
    a, c, p = aa.copy(), chi.copy(), pos.copy()
    e, t = ctx.block_io(a, c, p, 0, k=8, uniform_n_res=n_res)
    assert np.array_equal(a, aa) and np.array_equal(c, chi) and np.array_equal(p, pos)
    assert np.array_equal(e, ctx.score_state())
    assert np.array_equal(t[0], np.argsort(e, kind="stable")[:8])
    e0, t0 = ctx.block_io(a, c, p, 5, k=0, uniform_n_res=n_res)
    assert t0 is None and np.all(np.isfinite(e0))
    for kw in ({"n_steps": -1, "k": 8}, {"n_steps": 5, "k": 2000}):
        with pytest.raises(pkg.BinderError) as err:
            ctx.block_io(aa.copy(), chi.copy(), pos.copy(), kw["n_steps"], k=kw["k"], uniform_n_res=n_res)
        assert err.value.name == "BINDER_ERR_ARG"
    bad = aa.copy()
    bad[3] = 20
    with pytest.raises(pkg.BinderError) as err:
        ctx.block_io(bad, chi.copy(), pos.copy(), 5, k=8, uniform_n_res=n_res)
    assert err.value.name == "BINDER_ERR_ARG"


def _seg_topk(e, ag_id, n_seg, k):
    """Per antigen, the stable top-k of its candidates' energies (NaN last), -1 padded."""
    out = np.full((n_seg, k), -1, np.int64)
    for a in range(n_seg):
        idx = np.nonzero(ag_id == a)[0]
        key = np.where(np.isnan(e[idx]), np.inf, e[idx])
        o = idx[np.lexsort((idx, np.isnan(e[idx]), key))][:k]
        out[a, :len(o)] = o
    return out


@pytest.mark.parametrize("n_cand,k,dup", [(3000, 64, True), (3000, 1, False), (1000, 17, True), (5000, 64, False)])
def test_fused_selection_one_segment(ctx, oracle, pkg, n_cand, k, dup):
    """Scoring + selection of the block (candidate sums and top-k in one launch when
    k <= 64 and the segment holds at most 4096 candidates, 128 per CTA, the
    segment's last CTA merging; 5000 candidates take the two-launch path): the
    stable top-k of the returned energies, ties (duplicated candidates) by index,
    on repeated calls and through the graph."""
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg, n_cand=n_cand)
    if dup:  # candidates 2j and 2j + 1 identical: equal energies
        for c in range(0, n_cand - 1, 2):
            sl, sl2 = slice(c * n_res, (c + 1) * n_res), slice((c + 1) * n_res, (c + 2) * n_res)
            aa[sl2], chi[sl2], pos[sl2] = aa[sl], chi[sl], pos[sl]
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    for flags in (0, pkg.FLAG_GRAPH):
        ctx.set_params(pkg.Params.defaults(shell_radius=ctx.params.shell_radius, seed=5, flags=flags))
        for b in range(2):
            e, top = ctx.block(5 * b, 5 * b, k=k)
            assert np.array_equal(top, _seg_topk(e, np.zeros(n_cand, int), 1, k))
            assert np.array_equal(top[0], ctx.topk(e, k))
            assert np.array_equal(e, ctx.score_state())
    if dup:
        assert len(np.unique(e)) <= (n_cand + 1) // 2


def test_fused_selection_segments(ctx, pkg):
    """Eight antigens, ragged candidates: each segment's stable top-k; a segment with
    fewer candidates than k is padded with -1."""
    cfg = pkg.workloads.config2(n_cand=1200)
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=26.0, seed=6))
    for ag_aa, ag_ca in cfg["antigens"]:
        p_a, _ = ctx.build_residues(ag_ca, ag_aa)
        ctx.add_antigen(ag_aa, p_a)
    pop = cfg["pop"]
    ag_id = pop.antigen_id.copy()
    ag_id[ag_id == 7] = 6  # antigen 7 without candidates, antigen 6 with twice as many
    keep = np.ones(len(ag_id), bool)
    keep[np.nonzero(ag_id == 0)[0][40:]] = False  # antigen 0: 40 candidates < k
    off = np.concatenate([[0], np.cumsum(pop.n_res)])
    rs = np.concatenate([np.arange(off[c], off[c + 1]) for c in np.nonzero(keep)[0]])
    pos, chi = ctx.build_residues(pop.ca[rs], pop.aa[rs])
    n_res, ag_k = pop.n_res[keep], ag_id[keep]
    ctx.state_upload(pop.aa[rs], chi, pos, n_res=n_res, antigen_id=ag_k)
    for k in (64, 50):
        e, top = ctx.block(10, 0, k=k, n_segments=8)
        assert np.array_equal(top, _seg_topk(e, ag_k, 8, k))
        assert np.all(top[7] == -1) and np.sum(top[0] >= 0) == 40


def test_enqueued_blocks_pipeline(ctx, oracle, pkg):
    """Enqueued blocks (binder_block without outputs, graph on) sum and select each
    block's energies beside the next block's gradient steps; binder_block_fetch, or any
    other call, runs the last block's selection first.  Results equal the synchronous
    blocks', whatever comes between."""
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg, n_cand=512, flags=pkg.FLAG_GRAPH)
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    sync = [ctx.block(10, 10 * b, k=64) for b in range(5)]
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    for b in range(5):
        ctx.block_async(10, 10 * b, 64)
    e, top = ctx.block_fetch(64)
    assert np.array_equal(e, sync[4][0]) and np.array_equal(top, sync[4][1])
    # a call between the enqueued blocks and the fetch (the selection runs before it)
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    for b in range(3):
        ctx.block_async(10, 10 * b, 64)
    assert np.array_equal(ctx.score_state(), sync[2][0])
    e, top = ctx.block_fetch(64)
    assert np.array_equal(e, sync[2][0]) and np.array_equal(top, sync[2][1])
    # k changes between enqueued blocks; a synchronous block after enqueued ones
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    ctx.block_async(10, 0, 64)
    ctx.block_async(10, 10, 16)
    e, top = ctx.block_fetch(16)
    assert np.array_equal(e, sync[1][0]) and np.array_equal(top[0], sync[1][1][0][:16])
    ctx.state_upload(aa, chi, pos, uniform_n_res=n_res)
    ctx.block_async(10, 0, 64)
    e, top = ctx.block(10, 10, k=64)
    assert np.array_equal(e, sync[1][0]) and np.array_equal(top, sync[1][1])


def test_block_io_graph_with_pinned_arrays(ctx, oracle, pkg):
    """binder_block_io with pinned host arrays runs as one CUDA graph (copies in, block,
    copies out): the same energies, survivors and written-back residues as with
    pageable arrays (launches one by one), on repeated calls and a new population."""
    import torch
    aa, chi, pos, n_res = _setup(ctx, oracle, pkg, n_cand=256, flags=pkg.FLAG_GRAPH)
    chi, pos = np.array(chi, np.float32), np.array(pos, np.float32)
    pa = torch.empty(aa.shape, dtype=torch.uint8, pin_memory=True).numpy()
    pc = torch.empty(chi.shape, dtype=torch.float32, pin_memory=True).numpy()
    pp = torch.empty(pos.shape, dtype=torch.float32, pin_memory=True).numpy()
    pt = torch.empty(64, dtype=torch.int32, pin_memory=True).numpy()
    a, c, p = aa.copy(), chi.copy(), pos.copy()
    pa[:], pc[:], pp[:] = aa, chi, pos
    for step in range(3):
        e0, t0 = ctx.block_io(a, c, p, 10, k=64, uniform_n_res=n_res)
        e1, t1 = ctx.block_io(pa, pc, pp, 10, k=64, uniform_n_res=n_res, out_top=pt)
        assert np.array_equal(e0, e1) and np.array_equal(t0, t1) and np.array_equal(t0[0], pt)
        assert np.array_equal(a, pa) and np.array_equal(c, pc) and np.array_equal(p, pp)
    rng = np.random.default_rng(4)
    pp[:] = pos + rng.normal(scale=0.05, size=pos.shape).astype(np.float32)
    p = pp.copy()
    e0, t0 = ctx.block_io(a, c, p, 5, k=64, uniform_n_res=n_res)
    e1, t1 = ctx.block_io(pa, pc, pp, 5, k=64, uniform_n_res=n_res, out_top=pt)
    assert np.array_equal(e0, e1) and np.array_equal(t0, t1) and np.array_equal(p, pp)
