"""Failure paths made on the host or by a bounded wait, never by a GPU fault.

  * A device wait that runs out (a barrier nothing arrives on, a few thousand
    polls) returns BINDER_ERR_TIMEOUT, and the context keeps working.
  * An injected device-allocation failure surfaces as BINDER_ERR_OOM from the
    entry point that allocates, and the next call succeeds."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(ctx, pkg):
    L = pkg.lib()
    t0 = time.perf_counter()
    st = L.binder_selftest_wait(ctx._h, 4096)
    assert st == 4  # BINDER_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    assert b"timed out" in L.binder_last_error(ctx._h)
    # the context (and its stream) still runs kernels
    ctx.mlp_set_params(pkg.mlp_init_params(0))
    out = ctx.mlp_forward(np.zeros((4, pkg.MLP_IN), np.float32))
    assert out.shape == (4, 25) and np.all(np.isfinite(out))


def test_injected_allocation_failure_reports_oom(pkg):
    c = pkg.GpuContext.create(0)
    try:
        cfg = pkg.workloads.config0()
        ag_aa, ag_ca = cfg["antigens"][0]
        ag_pos, _ = c.build_residues(ag_ca, ag_aa)
        c.add_antigen(ag_aa, ag_pos)
        pop = cfg["pop"]
        pos, chi = c.build_residues(pop.ca, pop.aa)
        pkg.lib().binder_debug_fail_alloc(0)
        with pytest.raises(pkg.BinderError) as ei:
            c.state_upload(pop.aa, chi, pos, uniform_n_res=int(pop.n_res[0]))
        assert ei.value.status == 3  # BINDER_ERR_OOM
        c.state_upload(pop.aa, chi, pos, uniform_n_res=int(pop.n_res[0]))  # recovers
        a, _, p = c.state_download()
        assert np.array_equal(a, pop.aa) and np.array_equal(p, pos)
    finally:
        pkg.lib().binder_debug_fail_alloc(-1)
        c.close()
