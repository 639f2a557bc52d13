"""The Fv two-chain engine on the GPU vs the CPU oracle, through the C ABI: the
run_fv iteration loop (diffusion.rs:791-812) of VH3-23 / IGKV1-39 germline
scaffolds with random CDRs (germline.rs) placed beside the config-1 antigen as
run_fv places them.  Each iteration steps the heavy chains against the light
chains, then the light chains against the stepped heavy chains (fv_chain_step,
diffusion.rs:560-698), and keeps the pair whose fv_energy (diffusion.rs:541-547)
is lowest.  Chains bit-exact in both Metropolis accumulation modes; best energies
within 1e-5 relative of the oracle's f64 fv_energy; a candidate whose oracle run
met an elitist decision within 1e-5 (relative) of a tie may branch and is left
out of the bit-exact comparison (at most one of eight)."""
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 8


@pytest.mark.parametrize("acc", [0, 1])
def test_fv_run_matches_oracle(ctx, oracle, pkg, acc):
    cfg = pkg.workloads.config1(n_cand=4)
    ag_aa, ag_ca = cfg["antigens"][0]
    ag_pos, _ = oracle.build_residues(ag_ca, ag_aa)
    fv = pkg.workloads.config_fv(ag_ca, n_cand=8)
    chains = []
    for name in ("heavy", "light"):
        aa, ca, region = fv[name]
        pos, chi = oracle.build_residues(ca, aa)
        chains.append((aa.copy(), chi, pos, (region > 0).astype(np.uint8)))
    h, l = chains
    ctx.clear_antigens()
    ctx.set_params(pkg.Params.defaults(shell_radius=fv["target_radius"], seed=2024, accumulate=acc))
    ctx.add_antigen(ag_aa, ag_pos)
    ids = np.arange(8)
    ctx.fv_upload(h, l, cand_id=ids)
    e_gpu = ctx.fv_run(6)
    (gha, ghc, ghp), (gla, glc, glp) = ctx.fv_download()
    A = oracle.Antigen(ag_aa, ag_pos)
    prm = oracle.OrcParams.defaults(shell_radius=fv["target_radius"], seed=2024, accumulate=acc)
    h0 = tuple(x.copy() for x in h)
    e_orc, margin = A.fv_run(prm, h, l, 6, fv["target_radius"], cand_id=ids, acc64=True, threads=THREADS)
    clean = margin > 1e-5
    assert clean.sum() >= 7
    n_h, n_l = fv["n_heavy"], fv["n_light"]
    for c in np.nonzero(clean)[0]:
        sh, sl = slice(c * n_h, (c + 1) * n_h), slice(c * n_l, (c + 1) * n_l)
        assert np.array_equal(gha[sh], h[0][sh]) and np.array_equal(ghc[sh], h[1][sh]), c
        assert np.array_equal(ghp[sh], h[2][sh]), c
        assert np.array_equal(gla[sl], l[0][sl]) and np.array_equal(glp[sl], l[2][sl]), c
    assert np.all(rel_err(e_gpu[clean], e_orc[clean]) < 1e-5)
    # the search moved the chains, and only CDR positions changed amino acid
    assert not np.array_equal(ghp, h0[2])
    assert np.array_equal(gha[h0[3] == 0], h0[0][h0[3] == 0])
