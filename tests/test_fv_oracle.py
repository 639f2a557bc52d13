"""The Fv two-chain engine's inputs and the CPU oracle's restatement of it
(diffusion.rs:477-827, germline.rs): the germline scaffolds and their assembled
chains (germline.rs's own tests restated), the run_fv initial placement, and the
oracle's iteration loop (elitist: the best fv_energy never rises)."""
import numpy as np

from conftest import rel_err


def test_germline_tests_restated(pkg):
    wl = pkg.workloads
    for fw in (wl.VH_FRAMEWORK, wl.VL_FRAMEWORK):
        cdrs = [np.zeros(fw[k], np.uint8) for k in (1, 3, 5)]
        seq, region = wl.assemble_chain(fw, *cdrs)
        assert len(seq) == len(fw[0]) + fw[1] + len(fw[2]) + fw[3] + len(fw[4]) + fw[5] + len(fw[6])  # :136-154
        assert (region > 0).sum() == fw[1] + fw[3] + fw[5]                                          # :157-164
        assert "C" in fw[0] and "C" in fw[4]                                                       # :167-172
    assert len(wl.assemble_chain(wl.VH_FRAMEWORK, *[[0] * wl.VH_FRAMEWORK[k] for k in (1, 3, 5)])[0]) == 110


def test_fib_sphere_offsets_stay_within_their_target_radius(pkg):
    # diffusion.rs:1186-1195
    for i in range(20):
        d = np.linalg.norm(pkg.workloads.fib_sphere_offset(i, 20, 5.0))
        assert abs(d - 5.0) < 1e-3


def _fv_inputs(pkg, oracle, n_cand):
    cfg = pkg.workloads.config1(n_cand=4)
    ag_aa, ag_ca = cfg["antigens"][0]
    ag_pos, _ = oracle.build_residues(ag_ca, ag_aa)
    fv = pkg.workloads.config_fv(ag_ca, n_cand=n_cand)
    chains = []
    for name in ("heavy", "light"):
        aa, ca, region = fv[name]
        pos, chi = oracle.build_residues(ca, aa)
        chains.append((aa.copy(), chi, pos, (region > 0).astype(np.uint8)))
    return oracle.Antigen(ag_aa, ag_pos), fv, chains


def test_oracle_fv_run_is_elitist(pkg, oracle):
    A, fv, (h, l) = _fv_inputs(pkg, oracle, 2)
    n_h, n_l = fv["n_heavy"], fv["n_light"]
    e0 = [A.fv_energy(h[0][c * n_h:(c + 1) * n_h], h[2][c * n_h:(c + 1) * n_h], l[0][c * n_l:(c + 1) * n_l],
                      l[2][c * n_l:(c + 1) * n_l]) for c in range(2)]
    prm = oracle.OrcParams.defaults(seed=7)
    best, margin = A.fv_run(prm, h, l, 6, fv["target_radius"], cand_id=np.arange(2))
    assert np.all(best <= np.array(e0) + 1e-9)
    e1 = [A.fv_energy(h[0][c * n_h:(c + 1) * n_h], h[2][c * n_h:(c + 1) * n_h], l[0][c * n_l:(c + 1) * n_l],
                      l[2][c * n_l:(c + 1) * n_l]) for c in range(2)]
    assert np.all(rel_err(e1, best) < 1e-12)  # the chains left in place are the best pair
    # the framework sequence never changes (mutations only at CDR positions)
    assert np.array_equal(h[0][h[3] == 0], pkg.workloads.config_fv(np.zeros((1, 3), np.float32), 2)["heavy"][0][h[3] == 0])
