"""The reference's own unit tests (the only known-answer tests it has for this
path), restated against the CPU oracle.  Each test names the Rust test it
re-expresses; tolerances are the reference's."""
import numpy as np

from conftest import rel_err

A = {c: i for i, c in enumerate("ARNDCQEGHILKMFPSTWYV")}


def test_nerf_places_atom_at_correct_bond_length(oracle):
    # rotamer.rs:477-487
    d = oracle.place_atom([0, 0, 0], [1.5, 0, 0], [1.5, 1.4, 0], 1.52, 112.0, -60.0)
    assert abs(np.linalg.norm(d - np.float32([1.5, 1.4, 0])) - 1.52) < 1e-4


def test_rotamer_lib_non_empty_for_ile(oracle):
    # rotamer.rs:490-494
    assert len(oracle.rotamers(A["I"])) == 5


def test_build_ala_and_gly_residues(oracle):
    # allatom.rs:560-578
    assert len(oracle.topology(A["A"])) == 5
    assert len(oracle.topology(A["G"])) == 4
    pos, _ = oracle.build_residues([[10.0, 0, 0]], [A["A"]])
    assert len(oracle.flatten([A["A"]], pos)["x"]) == 5


def test_disulfide_zero_without_partner_and_beyond_cutoff(oracle):
    # allatom.rs:590-606
    pos, _ = oracle.build_residues([[0, 0, 0]], [A["C"]])
    assert oracle.disulfide([A["C"]], pos) == 0.0
    pos, _ = oracle.build_residues([[0, 0, 0], [50, 0, 0]], [A["C"], A["C"]])
    assert oracle.disulfide([A["C"], A["C"]], pos) == 0.0


def test_disulfide_matches_pairwise_gaussian_sum(oracle):
    # allatom.rs:610-639
    aa = [A["C"]] * 3
    pos, _ = oracle.build_residues([[0, 0, 0], [3.8, 0, 0], [7.6, 0, 0]], aa)
    sg = pos[:, 5, :].astype(np.float32)
    exp = np.float32(0)
    for i in range(3):
        for j in range(i + 1, 3):
            d = np.float32(np.sqrt(np.float32(np.sum((sg[i] - sg[j]) ** 2, dtype=np.float32))))
            if d > 4.0:
                continue
            z = (d - np.float32(2.05)) / np.float32(0.4)
            exp -= np.float32(4.0) * np.float32(np.exp(np.float32(-0.5) * z * z))
    assert abs(oracle.disulfide(aa, pos) - exp) < 1e-5


def _two_residue():
    # energy.rs:406-415: antigen Lys at origin + Leu at 5 A; antibody Asp at 3 A
    return [[0, 0, 0], [5, 0, 0]], [A["K"], A["L"]], [[3, 0, 0]], [A["D"]]


def test_grid_forces_match_brute_force(oracle):
    # energy.rs:418-441 (abs tol 1e-4, cell 10 A)
    ag, ag_aa, ab, ab_aa = _two_residue()
    fb = oracle.forces_cg_brute(ag, ag_aa, ab, ab_aa)
    fg = oracle.forces_cg_grid(10.0, ag, ag_aa, ab, ab_aa)
    for a, b in zip(fb, fg):
        assert np.all(np.abs(a - b) < 1e-4)


def test_opposite_charges_attract(oracle):
    # energy.rs:444-457
    ag, ag_aa, ab, ab_aa = _two_residue()
    fx, _, _ = oracle.forces_cg_brute(ag, ag_aa, ab, ab_aa)
    assert fx[0] < 0.0


def test_lj_repulsion_at_close_range(oracle):
    # energy.rs:459-473
    fx, _, _ = oracle.forces_cg_brute([[0, 0, 0]], [A["G"]], [[1, 0, 0]], [A["G"]])
    assert fx[0] > 0.0


def _cloud(xyz, types, q=None, hyd=None):
    xyz = np.float32(xyz).reshape(-1, 3)
    n = len(xyz)
    types = np.uint8(types)
    rmh = np.float32([1.908, 1.908, 1.908, 1.908, 1.908, 1.824, 1.824, 1.824, 1.824, 1.824, 1.6612, 1.6612, 1.721,
                      1.6837, 2.0, 2.0])[types]
    eps = np.float32([0.086, 0.086, 0.086, 0.086, 0.1094, 0.17, 0.17, 0.17, 0.17, 0.17, 0.21, 0.21, 0.2104, 0.17,
                      0.25, 0.25])[types]
    return dict(x=np.ascontiguousarray(xyz[:, 0]), y=np.ascontiguousarray(xyz[:, 1]),
                z=np.ascontiguousarray(xyz[:, 2]), q=np.float32(q if q is not None else np.zeros(n)), rmh=rmh,
                eps=eps, hyd=np.uint8(hyd if hyd is not None else np.zeros(n)), type=types,
                resi=np.zeros(n, np.uint32))


def test_hbond_well_depth_and_decay(oracle):
    # energy.rs:475-491: N (donor) vs O (acceptor); well depth -1.5 at 2.9 A, 0 beyond 5 A
    ag = _cloud([[0, 0, 0]], [10])
    for r, lo, hi in [(2.9, -1.5 - 1e-5, -1.5 + 1e-5)]:
        e = oracle.energy_atoms32(ag, _cloud([[r, 0, 0]], [5]))
        assert lo < e[3] < hi
    e_near = oracle.energy_atoms32(ag, _cloud([[2.9, 0, 0]], [5]))[3]
    e_far = oracle.energy_atoms32(ag, _cloud([[3.9, 0, 0]], [5]))[3]
    e_out = oracle.energy_atoms32(ag, _cloud([[np.sqrt(26.0), 0, 0]], [5]))[3]
    assert e_near < e_far and e_out == 0.0


def test_atom_breakdown_sums_to_total(oracle):
    # energy.rs:495-507: Asp antigen at origin, Lys antibody at 3 A
    ag_pos, _ = oracle.build_residues([[0, 0, 0]], [A["D"]])
    ab_pos, _ = oracle.build_residues([[3, 0, 0]], [A["K"]])
    ag = oracle.flatten([A["D"]], ag_pos)
    ab = oracle.flatten([A["K"]], ab_pos)
    b = oracle.energy_atoms32(ag, ab)
    b64, _ = oracle.energy_atoms64(ag, ab)
    assert np.all(rel_err(b, b64, floor=1e-3) < 1e-4)


def test_query_finds_nearby_atom(oracle):
    # spatial.rs:82-87
    off, idx = oracle.grid_neighbors(10.0, [0, 50, 100], [0, 50, 100], [0, 50, 100], [1.0], [1.0], [1.0])
    assert 0 in idx and 1 not in idx


def test_eef1_burial_signs(oracle):
    # solvation.rs:100-118 restated through the full breakdown: two aliphatic CT atoms
    # (dg_ref < 0 in the table) and two carbonyl O (dg_ref < 0): polar burial raises energy
    e = oracle.energy_atoms32(_cloud([[0, 0, 0]], [10]), _cloud([[3, 0, 0]], [10]))
    assert e[4] > 0.0


def _straight_chain(oracle, start, n, aa="A"):
    """straight_chain_at (diffusion.rs:1113-1120): n residues on a straight Calpha
    trace from `start`, 3.8 A apart along x, built by protein_from_ca_trace."""
    ca = np.float32([[start[0] + i * np.float32(3.8), start[1], start[2]] for i in range(n)])
    seq = np.full(n, A[aa], np.uint8)
    pos, chi = oracle.build_residues(ca, seq)
    return seq, chi, pos


def test_minimize_never_increases_true_partner_energy(oracle):
    # diffusion.rs:1123-1140: an antibody placed on top of its partner, 50 steps
    p_aa, _, p_pos = _straight_chain(oracle, [0.0, 0.0, 0.0], 6)
    aa, chi, pos = _straight_chain(oracle, [0.2, 0.2, 0.2], 6)
    Ag = oracle.Antigen(p_aa, p_pos)
    for acc64 in (False, True):  # the reference's f32 energies, and their f64 re-evaluation
        before = Ag.minimize(aa.copy(), chi.copy(), pos.copy(), 6, 0, acc64=acc64)[0]
        a2, c2, p2 = aa.copy(), chi.copy(), pos.copy()
        after = Ag.minimize(a2, c2, p2, 6, 50, acc64=acc64)[0]
        assert after <= before + 1e-3
        final = Ag.minimize(a2.copy(), c2.copy(), p2.copy(), 6, 0, acc64=acc64)[0]
        assert final == after  # the returned energy is the final structure's


def test_minimize_is_a_noop_with_zero_steps(oracle):
    # diffusion.rs:1143-1153
    p_aa, _, p_pos = _straight_chain(oracle, [0.0, 0.0, 0.0], 4)
    aa, chi, pos = _straight_chain(oracle, [20.0, 20.0, 20.0], 4)
    Ag = oracle.Antigen(p_aa, p_pos)
    pos0 = pos.copy()
    before = Ag.score_slots64(aa, pos, 4, full=True)[0]
    after = Ag.minimize(aa, chi, pos, 4, 0)[0]
    assert after == before and np.array_equal(pos, pos0)


def test_affinity_maturation_never_worsens_the_score(oracle):
    # diffusion.rs:1156-1172 (every residue mutable there; here the interface
    # residues, as main.rs:342-344 chooses them: the 8 A chain is all interface)
    g_aa, _, g_pos = _straight_chain(oracle, [0.0, 0.0, 0.0], 6)
    aa, chi, pos = _straight_chain(oracle, [8.0, 0.0, 0.0], 6)
    Ag = oracle.Antigen(g_aa, g_pos)
    before = Ag.score_slots64(aa, pos, 6, full=True)[0]
    after, kept = Ag.affinity_maturation(aa, chi, pos, 6)
    assert after[0] <= before + 1e-3
    assert abs(after[0] - Ag.score_slots64(aa, pos, 6, full=True)[0]) < 1e-3
    assert kept[0] >= 1 and not np.all(aa == A["A"])


def test_validation_restates_reference_tests(oracle):
    # validate.rs:149-175
    aa, chi, pos = _straight_chain(oracle, [0.0, 0.0, 0.0], 6)
    assert oracle.validate(aa, pos)[0] == 0  # no clashes in a well-spaced extended chain
    ca = np.float32([[0.0, 0.0, 0.0], [3.8, 0.0, 0.0], [0.05, 0.05, 0.05]])
    seq = np.zeros(3, np.uint8)
    p, _ = oracle.build_residues(ca, seq)
    assert oracle.validate(seq, p)[0] > 0  # residues 0 and 2 on top of each other
    aa, chi, pos = _straight_chain(oracle, [0.0, 0.0, 0.0], 5)
    cl, ra = oracle.validate(aa, pos)
    assert 0 <= ra <= 3  # at most the n - 2 residues with both torsions
