"""The transcribed force-field tables of the oracle and of the CUDA library equal
the reference source (tests/golden/reference_tables.json, parsed from
amber.rs / rotamer.rs / atom.rs by tests/golden/gen_reference_tables.py)."""
import numpy as np
import pytest


def test_golden_shapes(golden):
    # reference tests: ALA has 5 heavy atoms, GLY 4 (allatom.rs:560-578); ILE has 5 rotamers (rotamer.rs:490-494)
    n = [len(r["atoms"]) for r in golden["residues"]]
    assert n[0] == 5 and n[7] == 4 and max(n) == 14 and n[17] == 14
    assert len(golden["rotamers"][9]) == 5
    assert golden["rotamers"][0] == [] and golden["rotamers"][7] == []
    assert all(r["ca_idx"] == 1 for r in golden["residues"])
    # every residue's atom count = backbone (4, or 5 with CB) + side-chain build program
    for a, r in enumerate(golden["residues"]):
        nb = 4 if a == 7 else 5
        assert len(r["atoms"]) == nb + len(golden["sidechain_defs"][a])


def test_oracle_tables(oracle, golden):
    for a, r in enumerate(golden["residues"]):
        topo = oracle.topology(a)
        assert len(topo) == len(r["atoms"])
        for (q, t, h), g in zip(topo, r["atoms"]):
            assert np.float32(q) == np.float32(g["charge"]) and t == g["type"] and h == g["hydrophobic"]
        rots = oracle.rotamers(a)
        assert len(rots) == len(golden["rotamers"][a])
        for got, exp in zip(rots, golden["rotamers"][a]):
            assert np.array_equal(np.float32(got), np.float32(exp))
        q, e, s, h = oracle.residue_level(a)
        rl = golden["residue_level"]
        assert (np.float32(q), np.float32(e), np.float32(s), h) == (
            np.float32(rl["charge"][a]), np.float32(rl["lj_epsilon"][a]), np.float32(rl["lj_sigma"][a]),
            rl["hydrophobic"][a])
    for t in range(16):
        r, e = oracle.amber_nb(t)
        assert (np.float32(r), np.float32(e)) == tuple(np.float32(golden["amber_nb"][t]))


def test_library_tables(pkg, golden):
    T = pkg.tables()
    for a, r in enumerate(golden["residues"]):
        n = len(r["atoms"])
        assert T.n_atoms[a] == n
        assert np.array_equal(T.charge[a, :n], np.float32([x["charge"] for x in r["atoms"]]))
        assert np.array_equal(T.atom_type[a, :n], [x["type"] for x in r["atoms"]])
        assert np.array_equal(T.hydrophobic[a, :n], [x["hydrophobic"] for x in r["atoms"]])
        rots = golden["rotamers"][a]
        assert T.n_rot[a] == len(rots)
        for i, row in enumerate(rots):
            assert np.array_equal(T.rot_chi[a, i], np.float32(row[:4]))
        rl = golden["residue_level"]
        assert np.array_equal(T.residue_level[a], np.float32([rl["charge"][a], rl["lj_epsilon"][a],
                                                              rl["lj_sigma"][a], rl["hydrophobic"][a]]))
    assert np.array_equal(T.r_min_half, np.float32([x[0] for x in golden["amber_nb"]]))
    assert np.array_equal(T.epsilon, np.float32([x[1] for x in golden["amber_nb"]]))
    assert np.array_equal(T.hbond & 1, np.array(golden["hbond_donor"], int))
    assert np.array_equal(T.hbond >> 1, np.array(golden["hbond_acceptor"], int))
    assert np.array_equal(T.eef1, np.float32(golden["eef1"]))


def test_default_params_are_reference_constants(pkg, golden):
    p = pkg.Params.defaults()
    d = golden["diffusion_consts"]
    for name, key in [("step", "STEP"), ("noise_base", "NOISE_BASE"), ("t_hot", "T_HOT"), ("t_cold", "T_COLD"),
                      ("mutation_p", "MUTATION_P"), ("rotamer_move_p", "ROTAMER_MOVE_P"),
                      ("backbone_move_p", "BACKBONE_MOVE_P"), ("max_torsion_deg", "MAX_TORSION_DEG"),
                      ("iface_cutoff_sq", "IFACE_CUTOFF_SQ"), ("shell_radius", "INIT_RADIUS"),
                      ("max_disp", "MAX_DISP"), ("restraint_k", "RESTRAINT_K")]:
        assert np.float32(getattr(p, name)) == np.float32(d[key]), name
    assert p.ca_cell == 10.0


@pytest.mark.parametrize("aa", range(20))
def test_sidechain_programs_reference_backbone_or_earlier_atoms(golden, aa):
    for k, d in enumerate(golden["sidechain_defs"][aa]):
        assert max(d["ref"]) < 5 + k
