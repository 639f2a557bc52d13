"""The reference's input and output formats (pdb.rs, report.rs), host code of the
library called through the C ABI (no GPU needed): the CA-only PDB reader, the
one-letter peptide builder, the CA-only / all-atom / multi-chain PDB writers and the
FASTA / JSON / CSV report writers.  Expected texts follow the reference's format
strings column by column; report.rs's own unit tests are restated."""
import numpy as np
import pytest


def _record(serial, name, res, chain, seq, x, y, z):
    # pdb.rs:105-106: "ATOM  {:5} {:<4} {:3} {:1}{:4}    {:8.3}{:8.3}{:8.3}  1.00  0.00           C"
    return f"ATOM  {serial:5d} {name:<4} {res:<3} {chain}{seq:4d}    {x:8.3f}{y:8.3f}{z:8.3f}  1.00  0.00           C"


def test_write_pdb_ca_exact_columns(pkg):
    xyz = np.float32([[1.0, 2.0, 3.0], [-10.25, 0.5, 123.4567]])
    out = pkg.write_pdb_ca(xyz, [0, 8], chain="H")
    assert out.splitlines() == [
        "ATOM      1  CA  ALA H   1       1.000   2.000   3.000  1.00  0.00           C",
        "ATOM      2  CA  HIS H   2     -10.250   0.500 123.457  1.00  0.00           C",
        "END"]


def test_pdb_roundtrip_and_reader_rules(pkg):
    rng = np.random.default_rng(3)
    xyz = rng.uniform(-99, 99, size=(40, 3)).astype(np.float32)
    aa = rng.integers(0, 20, 40).astype(np.uint8)
    got_xyz, got_aa = pkg.parse_pdb(pkg.write_pdb_ca(xyz, aa))
    assert np.array_equal(got_aa, aa)
    assert np.allclose(got_xyz, xyz, atol=5e-4)
    text = "\r\n".join([
        "HEADER    TEST",
        _record(1, " N  ", "ALA", "A", 1, 0, 0, 0),           # not a CA: skipped
        "HETATM    2  CA  HID A   2       1.000   2.000   3.000",  # HETATM, HID -> His
        "ATOM      3  CA  HIP A   3       4.000   5.000   6.000",
        "ATOM      4  CA  XYZ A   4       abc     7.500   8.500",  # unknown name -> Gly, bad x -> 0
        "ATOM      5  CA  TRP A   5       1.5",                    # short line: y, z absent -> 0
        "ATOM      6  CB  TRP A   5       9.000   9.000   9.000",
    ]) + "\n"
    got_xyz, got_aa = pkg.parse_pdb(text)
    assert got_aa.tolist() == [8, 8, 7, 17]
    assert np.array_equal(got_xyz, np.float32([[1, 2, 3], [4, 5, 6], [0, 7.5, 8.5], [0, 0, 0]]))
    with pytest.raises(pkg.BinderError) as e:
        pkg.parse_pdb("HEADER only\nEND\n")
    assert e.value.status == 1  # EmptyInput
    with pytest.raises(pkg.BinderError) as e:
        pkg.parse_pdb(path="/nonexistent/dir/x.pdb")
    assert e.value.status == 10  # BINDER_ERR_IO


def test_parse_pdb_file(pkg, tmp_path):
    xyz = np.float32([[1, 2, 3], [4, 5, 6]])
    f = tmp_path / "ag.pdb"
    f.write_text(pkg.write_pdb_ca(xyz, [5, 6]))
    got_xyz, got_aa = pkg.parse_pdb(path=f)
    assert got_aa.tolist() == [5, 6] and np.array_equal(got_xyz, xyz)


def test_parse_peptide(pkg):
    xyz, aa = pkg.parse_peptide("ACdw")
    assert aa.tolist() == [0, 4, 3, 17]
    n = np.float32(4)
    exp = np.array([(np.float32(i) - n * np.float32(0.5)) * np.float32(3.8) for i in range(4)], np.float32)
    assert np.array_equal(xyz[:, 0], exp) and not xyz[:, 1:].any()
    for bad in ("", "ACX1"):
        with pytest.raises(pkg.BinderError):
            pkg.parse_peptide(bad)


def test_write_pdb_allatom_and_multi(pkg, oracle):
    aa = np.uint8([7, 17, 0])  # Gly (4 atoms), Trp (14), Ala (5)
    ca = np.float32([[0, 0, 0], [3.8, 0, 0], [7.6, 0, 0]])
    pos, _ = oracle.build_residues(ca, aa)
    lines = pkg.write_pdb_allatom(aa, pos, chain="L").splitlines()
    assert len(lines) == 4 + 14 + 5 + 1 and lines[-1] == "END"
    p = pos[1, 13]
    assert lines[4 + 13] == _record(18, " CH2", "TRP", "L", 2, *map(float, p))
    assert lines[0] == _record(1, " N  ", "GLY", "L", 1, *map(float, pos[0, 0]))
    multi = pkg.write_pdb_multi([(aa[:2], pos[:2], "H"), (aa[2:], pos[2:], "L")]).splitlines()
    assert multi[18] == "TER" and multi[-2] == "TER" and multi[-1] == "END"
    assert multi[19] == _record(19, " N  ", "ALA", "L", 1, *map(float, pos[2, 0]))
    assert len(multi) == 4 + 14 + 1 + 5 + 1 + 1


def _sample(pkg, **kw):
    d = dict(rank=1, sequence="ACDEFG", energy=-12.5, entropy_penalty=5.7, dg_corrected=-6.8, net_charge=2,
             aggregation_risk=False, n_interface=4, clashes=0, rama_outliers=1)
    d.update(kw)
    return pkg.CandidateReport.make(**d)


def test_report_writers_restate_reference_tests(pkg):
    # report.rs:138-178
    out = pkg.write_fasta([_sample(pkg)])
    assert ">candidate_1" in out and "ACDEFG" in out
    out = pkg.write_fasta([_sample(pkg, light_sequence="HIKLMN")])
    assert "_VH" in out and "_VL" in out and "HIKLMN" in out
    out = pkg.write_json([_sample(pkg), _sample(pkg)])
    assert out.startswith("[") and out.rstrip().endswith("]")
    assert out.count("{") == 2 and out.count("}") == 2
    lines = pkg.write_csv([_sample(pkg), _sample(pkg)]).splitlines()
    assert len(lines) == 3 and lines[0].startswith("rank,")


def test_report_writers_exact_text(pkg):
    a = _sample(pkg)
    b = _sample(pkg, rank=2, sequence='Q"W', light_sequence="E\\R", energy=-3.25, aggregation_risk=True,
                clashes=None, rama_outliers=None)
    assert pkg.write_fasta([a, b]) == (">candidate_1 E=-12.5000\nACDEFG\n>candidate_2_VH E=-3.2500\nQ\"W\n"
                                       ">candidate_2_VL E=-3.2500\nE\\R\n")
    f32 = lambda v: float(np.float32(v))  # noqa: E731 (the report holds f32)
    assert pkg.write_json([a, b]) == (
        "[\n  {\n    \"rank\": 1,\n    \"sequence\": \"ACDEFG\",\n    \"light_sequence\": null,\n"
        f"    \"energy\": {f32(-12.5):.6f},\n    \"entropy_penalty\": {f32(5.7):.6f},\n"
        f"    \"dg_corrected\": {f32(-6.8):.6f},\n    \"net_charge\": 2,\n    \"aggregation_risk\": false,\n"
        "    \"n_interface\": 4,\n    \"clashes\": 0,\n    \"rama_outliers\": 1\n  },\n"
        "  {\n    \"rank\": 2,\n    \"sequence\": \"Q\\\"W\",\n    \"light_sequence\": \"E\\\\R\",\n"
        f"    \"energy\": {f32(-3.25):.6f},\n    \"entropy_penalty\": {f32(5.7):.6f},\n"
        f"    \"dg_corrected\": {f32(-6.8):.6f},\n    \"net_charge\": 2,\n    \"aggregation_risk\": true,\n"
        "    \"n_interface\": 4,\n    \"clashes\": null,\n    \"rama_outliers\": null\n  }\n]\n")
    assert pkg.write_csv([a, b]).splitlines() == [
        "rank,sequence,light_sequence,energy,entropy_penalty,dg_corrected,net_charge,aggregation_risk,n_interface,"
        "clashes,rama_outliers",
        f"1,\"ACDEFG\",\"\",{f32(-12.5):.6f},{f32(5.7):.6f},{f32(-6.8):.6f},2,false,4,0,1",
        f"2,\"Q\"\"W\",\"E\\R\",{f32(-3.25):.6f},{f32(5.7):.6f},{f32(-6.8):.6f},2,true,4,,"]
    assert pkg.write_json([]) == "[\n]\n" and pkg.write_fasta([]) == ""
