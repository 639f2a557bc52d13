"""Generate csrc/binder_tables.inc (packed force-field tables for the CUDA library)
from tests/golden/reference_tables.json, which is parsed from the reference's
amber.rs / rotamer.rs / atom.rs source text.

Layout (all indexed by AminoAcid order of atom.rs:4-25):
  BT_TOPO_N[20]            heavy atoms per residue (amber.rs:126-351)
  BT_SLOT_Q/TYPE/HYD[20][14]  per-slot partial charge, AMBER type, hydrophobic flag
  BT_NB[16][2]             r_min_half, epsilon per AMBER type (amber.rs:46-63)
  BT_HB[16]                bit0 donor, bit1 acceptor (amber.rs:72-84)
  BT_EEF1[16][3]           dg_ref, vol, lambda (amber.rs:414-431)
  BT_ROT_N[20], BT_ROT_CHI[20][5][4]   rotamer chi tuples (rotamer.rs:33-184)
  BT_SC_N[20], BT_SC_REF[20][9][4] (a,b,c,chi_idx), BT_SC_GEOM[20][9][3] (bond,angle,dih)
                           side-chain build programs (rotamer.rs:288-430)
  BT_RES[20][4]            residue-level charge, epsilon, sigma, hydrophobic (atom.rs:55-104)
  BT_SLOT_NAME[20][14][5]  PDB atom name of every slot (amber.rs:126-351)
  BT_AA3[20][4]            three-letter residue names (atom.rs:114-120)

Usage: python de-novo-antigen-binder_b200/csrc/gen_tables.py
"""
import json
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE.parents[1] / "tests" / "golden" / "reference_tables.json"
OUT = HERE / "binder_tables.inc"


def f(v):
    return repr(float(v)) + "f"


def pad(seq, n, fill):
    seq = list(seq)
    return seq + [fill] * (n - len(seq))


def main():
    t = json.loads(SRC.read_text())
    res = t["residues"]
    L = ["// Generated by csrc/gen_tables.py from tests/golden/reference_tables.json", ""]
    L.append("static const int BT_TOPO_N[20] = {%s};" % ", ".join(str(len(r["atoms"])) for r in res))
    L.append("static const float BT_SLOT_Q[20][14] = {")
    L += ["  {%s}," % ", ".join(f(v) for v in pad([a["charge"] for a in r["atoms"]], 14, 0.0)) for r in res]
    L.append("};")
    L.append("static const unsigned char BT_SLOT_TYPE[20][14] = {")
    L += ["  {%s}," % ", ".join(str(v) for v in pad([a["type"] for a in r["atoms"]], 14, 0)) for r in res]
    L.append("};")
    L.append("static const unsigned char BT_SLOT_HYD[20][14] = {")
    L += ["  {%s}," % ", ".join(str(v) for v in pad([a["hydrophobic"] for a in r["atoms"]], 14, 0)) for r in res]
    L.append("};")
    L.append("static const float BT_NB[16][2] = {%s};" % ", ".join("{%s, %s}" % (f(a), f(b)) for a, b in t["amber_nb"]))
    L.append("static const unsigned char BT_HB[16] = {%s};" % ", ".join(
        str(int(d) | (int(a) << 1)) for d, a in zip(t["hbond_donor"], t["hbond_acceptor"])))
    L.append("static const float BT_EEF1[16][3] = {%s};" % ", ".join(
        "{%s, %s, %s}" % tuple(f(v) for v in row) for row in t["eef1"]))
    rots = t["rotamers"]
    L.append("static const int BT_ROT_N[20] = {%s};" % ", ".join(str(len(r)) for r in rots))
    L.append("static const float BT_ROT_CHI[20][5][4] = {")
    for r in rots:
        rows = [row[:4] for row in r] + [[0.0] * 4] * (5 - len(r))
        L.append("  {%s}," % ", ".join("{%s}" % ", ".join(f(v) for v in row) for row in rows))
    L.append("};")
    sc = t["sidechain_defs"]
    L.append("static const int BT_SC_N[20] = {%s};" % ", ".join(str(len(d)) for d in sc))
    L.append("static const unsigned char BT_SC_REF[20][9][4] = {")
    for d in sc:
        rows = [x["ref"] + [x["chi_idx"]] for x in d] + [[0, 0, 0, 255]] * (9 - len(d))
        L.append("  {%s}," % ", ".join("{%d, %d, %d, %d}" % tuple(row) for row in rows))
    L.append("};")
    L.append("static const float BT_SC_GEOM[20][9][3] = {")
    for d in sc:
        rows = [[x["bond"], x["angle"], x["dihedral_fixed"]] for x in d] + [[0.0] * 3] * (9 - len(d))
        L.append("  {%s}," % ", ".join("{%s}" % ", ".join(f(v) for v in row) for row in rows))
    L.append("};")
    rl = t["residue_level"]
    L.append("static const float BT_RES[20][4] = {%s};" % ", ".join(
        "{%s, %s, %s, %s}" % (f(q), f(e), f(s), f(h)) for q, e, s, h in zip(
            rl["charge"], rl["lj_epsilon"], rl["lj_sigma"], rl["hydrophobic"])))
    L.append("static const char BT_SLOT_NAME[20][14][5] = {")
    L += ["  {%s}," % ", ".join('"%s"' % a["name"] for a in r["atoms"]) for r in res]
    L.append("};")
    # AminoAcid::three_letter (atom.rs:114-120): the enum names in upper case
    L.append("static const char BT_AA3[20][4] = {%s};" % ", ".join('"%s"' % n.upper() for n in t["amino_acids"]))
    OUT.write_text("\n".join(L) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
