"""Generate oracle/oracle_tables.inc from tests/golden/reference_tables.json.

The JSON is parsed from the reference's Rust source text (amber.rs, rotamer.rs,
atom.rs) by tests/golden/gen_reference_tables.py; this script only re-lays the
numbers out as C arrays for the oracle.  Float literals are printed with enough
digits to round-trip exactly to the same f32 the Rust literal denotes.

Usage: python oracle/gen_tables.py
"""
import json
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "golden" / "reference_tables.json"
OUT = Path(__file__).with_name("oracle_tables.inc")


def f(v):
    s = repr(float(v))
    return s + "f"


def main():
    t = json.loads(SRC.read_text())
    L = ["// Generated by oracle/gen_tables.py from tests/golden/reference_tables.json.",
         "// Source of the numbers: reference src/amber.rs, src/rotamer.rs, src/atom.rs.", ""]
    L.append("static const float T_NB[16][2] = {  // AMBER_NB r_min_half, epsilon (amber.rs:46-63)")
    L += ["  {%s, %s}," % (f(a), f(b)) for a, b in t["amber_nb"]]
    L.append("};")
    L.append("static const unsigned char T_HB_DONOR[16] = {%s};  // amber.rs:72-77" %
             ", ".join(str(int(v)) for v in t["hbond_donor"]))
    L.append("static const unsigned char T_HB_ACC[16] = {%s};  // amber.rs:79-84" %
             ", ".join(str(int(v)) for v in t["hbond_acceptor"]))
    L.append("static const float T_EEF1[16][3] = {  // dg_ref, vol, lambda (amber.rs:414-431)")
    L += ["  {%s, %s, %s}," % tuple(f(v) for v in row) for row in t["eef1"]]
    L.append("};")
    res = t["residues"]
    L.append("static const int T_TOPO_N[20] = {%s};" % ", ".join(str(len(r["atoms"])) for r in res))
    L.append("static const int T_TOPO_CA[20] = {%s};" % ", ".join(str(r["ca_idx"]) for r in res))
    L.append("static const int T_TOPO_NCHI[20] = {%s};" % ", ".join(str(r["n_chi"]) for r in res))
    L.append("static const unsigned char T_TOPO_TYPE[20][14] = {  // amber.rs:126-351")
    L += ["  {%s}," % ", ".join(str(a["type"]) for a in r["atoms"]) for r in res]
    L.append("};")
    L.append("static const float T_TOPO_Q[20][14] = {")
    L += ["  {%s}," % ", ".join(f(a["charge"]) for a in r["atoms"]) for r in res]
    L.append("};")
    L.append("static const unsigned char T_TOPO_HYD[20][14] = {")
    L += ["  {%s}," % ", ".join(str(a["hydrophobic"]) for a in r["atoms"]) for r in res]
    L.append("};")
    L.append("static const char* const T_TOPO_NAME[20][14] = {")
    L += ["  {%s}," % ", ".join('"%s"' % a["name"] for a in r["atoms"]) for r in res]
    L.append("};")
    rots = t["rotamers"]
    L.append("static const int T_ROT_N[20] = {%s};  // rotamer.rs:163-184" % ", ".join(str(len(r)) for r in rots))
    L.append("static const float T_ROT[20][5][5] = {  // chi1..chi4, probability (rotamer.rs:33-160)")
    for r in rots:
        if not r:
            L.append("  {},")
        else:
            L.append("  {%s}," % ", ".join("{%s}" % ", ".join(f(v) for v in row) for row in r))
    L.append("};")
    sc = t["sidechain_defs"]
    L.append("struct TScDef { int a, b, c; float bond, angle, dih; int chi; };")
    L.append("static const int T_SC_N[20] = {%s};  // rotamer.rs:409-430" % ", ".join(str(len(d)) for d in sc))
    L.append("static const TScDef T_SC[20][9] = {  // rotamer.rs:288-406")
    for d in sc:
        if not d:
            L.append("  {},")
        else:
            L.append("  {%s}," % ", ".join("{%d, %d, %d, %s, %s, %s, %d}" % (
                x["ref"][0], x["ref"][1], x["ref"][2], f(x["bond"]), f(x["angle"]),
                f(x["dihedral_fixed"]), x["chi_idx"]) for x in d))
    L.append("};")
    rl = t["residue_level"]
    L.append("static const float T_RES_Q[20] = {%s};  // atom.rs:55-63" % ", ".join(f(v) for v in rl["charge"]))
    L.append("static const float T_RES_EPS[20] = {%s};  // atom.rs:66-77" % ", ".join(f(v) for v in rl["lj_epsilon"]))
    L.append("static const float T_RES_SIG[20] = {%s};  // atom.rs:80-91" % ", ".join(f(v) for v in rl["lj_sigma"]))
    L.append("static const unsigned char T_RES_HYD[20] = {%s};  // atom.rs:93-104" %
             ", ".join(str(v) for v in rl["hydrophobic"]))
    OUT.write_text("\n".join(L) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
