"""Extract the force-field, topology and rotamer tables from the reference's Rust
source text into ``reference_tables.json``.

The reference (a Rust crate) cannot be compiled in this environment, so its
numeric tables are pinned by parsing the source files as text.  The JSON it
writes is the golden fixture the oracle's and the CUDA library's transcribed
tables are checked against (``tests/test_tables.py``).

Sources parsed (paths inside the reference project):
  src/amber.rs     AMBER_NB (:46-63), HBOND_DONOR/ACCEPTOR (:72-84),
                   residue atom lists (:126-351), RESIDUE_TOPOLOGY (:357-378),
                   EEF1 (:414-431)
  src/rotamer.rs   ROT_* (:33-160), ROTAMER_LIB order (:163-184),
                   BD_* (:288-406), SIDECHAIN_DEFS order (:409-430)
  src/atom.rs      AminoAcid enum order (:4-25), charge/lj_epsilon/lj_sigma/
                   is_hydrophobic (:55-104)
  src/energy.rs    scalar constants (:13-27)
  src/diffusion.rs scalar hyper-parameters (:30-83)
  src/allatom.rs   ideal-backbone bond lengths (:494-497)

Usage:  python tests/golden/gen_reference_tables.py <reference_root>

reference_root is the directory of the reference crate (the one holding src/).
"""
import json
import re
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit("usage: gen_reference_tables.py <reference_root>")
REF = Path(sys.argv[1])
OUT = Path(__file__).with_name("reference_tables.json")

AA_NAMES = ["Ala", "Arg", "Asn", "Asp", "Cys", "Gln", "Glu", "Gly", "His", "Ile",
            "Leu", "Lys", "Met", "Phe", "Pro", "Ser", "Thr", "Trp", "Tyr", "Val"]
THREE = ["ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE",
         "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"]

NUM = r"-?\d+(?:\.\d+)?"


def read(rel):
    return (REF / rel).read_text()


def parse_atom_types(src):
    body = re.search(r"pub enum AtomType \{(.*?)\}", src, re.S).group(1)
    return [m.group(1) for m in re.finditer(r"^\s*(\w+)\s*=\s*\d+", body, re.M)]


def parse_amber_nb(src):
    body = re.search(r"pub static AMBER_NB.*?=\s*\[(.*?)\];", src, re.S).group(1)
    rows = re.findall(r"r_min_half:\s*(" + NUM + r"),\s*epsilon:\s*(" + NUM + r")", body)
    return [[float(a), float(b)] for a, b in rows]


def parse_bool_table(src, name):
    body = re.search(r"pub static " + name + r".*?=\s*\[(.*?)\];", src, re.S).group(1)
    body = re.sub(r"//[^\n]*", "", body)
    return [w == "true" for w in re.findall(r"\b(true|false)\b", body)]


def parse_eef1(src):
    body = re.search(r"pub static EEF1.*?=\s*\[(.*?)\];", src, re.S).group(1)
    rows = re.findall(r"dg_ref:\s*(" + NUM + r"),\s*vol:\s*(" + NUM + r"),\s*lambda:\s*(" + NUM + r")", body)
    return [[float(a), float(b), float(c)] for a, b, c in rows]


def parse_residue_atoms(src, types):
    out = {}
    for three in THREE:
        body = re.search(r"static " + three + r"_ATOMS: &\[ResAtom\] = &\[(.*?)\];", src, re.S).group(1)
        atoms = []
        for m in re.finditer(r'atom!\("([^"]+)",\s*(\w+),\s*(' + NUM + r')(,\s*H)?\)', body):
            atoms.append({"name": m.group(1), "type": types.index(m.group(2)),
                          "charge": float(m.group(3)), "hydrophobic": 1 if m.group(4) else 0})
        out[three] = atoms
    return out


def parse_topology(src):
    body = re.search(r"pub static RESIDUE_TOPOLOGY.*?=\s*\[(.*?)\];", src, re.S).group(1)
    rows = re.findall(r"atoms:\s*(\w+)_ATOMS,\s*ca_idx:\s*(\d+),\s*n_chi:\s*(\d+)", body)
    return [{"atoms": a, "ca_idx": int(c), "n_chi": int(n)} for a, c, n in rows]


def parse_rotamers(src):
    rot = {}
    for three in THREE:
        body = re.search(r"static ROT_" + three + r": &\[Rotamer\] = &\[(.*?)\];", src, re.S).group(1)
        rows = re.findall(r"Rotamer::new\(\s*(" + NUM + r"),\s*(" + NUM + r"),\s*(" + NUM + r"),\s*("
                          + NUM + r"),\s*(" + NUM + r")\)", body)
        rot[three] = [[float(v) for v in r] for r in rows]
    order = re.search(r"pub static ROTAMER_LIB.*?=\s*\[(.*?)\];", src, re.S).group(1)
    names = re.findall(r"ROT_(\w+)", order)
    return [rot[n] for n in names]


def parse_bonddefs(src):
    defs = {}
    for three in THREE:
        body = re.search(r"static BD_" + three + r": &\[BondDef\] = &\[(.*?)\];", src, re.S).group(1)
        body = re.sub(r"//[^\n]*", "", body)
        rows = []
        for m in re.finditer(r"BondDef::(chi|fixed)\(\s*(\d+),\s*(\d+),\s*(\d+),\s*(" + NUM + r"),\s*("
                             + NUM + r"),\s*(" + NUM + r")\s*\)", body):
            kind, a, b, c, bl, ang, last = m.groups()
            if kind == "chi":
                rows.append({"ref": [int(a), int(b), int(c)], "bond": float(bl), "angle": float(ang),
                             "dihedral_fixed": 0.0, "chi_idx": int(last)})
            else:
                rows.append({"ref": [int(a), int(b), int(c)], "bond": float(bl), "angle": float(ang),
                             "dihedral_fixed": float(last), "chi_idx": 255})
        defs[three] = rows
    order = re.search(r"pub static SIDECHAIN_DEFS.*?=\s*\[(.*?)\];", src, re.S).group(1)
    names = re.findall(r"BD_(\w+)", order)
    return [defs[n] for n in names]


def parse_match_fn(src, fn):
    """Parse a `match self { A | B => v, ... _ => d }` residue-level table."""
    body = re.search(r"pub fn " + fn + r"\(self\) -> f32 \{\s*match self \{(.*?)\n\s*\}\s*\n\s*\}", src, re.S).group(1)
    default = None
    val = {}
    for m in re.finditer(r"([\w:| ]+?)\s*=>\s*(" + NUM + r")", body):
        lhs, v = m.group(1).strip(), float(m.group(2))
        if lhs == "_":
            default = v
            continue
        for name in re.findall(r"AminoAcid::(\w+)", lhs):
            val[name] = v
    return [val.get(n, default) for n in AA_NAMES]


def parse_hydrophobic(src):
    body = re.search(r"pub fn is_hydrophobic\(self\) -> bool \{(.*?)\n    \}", src, re.S).group(1)
    names = set(re.findall(r"AminoAcid::(\w+)", body))
    return [1 if n in names else 0 for n in AA_NAMES]


def parse_consts(src, names):
    out = {}
    for n in names:
        m = re.search(r"const " + n + r":\s*\w+\s*=\s*(" + NUM + r")", src)
        out[n] = float(m.group(1))
    return out


def main():
    amber = read("src/amber.rs")
    rot = read("src/rotamer.rs")
    atom = read("src/atom.rs")
    energy = read("src/energy.rs")
    diffusion = read("src/diffusion.rs")
    allatom = read("src/allatom.rs")
    solv = read("src/solvation.rs")

    types = parse_atom_types(amber)
    enum_body = re.search(r"pub enum AminoAcid \{(.*?)\}", atom, re.S).group(1)
    aa_order = re.findall(r"^\s*(\w+)", enum_body, re.M)
    assert aa_order == AA_NAMES, aa_order

    residues = parse_residue_atoms(amber, types)
    topo = parse_topology(amber)
    assert [t["atoms"] for t in topo] == THREE

    out = {
        "source": "reference src/{amber,rotamer,atom,energy,diffusion,allatom,solvation}.rs (parsed as text)",
        "amino_acids": AA_NAMES,
        "atom_types": types,
        "amber_nb": parse_amber_nb(amber),
        "hbond_donor": parse_bool_table(amber, "HBOND_DONOR"),
        "hbond_acceptor": parse_bool_table(amber, "HBOND_ACCEPTOR"),
        "eef1": parse_eef1(amber),
        "residues": [{"atoms": residues[t["atoms"]], "ca_idx": t["ca_idx"], "n_chi": t["n_chi"]} for t in topo],
        "rotamers": parse_rotamers(rot),
        "sidechain_defs": parse_bonddefs(rot),
        "residue_level": {
            "charge": parse_match_fn(atom, "charge"),
            "lj_epsilon": parse_match_fn(atom, "lj_epsilon"),
            "lj_sigma": parse_match_fn(atom, "lj_sigma"),
            "hydrophobic": parse_hydrophobic(atom),
        },
        "energy_consts": parse_consts(energy, ["COULOMB_K", "CUTOFF_SQ", "MIN_R_SQ", "HYDRO_CUTOFF_SQ",
                                               "HYDRO_BONUS", "HB_R0", "HB_SIGMA", "HB_DEPTH", "HB_CUTOFF_SQ"]),
        "diffusion_consts": parse_consts(diffusion, [
            "AA_POPULATION", "GPU_STEPS", "CPU_STEPS", "TOP_K", "STEP", "NOISE_BASE", "T_HOT", "T_COLD",
            "MUTATION_P", "ROTAMER_MOVE_P", "BACKBONE_MOVE_P", "MAX_TORSION_DEG", "IFACE_CUTOFF_SQ",
            "INIT_RADIUS", "MAX_DISP", "RESTRAINT_K"]),
        "backbone_consts": parse_consts(allatom, ["N_CA_BOND", "CA_C_BOND", "C_O_BOND", "CA_CB_BOND"]),
        "solvation_consts": {"PI32": float(re.search(r"const PI32: f32 = (" + NUM + r")", solv.replace("_", "")).group(1)),
                             "SOLV_CUTOFF": float(re.search(r"SOLV_CUTOFF: f32 = (" + NUM + r")", solv).group(1))},
    }
    assert len(out["amber_nb"]) == 16 and len(out["eef1"]) == 16
    assert len(out["hbond_donor"]) == 16 and len(out["hbond_acceptor"]) == 16
    assert all(len(r) == 5 or len(r) == 0 for r in out["rotamers"])
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
