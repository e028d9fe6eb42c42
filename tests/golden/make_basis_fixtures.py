"""Writes tests/golden/h2o_basis_sets.json: the H and O entries of three
Gaussian94 basis files and two H2O geometries with their golden energies,
read from the reference source tree (test infrastructure, run where the
reference is present; the JSON travels with the repository):

* cc-pVDZ   from the reference's data/basis/cc-pvdz.gbs (the H2O case run by
            the reference, O at (0,0,0), H at (+-0.757, 0.587, 0) Angstrom);
* STO-3G and aug-cc-pVDZ from the basis library of the libint2 sources
            vendored in the reference (include/libint2/evaleev/...), with
            libint2's own Hartree-Fock tests: tests/hartree-fock/h2o.xyz in
            STO-3G must give E_RHF = -74.942080057698 Eh (tolerance 1e-11,
            hartree-fock-validate.py), h2o_rotated.xyz in aug-cc-pVDZ
            -76.003354058454 Eh (5e-12, hartree-fock++-validate.py); both
            convert Angstrom with the CODATA 2010 Bohr radius 0.52917721092.

    python tests/golden/make_basis_fixtures.py [REFERENCE_TREE]
"""
import glob
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def element_block(text, el):
    """The lines of one element's entry of a Gaussian94 file."""
    lines = text.splitlines()
    out, on = [], False
    for ln in lines:
        parts = ln.split()
        if not on and len(parts) == 2 and parts[0] == el and parts[1] == "0":
            on = True
            out.append(ln.strip())
            continue
        if on:
            out.append(ln.rstrip())
            if ln.startswith("****"):
                break
    return "\n".join(out)


def read_xyz(path):
    lines = open(path).read().splitlines()
    n = int(lines[0].split()[0])
    atoms = []
    for ln in lines[2:2 + n]:
        p = ln.split()
        atoms.append([p[0], float(p[1]), float(p[2]), float(p[3])])
    return atoms


def golden(path, pattern):
    m = re.search(pattern, open(path).read())
    return float(m.group(1))


def main(ref):
    libint = glob.glob(os.path.join(ref, "include", "libint2", "evaleev", "libint-*", "*"))
    libint = [d for d in libint if os.path.isdir(os.path.join(d, "lib", "basis"))][0]
    hf = os.path.join(libint, "tests", "hartree-fock")
    lb = os.path.join(libint, "lib", "basis")
    # libint2 builds aug-cc-pVDZ from its cc-pvdz.g94 plus the diffuse shells
    # of augmentation-cc-pvdz.g94, appended per atom
    files = {
        "cc-pvdz": [os.path.join(ref, "data", "basis", "cc-pvdz.gbs")],
        "sto-3g": [os.path.join(lb, "sto-3g.g94")],
        "aug-cc-pvdz": [os.path.join(lb, "cc-pvdz.g94"), os.path.join(lb, "augmentation-cc-pvdz.g94")],
    }
    out = {"basis": {}, "cases": {}}
    for name, paths in files.items():
        texts = [open(pth).read() for pth in paths]
        blocks = []
        for el in ("H", "O"):
            parts = [element_block(t, el).splitlines() for t in texts]
            # one entry: the header of the first, the shells of all, one terminator
            merged = [parts[0][0]] + [ln for pt in parts for ln in pt[1:] if not ln.startswith("****")] + ["****"]
            blocks.append("\n".join(merged))
        out["basis"][name] = {"source": [os.path.relpath(pth, ref) for pth in paths], "spherical": True,
                              "g94": "****\n" + "\n".join(blocks) + "\n"}
    bohr2010 = 0.52917721092
    out["cases"]["libint_h2o_sto3g"] = {
        "basis": "sto-3g", "atoms": read_xyz(os.path.join(hf, "h2o.xyz")), "angstrom_to_bohr": 1.0 / bohr2010,
        "e_rhf": golden(os.path.join(hf, "hartree-fock-validate.py"), r"eref\s*=\s*([-\d.eE+]+)"),
        "tolerance": 1e-11, "source": "libint2 tests/hartree-fock (hartree-fock.cc, h2o.xyz)"}
    out["cases"]["libint_h2o_rotated_augccpvdz"] = {
        "basis": "aug-cc-pvdz", "atoms": read_xyz(os.path.join(hf, "h2o_rotated.xyz")),
        "angstrom_to_bohr": 1.0 / bohr2010,
        "e_rhf": golden(os.path.join(hf, "hartree-fock++-validate.py"), r"eref\s*=\s*\[\s*([-\d.eE+]+)"),
        "tolerance": 5e-12, "source": "libint2 tests/hartree-fock (hartree-fock++.cc, h2o_rotated.xyz)"}
    out["cases"]["mshqc_h2o_ccpvdz"] = {
        "basis": "cc-pvdz", "atoms": [["O", 0.0, 0.0, 0.0], ["H", 0.757, 0.587, 0.0], ["H", -0.757, 0.587, 0.0]],
        "angstrom_to_bohr": 1.88972612457, "e_rhf": None, "tolerance": None,
        "source": "benchmark configuration 1 (H2O, cc-pVDZ from data/basis of the reference)"}
    dst = os.path.join(HERE, "h2o_basis_sets.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MSHQC_REFERENCE", "/root/reference"))
