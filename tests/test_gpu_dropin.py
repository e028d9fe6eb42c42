"""The reference's own C++ classes on this library: a program written against
the reference's public API (Molecule, BasisSet, IntegralEngine, RHF,
CholeskyERI, CholeskyRMP2, CholeskyUMP2, CholeskyOMP2; include/mshqc/*.h),
linked with the reference's molecule/basis/RHF sources and with the drop-in
library (mshqc_b200/dropin) in place of its integral, Cholesky and MP2
sources (tests/dropin, built where the reference is present), runs H2O in
cc-pVDZ in a child process.  Against the reference's own CholeskyRMP2
(oracle/_ref) on the vectors and orbitals the program produced: E_corr to
1e-9 Eh and the stored t2 (CholeskyRMP2Result::t2) to 1e-12 of its largest
element; the closed-shell UMP2 split ss_aa = ss_bb and total = RMP2; the OMP2
loop runs."""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from oracle import ref

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CHECK = os.path.join(HERE, "dropin", "_build", "libdropin_check.so")

CHILD = r'''
import ctypes, json, sys
import numpy as np
lib = ctypes.CDLL(sys.argv[1])
lib.dropin_last_error.restype = ctypes.c_char_p
d = json.load(open(sys.argv[2]))
atoms = d["atoms"]
Z = (ctypes.c_int * len(atoms))(*[{"H": 1, "O": 8}[a[0]] for a in atoms])
xyz = np.ascontiguousarray([[a[1], a[2], a[3]] for a in atoms], dtype=np.float64)
N, maxv = 24, 600
out = np.zeros(14); C = np.zeros(N * N); eps = np.zeros(N); L = np.zeros(maxv * N * N); t2 = np.zeros(5 * 5 * 19 * 19)
p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
rc = lib.dropin_closed_shell(len(atoms), Z, p(xyz), sys.argv[3].encode(), b"cc-pvdz", ctypes.c_double(1e-6),
                             p(out), p(C), p(eps), p(L), maxv, p(t2))
if rc != 0:
    print("ERROR", lib.dropin_last_error().decode()); sys.exit(1)
M = int(out[2])
np.savez(sys.argv[4], out=out, C=C.reshape(N, N, order="F"), eps=eps, L=L[:M * N * N].reshape(M, N * N),
         t2=t2.reshape(5, 5, 19, 19, order="F"))
'''


@pytest.mark.skipif(not (os.path.exists(CHECK) and ref.available()), reason="drop-in check or oracle not built")
def test_reference_api_program_on_the_gpu(tmp_path):
    fix = json.load(open(os.path.join(HERE, "golden", "h2o_basis_sets.json")))
    case = fix["cases"]["mshqc_h2o_ccpvdz"]
    bdir = tmp_path / "basis"
    bdir.mkdir()
    (bdir / "cc-pvdz.gbs").write_text("spherical\n\n" + fix["basis"]["cc-pvdz"]["g94"])
    cfile = tmp_path / "case.json"
    cfile.write_text(json.dumps(case))
    res = tmp_path / "out.npz"
    r = subprocess.run([sys.executable, "-c", CHILD, CHECK, str(cfile), str(bdir), str(res)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    z = np.load(res)
    out = z["out"]
    o = int(out[3])
    orc = ref.rmp2(z["L"], z["C"], z["eps"], o, want_t2=True)
    print(f"\ndrop-in H2O/cc-pVDZ: E_SCF {out[0]:.12f}, RMP2 {out[1]:.12f} ({int(out[2])} vectors), reference "
          f"CholeskyRMP2 on the same vectors {orc['e_corr']:.12f}; UMP2 {out[5]:.10f} {out[6]:.10f} "
          f"{out[7]:.10f}; OMP2 {out[9]:.10f} after {int(out[10])} iterations")
    assert abs(out[1] - orc["e_corr"]) <= 1e-9
    assert np.max(np.abs(z["t2"] - orc["t2"])) <= 1e-12 * np.max(np.abs(orc["t2"]))
    assert abs(out[5] - out[6]) <= 1e-12 and abs(out[8] - out[1]) <= 1e-10
    assert int(out[10]) >= 1 and np.isfinite(out[9])
