"""Benchmark configuration 1: H2O (O at (0,0,0), H at (+-0.757, 0.587, 0)
Angstrom), cc-pVDZ (24 functions, 5 occupied, frozen core off), Cholesky
threshold 1e-6 on the AO ERI matrix, RHF converged to 1e-12 in the energy.

The AO integrals come from this library's host engine (libint2, which the
reference uses, is absent; the engine itself is pinned by libint2's own
H2O golden energies in tests/test_ao_integrals.py), so parity is stated given
identical integrals: the reference's own RHF and CholeskyRMP2 (constructor
1, decomposing the ERI tensor itself; oracle/_ref) against the GPU
decomposition (mshqc_cd_cholesky_decompose, first-argmax pivots) and the GPU
CD-RMP2 energy with the reference's RHF orbitals: the same number of
vectors, FP64 energy to 1e-9 Eh, mixed precision to 1 uEh."""
import json
import os

import numpy as np
import pytest

from mshqc_b200 import ao, capi
from oracle import ref

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_config1_h2o_ccpvdz_against_reference_cdrmp2():
    fix = json.load(open(os.path.join(HERE, "golden", "h2o_basis_sets.json")))
    case = fix["cases"]["mshqc_h2o_ccpvdz"]
    mol = ao.Molecule.from_angstrom(case["atoms"], case["angstrom_to_bohr"])
    bs = ao.BasisSet.from_g94(fix["basis"]["cc-pvdz"]["g94"], mol)
    eng = ao.IntegralEngine(mol, bs)
    S, T, V, g = eng.compute_overlap(), eng.compute_kinetic(), eng.compute_nuclear(), eng.compute_eri()
    r = ref.rhf_cdrmp2(mol.Z, mol.xyz, S, T, V, g, chol_thr=1e-6)
    assert r["converged"]
    N, o = eng.nbasis, r["nocc"]
    with capi.Context(0) as ctx:
        L = ctx.cholesky_decompose(g, 1e-6)
        conv = ctx.decompose_converged
        ctx.set_orbitals(capi.ALPHA, r["C"], r["eps"], o)
        e64 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
        e3 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)["total"]
    M = L.shape[0]
    print(f"\nconfig 1: N={N} o={o}; reference E_SCF {r['e_scf']:.12f} E_corr {r['e_corr']:.12f} "
          f"({r['n_vectors']} vectors); GPU {M} vectors, FP64 error {abs(e64 - r['e_corr']):.2e} Eh, "
          f"mixed error {abs(e3 - r['e_corr']) * 1e6:.4f} uEh")
    assert conv
    assert M == r["n_vectors"]
    assert abs(e64 - r["e_corr"]) <= 1e-9
    assert abs(e3 - r["e_corr"]) <= 1e-6


def test_config1_integral_direct_decomposition():
    """The integral-direct decomposition (mshqc_cd_cholesky_direct: ERI
    diagonal and columns from the host engine, the vectors on the GPU, the
    reference's DirectCholesky of src/integrals/cholesky_direct.cc) against the
    decomposition of the full ERI tensor.  The two need not pick the same
    pivots: H2O's diagonal is full of ties ((mn|mn) = (nm|nm) always, and the
    two H atoms are equivalent; 166 of the 182 steps choose among near-equal
    maxima), so the first argmax depends on the last bit of each diagonal
    update and the vectors may come out in another order or basis.  What they
    represent must agree: the same number of vectors, each set reproducing
    the ERI matrix within the stopping threshold (the residual is positive
    semidefinite, so its largest entry is its largest diagonal element), and
    the same CD-RMP2 energy to 1e-10 Eh."""
    fix = json.load(open(os.path.join(HERE, "golden", "h2o_basis_sets.json")))
    case = fix["cases"]["mshqc_h2o_ccpvdz"]
    mol = ao.Molecule.from_angstrom(case["atoms"], case["angstrom_to_bohr"])
    bs = ao.BasisSet.from_g94(fix["basis"]["cc-pvdz"]["g94"], mol)
    eng = ao.IntegralEngine(mol, bs)
    g = eng.compute_eri()
    S, T, V = eng.compute_overlap(), eng.compute_kinetic(), eng.compute_nuclear()
    s, U = np.linalg.eigh(S)
    X = U @ np.diag(s ** -0.5) @ U.T
    e, C = np.linalg.eigh(X.T @ (T + V) @ X)
    C = X @ C                                     # core-Hamiltonian orbitals suffice here
    with capi.Context(0) as ctx:
        Lf = ctx.cholesky_decompose(g, 1e-6)
        ctx.set_orbitals(capi.ALPHA, C, e, 5)
        ef = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
        Ld = ctx.cholesky_direct(bs, 1e-6)
        ctx.set_orbitals(capi.ALPHA, C, e, 5)
        ed = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
    G = g.reshape(Lf.shape[1], Lf.shape[1])
    res_d = np.max(np.abs(G - Ld.T @ Ld))
    res_f = np.max(np.abs(G - Lf.T @ Lf))
    print(f"\nintegral-direct: {Ld.shape[0]} vectors (full tensor: {Lf.shape[0]}), max |G - L^T L| "
          f"{res_d:.2e} ({res_f:.2e}), energy difference {abs(ed - ef):.2e} Eh")
    assert Ld.shape == Lf.shape
    assert res_d <= 1e-6 and res_f <= 1e-6
    assert abs(ed - ef) <= 1e-10
