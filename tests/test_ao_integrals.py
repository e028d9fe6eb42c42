"""Host AO integral engine (mshqc_ao_*, mshqc_b200/ao.py), no GPU needed.

Pinned by libint2's own Hartree-Fock tests as vendored in the reference
(tests/golden/h2o_basis_sets.json, written by make_basis_fixtures.py): the RHF
energy of H2O in STO-3G (-74.942080057698 Eh, tolerance 1e-11) and of rotated
H2O in aug-cc-pVDZ (-76.003354058454 Eh, 5e-12; d shells as solid
harmonics, diffuse functions) from S, T, V and the ERI tensor of this engine
with a plain DIIS RHF here.  Plus invariants: orthogonal solid harmonics
within a shell with the norm of its x^l component, the reference's
coefficient normalization, symmetric one-electron matrices, the eight-fold ERI
symmetry, the ERI diagonal and columns against the full tensor, translation
invariance, and the reference's own RHF + CD-RMP2 (oracle/_ref) on the
configuration-1 molecule against the RHF energy here."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

from mshqc_b200 import ao, capi

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "h2o_basis_sets.json")))


def setup_case(name, shift=(0.0, 0.0, 0.0)):
    case = FIX["cases"][name]
    mol = ao.Molecule.from_angstrom(case["atoms"], case["angstrom_to_bohr"])
    mol.xyz = mol.xyz + np.asarray(shift)
    bs = ao.BasisSet.from_g94(FIX["basis"][case["basis"]]["g94"], mol)
    return case, mol, ao.IntegralEngine(mol, bs)


def rhf(S, H, eri, nocc, enuc, conv=1e-13, maxit=300):
    """Closed-shell SCF with DIIS (test infrastructure)."""
    s, U = np.linalg.eigh(S)
    X = U @ np.diag(s ** -0.5) @ U.T
    e, C = np.linalg.eigh(X.T @ H @ X)
    C = X @ C
    D = C[:, :nocc] @ C[:, :nocc].T
    E_old, Fs, errs = 0.0, [], []
    for it in range(maxit):
        F = H + 2 * np.einsum("pqrs,rs->pq", eri, D) - np.einsum("prqs,rs->pq", eri, D)
        E = float(np.sum(D * (H + F))) + enuc
        Fs = (Fs + [F])[-8:]
        errs = (errs + [F @ D @ S - S @ D @ F])[-8:]
        n = len(Fs)
        B = -np.ones((n + 1, n + 1))
        B[n, n] = 0.0
        for i in range(n):
            for j in range(n):
                B[i, j] = np.sum(errs[i] * errs[j])
        rhs = np.zeros(n + 1)
        rhs[n] = -1.0
        c = np.linalg.solve(B, rhs)[:n]
        e, C = np.linalg.eigh(X.T @ sum(ci * Fi for ci, Fi in zip(c, Fs)) @ X)
        C = X @ C
        Dn = C[:, :nocc] @ C[:, :nocc].T
        if abs(E - E_old) < conv and np.max(np.abs(Dn - D)) < 1e-10:
            return E, C, e
        D, E_old = Dn, E
    raise RuntimeError("SCF did not converge")


def scf_energy(eng, mol):
    S, T, V = eng.compute_overlap(), eng.compute_kinetic(), eng.compute_nuclear()
    return rhf(S, T + V, eng.compute_eri(), mol.n_electrons() // 2, eng.nuclear_repulsion_energy())


@pytest.mark.parametrize("name", ["libint_h2o_sto3g", "libint_h2o_rotated_augccpvdz"])
def test_rhf_energy_matches_libint_golden(name):
    case, mol, eng = setup_case(name)
    E, _, _ = scf_energy(eng, mol)
    assert abs(E - case["e_rhf"]) <= case["tolerance"], (E, case["e_rhf"])


@pytest.mark.parametrize("l", [1, 2, 3, 4])
def test_pure_shell_components_orthogonal_with_the_norm_of_x_l(l):
    """Solid harmonics of one shell are orthogonal and each has the norm of
    the shell's x^l Cartesian component (the convention of the Cartesian ->
    solid-harmonic transform the reference gets from libint2)."""
    mol = ao.Molecule(np.array([0.0]), np.zeros((1, 3)), ["X"])
    e = np.array([3.1, 0.9, 0.21])
    c = np.array([0.3, 0.5, 0.4])
    pure = ao.BasisSet({"X": [(l, e, c)]}, mol, spherical=True)
    cart = ao.BasisSet({"X": [(l, e, c)]}, mol, spherical=False)
    S = ao.IntegralEngine(mol, pure).compute_overlap()
    xl = ao.IntegralEngine(mol, cart).compute_overlap()[0, 0]
    assert S.shape == (2 * l + 1, 2 * l + 1)
    assert np.max(np.abs(S - xl * np.eye(2 * l + 1))) < 1e-13 * xl


def test_normalization_follows_the_reference_shell():
    """mshqc_ao_normalize_shell is the reference's Shell::normalize
    (src/core/basis.cc:82-104): coefficients times the x^l primitive norms,
    then divided by sqrt(sum c_i c_j (2 sqrt(a_i a_j)/(a_i + a_j))^(l+3/2))
    of those products -- which leaves a one-primitive shell's coefficient at
    1 on the raw Gaussian (the reference hands these to libint2 without
    renormalization, so its basis functions are not unit-norm in general;
    energies do not depend on that scaling)."""
    for l in (0, 1, 2):
        assert abs(ao.normalize_shell(l, [0.727], [1.0])[0] - 1.0) < 1e-15
    e, c, l = np.array([13.01, 1.962, 0.4446]), np.array([0.019685, 0.137977, 0.478148]), 0
    n = np.array([(2 * a / np.pi) ** 0.75 * (4 * a) ** (l / 2) for a in e])
    cc = c * n
    r = (2 * np.sqrt(np.outer(e, e)) / np.add.outer(e, e)) ** (l + 1.5)
    expect = cc / np.sqrt(cc @ r @ cc)
    assert np.max(np.abs(ao.normalize_shell(l, e, c) - expect)) < 1e-15


def test_symmetries_diagonal_and_columns():
    _, mol, eng = setup_case("mshqc_h2o_ccpvdz")
    N = eng.nbasis
    assert N == 24
    for M in (eng.compute_overlap(), eng.compute_kinetic(), eng.compute_nuclear()):
        assert np.max(np.abs(M - M.T)) < 1e-14
    g = eng.compute_eri()
    for perm in [(1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1)]:
        assert np.max(np.abs(g - g.transpose(perm))) < 1e-14
    gm = g.reshape(N * N, N * N)
    assert np.max(np.abs(eng.compute_eri_diagonal() - np.diag(gm))) < 1e-14
    for piv in (0, 37, N * N - 1):
        assert np.max(np.abs(eng.compute_eri_column(piv) - gm[:, piv])) < 1e-14
    # positive semidefinite ERI matrix (the Cholesky decomposition needs it)
    assert np.linalg.eigvalsh(gm).min() > -1e-12


def test_translation_invariance():
    _, mol0, e0 = setup_case("mshqc_h2o_ccpvdz")
    _, mol1, e1 = setup_case("mshqc_h2o_ccpvdz", shift=(0.7, -1.3, 2.1))
    for f in ("compute_overlap", "compute_kinetic", "compute_nuclear"):
        assert np.max(np.abs(getattr(e0, f)() - getattr(e1, f)())) < 1e-12
    assert np.max(np.abs(e0.compute_eri() - e1.compute_eri())) < 1e-12
    assert abs(e0.nuclear_repulsion_energy() - e1.nuclear_repulsion_energy()) < 1e-12


def test_reference_rhf_and_cdrmp2_on_these_integrals():
    """Configuration 1 on the CPU: the reference's RHF (src/scf/rhf.cc) on
    these integrals agrees with the RHF here; its CholeskyRMP2 gives a
    finite correlation energy of the expected size."""
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    _, mol, eng = setup_case("mshqc_h2o_ccpvdz")
    S, T, V, g = eng.compute_overlap(), eng.compute_kinetic(), eng.compute_nuclear(), eng.compute_eri()
    E, _, _ = rhf(S, T + V, g, 5, eng.nuclear_repulsion_energy())
    r = ref.rhf_cdrmp2(mol.Z, mol.xyz, S, T, V, g)
    assert r["converged"] and r["nocc"] == 5
    assert abs(r["e_scf"] - E) < 1e-9
    assert -0.25 < r["e_corr"] < -0.15
    assert 24 < r["n_vectors"] <= 300


def test_ao_symbols_exported():
    lib = ctypes.CDLL(capi.LIB_PATH)
    txt = open(os.path.join(os.path.dirname(HERE), "include", "mshqc_ao.h")).read()
    names = sorted(set(re.findall(r"MSHQC_AO_API\s+[\w\s\*]*?\b(mshqc_ao_\w+)\s*\(", txt)))
    assert len(names) >= 7
    assert not [n for n in names if not hasattr(lib, n)]
