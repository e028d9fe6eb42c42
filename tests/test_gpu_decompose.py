"""Pivoted Cholesky decomposition of the ERI matrix on the GPU
(mshqc_cd_cholesky_decompose) against the reference's CholeskyERI::decompose
(golden fixture) and the oracle; the decomposed vectors then drive the MP2
energy like uploaded ones.  Tolerance 1e-12 absolute on the vectors (same
operations, the reference build may fuse multiply-adds)."""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc

pytestmark = pytest.mark.gpu


def eri_from_vectors(Lv, N):
    """A symmetric positive semidefinite ERI-like tensor (ij|kl) = sum_Q
    L^Q_ij L^Q_kl from symmetric vectors."""
    E = Lv.T @ Lv
    return E.reshape(N, N, N, N)


def test_decompose_vs_reference(golden):
    g = golden("cholesky_decompose_n8")
    with capi.Context(0) as c:
        Lv = c.cholesky_decompose(g["eri"], float(g["threshold"]))
        assert c.decompose_converged
    assert Lv.shape == g["L"].shape
    assert np.max(np.abs(Lv - g["L"])) <= 1e-12


def test_decompose_vs_oracle_and_energy():
    N, o, M = 12, 3, 40
    inp = syn.make_inputs(N, o, M, seed=4)
    eri = eri_from_vectors(inp.L, N)
    ref = orc.cholesky_decompose(eri, 1e-8)
    with capi.Context(0) as c:
        Lv = c.cholesky_decompose(eri, 1e-8)
        assert Lv.shape == ref.shape
        assert np.max(np.abs(Lv - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))
        c.set_orbitals(capi.ALPHA, inp.alpha.C, inp.alpha.eps, o)
        e_dec = c.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
        c.set_vectors(Lv)
        c.set_orbitals(capi.ALPHA, inp.alpha.C, inp.alpha.eps, o)
        e_up = c.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
    assert e_dec == e_up
    # the decomposition reproduces the ERIs to the threshold
    n2 = N * N
    assert np.max(np.abs(Lv.T @ Lv - eri.reshape(n2, n2))) < 10 * 1e-8 * np.max(np.abs(eri))


def test_decompose_below_threshold_gives_no_vectors():
    eri = np.zeros((4, 4, 4, 4))
    with capi.Context(0) as c:
        Lv = c.cholesky_decompose(eri, 1e-6)
    assert Lv.shape == (0, 16)
