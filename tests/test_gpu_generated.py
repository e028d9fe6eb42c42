"""Cholesky vectors generated on the device (mshqc_cd_gen_vectors) against
the same recipe drawn by the numpy restatement and uploaded: energies and
gradients agree to 1e-12 relative (the generator's log/cos may differ from
numpy's by an ulp), with the vectors generated in one chunk or in chunks of
7 (the chunked dE/dC_occ accumulation)."""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

N, O, M, SEED = 44, 6, 101, 77


@pytest.fixture(scope="module")
def inputs():
    orb = syn.make_orbitals(N, O, 5)
    sigma = syn.twin_sigma(N, O, M, orb.eps)
    return orb, sigma, syn.make_vectors_philox(N, M, SEED, sigma)


def run(setup, orb, precision):
    with capi.Context(0) as c:
        setup(c)
        c.set_orbitals(capi.ALPHA, orb.C, orb.eps, O)
        e = c.mp2_energy(capi.RESTRICTED, precision)
        g = c.mp2_gradient(capi.RESTRICTED, precision)
    return e, g


@pytest.mark.parametrize("chunk", [None, "7"])
def test_generated_matches_uploaded(inputs, monkeypatch, chunk):
    orb, sigma, L = inputs
    if chunk:
        monkeypatch.setenv("MSHQC_CD_GEN_CHUNK", chunk)
    e_up, g_up = run(lambda c: c.set_vectors(L), orb, capi.FP64)
    e_gen, g_gen = run(lambda c: c.gen_vectors(N, M, SEED, sigma), orb, capi.FP64)
    assert abs(e_gen["total"] - e_up["total"]) <= 1e-12 * abs(e_up["total"])
    assert abs(g_gen.energy["total"] - g_up.energy["total"]) <= 1e-12 * abs(e_up["total"])
    assert np.max(np.abs(g_gen.dC_a - g_up.dC_a)) <= 1e-12 * np.max(np.abs(g_up.dC_a))
    assert np.max(np.abs(g_gen.deps_a - g_up.deps_a)) <= 1e-12 * np.max(np.abs(g_up.deps_a))


def test_generated_mixed_close_to_fp64(inputs):
    orb, sigma, _ = inputs
    _, g64 = run(lambda c: c.gen_vectors(N, M, SEED, sigma), orb, capi.FP64)
    _, g3 = run(lambda c: c.gen_vectors(N, M, SEED, sigma), orb, capi.FP16X3)
    assert abs(g3.energy["total"] - g64.energy["total"]) <= 1e-6
    assert np.max(np.abs(g3.dC_a - g64.dC_a)) <= 1e-6


def test_omp2_refuses_generated_vectors(inputs):
    orb, sigma, _ = inputs
    with capi.Context(0) as c:
        c.gen_vectors(N, M, SEED, sigma)
        c.set_orbitals(capi.ALPHA, orb.C, orb.eps, O)
        c.set_orbitals(capi.BETA, orb.C, orb.eps, O)
        c.set_core_hamiltonian(np.eye(N))
        with pytest.raises(capi.CDError) as err:
            c.omp2_pieces()
        assert err.value.code == capi.ERR_UNSUPPORTED
