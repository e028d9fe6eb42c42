"""Exact MP2 gradient on the GPU (dE/dC, dE/deps, the energy of the same
pass) vs the CPU oracle and vs central finite differences of the GPU energy.

Tolerances: FP64 path 1e-10 of the largest element (different summation
order, FP64 throughout); orbital-rotation finite differences (step 1e-4)
1e-6 absolute on scaled-twin inputs.
"""
import numpy as np
import pytest
import scipy.linalg

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def twin(N, o, M, seed, nocc_beta=None):
    base = syn.make_inputs(N, o, M, seed=seed, nocc_beta=nocc_beta)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    return syn.make_inputs(N, o, M, seed=seed, sigma=sig, nocc_beta=nocc_beta)


@pytest.mark.parametrize("N,o,M,seed", [(24, 5, 60, 1), (29, 7, 61, 4), (70, 9, 150, 2)])
def test_restricted_fp64_gradient_vs_oracle(ctx, N, o, M, seed):
    inp = syn.make_inputs(N, o, M, seed=seed)
    a = inp.alpha
    ref = orc.restricted_gradient(inp.L, a.C, a.eps, o)
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    g = ctx.mp2_gradient(capi.RESTRICTED, capi.FP64)
    assert abs(g.energy["total"] - ref["E"]) <= 1e-12 * abs(ref["E"])
    assert np.max(np.abs(g.dC_a - ref["dC"])) <= 1e-10 * np.max(np.abs(ref["dC"]))
    assert np.max(np.abs(g.deps_a - ref["deps"])) <= 1e-10 * np.max(np.abs(ref["deps"]))


def test_restricted_fp64_orbital_gradient_fd(ctx):
    N, o, M = 48, 6, 120
    inp = twin(N, o, M, seed=8)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    g = ctx.mp2_gradient(capi.RESTRICTED, capi.FP64)
    kg = orc.orbital_gradient(a.C, g.dC_a, o)
    h = 1e-4
    for (ai, ii) in [(0, 0), (7, 3), (30, 5)]:
        K = np.zeros((N, N))
        K[o + ai, ii], K[ii, o + ai] = 1.0, -1.0
        ctx.set_orbitals(capi.ALPHA, a.C @ scipy.linalg.expm(-h * K), a.eps, o)
        ep = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
        ctx.set_orbitals(capi.ALPHA, a.C @ scipy.linalg.expm(h * K), a.eps, o)
        em = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
        fd = (ep - em) / (2 * h)
        assert abs(fd - kg[ai, ii]) <= 1e-6, (ai, ii, fd, kg[ai, ii])


# Mixed precision: the same derivatives from the tensor-core path (exact
# fixed-point amplitude pass, Gamma GEMM with round-to-nearest promotion).
# Tolerance on scaled-twin inputs: max |d dE/dC|, max |d dE/deps| <= 1e-6,
# energy <= 1 micro-Eh.
@pytest.mark.parametrize("N,o,M,seed", [(60, 8, 150, 3), (131, 14, 300, 5), (257, 21, 640, 6)])
def test_restricted_mixed_gradient_vs_fp64(ctx, N, o, M, seed):
    inp = twin(N, o, M, seed=seed)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    g64 = ctx.mp2_gradient(capi.RESTRICTED, capi.FP64)
    g3 = ctx.mp2_gradient(capi.RESTRICTED, capi.FP16X3)
    assert abs(g3.energy["total"] - g64.energy["total"]) <= 1e-6
    assert np.max(np.abs(g3.dC_a - g64.dC_a)) <= 1e-6, np.max(np.abs(g3.dC_a - g64.dC_a))
    assert np.max(np.abs(g3.deps_a - g64.deps_a)) <= 1e-6, np.max(np.abs(g3.deps_a - g64.deps_a))


def test_restricted_mixed_gradient_vs_oracle(ctx):
    N, o, M = 48, 6, 120
    inp = twin(N, o, M, seed=8)
    a = inp.alpha
    ref = orc.restricted_gradient(inp.L, a.C, a.eps, o)
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    g = ctx.mp2_gradient(capi.RESTRICTED, capi.FP16X3)
    assert abs(g.energy["total"] - ref["E"]) <= 1e-6
    assert np.max(np.abs(g.dC_a - ref["dC"])) <= 1e-6
    assert np.max(np.abs(g.deps_a - ref["deps"])) <= 1e-6
