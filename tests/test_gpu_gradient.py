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
    ctx.set_orbitals(capi.ALPHA, a.C, a.eps, o)      # mixed transform (int8 slices), not the FP64 one
    g3 = ctx.mp2_gradient(capi.RESTRICTED, capi.FP16X3)
    assert abs(g3.energy["total"] - g64.energy["total"]) <= 1e-6
    assert np.max(np.abs(g3.dC_a - g64.dC_a)) <= 1e-6, np.max(np.abs(g3.dC_a - g64.dC_a))
    assert np.max(np.abs(g3.deps_a - g64.deps_a)) <= 1e-6, np.max(np.abs(g3.deps_a - g64.deps_a))


def test_gradient_torch_defaults_to_context_gpu(ctx):
    import torch
    inp = twin(40, 5, 90, seed=12)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, 5)
    g = ctx.mp2_gradient(capi.RESTRICTED, capi.FP64)
    gt = ctx.mp2_gradient_torch(capi.RESTRICTED, capi.FP64)
    assert gt.dC_a.is_cuda and gt.dC_a.device.index == ctx.device
    assert np.array_equal(gt.dC_a.cpu().numpy(), g.dC_a)
    # dE/deps sums per-block partials in launch order: equal to rounding
    assert np.allclose(gt.deps_a.cpu().numpy(), g.deps_a, rtol=1e-12, atol=1e-15)


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


# ---------------------------------------------------------------------------
# Unrestricted (CD-UMP2 energy, the OMP2 step): dE/dC and dE/deps per spin.
# ---------------------------------------------------------------------------
def set_unrestricted(ctx, inp):
    A, B = inp.alpha, inp.beta
    ctx.set_vectors(inp.L)
    ctx.set_orbitals(capi.ALPHA, A.C, A.eps, A.nocc)
    ctx.set_orbitals(capi.BETA, B.C, B.eps, B.nocc)


def maxrel(x, ref):
    return np.max(np.abs(x - ref)) / np.max(np.abs(ref))


@pytest.mark.parametrize("N,oa,ob,M,seed", [(26, 6, 5, 70, 1), (45, 7, 4, 101, 2), (80, 9, 8, 190, 3)])
def test_unrestricted_fp64_gradient_vs_oracle(ctx, N, oa, ob, M, seed):
    inp = syn.make_inputs(N, oa, M, seed=seed, nocc_beta=ob)
    A, B = inp.alpha, inp.beta
    ref = orc.unrestricted_gradient(inp.L, A.C, B.C, A.eps, B.eps, oa, ob)
    set_unrestricted(ctx, inp)
    g = ctx.mp2_gradient(capi.UNRESTRICTED, capi.FP64)
    for key in ("ss_aa", "ss_bb", "os"):
        assert abs(g.energy[key] - ref[key]) <= 1e-12 * abs(ref[key]), key
    assert abs(g.energy["total"] - ref["E"]) <= 1e-12 * abs(ref["E"])
    assert maxrel(g.dC_a, ref["dC_a"]) <= 1e-10
    assert maxrel(g.dC_b, ref["dC_b"]) <= 1e-10
    assert maxrel(g.deps_a, ref["deps_a"]) <= 1e-10
    assert maxrel(g.deps_b, ref["deps_b"]) <= 1e-10


def test_unrestricted_energy_matches_energy_entry(ctx):
    inp = twin(64, 8, 160, seed=5, nocc_beta=6)
    set_unrestricted(ctx, inp)
    e = ctx.mp2_energy(capi.UNRESTRICTED, capi.FP64)
    g = ctx.mp2_gradient(capi.UNRESTRICTED, capi.FP64)
    for key in ("ss_aa", "ss_bb", "os", "total"):
        assert abs(g.energy[key] - e[key]) <= 1e-12 * abs(e[key]) + 1e-15, key


def test_unrestricted_closed_shell_limit(ctx):
    """C_a = C_b, equal occupations: dE/dC_a + dE/dC_b equals the restricted
    dE/dC (FP64 and mixed)."""
    N, o, M = 70, 8, 170
    inp = twin(N, o, M, seed=9)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    r = ctx.mp2_gradient(capi.RESTRICTED, capi.FP64)
    ctx.set_orbitals(capi.BETA, a.C, a.eps, o)
    for prec, tol in ((capi.FP64, 1e-10), (capi.FP16X3, 1e-6)):
        u = ctx.mp2_gradient(capi.UNRESTRICTED, prec)
        scale = 1.0 if prec == capi.FP16X3 else np.max(np.abs(r.dC_a))
        assert abs(u.energy["total"] - r.energy["total"]) <= (1e-12 if prec == capi.FP64 else 1e-6)
        assert np.max(np.abs(u.dC_a + u.dC_b - r.dC_a)) <= tol * scale
        assert np.max(np.abs(u.deps_a + u.deps_b - r.deps_a)) <= tol * (1.0 if prec == capi.FP16X3
                                                                          else np.max(np.abs(r.deps_a)))


def test_unrestricted_orbital_gradient_fd(ctx):
    """g_ai of each spin from the GPU dE/dC against central differences of the
    GPU UMP2 energy under C_s -> C_s exp(-h K) (step 1e-4)."""
    N, oa, ob, M = 40, 6, 4, 100
    inp = twin(N, oa, M, seed=11, nocc_beta=ob)
    A, B = inp.alpha, inp.beta
    set_unrestricted(ctx, inp)
    g = ctx.mp2_gradient(capi.UNRESTRICTED, capi.FP64)
    h = 1e-4
    for spin, S, o, dC in ((capi.ALPHA, A, oa, g.dC_a), (capi.BETA, B, ob, g.dC_b)):
        kg = orc.orbital_gradient(S.C, dC, o)
        for (ai, ii) in [(0, 0), (5, o - 1), (20, 1)]:
            K = np.zeros((N, N))
            K[o + ai, ii], K[ii, o + ai] = 1.0, -1.0
            ctx.set_orbitals(spin, S.C @ scipy.linalg.expm(-h * K), S.eps, o)
            ep = ctx.mp2_energy(capi.UNRESTRICTED, capi.FP64)["total"]
            ctx.set_orbitals(spin, S.C @ scipy.linalg.expm(h * K), S.eps, o)
            em = ctx.mp2_energy(capi.UNRESTRICTED, capi.FP64)["total"]
            ctx.set_orbitals(spin, S.C, S.eps, o)
            fd = (ep - em) / (2 * h)
            assert abs(fd - kg[ai, ii]) <= 1e-6, (spin, ai, ii, fd, kg[ai, ii])


@pytest.mark.parametrize("N,oa,ob,M,seed", [(60, 8, 7, 150, 3), (131, 14, 11, 300, 5), (210, 19, 17, 520, 6)])
def test_unrestricted_mixed_gradient_vs_fp64(ctx, N, oa, ob, M, seed):
    inp = twin(N, oa, M, seed=seed, nocc_beta=ob)
    set_unrestricted(ctx, inp)
    g64 = ctx.mp2_gradient(capi.UNRESTRICTED, capi.FP64)
    set_unrestricted(ctx, inp)                        # mixed transforms of both spins
    g3 = ctx.mp2_gradient(capi.UNRESTRICTED, capi.FP16X3)
    for key in ("ss_aa", "ss_bb", "os", "total"):
        assert abs(g3.energy[key] - g64.energy[key]) <= 1e-6, key
    for x, y in ((g3.dC_a, g64.dC_a), (g3.dC_b, g64.dC_b), (g3.deps_a, g64.deps_a), (g3.deps_b, g64.deps_b)):
        assert np.max(np.abs(x - y)) <= 1e-6, np.max(np.abs(x - y))


# Block pairs: the mixed backward splits the occupied orbitals into blocks
# and, for the restricted and same-spin passes, computes only block pairs
# I <= J (the (j, i) amplitudes are the transposes of the (i, j) ones).
# Small blocks force several block pairs, mirrored ones included.
@pytest.mark.parametrize("block", ["3", "5"])
def test_restricted_mixed_gradient_block_pairs(ctx, monkeypatch, block):
    N, o, M = 120, 13, 280
    inp = twin(N, o, M, seed=31)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    g64 = ctx.mp2_gradient(capi.RESTRICTED, capi.FP64)
    one = ctx.mp2_gradient(capi.RESTRICTED, capi.FP16X3)
    monkeypatch.setenv("MSHQC_CD_BWD_BLOCK", block)
    g3 = ctx.mp2_gradient(capi.RESTRICTED, capi.FP16X3)
    assert abs(g3.energy["total"] - g64.energy["total"]) <= 1e-6
    assert abs(g3.energy["total"] - one.energy["total"]) <= 1e-9
    assert np.max(np.abs(g3.dC_a - g64.dC_a)) <= 1e-6
    assert np.max(np.abs(g3.deps_a - g64.deps_a)) <= 1e-6
    assert np.max(np.abs(g3.dC_a - one.dC_a)) <= 1e-7


def test_unrestricted_mixed_gradient_block_pairs(ctx, monkeypatch):
    inp = twin(100, 11, 240, seed=33, nocc_beta=9)
    set_unrestricted(ctx, inp)
    g64 = ctx.mp2_gradient(capi.UNRESTRICTED, capi.FP64)
    monkeypatch.setenv("MSHQC_CD_BWD_BLOCK", "4")
    g3 = ctx.mp2_gradient(capi.UNRESTRICTED, capi.FP16X3)
    for key in ("ss_aa", "ss_bb", "os", "total"):
        assert abs(g3.energy[key] - g64.energy[key]) <= 1e-6, key
    for x, y in ((g3.dC_a, g64.dC_a), (g3.dC_b, g64.dC_b), (g3.deps_a, g64.deps_a), (g3.deps_b, g64.deps_b)):
        assert np.max(np.abs(x - y)) <= 1e-6, np.max(np.abs(x - y))
