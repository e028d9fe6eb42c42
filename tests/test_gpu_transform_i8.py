"""Half transform of the mixed path on the int8 tensor cores (ozaki_i8.cuh:
every operand row cut into five 7-bit slices under a per-row power of two,
exact int32 products, FP64 combination) against the CPU oracle and the FP64
path.

The slice products carry an error of about 2^-31 of (row max x row max) per
term, so the transformed vectors agree with the FP64 ones to
REL_TOL = 2e-8 of max |B| (the FP64 path: 1e-13).  An FP64 request after a
mixed one recomputes the vectors in FP64; MSHQC_CD_TRANSFORM=f64 sends the
mixed path through the FP64 transform, =i8 (set for every test here: these
sizes are below N = 512, where the library itself switches the forward
transform to the int8 products) through the int8 one.
"""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc

pytestmark = pytest.mark.gpu

REL_TOL = 2e-8


@pytest.fixture(autouse=True)
def int8_forward(monkeypatch):
    """These sizes are below the one from which the library takes the int8
    forward transform by itself: force it (tests that switch it off set
    MSHQC_CD_TRANSFORM=f64 over this)."""
    monkeypatch.setenv("MSHQC_CD_TRANSFORM", "i8")


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def rel_err(B, Bref):
    return np.max(np.abs(B - Bref)) / np.max(np.abs(Bref))


@pytest.mark.parametrize("name", ["rmp2_ragged_n29_o7_m61", "rmp2_n32_o6_m96", "rmp2_single_occupied"])
def test_mixed_transform_vs_oracle(ctx, golden, name):
    g = golden(name)
    o = int(g["nocc"])
    ctx.set_vectors(g["L"]).set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    B = ctx.transform(capi.ALPHA, capi.FP16X3)
    Bref = orc.transform(g["L"], g["C"], o)
    assert B.shape == Bref.shape
    assert rel_err(B, Bref) <= REL_TOL
    # an FP64 request does not reuse the int8-slice vectors
    B64 = ctx.transform(capi.ALPHA, capi.FP64)
    assert np.max(np.abs(B64 - Bref)) <= 1e-13 * np.max(np.abs(Bref))


@pytest.mark.parametrize("N,o,M", [(257, 19, 515), (300, 30, 1200), (161, 1, 97), (96, 95, 33)])
def test_mixed_transform_vs_fp64(ctx, N, o, M):
    inp = syn.make_inputs(N, o, M, seed=N + o)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    B64 = ctx.transform(capi.ALPHA, capi.FP64)
    ctx.set_orbitals(capi.ALPHA, a.C, a.eps, o)    # drop the FP64 vectors
    B8 = ctx.transform(capi.ALPHA, capi.FP16X3)
    assert rel_err(B8, B64) <= REL_TOL, rel_err(B8, B64)


def test_env_switch_selects_fp64_transform(ctx, monkeypatch):
    inp = syn.make_inputs(120, 12, 300, seed=5)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, 12)
    B64 = ctx.transform(capi.ALPHA, capi.FP64)
    monkeypatch.setenv("MSHQC_CD_TRANSFORM", "f64")
    ctx.set_orbitals(capi.ALPHA, a.C, a.eps, 12)
    B = ctx.transform(capi.ALPHA, capi.FP16X3)
    assert np.array_equal(B, B64)


@pytest.mark.parametrize("chunk", [None, "7"])
def test_generated_vectors_mixed_transform(monkeypatch, chunk):
    N, o, M, seed = 70, 9, 130, 11
    if chunk:
        monkeypatch.setenv("MSHQC_CD_GEN_CHUNK", chunk)
    orb = syn.make_orbitals(N, o, 3)
    L = syn.make_vectors_philox(N, M, seed, 0.01)
    with capi.Context(0) as c:
        c.gen_vectors(N, M, seed, 0.01)
        c.set_orbitals(capi.ALPHA, orb.C, orb.eps, o)
        B = c.transform(capi.ALPHA, capi.FP16X3)
    Bref = orc.transform(L, orb.C, o)
    assert rel_err(B, Bref) <= REL_TOL


def test_mixed_energy_with_int8_transform_vs_fp64(ctx):
    N, o, M = 200, 20, 800
    base = syn.make_inputs(N, o, M, seed=9)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    inp = syn.make_inputs(N, o, M, seed=9, sigma=sig)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    e3 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)
    e64 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)
    assert abs(e3["total"] - e64["total"]) <= 1e-6


# The backward's transposed transforms of the mixed path run on the same
# int8 products (dC_vir over batches of occupied orbitals, W with C_vir
# shared, dC_occ over batches of Q).  dE/dC agrees with the FP64 path to the
# mixed-path tolerance 1e-6, with stored vectors, generated vectors in one
# chunk or in chunks of 7, and with the int8 transforms switched off.
def twin_inputs(N, o, M, seed):
    base = syn.make_inputs(N, o, M, seed=seed)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    return syn.make_inputs(N, o, M, seed=seed, sigma=sig)


@pytest.mark.parametrize("switch", [None, "f64"])
def test_mixed_gradient_int8_transposed_vs_fp64(ctx, monkeypatch, switch):
    N, o, M = 150, 17, 380
    inp = twin_inputs(N, o, M, seed=21)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    g64 = ctx.mp2_gradient(capi.RESTRICTED, capi.FP64)
    if switch:
        monkeypatch.setenv("MSHQC_CD_TRANSFORM", switch)
    else:
        monkeypatch.delenv("MSHQC_CD_TRANSFORM")      # the library's own choice at this size
    ctx.set_orbitals(capi.ALPHA, a.C, a.eps, o)
    g3 = ctx.mp2_gradient(capi.RESTRICTED, capi.FP16X3)
    assert abs(g3.energy["total"] - g64.energy["total"]) <= 1e-6
    assert np.max(np.abs(g3.dC_a - g64.dC_a)) <= 1e-6
    assert np.max(np.abs(g3.deps_a - g64.deps_a)) <= 1e-6


@pytest.mark.parametrize("chunk", [None, "7"])
def test_generated_mixed_gradient_vs_fp64(monkeypatch, chunk):
    N, o, M, seed = 64, 8, 150, 4
    if chunk:
        monkeypatch.setenv("MSHQC_CD_GEN_CHUNK", chunk)
    orb = syn.make_orbitals(N, o, 7)
    sigma = syn.twin_sigma(N, o, M, orb.eps)
    out = {}
    for prec in (capi.FP64, capi.FP16X3):
        with capi.Context(0) as c:
            c.gen_vectors(N, M, seed, sigma)
            c.set_orbitals(capi.ALPHA, orb.C, orb.eps, o)
            out[prec] = c.mp2_gradient(capi.RESTRICTED, prec)
    g64, g3 = out[capi.FP64], out[capi.FP16X3]
    assert abs(g3.energy["total"] - g64.energy["total"]) <= 1e-6
    assert np.max(np.abs(g3.dC_a - g64.dC_a)) <= 1e-6
