"""Mixed-precision path (scaled FP16x3 on tcgen05: exact FP32 accumulation of
fixed-point products, FP64 denominators and sums) vs the FP64 path, the CPU
oracle and the reference fixtures.

The mixed path represents every MO row (i,a) in fixed point with one
power-of-two scale (step 2^-17 of the row maximum) and accumulates the
integer products exactly on the tensor cores, so its error is the
round-to-nearest representation error: random, unbiased, and averaging down
as o*v grows.

Tolerances:
  * scaled-twin inputs (|E_corr| ~ 0.05 o Eh): |dE| <= 1 micro-Eh absolute;
  * raw recipe, the reference fixtures (N <= 32, M <= 100, rows spanning six
    decades over Q): |dE| / |E| <= 5e-6;
  * raw recipe, N >= 100: |dE| / |E| <= 1e-6.
"""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc

pytestmark = pytest.mark.gpu

ABS_TOL_TWIN = 1e-6     # Eh
REL_TOL_RAW_SMALL = 5e-6
REL_TOL_RAW = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def twin_inputs(N, o, M, seed, nocc_beta=None):
    base = syn.make_inputs(N, o, M, seed=seed, nocc_beta=nocc_beta)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    return syn.make_inputs(N, o, M, seed=seed, sigma=sig, nocc_beta=nocc_beta)


@pytest.mark.parametrize("name", ["rmp2_n24_o5_m60", "rmp2_n32_o6_m96", "rmp2_ragged_n29_o7_m61",
                                  "rmp2_zero_denominators", "rmp2_single_occupied"])
def test_restricted_raw_vs_reference(ctx, golden, name):
    g = golden(name)
    o = int(g["nocc"])
    ctx.set_vectors(g["L"]).set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    e = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)
    ref = float(g["e_corr"])
    assert abs(e["total"] - ref) <= REL_TOL_RAW_SMALL * abs(ref), (e["total"], ref)
    assert abs(e["os"] - float(g["ump2_os"])) <= REL_TOL_RAW_SMALL * abs(float(g["ump2_os"]))


def test_restricted_twin_fixture_abs(ctx, golden):
    g = golden("rmp2_twin_n28_o5_m80")
    o = int(g["nocc"])
    ctx.set_vectors(g["L"]).set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    e = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)
    assert abs(e["total"] - float(g["e_corr"])) <= ABS_TOL_TWIN


@pytest.mark.parametrize("N,o,M", [(160, 16, 640), (300, 30, 1200), (257, 19, 515)])
def test_restricted_twin_vs_fp64(ctx, N, o, M):
    inp = twin_inputs(N, o, M, seed=N)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    e64 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)
    e3 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)
    assert abs(e3["total"] - e64["total"]) <= ABS_TOL_TWIN, (e3["total"], e64["total"])
    assert abs(e3["os"] - e64["os"]) <= ABS_TOL_TWIN
    # pair energies agree too
    ctx.mp2_energy(capi.RESTRICTED, capi.FP64)
    P64 = ctx.pair_energies(0)
    ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)
    P3 = ctx.pair_energies(0)
    assert np.max(np.abs(P3 - P64)) <= ABS_TOL_TWIN


@pytest.mark.parametrize("name", ["ump2_n26_o6_5_m70", "ump2_n20_o4_3_m50"])
def test_unrestricted_raw_vs_reference(ctx, golden, name):
    g = golden(name)
    na, nb = int(g["nocc_a"]), int(g["nocc_b"])
    ctx.set_vectors(g["L"])
    ctx.set_orbitals(capi.ALPHA, g["Ca"], g["ea"], na)
    ctx.set_orbitals(capi.BETA, g["Cb"], g["eb"], nb)
    e = ctx.mp2_energy(capi.UNRESTRICTED, capi.FP16X3)
    for k in ("ss_aa", "ss_bb", "os"):
        assert abs(e[k] - float(g[k])) <= REL_TOL_RAW_SMALL * abs(float(g[k])), k


def test_unrestricted_twin_vs_fp64(ctx):
    N, oa, ob, M = 200, 20, 18, 800
    inp = twin_inputs(N, oa, M, seed=4, nocc_beta=ob)
    ctx.set_vectors(inp.L)
    ctx.set_orbitals(capi.ALPHA, inp.alpha.C, inp.alpha.eps, oa)
    ctx.set_orbitals(capi.BETA, inp.beta.C, inp.beta.eps, ob)
    e64 = ctx.mp2_energy(capi.UNRESTRICTED, capi.FP64)
    e3 = ctx.mp2_energy(capi.UNRESTRICTED, capi.FP16X3)
    for k in ("ss_aa", "ss_bb", "os", "total"):
        assert abs(e3[k] - e64[k]) <= ABS_TOL_TWIN, (k, e3[k], e64[k])


def test_mixed_vs_oracle_medium(ctx):
    N, o, M = 200, 25, 700
    inp = twin_inputs(N, o, M, seed=12)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    e3 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)
    B = orc.transform(inp.L, a.C, o)
    E, _ = orc.rmp2_energy(B, a.eps, o)
    assert abs(e3["total"] - E) <= ABS_TOL_TWIN


@pytest.mark.parametrize("N,o,M", [(160, 16, 640), (211, 23, 901)])
def test_restricted_raw_medium_vs_fp64(ctx, N, o, M):
    inp = syn.make_inputs(N, o, M, seed=N + 1)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    e64 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
    e3 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)["total"]
    assert abs(e3 - e64) <= REL_TOL_RAW * abs(e64), (e3, e64)


def test_mixed_deterministic(ctx, golden):
    g = golden("rmp2_n32_o6_m96")
    o = int(g["nocc"])
    ctx.set_vectors(g["L"]).set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    e1 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)["total"]
    ctx.set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    e2 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)["total"]
    assert e1 == e2
