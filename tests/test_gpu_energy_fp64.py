"""FP64 CUDA path vs the reference (golden fixtures) and the CPU oracle.

Tolerance: relative 1e-12 on energies (different summation order than the
reference; both are FP64), 1e-12 of the largest element on arrays.
"""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc

pytestmark = pytest.mark.gpu

RESTRICTED = ["rmp2_n24_o5_m60", "rmp2_n32_o6_m96", "rmp2_twin_n28_o5_m80",
              "rmp2_ragged_n29_o7_m61", "rmp2_zero_denominators", "rmp2_single_occupied"]
REL = 1e-12


def close(x, ref, rel=REL, atol=1e-14):
    return abs(x - ref) <= rel * abs(ref) + atol


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", RESTRICTED)
def test_rmp2_energy_vs_reference(ctx, golden, name):
    g = golden(name)
    o = int(g["nocc"])
    ctx.set_vectors(g["L"]).set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    e = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)
    assert close(e["total"], float(g["e_corr"])), (e["total"], float(g["e_corr"]))
    # same/opposite-spin split of the closed-shell energy = CD-UMP2 with C_a = C_b
    assert close(e["os"], float(g["ump2_os"]), 1e-11)
    assert close(e["ss_aa"], float(g["ump2_ss_aa"]), 1e-11, 1e-13)


@pytest.mark.parametrize("name", RESTRICTED)
def test_closed_shell_unrestricted_vs_reference(ctx, golden, name):
    g = golden(name)
    o = int(g["nocc"])
    ctx.set_vectors(g["L"])
    ctx.set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    ctx.set_orbitals(capi.BETA, g["C"], g["eps"], o)
    e = ctx.mp2_energy(capi.UNRESTRICTED, capi.FP64)
    assert close(e["ss_aa"], float(g["ump2_ss_aa"]), REL, 1e-13)
    assert close(e["ss_bb"], float(g.get("ump2_ss_bb", g["ump2_ss_aa"])), REL, 1e-13)
    assert close(e["os"], float(g["ump2_os"]))
    assert close(e["total"], float(g["e_corr"]), 1e-11)


@pytest.mark.parametrize("name", ["ump2_n26_o6_5_m70", "ump2_n20_o4_3_m50"])
def test_open_shell_ump2_vs_reference(ctx, golden, name):
    g = golden(name)
    na, nb = int(g["nocc_a"]), int(g["nocc_b"])
    ctx.set_vectors(g["L"])
    ctx.set_orbitals(capi.ALPHA, g["Ca"], g["ea"], na)
    ctx.set_orbitals(capi.BETA, g["Cb"], g["eb"], nb)
    e = ctx.mp2_energy(capi.UNRESTRICTED, capi.FP64)
    for k in ("ss_aa", "ss_bb", "os"):
        assert close(e[k], float(g[k])), (k, e[k], float(g[k]))
    assert close(e["total"], float(g["e_corr"]))


def test_transform_vs_oracle(ctx, golden):
    g = golden("rmp2_ragged_n29_o7_m61")
    o = int(g["nocc"])
    ctx.set_vectors(g["L"]).set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    B = ctx.transform(capi.ALPHA, capi.FP64)
    Bref = orc.transform(g["L"], g["C"], o)
    assert B.shape == Bref.shape
    assert np.max(np.abs(B - Bref)) <= 1e-13 * np.max(np.abs(Bref))


def test_pair_energies_vs_oracle(ctx, golden):
    g = golden("rmp2_n32_o6_m96")
    o = int(g["nocc"])
    ctx.set_vectors(g["L"]).set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    e = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)
    P = ctx.pair_energies(0)
    B = orc.transform(g["L"], g["C"], o)
    _, Pref = orc.rmp2_energy(B, g["eps"], o)
    assert np.max(np.abs(P - Pref)) <= 1e-12 * np.max(np.abs(Pref))
    assert close(P.sum(), e["total"])


@pytest.mark.parametrize("N,o,M", [(96, 12, 300), (130, 17, 257)])
def test_medium_sizes_vs_oracle(ctx, N, o, M):
    inp = syn.make_inputs(N, o, M, seed=N)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    e = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)
    B = orc.transform(inp.L, a.C, o)
    E, _ = orc.rmp2_energy(B, a.eps, o)
    assert close(e["total"], E), (e["total"], E)


def test_packed_layout_and_q_rotation_invariance(ctx):
    """E is invariant under an orthogonal rotation of the Cholesky index Q;
    the packed upper-triangle upload gives the same energy as the full one."""
    N, o, M = 40, 6, 90
    inp = syn.make_inputs(N, o, M, seed=9)
    a = inp.alpha
    ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    e0 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
    rng = np.random.default_rng(1)
    R, _ = np.linalg.qr(rng.standard_normal((M, M)))
    Lr = R.T @ inp.L
    ctx.set_vectors(Lr).set_orbitals(capi.ALPHA, a.C, a.eps, o)
    e1 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
    assert close(e1, e0, 1e-11)
    iu = np.triu_indices(N)
    packed = inp.L.reshape(M, N, N)[:, iu[0], iu[1]]
    ctx.set_vectors(packed, nbf=N, layout="packed").set_orbitals(capi.ALPHA, a.C, a.eps, o)
    e2 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
    assert close(e2, e0)


def test_deterministic(ctx, golden):
    g = golden("rmp2_n32_o6_m96")
    o = int(g["nocc"])
    ctx.set_vectors(g["L"]).set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    e1 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
    ctx.set_orbitals(capi.ALPHA, g["C"], g["eps"], o)   # forces a new transform
    e2 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
    assert e1 == e2


def test_error_statuses(ctx, golden):
    g = golden("rmp2_n24_o5_m60")
    fresh = capi.Context(0)
    try:
        with pytest.raises(capi.CDError) as ex:
            fresh.mp2_energy(capi.RESTRICTED, capi.FP64)
        assert ex.value.code == capi.ERR_STATE
        fresh.set_vectors(g["L"])
        eps = g["eps"].copy()
        eps[3] = np.nan
        with pytest.raises(capi.CDError) as ex:
            fresh.set_orbitals(capi.ALPHA, g["C"], eps, 5)
        assert ex.value.code == capi.ERR_NUMERIC
        with pytest.raises(capi.CDError) as ex:
            fresh.set_orbitals(capi.ALPHA, g["C"], g["eps"], 24)
        assert ex.value.code == capi.ERR_ARG
        fresh.set_orbitals(capi.ALPHA, g["C"], g["eps"], 5)
        with pytest.raises(capi.CDError) as ex:
            fresh.mp2_energy(capi.UNRESTRICTED, capi.FP64)   # beta never set
        assert ex.value.code == capi.ERR_STATE
        # the context is still usable after the errors
        e = fresh.mp2_energy(capi.RESTRICTED, capi.FP64)
        assert close(e["total"], float(g["e_corr"]))
    finally:
        fresh.close()
