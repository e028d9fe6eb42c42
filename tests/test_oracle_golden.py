"""The CPU restatement (oracle/cdmp2_oracle.py) against golden fixtures
produced by the reference's own code (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle import cdmp2_oracle as orc

RESTRICTED = ["rmp2_n24_o5_m60", "rmp2_n32_o6_m96", "rmp2_twin_n28_o5_m80",
              "rmp2_ragged_n29_o7_m61", "rmp2_zero_denominators", "rmp2_single_occupied"]


@pytest.mark.parametrize("name", RESTRICTED)
def test_rmp2_energy_matches_reference(golden, name):
    g = golden(name)
    o = int(g["nocc"])
    B = orc.transform(g["L"], g["C"], o)
    E, pair = orc.rmp2_energy(B, g["eps"], o)
    assert abs(E - g["e_corr"]) <= 1e-12 * abs(g["e_corr"]) + 1e-14
    # pair energies are symmetric and sum to the total
    assert np.allclose(pair, pair.T, rtol=1e-12, atol=1e-14)
    assert abs(pair.sum() - E) <= 1e-12 * abs(E) + 1e-14


@pytest.mark.parametrize("name", RESTRICTED)
def test_closed_shell_ump2_matches_reference(golden, name):
    g = golden(name)
    o = int(g["nocc"])
    B = orc.transform(g["L"], g["C"], o, convention="ump2")
    u = orc.ump2_energies(B, B, g["eps"], g["eps"], o, o)
    assert abs(u["ss_aa"] - g["ump2_ss_aa"]) <= 1e-12 * abs(g["ump2_ss_aa"]) + 1e-14
    assert abs(u["os"] - g["ump2_os"]) <= 1e-12 * abs(g["ump2_os"]) + 1e-14
    # RMP2 = UMP2(C_a = C_b) identity
    assert abs(u["e_corr"] - g["e_corr"]) <= 1e-11 * abs(g["e_corr"]) + 1e-14


def test_rmp2_amplitudes_match_reference(golden):
    g = golden("rmp2_n24_o5_m60")
    o = int(g["nocc"])
    B = orc.transform(g["L"], g["C"], o)
    t2 = orc.rmp2_t2(B, g["eps"], o)
    assert np.max(np.abs(t2 - g["t2"])) <= 1e-12 * np.max(np.abs(g["t2"]))


def test_single_occupied_same_spin_vanishes(golden):
    g = golden("rmp2_single_occupied")
    assert g["ump2_ss_aa"] == 0.0
    B = orc.transform(g["L"], g["C"], 1)
    u = orc.ump2_energies(B, B, g["eps"], g["eps"], 1, 1)
    assert u["ss_aa"] == 0.0


@pytest.mark.parametrize("name", ["ump2_n26_o6_5_m70", "ump2_n20_o4_3_m50"])
def test_open_shell_ump2_and_omp2_pieces(golden, name):
    g = golden(name)
    na, nb = int(g["nocc_a"]), int(g["nocc_b"])
    Ba = orc.transform(g["L"], g["Ca"], na, convention="ump2")
    Bb = orc.transform(g["L"], g["Cb"], nb, convention="ump2")
    u = orc.ump2_energies(Ba, Bb, g["ea"], g["eb"], na, nb)
    for k in ("ss_aa", "ss_bb", "os", "e_corr"):
        assert abs(u[k] - g[k]) <= 1e-12 * abs(g[k]) + 1e-14, k
    p = orc.omp2_pieces(g["L"], g["H"], g["Ca"], g["Cb"], g["ea"], g["eb"], na, nb)
    assert abs(p["e_mp2"] - g["omp2_e_mp2"]) <= 1e-12 * abs(g["omp2_e_mp2"])
    assert abs(p["e_mp2"] - g["e_corr"]) <= 1e-11 * abs(g["e_corr"])
    for k in ("Goo_a", "Gvv_a", "Goo_b", "Gvv_b", "F_a", "F_b", "w_a", "w_b"):
        scale = max(1.0, np.max(np.abs(g[k])))
        assert np.max(np.abs(p[k] - g[k])) <= 1e-12 * scale, k


def test_omp2_loop_matches_reference(golden):
    g = golden("omp2_loop_twin_n20_o4_m50")
    o = int(g["nocc"])
    r = orc.omp2(g["L"], g["H"], g["C"], g["C"], g["eps"], g["eps"], o, o,
                 e_scf=float(g["e_scf"]))
    assert r["iterations"] == int(g["iterations"])
    assert r["converged"] == bool(g["converged"])
    assert abs(r["e_corr"] - g["e_corr"]) <= 1e-12
    assert abs(r["e_total"] - g["e_total"]) <= 1e-12
    assert np.max(np.abs(r["C_alpha"] - g["C_alpha"])) <= 1e-12


def test_cholesky_decompose_matches_reference(golden):
    g = golden("cholesky_decompose_n8")
    Lv = orc.cholesky_decompose(g["eri"], float(g["threshold"]))
    assert Lv.shape == g["L"].shape
    assert np.max(np.abs(Lv - g["L"])) <= 1e-12
    # reconstruction error below the threshold
    n2 = int(g["N"]) ** 2
    R = Lv.T @ Lv
    assert np.max(np.abs(R - g["eri"].reshape(n2, n2))) < 10 * float(g["threshold"])
