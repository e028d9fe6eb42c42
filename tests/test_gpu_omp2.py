"""CD-OMP2 on the GPU (FP64) against the reference: one gradient evaluation
(energy, G_oo, G_vv, generalized Fock, w_ai) on the golden fixtures made by
the reference's own CholeskyOMP2, and the whole orbital-rotation loop.

Tolerances: 1e-10 of the largest element for matrices, 1e-11 relative for
energies (FP64 throughout, different summation order); the loop's orbitals
after several rotations 1e-9.
"""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def close_mat(x, ref, rel=1e-10):
    return np.max(np.abs(x - ref)) <= rel * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("name", ["ump2_n26_o6_5_m70", "ump2_n20_o4_3_m50"])
def test_omp2_pieces_vs_reference(ctx, golden, name):
    g = golden(name)
    na, nb = int(g["nocc_a"]), int(g["nocc_b"])
    ctx.set_vectors(g["L"])
    ctx.set_orbitals(capi.ALPHA, g["Ca"], g["ea"], na)
    ctx.set_orbitals(capi.BETA, g["Cb"], g["eb"], nb)
    ctx.set_core_hamiltonian(g["H"])
    p = ctx.omp2_pieces()
    assert abs(p["e_mp2"] - g["omp2_e_mp2"]) <= 1e-11 * abs(g["omp2_e_mp2"])
    for k in ("Goo_a", "Gvv_a", "Goo_b", "Gvv_b", "F_a", "F_b", "w_a", "w_b"):
        assert close_mat(p[k], g[k]), (k, np.max(np.abs(p[k] - g[k])))


def test_omp2_pieces_vs_oracle_larger(ctx):
    N, na, nb, M = 90, 9, 7, 220
    base = syn.make_inputs(N, na, M, seed=13, nocc_beta=nb)
    sig = syn.twin_sigma(N, na, M, base.alpha.eps)
    inp = syn.make_inputs(N, na, M, seed=13, sigma=sig, nocc_beta=nb)
    H = syn.default_core_hamiltonian(inp)
    A, B = inp.alpha, inp.beta
    ref = orc.omp2_pieces(inp.L, H, A.C, B.C, A.eps, B.eps, na, nb)
    ctx.set_vectors(inp.L)
    ctx.set_orbitals(capi.ALPHA, A.C, A.eps, na)
    ctx.set_orbitals(capi.BETA, B.C, B.eps, nb)
    ctx.set_core_hamiltonian(H)
    p = ctx.omp2_pieces()
    assert abs(p["e_mp2"] - ref["e_mp2"]) <= 1e-11 * abs(ref["e_mp2"])
    for k in ("Goo_a", "Gvv_a", "Goo_b", "Gvv_b", "F_a", "F_b", "w_a", "w_b"):
        assert close_mat(p[k], ref[k]), (k, np.max(np.abs(p[k] - ref[k])))


def test_omp2_loop_vs_reference(ctx, golden):
    """The reference's CholeskyOMP2::compute on a closed shell (beta follows
    alpha), run to convergence by the reference itself."""
    g = golden("omp2_loop_twin_n20_o4_m50")
    o = int(g["nocc"])
    ctx.set_vectors(g["L"])
    ctx.set_orbitals(capi.ALPHA, g["C"], g["eps"], o)
    ctx.set_orbitals(capi.BETA, g["C"], g["eps"], o)
    ctx.set_core_hamiltonian(g["H"])
    r = ctx.omp2(e_scf=float(g["e_scf"]))
    assert r["iterations"] == int(g["iterations"])
    assert r["converged"] == bool(g["converged"])
    assert abs(r["energy_mp2_corr"] - g["e_corr"]) <= 1e-11
    assert abs(r["energy_total"] - g["e_total"]) <= 1e-11
    assert np.max(np.abs(r["C_alpha"] - g["C_alpha"])) <= 1e-9
    assert np.max(np.abs(r["C_beta"] - g["C_alpha"])) <= 1e-9


def test_omp2_open_shell_loop_vs_oracle(ctx):
    """Open shell (nocc_alpha != nocc_beta: alpha and beta rotated
    separately), six iterations from common spatial orbitals."""
    N, na, nb, M = 30, 5, 3, 80
    base = syn.make_inputs(N, na, M, seed=17)
    sig = syn.twin_sigma(N, na, M, base.alpha.eps)
    inp = syn.make_inputs(N, na, M, seed=17, sigma=sig)
    A = inp.alpha
    B = syn.SpinOrbitals(A.C, A.eps, nb)
    H = syn.default_core_hamiltonian(syn.CDInputs(N=N, M=M, L=inp.L, alpha=A, beta=B))
    ref = orc.omp2(inp.L, H, A.C, B.C, A.eps, B.eps, na, nb, e_scf=-2.0, max_iter=6)
    ctx.set_vectors(inp.L)
    ctx.set_orbitals(capi.ALPHA, A.C, A.eps, na)
    ctx.set_orbitals(capi.BETA, B.C, B.eps, nb)
    ctx.set_core_hamiltonian(H)
    r = ctx.omp2(max_iterations=6, e_scf=-2.0)
    assert r["iterations"] == ref["iterations"]
    assert r["converged"] == ref["converged"]
    assert abs(r["energy_mp2_corr"] - ref["e_corr"]) <= 1e-11
    assert abs(r["energy_total"] - ref["e_total"]) <= 1e-11
    assert np.max(np.abs(r["C_alpha"] - ref["C_alpha"])) <= 1e-9
    assert np.max(np.abs(r["C_beta"] - ref["C_beta"])) <= 1e-9


def test_omp2_requires_core_hamiltonian():
    with capi.Context(0) as c:
        inp = syn.make_inputs(12, 2, 20, seed=1, nocc_beta=2)
        c.set_vectors(inp.L)
        c.set_orbitals(capi.ALPHA, inp.alpha.C, inp.alpha.eps, 2)
        c.set_orbitals(capi.BETA, inp.beta.C, inp.beta.eps, 2)
        with pytest.raises(capi.CDError) as err:
            c.omp2_pieces()
        assert err.value.code == capi.ERR_STATE
