"""mshqc's Python API (mshqc_b200._mshqc) on the GPU, used the way the
reference's scripts use its classes: CholeskyERI -> CholeskyRMP2 /
CholeskyUMP2 / CholeskyOMP2 -> compute(), against the reference's own
results (golden fixtures made by running it).  Energies 1e-12 relative
(1e-11 for the OMP2 loop), orbitals 1e-9; the stored t2 of
CholeskyRMP2Result and CholeskyUMP2's t2 / L_ia (what the reference's MP3
classes read) 1e-12 of their largest element."""
import numpy as np
import pytest

from mshqc_b200 import _mshqc as mshqc
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc

pytestmark = pytest.mark.gpu


class Integrals:
    """The two integral-engine calls the Cholesky-MP2 classes make."""

    def __init__(self, H=None, eri=None):
        self.H, self.eri = H, eri

    def compute_core_hamiltonian(self):
        return self.H

    def compute_eri(self):
        return self.eri


def scf(C, eps, na, Cb=None, eb=None, nb=None, e_total=0.0):
    r = mshqc.SCFResult()
    r.C_alpha, r.orbital_energies_alpha, r.n_occ_alpha = C, eps, na
    r.C_beta = C if Cb is None else Cb
    r.orbital_energies_beta = eps if eb is None else eb
    r.n_occ_beta = na if nb is None else nb
    r.energy_total = e_total
    return r


def quiet(cfg):
    cfg.print_level = 0
    return cfg


@pytest.mark.parametrize("name", ["rmp2_n24_o5_m60", "rmp2_ragged_n29_o7_m61", "rmp2_twin_n28_o5_m80"])
def test_cholesky_rmp2_vs_reference(golden, name):
    g = golden(name)
    N, o = int(g["N"]), int(g["nocc"])
    chol = mshqc.CholeskyERI(1e-6)
    chol.set_vectors(g["L"])
    res = mshqc.CholeskyRMP2(None, N, None, scf(g["C"], g["eps"], o, e_total=-1.5),
                             quiet(mshqc.CholeskyRMP2Config()), chol).compute()
    assert abs(res.e_corr - g["e_corr"]) <= 1e-12 * abs(g["e_corr"])
    assert res.e_total == res.e_rhf + res.e_corr and res.e_rhf == -1.5
    assert (res.n_occ, res.n_virt, res.n_chol_vectors) == (o, N - o, g["L"].shape[0])
    # the stored amplitudes and vectors the reference's CholeskyRMP3 reads
    if "t2" in g:
        assert res.t2.shape == g["t2"].shape
        assert np.max(np.abs(res.t2 - g["t2"])) <= 1e-12 * np.max(np.abs(g["t2"]))
    assert len(res.chol_vectors) == g["L"].shape[0]
    assert np.array_equal(res.chol_vectors[0], g["L"][0])


@pytest.mark.parametrize("name", ["ump2_n26_o6_5_m70", "ump2_n20_o4_3_m50"])
def test_cholesky_ump2_vs_reference(golden, name):
    g = golden(name)
    N, na, nb = int(g["N"]), int(g["nocc_a"]), int(g["nocc_b"])
    chol = mshqc.CholeskyERI()
    chol.set_vectors(g["L"])
    res = mshqc.CholeskyUMP2(scf(g["Ca"], g["ea"], na, g["Cb"], g["eb"], nb), N, None,
                             quiet(mshqc.CholeskyUMP2Config()), chol).compute()
    for attr, key in (("e_corr_ss_aa", "ss_aa"), ("e_corr_ss_bb", "ss_bb"), ("e_corr_os", "os"),
                      ("e_corr_total", "e_corr")):
        assert abs(getattr(res, attr) - g[key]) <= 1e-12 * abs(g[key]) + 1e-14, attr
    assert res.n_cholesky_vectors == g["L"].shape[0]
    # the MO vectors and amplitudes the reference's CholeskyUMP3 reads
    u = mshqc.CholeskyUMP2(scf(g["Ca"], g["ea"], na, g["Cb"], g["eb"], nb), N, None,
                           quiet(mshqc.CholeskyUMP2Config()), chol)
    u.compute()
    u.compute_t2_amplitudes()
    Ba = orc.transform(g["L"], g["Ca"], na)
    Bb = orc.transform(g["L"], g["Cb"], nb)
    assert len(u.L_ia_alpha) == g["L"].shape[0] and len(u.L_ia_beta) == g["L"].shape[0]
    assert np.max(np.abs(np.stack(u.L_ia_alpha, axis=-1) - Ba)) <= 1e-12 * np.max(np.abs(Ba))
    ea, eb = g["ea"], g["eb"]
    for t, X, Y, ex, ey, ox, oy in ((u.t2_aa, Ba, Ba, ea, ea, na, na), (u.t2_bb, Bb, Bb, eb, eb, nb, nb),
                                    (u.t2_ab, Ba, Bb, ea, eb, na, nb)):
        gg = np.einsum("iaQ,jbQ->ijab", X, Y)
        D = (ex[:ox, None, None, None] + ey[None, :oy, None, None] - ex[None, None, ox:, None]
             - ey[None, None, None, oy:])
        assert np.max(np.abs(t - gg / D)) <= 1e-12 * np.max(np.abs(gg / D))


def test_cholesky_omp2_vs_reference(golden):
    g = golden("omp2_loop_twin_n20_o4_m50")
    o = int(g["nocc"])
    chol = mshqc.CholeskyERI()
    chol.set_vectors(g["L"])
    r = scf(g["C"], g["eps"], o, e_total=float(g["e_scf"]))
    res = mshqc.CholeskyOMP2(None, None, Integrals(H=g["H"]), r, quiet(mshqc.CholeskyOMP2Config()), chol).compute()
    assert res.iterations == int(g["iterations"]) and res.converged == bool(g["converged"])
    assert abs(res.energy_mp2_corr - g["e_corr"]) <= 1e-11
    assert abs(res.energy_total - g["e_total"]) <= 1e-11
    assert np.max(np.abs(res.C_alpha - g["C_alpha"])) <= 1e-9
    assert np.array_equal(res.orbital_energies_alpha, g["eps"])


def test_decompose_inside_constructor():
    """Constructor 1: the class decomposes integrals.compute_eri() itself."""
    N, o, M = 14, 3, 50
    inp = syn.make_inputs(N, o, M, seed=6)
    eri = (inp.L.T @ inp.L).reshape(N, N, N, N)
    cfg = quiet(mshqc.CholeskyRMP2Config())
    cfg.cholesky_threshold = 1e-10
    res = mshqc.CholeskyRMP2(None, N, Integrals(eri=eri), scf(inp.alpha.C, inp.alpha.eps, o), cfg).compute()
    Lv = orc.cholesky_decompose(eri, 1e-10)
    ref = orc.rmp2_energy(orc.transform(Lv, inp.alpha.C, o), inp.alpha.eps, o)[0]
    assert abs(res.e_corr - ref) <= 1e-11 * abs(ref)
    assert res.n_chol_vectors == Lv.shape[0]


def test_mixed_precision_config():
    N, o, M = 90, 9, 220
    base = syn.make_inputs(N, o, M, seed=8)
    inp = syn.make_inputs(N, o, M, seed=8, sigma=syn.twin_sigma(N, o, M, base.alpha.eps))
    chol = mshqc.CholeskyERI()
    chol.set_vectors(inp.L)
    r = scf(inp.alpha.C, inp.alpha.eps, o)
    e = {}
    for prec in (0, 1):
        cfg = quiet(mshqc.CholeskyRMP2Config())
        cfg.precision = prec
        e[prec] = mshqc.CholeskyRMP2(None, N, None, r, cfg, chol).compute().e_corr
    assert abs(e[1] - e[0]) <= 1e-6


def test_omp2_empty_vectors_raise():
    with pytest.raises(RuntimeError):
        mshqc.CholeskyOMP2(None, None, Integrals(H=np.eye(4)), scf(np.eye(4), np.arange(4.0), 1),
                           quiet(mshqc.CholeskyOMP2Config()), mshqc.CholeskyERI())
