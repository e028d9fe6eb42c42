"""The oracle's exact MP2 derivatives (restricted and unrestricted) against
central finite differences of the oracle energy: dE/dC, dE/deps and the
orbital-rotation gradient dE/dkappa for C -> C exp(-kappa)."""
import numpy as np
import pytest
import scipy.linalg

from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc


def e_restricted(L, C, eps, o):
    return orc.rmp2_energy(orc.transform(L, C, o), eps, o)[0]


def e_unrestricted(L, Ca, Cb, ea, eb, na, nb):
    Ba = orc.transform(L, Ca, na)
    Bb = orc.transform(L, Cb, nb)
    return orc.ump2_energies(Ba, Bb, ea, eb, na, nb)["e_corr"]


@pytest.fixture(scope="module")
def small():
    base = syn.make_inputs(14, 3, 30, seed=21)
    sig = syn.twin_sigma(14, 3, 30, base.alpha.eps)
    return syn.make_inputs(14, 3, 30, seed=21, sigma=sig, nocc_beta=2)


def test_restricted_dC_deps_fd(small):
    inp = small
    a = inp.alpha
    g = orc.restricted_gradient(inp.L, a.C, a.eps, a.nocc)
    assert abs(g["E"] - e_restricted(inp.L, a.C, a.eps, a.nocc)) < 1e-12 * abs(g["E"])
    h = 1e-5
    rng = np.random.default_rng(0)
    for _ in range(6):
        mu, p = rng.integers(0, inp.N, 2)
        Cp, Cm = a.C.copy(), a.C.copy()
        Cp[mu, p] += h
        Cm[mu, p] -= h
        fd = (e_restricted(inp.L, Cp, a.eps, a.nocc) - e_restricted(inp.L, Cm, a.eps, a.nocc)) / (2 * h)
        assert abs(fd - g["dC"][mu, p]) < 1e-7 * max(1.0, abs(fd)), (mu, p, fd, g["dC"][mu, p])
    for k in [0, 1, 2, 5, 9, 13]:
        ep, em = a.eps.copy(), a.eps.copy()
        ep[k] += h
        em[k] -= h
        fd = (e_restricted(inp.L, a.C, ep, a.nocc) - e_restricted(inp.L, a.C, em, a.nocc)) / (2 * h)
        assert abs(fd - g["deps"][k]) < 1e-7 * max(1.0, abs(fd)), (k, fd, g["deps"][k])


def test_restricted_orbital_gradient_fd(small):
    inp = small
    a = inp.alpha
    o, N = a.nocc, inp.N
    g = orc.restricted_gradient(inp.L, a.C, a.eps, o)
    kap_grad = orc.orbital_gradient(a.C, g["dC"], o)       # (v, o)
    h = 1e-4
    for (ai, ii) in [(0, 0), (3, 1), (10, 2)]:
        K = np.zeros((N, N))
        K[o + ai, ii] = 1.0
        K[ii, o + ai] = -1.0
        Ep = e_restricted(inp.L, a.C @ scipy.linalg.expm(-h * K), a.eps, o)
        Em = e_restricted(inp.L, a.C @ scipy.linalg.expm(h * K), a.eps, o)
        fd = (Ep - Em) / (2 * h)
        assert abs(fd - kap_grad[ai, ii]) < 1e-6 * max(1.0, abs(fd)), (ai, ii, fd, kap_grad[ai, ii])


def test_unrestricted_fd(small):
    inp = small
    A, B = inp.alpha, inp.beta
    g = orc.unrestricted_gradient(inp.L, A.C, B.C, A.eps, B.eps, A.nocc, B.nocc)
    E0 = e_unrestricted(inp.L, A.C, B.C, A.eps, B.eps, A.nocc, B.nocc)
    assert abs(g["E"] - E0) < 1e-12 * abs(E0)
    h = 1e-5
    rng = np.random.default_rng(1)
    for spin in ("a", "b"):
        for _ in range(4):
            mu, p = rng.integers(0, inp.N, 2)
            Ca, Cb = A.C.copy(), B.C.copy()
            X = Ca if spin == "a" else Cb
            X[mu, p] += h
            Ep = e_unrestricted(inp.L, Ca, Cb, A.eps, B.eps, A.nocc, B.nocc)
            X[mu, p] -= 2 * h
            Em = e_unrestricted(inp.L, Ca, Cb, A.eps, B.eps, A.nocc, B.nocc)
            fd = (Ep - Em) / (2 * h)
            an = g["dC_" + spin][mu, p]
            assert abs(fd - an) < 1e-7 * max(1.0, abs(fd)), (spin, mu, p, fd, an)
        for k in [0, 1, 4, 12]:
            ea, eb = A.eps.copy(), B.eps.copy()
            X = ea if spin == "a" else eb
            X[k] += h
            Ep = e_unrestricted(inp.L, A.C, B.C, ea, eb, A.nocc, B.nocc)
            X[k] -= 2 * h
            Em = e_unrestricted(inp.L, A.C, B.C, ea, eb, A.nocc, B.nocc)
            fd = (Ep - Em) / (2 * h)
            an = g["deps_" + spin][k]
            assert abs(fd - an) < 1e-7 * max(1.0, abs(fd)), (spin, k, fd, an)


def test_closed_shell_limits_agree(small):
    """With C_a = C_b and equal occupations the unrestricted derivatives sum
    to the restricted ones (dE/dC_a + dE/dC_b = dE/dC)."""
    inp = small
    a = inp.alpha
    r = orc.restricted_gradient(inp.L, a.C, a.eps, a.nocc)
    u = orc.unrestricted_gradient(inp.L, a.C, a.C, a.eps, a.eps, a.nocc, a.nocc)
    assert abs(r["E"] - u["E"]) < 1e-12 * abs(r["E"])
    assert np.max(np.abs(u["dC_a"] + u["dC_b"] - r["dC"])) < 1e-11 * np.max(np.abs(r["dC"]))
    assert np.max(np.abs(u["deps_a"] + u["deps_b"] - r["deps"])) < 1e-11 * np.max(np.abs(r["deps"]))
