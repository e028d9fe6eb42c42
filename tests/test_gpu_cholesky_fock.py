"""Cholesky Fock builds on the GPU (mshqc_cd_cholesky_fock) against the
reference's own CholeskyRHF::build_fock (src/scf/cholesky_rhf.cc:99-137) and
CholeskyUHF::build_fock_cholesky (src/scf/cholesky_uhf.cc:77-103), compiled
into oracle/_ref, and against numpy's J and K: FP64 throughout, so 1e-12 of
the largest entry.  One vector is scaled below the reference's exchange
screening norm (1e-8) so that the screened and unscreened RHF builds
differ; the generated-vector case runs in chunks of 7."""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import ref

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

N, M = 40, 150


def sym_vectors(seed, n=N, m=M):
    rng = np.random.default_rng(seed)
    L = rng.standard_normal((m, n, n)) * 0.05
    L = L + L.transpose(0, 2, 1)
    L[5] *= 1e-9                     # Frobenius norm below 1e-8: screened out of K
    return L.reshape(m, n * n)


def densities(seed, n=N, oa=7, ob=5):
    rng = np.random.default_rng(seed)
    C, _ = np.linalg.qr(rng.standard_normal((n, n)))
    H = rng.standard_normal((n, n))
    return C[:, :oa] @ C[:, :oa].T, C[:, :ob] @ C[:, :ob].T, 0.5 * (H + H.T)


def numpy_jk(L, Ptot, Ps, screen=False):
    Ls = L.reshape(-1, N, N)
    keep = [q for q in range(Ls.shape[0]) if not screen or np.linalg.norm(Ls[q]) > 1e-8]
    J = np.einsum("q,qmn->mn", np.einsum("qmn,mn->q", Ls, Ptot), Ls)
    K = [sum(Ls[q] @ P @ Ls[q] for q in keep) for P in Ps]
    return J, K


def close(x, y, tol=1e-12):
    return np.max(np.abs(x - y)) <= tol * max(1.0, np.max(np.abs(y)))


@needs_ref
@pytest.mark.parametrize("screen", [True, False])
def test_rhf_fock_matches_reference(screen):
    L = sym_vectors(3)
    Pa, _, H = densities(4)
    P = 2.0 * Pa                                  # CholeskyRHF::build_density
    with capi.Context(0) as ctx:
        ctx.set_vectors(L)
        out = ctx.cholesky_fock(H, P, screen_exchange=screen)
    F_ref = ref.cholesky_fock(L, H, P, screen_exchange=screen)
    J, (K,) = numpy_jk(L, P, [P], screen)
    assert close(out["F_a"], F_ref)
    assert close(out["J"], J) and close(out["K_a"], K)
    assert close(out["F_a"], H + J - 0.5 * K)


@needs_ref
def test_uhf_fock_matches_reference():
    L = sym_vectors(5)
    Pa, Pb, H = densities(6)
    with capi.Context(0) as ctx:
        ctx.set_vectors(L)
        out = ctx.cholesky_fock(H, Pa, Pb)
    Fa_ref, Fb_ref = ref.cholesky_fock(L, H, Pa, Pb)
    J, (Ka, Kb) = numpy_jk(L, Pa + Pb, [Pa, Pb])
    assert close(out["F_a"], Fa_ref) and close(out["F_b"], Fb_ref)
    assert close(out["J"], J) and close(out["K_a"], Ka) and close(out["K_b"], Kb)


def test_generated_vectors_in_chunks(monkeypatch):
    """Vectors generated on the device chunk by chunk give the Fock matrices
    of the same recipe drawn by numpy and uploaded."""
    monkeypatch.setenv("MSHQC_CD_GEN_CHUNK", "7")
    n, m, seed = 36, 50, 21
    orb = syn.make_orbitals(n, 5, 2)
    sigma = syn.twin_sigma(n, 5, m, orb.eps)
    L = syn.make_vectors_philox(n, m, seed, sigma)
    Pa, Pb, H = densities(8, n, 5, 4)
    with capi.Context(0) as ctx:
        ctx.gen_vectors(n, m, seed, sigma)
        gen = ctx.cholesky_fock(H, Pa, Pb)
    with capi.Context(0) as ctx:
        ctx.set_vectors(L)
        up = ctx.cholesky_fock(H, Pa, Pb)
    for k in ("J", "K_a", "K_b", "F_a", "F_b"):
        assert close(gen[k], up[k]), k


def test_argument_errors():
    """nspin outside 1..2, a missing beta density and a Fock matrix without H
    are refused before any device work."""
    lib = capi.load_library()
    Pa, _, H = densities(2, 8, 3, 2)
    F = np.empty((8, 8))
    with capi.Context(0) as ctx:
        ctx.set_vectors(sym_vectors(1, 8, 10))
        p = lambda a: a.ctypes.data_as(capi.ctypes.c_void_p)
        assert lib.mshqc_cd_cholesky_fock(ctx._h, 3, p(Pa), None, p(H), 0, p(F), None, None, None, None,
                                          capi.HOST) != 0
        assert lib.mshqc_cd_cholesky_fock(ctx._h, 2, p(Pa), None, p(H), 0, p(F), None, None, None, None,
                                          capi.HOST) != 0
        assert lib.mshqc_cd_cholesky_fock(ctx._h, 1, p(Pa), None, None, 0, p(F), None, None, None, None,
                                          capi.HOST) != 0
