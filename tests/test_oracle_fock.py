"""The reference's Cholesky Fock builds as compiled into oracle/_ref
(CholeskyRHF::build_fock, src/scf/cholesky_rhf.cc:99-137, and
CholeskyUHF::build_fock_cholesky, src/scf/cholesky_uhf.cc:77-103) against the
textbook J and K: F = H + J - K/2 (RHF, total density, vectors of norm
<= 1e-8 screened out of K when asked) and F_s = H + J - K_s (UHF).  This pins
the checker the GPU Fock test compares with."""
import numpy as np
import pytest

from oracle import ref

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")

N, M = 14, 40


def inputs(seed):
    rng = np.random.default_rng(seed)
    L = rng.standard_normal((M, N, N)) * 0.1
    L = L + L.transpose(0, 2, 1)
    L[3] *= 1e-9
    C, _ = np.linalg.qr(rng.standard_normal((N, N)))
    H = rng.standard_normal((N, N))
    return L, C[:, :4] @ C[:, :4].T, C[:, :3] @ C[:, :3].T, 0.5 * (H + H.T)


def jk(L, Ptot, P, screen):
    keep = [q for q in range(M) if not screen or np.linalg.norm(L[q]) > 1e-8]
    J = sum(np.sum(L[q] * Ptot) * L[q] for q in range(M))
    K = sum(L[q] @ P @ L[q] for q in keep)
    return J, K


@needs_ref
@pytest.mark.parametrize("screen", [True, False])
def test_reference_rhf_fock(screen):
    L, Pa, _, H = inputs(1)
    P = 2.0 * Pa
    F = ref.cholesky_fock(L.reshape(M, N * N), H, P, screen_exchange=screen)
    J, K = jk(L, P, P, screen)
    assert np.max(np.abs(F - (H + J - 0.5 * K))) <= 1e-12 * np.max(np.abs(F))


@needs_ref
def test_reference_uhf_fock():
    L, Pa, Pb, H = inputs(2)
    Fa, Fb = ref.cholesky_fock(L.reshape(M, N * N), H, Pa, Pb)
    for P, F in ((Pa, Fa), (Pb, Fb)):
        J, K = jk(L, Pa + Pb, P, False)
        assert np.max(np.abs(F - (H + J - K))) <= 1e-12 * np.max(np.abs(F))
