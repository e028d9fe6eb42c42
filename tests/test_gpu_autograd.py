"""The torch.autograd.Function of mshqc_b200.autograd.

* its gradients are the library's exact dE/dC, dE/deps;
* unrestricted orbital rotations: the autograd gradient with respect to
  kappa (C_s -> C_s exp(-kappa_s), kappa_s antisymmetric, occupied-virtual
  block) against central finite differences (step 1e-4) of the FP64 energy
  along 64 random directions, tolerance 1e-6 on scaled-twin inputs;
* the mixed-precision gradient within 1e-6 of the FP64 one.
"""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0)
    yield c
    c.close()


def twin(N, o, M, seed, nocc_beta=None):
    base = syn.make_inputs(N, o, M, seed=seed, nocc_beta=nocc_beta)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    return syn.make_inputs(N, o, M, seed=seed, sigma=sig, nocc_beta=nocc_beta)


def t(x):
    return torch.from_numpy(np.ascontiguousarray(x)).to(DEV)


def test_restricted_autograd_matches_library_gradient(ctx):
    from mshqc_b200.autograd import mp2_energy
    inp = twin(70, 8, 170, seed=21)
    a = inp.alpha
    ctx.set_vectors(inp.L)
    ctx.set_orbitals(capi.ALPHA, a.C, a.eps, a.nocc)
    ref = ctx.mp2_gradient(capi.RESTRICTED, capi.FP64)
    C = t(a.C).requires_grad_(True)
    eps = t(a.eps).requires_grad_(True)
    E = mp2_energy(ctx, C, eps, a.nocc)
    (2.0 * E).backward()
    assert abs(E.item() - ref.energy["total"]) <= 1e-14 * abs(ref.energy["total"])
    assert np.max(np.abs(C.grad.cpu().numpy() - 2.0 * ref.dC_a)) <= 1e-14 * np.max(np.abs(ref.dC_a))
    assert np.max(np.abs(eps.grad.cpu().numpy() - 2.0 * ref.deps_a)) <= 1e-14 * np.max(np.abs(ref.deps_a))


def rotated(C0, kappa, o):
    """C0 exp(-K) with K antisymmetric, K[o+a, i] = kappa[a, i]."""
    N = C0.shape[0]
    K = torch.zeros((N, N), dtype=torch.float64, device=C0.device)
    K[o:, :o] = kappa
    K = K - K.T
    return C0 @ torch.linalg.matrix_exp(-K)


def test_unrestricted_rotation_gradient_fd_64_directions(ctx):
    from mshqc_b200.autograd import mp2_energy
    N, oa, ob, M = 90, 10, 8, 220
    inp = twin(N, oa, M, seed=23, nocc_beta=ob)
    A, B = inp.alpha, inp.beta
    ctx.set_vectors(inp.L)
    Ca0, Cb0, ea, eb = t(A.C), t(B.C), t(A.eps), t(B.eps)

    def energy(ka, kb):
        return mp2_energy(ctx, rotated(Ca0, ka, oa), ea, oa, rotated(Cb0, kb, ob), eb, ob)

    ka = torch.zeros((N - oa, oa), dtype=torch.float64, device=DEV, requires_grad=True)
    kb = torch.zeros((N - ob, ob), dtype=torch.float64, device=DEV, requires_grad=True)
    energy(ka, kb).backward()
    ga, gb = ka.grad.clone(), kb.grad.clone()
    rng = np.random.default_rng(5)
    h = 1e-4
    worst = 0.0
    with torch.no_grad():
        for _ in range(64):
            da = t(rng.standard_normal((N - oa, oa)))
            db = t(rng.standard_normal((N - ob, ob)))
            nrm = float(torch.sqrt((da * da).sum() + (db * db).sum()))
            da, db = da / nrm, db / nrm
            ep = energy(h * da, h * db).item()
            em = energy(-h * da, -h * db).item()
            fd = (ep - em) / (2 * h)
            an = float((ga * da).sum() + (gb * db).sum())
            worst = max(worst, abs(fd - an))
    assert worst <= 1e-6, worst


def test_mixed_autograd_close_to_fp64(ctx):
    from mshqc_b200.autograd import mp2_energy
    inp = twin(131, 14, 300, seed=25, nocc_beta=12)
    A, B = inp.alpha, inp.beta
    ctx.set_vectors(inp.L)
    grads = {}
    for prec in ("fp64", "fp16x3"):
        Ca, Cb = t(A.C).requires_grad_(True), t(B.C).requires_grad_(True)
        E = mp2_energy(ctx, Ca, t(A.eps), A.nocc, Cb, t(B.eps), B.nocc, precision=prec)
        E.backward()
        grads[prec] = (E.item(), Ca.grad.cpu().numpy(), Cb.grad.cpu().numpy())
    e64, a64, b64 = grads["fp64"]
    e3, a3, b3 = grads["fp16x3"]
    assert abs(e3 - e64) <= 1e-6
    assert np.max(np.abs(a3 - a64)) <= 1e-6
    assert np.max(np.abs(b3 - b64)) <= 1e-6
