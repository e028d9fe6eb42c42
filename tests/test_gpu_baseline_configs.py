"""Parity at the benchmark configurations themselves (seeded synthetic
recipe of mshqc_b200/synthetic.py; |E_corr| of the raw recipe is ~1e8 Eh, so
absolute uEh errors are stated on its scaled twin L -> sigma L with
|E_corr| ~ 0.05 o Eh):

* N=400, o=40, M=1600 (CD-RMP2 energy): the FP64 GPU energy against the
  reference's own CholeskyRMP2 (oracle/_ref, src/mp2/cholesky_rmp2.cc:97-179)
  run in the same test, to 1e-9 Eh absolute and 1e-12 relative on the twin;
  the mixed-precision energy to <= 1 uEh of both; on the raw recipe FP64
  against the numpy oracle to 1e-12 relative and mixed to 1e-6 relative.
* N=1000, o=100, M=4000 (mixed CD-RMP2 energy, vectors generated on the
  device): mixed against FP64 GPU, <= 1 uEh on the twin, 1e-6 relative raw.
* N=600, o=60/58, M=2400 (differentiated CD-UMP2, separate alpha / beta
  orbitals): the mixed-precision backward through the torch.autograd.Function
  against central finite differences (step 1e-4) of the FP64 energy along 64
  random orbital rotations, tolerance 1e-6; and the OMP2 gradient w_ai of the
  GPU against the reference's CholeskyOMP2 (src/mp2/cholesky_omp2.cc:441-466)
  at N=180, o=18/17, M=720, where the reference's stored t2 stays small.
Each test prints the errors it measured.
"""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc
from oracle import ref

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def twin_sigma_for(N, o, M, seed):
    base = syn.make_orbitals(N, o, seed)
    return syn.twin_sigma(N, o, M, base.eps)


def twin(N, o, M, seed, nocc_beta=None):
    base = syn.make_inputs(N, o, M, seed=seed, nocc_beta=nocc_beta)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    return syn.make_inputs(N, o, M, seed=seed, sigma=sig, nocc_beta=nocc_beta)


@needs_ref
def test_config2_fp64_and_mixed_against_reference_cdrmp2():
    N, o, M = 400, 40, 1600
    inp = twin(N, o, M, seed=0)
    a = inp.alpha
    r = ref.rmp2(inp.L, a.C, a.eps, o)
    with capi.Context(0) as ctx:
        ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
        e64 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
        e3 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)["total"]
    d64, d3 = abs(e64 - r["e_corr"]), abs(e3 - r["e_corr"])
    print(f"\nconfig 2 twin: reference {r['e_corr']:.12f} Eh ({r['seconds']:.1f} s); "
          f"FP64 GPU error {d64:.2e} Eh ({d64 / abs(r['e_corr']):.1e} rel); mixed error {d3 * 1e6:.4f} uEh; "
          f"mixed - FP64 {abs(e3 - e64) * 1e6:.4f} uEh")
    assert d64 <= 1e-9
    assert d64 <= 1e-12 * abs(r["e_corr"])
    assert d3 <= 1e-6
    assert abs(e3 - e64) <= 1e-6


def test_config2_raw_recipe_against_numpy_oracle():
    N, o, M = 400, 40, 1600
    inp = syn.make_inputs(N, o, M, seed=0)
    a = inp.alpha
    E, _ = orc.rmp2_energy(orc.transform(inp.L, a.C, o), a.eps, o)
    with capi.Context(0) as ctx:
        ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
        e64 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
        e3 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)["total"]
    r64, r3 = abs(e64 - E) / abs(E), abs(e3 - E) / abs(E)
    print(f"\nconfig 2 raw: E {E:.10e}; FP64 rel {r64:.1e}; mixed rel {r3:.1e}")
    assert r64 <= 1e-12
    assert r3 <= 1e-6


@pytest.mark.parametrize("scaled", [True, False])
def test_config3_mixed_against_fp64(scaled):
    N, o, M, seed = 1000, 100, 4000, 3
    sigma = twin_sigma_for(N, o, M, seed) if scaled else 1.0
    orb = syn.make_orbitals(N, o, seed)
    with capi.Context(0) as ctx:
        ctx.gen_vectors(N, M, seed, sigma)
        ctx.set_orbitals(capi.ALPHA, orb.C, orb.eps, o)
        e64 = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)["total"]
        e3 = ctx.mp2_energy(capi.RESTRICTED, capi.FP16X3)["total"]
    d = abs(e3 - e64)
    print(f"\nconfig 3 {'twin' if scaled else 'raw'}: FP64 {e64:.12e} Eh; mixed - FP64 {d * 1e6:.4f} uEh "
          f"({d / abs(e64):.1e} rel)")
    if scaled:
        assert d <= 1e-6
    else:
        assert d <= 1e-6 * abs(e64)


def _rotated(C0, kappa, o):
    """C0 exp(-K), K antisymmetric with K[o + a, i] = kappa[a, i]."""
    N = C0.shape[0]
    K = torch.zeros((N, N), dtype=torch.float64, device=C0.device)
    K[o:, :o] = kappa
    K = K - K.T
    return C0 @ torch.linalg.matrix_exp(-K)


def test_config4_mixed_backward_against_fd_64_rotations():
    from mshqc_b200.autograd import mp2_energy
    N, oa, ob, M, seed = 600, 60, 58, 2400, 4
    sigma = twin_sigma_for(N, oa, M, seed)
    A = syn.make_orbitals(N, oa, seed)
    B = syn.make_orbitals(N, ob, seed + 7919)          # separate random orthogonal C_beta
    dev = "cuda:0"
    tt = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    Ca0, Cb0, ea, eb = tt(A.C), tt(B.C), tt(A.eps), tt(B.eps)
    with capi.Context(0) as ctx:
        ctx.gen_vectors(N, M, seed, sigma)

        def energy(ka, kb, precision):
            return mp2_energy(ctx, _rotated(Ca0, ka, oa), ea, oa, _rotated(Cb0, kb, ob), eb, ob,
                              precision=precision)

        ka = torch.zeros((N - oa, oa), dtype=torch.float64, device=dev, requires_grad=True)
        kb = torch.zeros((N - ob, ob), dtype=torch.float64, device=dev, requires_grad=True)
        energy(ka, kb, "fp16x3").backward()
        ga, gb = ka.grad.clone(), kb.grad.clone()
        rng = np.random.default_rng(5)
        h = 1e-4
        worst, biggest = 0.0, 0.0
        with torch.no_grad():
            for _ in range(64):
                da = tt(rng.standard_normal((N - oa, oa)))
                db = tt(rng.standard_normal((N - ob, ob)))
                nrm = float(torch.sqrt((da * da).sum() + (db * db).sum()))
                da, db = da / nrm, db / nrm
                ep = energy(h * da, h * db, "fp64").item()
                em = energy(-h * da, -h * db, "fp64").item()
                fd = (ep - em) / (2 * h)
                an = float((ga * da).sum() + (gb * db).sum())
                worst = max(worst, abs(fd - an))
                biggest = max(biggest, abs(fd))
    print(f"\nconfig 4: 64 rotations, max |FD - mixed backward| {worst:.2e} (largest |FD| {biggest:.2e})")
    assert worst <= 1e-6


@needs_ref
def test_config4_omp2_gradient_against_reference():
    N, oa, ob, M = 180, 18, 17, 720
    inp = twin(N, oa, M, seed=4, nocc_beta=ob)
    A, B = inp.alpha, inp.beta                             # separate random orthogonal C_alpha, C_beta
    H = syn.default_core_hamiltonian(inp)
    r = ref.omp2_pieces(inp.L, A.C, B.C, A.eps, B.eps, oa, ob, H)
    with capi.Context(0) as ctx:
        ctx.set_vectors(inp.L)
        ctx.set_orbitals(capi.ALPHA, A.C, A.eps, oa)
        ctx.set_orbitals(capi.BETA, B.C, B.eps, ob)
        ctx.set_core_hamiltonian(H)
        g = ctx.omp2_pieces()
    wa = 2.0 * g["F_a"][oa:, :oa]
    wb = 2.0 * g["F_b"][ob:, :ob]
    ea = np.max(np.abs(wa - r["w_a"])) / np.max(np.abs(r["w_a"]))
    eb = np.max(np.abs(wb - r["w_b"])) / np.max(np.abs(r["w_b"]))
    de = abs(g["e_mp2"] - r["e_mp2"])
    print(f"\nconfig 4 shape ratios at N={N}: E_mp2 error {de:.2e} Eh; w_ai relative error alpha {ea:.1e}, "
          f"beta {eb:.1e} (reference {r['seconds']:.1f} s)")
    assert de <= 1e-12 * abs(r["e_mp2"])
    assert ea <= 1e-10 and eb <= 1e-10
