"""Seeded synthetic Cholesky-MP2 inputs.

The recipe (used for every synthetic workload of this package):

* Cholesky vectors ``L^Q = s_Q * G^Q`` with ``G^Q = (X + X^T)/2``,
  ``X ~ N(0,1)`` (N x N), and ``s_Q = 10**(-6 Q / M)`` for ``Q = 0..M-1``.
  Stored as the reference's ``CholeskyERI`` does: M vectors of length N*N,
  index ``mu*N + nu`` (reference include/mshqc/integrals/cholesky_eri.h:81, :89-91).
* MO coefficients ``C``: the Q factor of the QR decomposition of a Gaussian
  N x N matrix (column-major on the C-ABI, Eigen convention).
* Occupied energies uniform in [-2.0, -0.3] Eh with the 4 lowest set to
  -20 Eh; virtual energies log-uniform in [0.05, 5] Eh; sorted ascending so
  that the first ``nocc`` columns of C are the occupied orbitals
  (``leftCols(nocc)`` in reference src/mp2/cholesky_rmp2.cc:77-78).
* ``sigma`` scales L (``L -> sigma*L``, E_corr scales as sigma**4).  The
  "scaled twin" picks sigma so that |E_corr| is about 0.05*o Eh, where an
  absolute micro-Hartree tolerance is meaningful.

Generation order is fixed so a seed reproduces bit-identical arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class SpinOrbitals:
    C: np.ndarray      # (N, N) float64, C[mu, p]
    eps: np.ndarray    # (N,) float64, ascending
    nocc: int


@dataclass
class CDInputs:
    N: int
    M: int
    L: np.ndarray                  # (M, N*N) float64, index mu*N+nu
    alpha: SpinOrbitals
    beta: SpinOrbitals | None = None
    sigma: float = 1.0
    seed: int = 0
    H: np.ndarray | None = field(default=None, repr=False)  # core Hamiltonian (optional)

    @property
    def restricted(self) -> bool:
        return self.beta is None


def scale_factors(M: int) -> np.ndarray:
    q = np.arange(M, dtype=np.float64)
    return 10.0 ** (-6.0 * q / M)


def _orbital_energies(rng: np.random.Generator, N: int, nocc: int) -> np.ndarray:
    n_low = min(4, nocc)
    occ = rng.uniform(-2.0, -0.3, size=nocc)
    occ.sort()
    occ[:n_low] = -20.0
    vir = np.exp(rng.uniform(math.log(0.05), math.log(5.0), size=N - nocc))
    vir.sort()
    return np.concatenate([occ, vir])


def _orthogonal(rng: np.random.Generator, N: int) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((N, N)))
    # fix the sign convention so the factor is unique for a given matrix
    q *= np.sign(np.diag(r))[None, :]
    return np.ascontiguousarray(q)


def make_vectors(rng: np.random.Generator, N: int, M: int, sigma: float = 1.0,
                 dtype=np.float64, chunk: int = 64) -> np.ndarray:
    """L as (M, N*N): L^Q = sigma * s_Q * (X + X^T)/2, X ~ N(0,1)."""
    s = scale_factors(M) * sigma
    L = np.empty((M, N * N), dtype=dtype)
    for q0 in range(0, M, chunk):
        q1 = min(M, q0 + chunk)
        X = rng.standard_normal((q1 - q0, N, N))
        G = 0.5 * (X + X.transpose(0, 2, 1))
        G *= s[q0:q1, None, None]
        L[q0:q1] = G.reshape(q1 - q0, N * N)
    return L


def make_inputs(N: int, nocc: int, M: int, seed: int = 0, sigma: float = 1.0,
                nocc_beta: int | None = None, dtype=np.float64) -> CDInputs:
    """Restricted inputs when ``nocc_beta`` is None, else separate alpha/beta
    orbitals (distinct random orthogonal C_alpha, C_beta) sharing L."""
    rng = np.random.default_rng(seed)
    L = make_vectors(rng, N, M, sigma, dtype=dtype)
    Ca = _orthogonal(rng, N)
    ea = _orbital_energies(rng, N, nocc)
    alpha = SpinOrbitals(Ca, ea, nocc)
    beta = None
    if nocc_beta is not None:
        Cb = _orthogonal(rng, N)
        eb = _orbital_energies(rng, N, nocc_beta)
        beta = SpinOrbitals(Cb, eb, nocc_beta)
    return CDInputs(N=N, M=M, L=L, alpha=alpha, beta=beta, sigma=sigma, seed=seed)


def mean_inverse_denominator(eps_occ_i, eps_vir_a, eps_occ_j, eps_vir_b,
                             samples: int = 1 << 20, seed: int = 12345) -> float:
    rng = np.random.default_rng(seed)
    i = rng.integers(0, len(eps_occ_i), samples)
    j = rng.integers(0, len(eps_occ_j), samples)
    a = rng.integers(0, len(eps_vir_a), samples)
    b = rng.integers(0, len(eps_vir_b), samples)
    d = eps_occ_i[i] + eps_occ_j[j] - eps_vir_a[a] - eps_vir_b[b]
    return float(np.mean(1.0 / d))


def twin_sigma(N: int, nocc: int, M: int, eps: np.ndarray,
               target_per_occ: float = 0.05) -> float:
    """sigma for which the recipe's expected |E_corr| is about target*o Eh.

    Model: B^Q_ia ~ N(0, s_Q^2/2) for an orthogonal C (the symmetrised
    Gaussian has off-diagonal variance 1/2 and is rotation invariant), so
    Var((ia|jb)) = sum_Q s_Q^4 / 4 and E ~ 2 o^2 v^2 Var <1/D>.
    """
    v = N - nocc
    s4 = float(np.sum(scale_factors(M) ** 4))
    var = s4 / 4.0
    inv_d = abs(mean_inverse_denominator(eps[:nocc], eps[nocc:], eps[:nocc], eps[nocc:]))
    e1 = 2.0 * nocc * nocc * v * v * var * inv_d
    return (target_per_occ * nocc / e1) ** 0.25


def default_core_hamiltonian(inp: CDInputs) -> np.ndarray:
    """H such that the reference-density Fock operator of spin alpha is
    C diag(eps) C^T (an orthonormal AO basis, S = I):
    H = C_a diag(eps_a) C_a^T - J[P_a + P_b] + K[P_a], with the Cholesky J/K of
    reference src/mp2/cholesky_omp2.cc:347-358."""
    N = inp.N
    a = inp.alpha
    b = inp.beta if inp.beta is not None else inp.alpha
    Pa = a.C[:, :a.nocc] @ a.C[:, :a.nocc].T
    Pb = b.C[:, :b.nocc] @ b.C[:, :b.nocc].T
    Ptot = Pa + Pb
    L3 = inp.L.reshape(inp.M, N, N)
    J = np.zeros((N, N))
    K = np.zeros((N, N))
    for q in range(inp.M):
        Lq = L3[q].T  # Eigen column-major map of the vector
        J += np.sum(Lq * Ptot) * Lq
        K += Lq @ Pa @ Lq
    F = (a.C * a.eps[None, :]) @ a.C.T
    return F - J + K


def make_vectors_device(N: int, M: int, seed: int, sigma: float, device, chunk: int = 64):
    """The same recipe as make_vectors, drawn on the device with a seeded
    torch (Philox) generator: L^Q = sigma s_Q (X + X^T)/2.  Returns an (M, N*N)
    float64 CUDA tensor.  Used for workloads too large to draw on the host;
    the stream differs from numpy's, the distribution is the same."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    s = torch.from_numpy(scale_factors(M) * sigma).to(device)
    L = torch.empty((M, N * N), dtype=torch.float64, device=device)
    for q0 in range(0, M, chunk):
        q1 = min(M, q0 + chunk)
        X = torch.randn((q1 - q0, N, N), dtype=torch.float64, device=device, generator=g)
        X = 0.5 * (X + X.transpose(1, 2))
        X *= s[q0:q1, None, None]
        L[q0:q1] = X.reshape(q1 - q0, N * N)
        del X
    return L


_PHILOX_M = (np.uint64(0xD2511F53), np.uint64(0xCD9E8D57))
_PHILOX_W = (np.uint32(0x9E3779B9), np.uint32(0xBB67AE85))
_MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr: np.ndarray, seed: int) -> tuple:
    """Philox4x32-10 (Salmon et al., SC 2011) of the 64-bit counters `ctr`
    (words (ctr_lo, ctr_hi, 0, 0)) under key `seed`; four uint32 arrays."""
    ctr = np.asarray(ctr, dtype=np.uint64)
    c0 = (ctr & _MASK32).astype(np.uint32)
    c1 = (ctr >> np.uint64(32)).astype(np.uint32)
    return philox4x32_10_words(c0, c1, np.zeros_like(c0), np.zeros_like(c0),
                               seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)


def philox4x32_10_words(c0, c1, c2, c3, key0: int, key1: int) -> tuple:
    """The ten Philox4x32 rounds on counter words c0..c3 (uint32 arrays) and
    key (key0, key1): per round (hi0, lo0) = M0 c0, (hi1, lo1) = M1 c2,
    c <- (hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0), then the key grows by the
    Weyl constants."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint32) for c in (c0, c1, c2, c3))
    k0 = np.uint32(key0)
    k1 = np.uint32(key1)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = _PHILOX_M[0] * c0.astype(np.uint64)
            p1 = _PHILOX_M[1] * c2.astype(np.uint64)
            hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & _MASK32).astype(np.uint32)
            hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & _MASK32).astype(np.uint32)
            c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
            k0 = np.uint32(k0 + _PHILOX_W[0])
            k1 = np.uint32(k1 + _PHILOX_W[1])
    return c0, c1, c2, c3


def philox_normal_pair(ctr: np.ndarray, seed: int) -> tuple:
    """Box-Muller pair of independent standard normals from one Philox block
    per counter: r = sqrt(-2 ln u1), (r cos 2 pi u2, r sin 2 pi u2), with u1
    from the first 64 output bits and u2 from the second."""
    c0, c1, c2, c3 = philox4x32_10(ctr, seed)
    a = (c0.astype(np.uint64) << np.uint64(32)) | c1.astype(np.uint64)
    b = (c2.astype(np.uint64) << np.uint64(32)) | c3.astype(np.uint64)
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
    u2 = ((b >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
    r = np.sqrt(-2.0 * np.log(u1))
    return r * np.cos(6.283185307179586 * u2), r * np.sin(6.283185307179586 * u2)


def philox_normal(ctr: np.ndarray, seed: int) -> np.ndarray:
    """The first (cosine) member of philox_normal_pair."""
    return philox_normal_pair(ctr, seed)[0]


def make_vectors_philox(N: int, M: int, seed: int, sigma: float = 1.0) -> np.ndarray:
    """The recipe as the library's device generator draws it
    (mshqc_cd_gen_vectors): for mu < nu one Philox block with counter
    (Q N + mu) N + nu gives the Box-Muller pair (X^Q_{mu nu}, X^Q_{nu mu}), the
    diagonal X^Q_{mu mu} is the cosine member of counter (Q N + mu) N + mu, and
    L^Q = sigma 10^(-6Q/M) (X + X^T)/2.  (M, N*N) float64; for small sizes."""
    s = scale_factors(M) * sigma
    L = np.empty((M, N * N), dtype=np.float64)
    mu = np.arange(N, dtype=np.uint64)[:, None]
    nu = np.arange(N, dtype=np.uint64)[None, :]
    for q in range(M):
        base = np.uint64(q) * np.uint64(N)
        Zc, Zs = philox_normal_pair((base + mu) * np.uint64(N) + nu, seed)
        X = np.triu(Zc, 1) + np.triu(Zs, 1).T + np.diag(np.diag(Zc))
        L[q] = (s[q] * (0.5 * (X + X.T))).reshape(N * N)
    return L


def make_orbitals(N: int, nocc: int, seed: int) -> SpinOrbitals:
    rng = np.random.default_rng(seed)
    return SpinOrbitals(_orthogonal(rng, N), _orbital_energies(rng, N, nocc), nocc)
