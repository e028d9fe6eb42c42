"""Generate the golden fixtures in this folder by running the REFERENCE's own
Cholesky-MP2 code (oracle/_ref/libmshqc_ref.so, built by `make -C oracle`
from the reference sources).  Inputs are stored alongside the outputs so the
fixtures do not depend on numpy's random streams.

    python tests/golden/make_golden.py

The reference ships no golden values of its own (its `python test/` scripts
only print), so these fixtures are the pins for the CPU restatement in
oracle/cdmp2_oracle.py and for the CUDA path.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mshqc_b200 import synthetic as syn  # noqa: E402
from oracle import ref  # noqa: E402


def _save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, sum(a.nbytes for a in map(np.asarray, arrays.values())), "bytes")


def restricted_case(name, N, o, M, seed, twin=False, t2=False):
    sigma = 1.0
    if twin:
        base = syn.make_inputs(N, o, M, seed=seed)
        sigma = syn.twin_sigma(N, o, M, base.alpha.eps)
    inp = syn.make_inputs(N, o, M, seed=seed, sigma=sigma)
    a = inp.alpha
    r = ref.rmp2(inp.L, a.C, a.eps, o, e_scf=-1.0, want_t2=t2)
    u = ref.ump2(inp.L, a.C, a.C, a.eps, a.eps, o, o, e_scf=-1.0)
    extra = dict(t2=r["t2"]) if t2 else {}
    _save(name, N=N, nocc=o, M=M, seed=seed, sigma=sigma, L=inp.L, C=a.C, eps=a.eps,
          e_corr=r["e_corr"], e_total=r["e_total"], ump2_ss_aa=u["ss_aa"],
          ump2_ss_bb=u["ss_bb"], ump2_os=u["os"], **extra)


def unrestricted_case(name, N, oa, ob, M, seed):
    inp = syn.make_inputs(N, oa, M, seed=seed, nocc_beta=ob)
    a, b = inp.alpha, inp.beta
    u = ref.ump2(inp.L, a.C, b.C, a.eps, b.eps, oa, ob, e_scf=-1.0)
    H = syn.default_core_hamiltonian(inp)
    p = ref.omp2_pieces(inp.L, a.C, b.C, a.eps, b.eps, oa, ob, H)
    _save(name, N=N, nocc_a=oa, nocc_b=ob, M=M, seed=seed, L=inp.L, Ca=a.C, Cb=b.C,
          ea=a.eps, eb=b.eps, H=H, ss_aa=u["ss_aa"], ss_bb=u["ss_bb"], os=u["os"],
          e_corr=u["e_corr"], omp2_e_mp2=p["e_mp2"], Goo_a=p["Goo_a"], Gvv_a=p["Gvv_a"],
          Goo_b=p["Goo_b"], Gvv_b=p["Gvv_b"], F_a=p["F_a"], F_b=p["F_b"], w_a=p["w_a"],
          w_b=p["w_b"])


def omp2_loop_case(name, N, o, M, seed):
    base = syn.make_inputs(N, o, M, seed=seed)
    sigma = syn.twin_sigma(N, o, M, base.alpha.eps)
    inp = syn.make_inputs(N, o, M, seed=seed, sigma=sigma)
    a = inp.alpha
    H = syn.default_core_hamiltonian(inp)
    r = ref.omp2(inp.L, a.C, a.C, a.eps, a.eps, o, o, H, e_scf=-1.0, max_iter=50)
    p = ref.omp2_pieces(inp.L, a.C, a.C, a.eps, a.eps, o, o, H)
    _save(name, N=N, nocc=o, M=M, seed=seed, sigma=sigma, L=inp.L, C=a.C, eps=a.eps, H=H,
          e_scf=-1.0, e_corr=r["e_corr"], e_total=r["e_total"], iterations=r["iterations"],
          converged=r["converged"], C_alpha=r["C_alpha"], w_a=p["w_a"], F_a=p["F_a"])


def degenerate_case(name):
    """Exactly zero denominators: the reference skips |D| < 1e-12 terms
    (src/mp2/cholesky_rmp2.cc:139, cholesky_ump2.cc:344)."""
    N, o, M = 10, 3, 30
    inp = syn.make_inputs(N, o, M, seed=7)
    a = inp.alpha
    eps = np.array([-1.0, 0.25, 0.5, 0.25, 0.5, 0.75, 1.0, 1.5, 2.0, 3.0])
    r = ref.rmp2(inp.L, a.C, eps, o, e_scf=0.0)
    u = ref.ump2(inp.L, a.C, a.C, eps, eps, o, o, e_scf=0.0)
    _save(name, N=N, nocc=o, M=M, L=inp.L, C=a.C, eps=eps, e_corr=r["e_corr"],
          ump2_ss_aa=u["ss_aa"], ump2_os=u["os"])


def single_occupied_case(name):
    """o = 1: the same-spin energy vanishes identically."""
    N, o, M = 12, 1, 40
    inp = syn.make_inputs(N, o, M, seed=11)
    a = inp.alpha
    r = ref.rmp2(inp.L, a.C, a.eps, o)
    u = ref.ump2(inp.L, a.C, a.C, a.eps, a.eps, o, o)
    _save(name, N=N, nocc=o, M=M, L=inp.L, C=a.C, eps=a.eps, e_corr=r["e_corr"],
          ump2_ss_aa=u["ss_aa"], ump2_os=u["os"])


def decompose_case(name):
    """Pivoted Cholesky (src/integrals/cholesky_eri.cc:40-203) of a synthetic
    8-fold-symmetric positive semidefinite ERI tensor of rank 40."""
    N, R = 8, 40
    rng = np.random.default_rng(5)
    X = rng.standard_normal((R, N, N))
    X = 0.5 * (X + X.transpose(0, 2, 1))
    X *= (10.0 ** (-3.0 * np.arange(R) / R))[:, None, None]
    eri = np.einsum("Pij,Pkl->ijkl", X, X)
    Lv = ref.cholesky_decompose(eri, 1e-6)
    _save(name, N=N, eri=eri, threshold=1e-6, L=Lv)


if __name__ == "__main__":
    if not ref.available():
        sys.exit("oracle/_ref/libmshqc_ref.so missing: run `make -C oracle` first")
    restricted_case("rmp2_n24_o5_m60", 24, 5, 60, seed=1, t2=True)
    restricted_case("rmp2_n32_o6_m96", 32, 6, 96, seed=2)
    restricted_case("rmp2_twin_n28_o5_m80", 28, 5, 80, seed=3, twin=True)
    restricted_case("rmp2_ragged_n29_o7_m61", 29, 7, 61, seed=4)
    unrestricted_case("ump2_n26_o6_5_m70", 26, 6, 5, 70, seed=5)
    unrestricted_case("ump2_n20_o4_3_m50", 20, 4, 3, 50, seed=2)
    omp2_loop_case("omp2_loop_twin_n20_o4_m50", 20, 4, 50, seed=3)
    degenerate_case("rmp2_zero_denominators")
    single_occupied_case("rmp2_single_occupied")
    decompose_case("cholesky_decompose_n8")
