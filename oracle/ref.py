"""Oracle test infrastructure -- NOT part of the product.

ctypes access to oracle/_ref/libmshqc_ref.so, the reference's own
Cholesky-MP2 classes compiled from its sources by oracle/Makefile
(CholeskyRMP2 src/mp2/cholesky_rmp2.cc, CholeskyUMP2 src/mp2/cholesky_ump2.cc,
CholeskyOMP2 src/mp2/cholesky_omp2.cc, CholeskyERI src/integrals/cholesky_eri.cc).

Only tests, the smoke check and bench.py's reference / cpu_baseline legs use
this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libmshqc_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(
                f"{LIB_PATH} missing: build it with `make -C oracle` where the "
                "reference sources are present")
        lib = ctypes.CDLL(LIB_PATH)
        lib.ref_last_error.restype = ctypes.c_char_p
        i, d = ctypes.c_int, ctypes.c_double
        lib.ref_rmp2.argtypes = [i, i, _dp, _dp, _dp, i, d, i, _dp, _dp]
        lib.ref_ump2.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, i, i, d, i, _dp]
        lib.ref_omp2_pieces.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, i, i, _dp, i,
                                        _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.ref_omp2.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, i, i, _dp, d, i, d, d, i,
                                 _dp, _ip, _dp, _dp]
        lib.ref_cholesky_decompose.argtypes = [i, _dp, d, i, _dp, _ip]
        lib.ref_omp2_mp2_part.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, i, i, i, _dp]
        lib.ref_rhf_cdrmp2.argtypes = [i, i, _dp, _dp, _dp, _dp, _dp, _dp, d, d, d, i, _dp, _dp, _dp, _ip]
        lib.ref_cholesky_fock.argtypes = [i, i, _dp, i, _dp, _dp, _dp, i, _dp, _dp]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _f(a):
    """column-major float64 copy (Eigen layout)"""
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _c(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference harness: " + _load().ref_last_error().decode())


def rmp2(L, C, eps, nocc, e_scf=0.0, nthreads=0, want_t2=False):
    """Returns dict(e_corr, e_total, seconds[, t2 (o,o,v,v)])."""
    lib = _load()
    L = _c(L)
    M = L.shape[0]
    N = C.shape[0]
    C = _f(C)
    eps = _c(eps)
    out = np.zeros(3)
    v = N - nocc
    t2 = np.zeros((nocc, nocc, v, v), order="F") if want_t2 else None
    _check(lib.ref_rmp2(N, M, _p(L), _p(C), _p(eps), nocc, e_scf, nthreads, _p(out),
                        _p(t2) if want_t2 else None))
    res = dict(e_corr=out[0], e_total=out[1], seconds=out[2])
    if want_t2:
        res["t2"] = np.asarray(t2)
    return res


def ump2(L, Ca, Cb, ea, eb, na, nb, e_scf=0.0, nthreads=0):
    """Returns dict(ss_aa, ss_bb, os, e_corr, e_total, seconds)."""
    lib = _load()
    L = _c(L)
    M = L.shape[0]
    N = Ca.shape[0]
    Ca, Cb = _f(Ca), _f(Cb)
    ea, eb = _c(ea), _c(eb)
    out = np.zeros(6)
    _check(lib.ref_ump2(N, M, _p(L), _p(Ca), _p(Cb), _p(ea), _p(eb), na, nb, e_scf,
                        nthreads, _p(out)))
    return dict(ss_aa=out[0], ss_bb=out[1], os=out[2], e_corr=out[3], e_total=out[4],
                seconds=out[5])


def omp2_pieces(L, Ca, Cb, ea, eb, na, nb, H, nthreads=0):
    """One OMP2 gradient evaluation (t2, E, OPDM, generalized Fock, w_ai)."""
    lib = _load()
    L = _c(L)
    M = L.shape[0]
    N = Ca.shape[0]
    va, vb = N - na, N - nb
    Ca, Cb, H = _f(Ca), _f(Cb), _f(H)
    ea, eb = _c(ea), _c(eb)
    e = np.zeros(2)
    Gooa = np.zeros((na, na), order="F")
    Gvva = np.zeros((va, va), order="F")
    Goob = np.zeros((nb, nb), order="F")
    Gvvb = np.zeros((vb, vb), order="F")
    Fa = np.zeros((N, N), order="F")
    Fb = np.zeros((N, N), order="F")
    wa = np.zeros((va, na), order="F")
    wb = np.zeros((vb, nb), order="F")
    _check(lib.ref_omp2_pieces(N, M, _p(L), _p(Ca), _p(Cb), _p(ea), _p(eb), na, nb,
                               _p(H), nthreads, _p(e), _p(Gooa), _p(Gvva), _p(Goob),
                               _p(Gvvb), _p(Fa), _p(Fb), _p(wa), _p(wb)))
    return dict(e_mp2=e[0], seconds=e[1], Goo_a=Gooa, Gvv_a=Gvva, Goo_b=Goob,
                Gvv_b=Gvvb, F_a=Fa, F_b=Fb, w_a=wa, w_b=wb)


def rhf_cdrmp2(Z, xyz, S, T, V, eri, chol_thr=1e-6, e_thr=1e-12, d_thr=1e-10, nthreads=0):
    """The reference's RHF (src/scf/rhf.cc) and CholeskyRMP2 constructor 1
    (decomposes the ERI tensor itself, src/mp2/cholesky_rmp2.cc:20-41) on the
    given AO integrals; atoms Z, xyz (bohr).  Returns dict(e_scf, e_corr,
    n_vectors, iterations, converged, C (N, N), eps (N,), nocc)."""
    lib = _load()
    N = S.shape[0]
    Zc, X = _c(Z), _c(np.asarray(xyz).reshape(-1))
    S, T, V = _f(S), _f(T), _f(V)
    E = _c(np.asarray(eri).reshape(-1))
    out = np.zeros(5)
    C = np.zeros((N, N), order="F")
    eps = np.zeros(N)
    nocc = ctypes.c_int(0)
    _check(lib.ref_rhf_cdrmp2(N, len(Zc), _p(Zc), _p(X), _p(S), _p(T), _p(V), _p(E), chol_thr, e_thr, d_thr,
                              nthreads, _p(out), _p(C), _p(eps), ctypes.byref(nocc)))
    return dict(e_scf=out[0], e_corr=out[1], n_vectors=int(out[2]), iterations=int(out[3]),
                converged=bool(out[4]), C=C, eps=eps, nocc=nocc.value)


def omp2_mp2_part(L, Ca, Cb, ea, eb, na, nb, nthreads=0):
    """The MP2 part of one OMP2 gradient evaluation (transforms, t2, E, OPDM of
    both spins), timed inside the reference: dict(e_mp2, seconds)."""
    lib = _load()
    L = _c(L)
    M = L.shape[0]
    N = Ca.shape[0]
    Ca, Cb = _f(Ca), _f(Cb)
    ea, eb = _c(ea), _c(eb)
    out = np.zeros(2)
    _check(lib.ref_omp2_mp2_part(N, M, _p(L), _p(Ca), _p(Cb), _p(ea), _p(eb), na, nb, nthreads, _p(out)))
    return dict(e_mp2=out[0], seconds=out[1])


def omp2(L, Ca, Cb, ea, eb, na, nb, H, e_scf=0.0, max_iter=50, e_thr=1e-6,
         g_thr=1e-5, nthreads=0):
    lib = _load()
    L = _c(L)
    M = L.shape[0]
    N = Ca.shape[0]
    Ca, Cb, H = _f(Ca), _f(Cb), _f(H)
    ea, eb = _c(ea), _c(eb)
    out = np.zeros(4)
    iters = np.zeros(2, dtype=np.int32)
    Ca_out = np.zeros((N, N), order="F")
    Cb_out = np.zeros((N, N), order="F")
    _check(lib.ref_omp2(N, M, _p(L), _p(Ca), _p(Cb), _p(ea), _p(eb), na, nb, _p(H),
                        e_scf, max_iter, e_thr, g_thr, nthreads, _p(out),
                        iters.ctypes.data_as(_ip), _p(Ca_out), _p(Cb_out)))
    return dict(e_corr=out[0], e_total=out[1], e_scf=out[2], seconds=out[3],
                iterations=int(iters[0]), converged=bool(iters[1]), C_alpha=Ca_out,
                C_beta=Cb_out)


def cholesky_decompose(eri, threshold):
    """eri: (N,N,N,N) array indexed eri[i,j,k,l] = (ij|kl)."""
    lib = _load()
    N = eri.shape[0]
    E = _f(eri)
    cap = N * N
    Lout = np.zeros((cap, N * N))
    m = ctypes.c_int(0)
    _check(lib.ref_cholesky_decompose(N, _p(E), threshold, cap, _p(Lout), ctypes.byref(m)))
    return Lout[: m.value].copy()


def cholesky_fock(L, H, Pa, Pb=None, screen_exchange=True):
    """The reference's Cholesky Fock build on vectors L (M, N*N): with one
    density the CholeskyRHF build (src/scf/cholesky_rhf.cc:99-137,
    F = H + J - K/2, P the total density), with two the CholeskyUHF build
    (src/scf/cholesky_uhf.cc:77-103, F_s = H + J - K_s).  Returns F or
    (F_a, F_b), column-major N x N arrays."""
    lib = _load()
    L = np.ascontiguousarray(L, dtype=np.float64)
    M, nn = L.shape
    N = int(round(nn ** 0.5))
    f = lambda x: np.asfortranarray(x, dtype=np.float64)
    H, Pa = f(H), f(Pa)
    Pb_ = f(Pb) if Pb is not None else Pa
    Fa = np.zeros((N, N), order="F")
    Fb = np.zeros((N, N), order="F")
    ptr = lambda a: a.ctypes.data_as(_dp)
    rc = lib.ref_cholesky_fock(N, M, ptr(L), 1 if Pb is None else 2, ptr(Pa), ptr(Pb_), ptr(H),
                               1 if screen_exchange else 0, ptr(Fa), ptr(Fb))
    if rc != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    return Fa if Pb is None else (Fa, Fb)
