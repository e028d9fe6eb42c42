"""ctypes binding of the C ABI in include/mshqc_cd.h (libmshqc_cuda.so).

This is the only way the Python side reaches the GPU: there is no CPU
fallback.  If the library is missing, importing this module still works (so
that CPU-only tooling can inspect it) but creating a Context raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libmshqc_cuda.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mshqc_cd.h")

OK = 0
ERR_ARG, ERR_STATE, ERR_CUDA, ERR_ALLOC, ERR_NUMERIC, ERR_UNSUPPORTED, ERR_TIMEOUT = (
    -1, -2, -3, -4, -5, -6, -7)
FP64, FP16X3 = 0, 1
RESTRICTED, UNRESTRICTED = 0, 1
LAYOUT_FULL, LAYOUT_PACKED = 0, 1
HOST, DEVICE = 0, 1
ALPHA, BETA = 0, 1

PRECISIONS = {"fp64": FP64, "fp16x3": FP16X3}


class CDError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Omp2Config(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_int), ("energy_threshold", ctypes.c_double),
                ("gradient_threshold", ctypes.c_double), ("e_scf", ctypes.c_double)]


class Omp2Result(ctypes.Structure):
    _fields_ = [("energy_scf", ctypes.c_double), ("energy_mp2_corr", ctypes.c_double),
                ("energy_total", ctypes.c_double), ("iterations", ctypes.c_int),
                ("converged", ctypes.c_int), ("ms_total", ctypes.c_double)]


class Energy(ctypes.Structure):
    _fields_ = [("ss_aa", ctypes.c_double), ("ss_bb", ctypes.c_double),
                ("os", ctypes.c_double), ("total", ctypes.c_double),
                ("ms_transform", ctypes.c_double), ("ms_energy", ctypes.c_double),
                ("ms_total", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = ctypes.c_void_p
_i32 = ctypes.c_int
_i64 = ctypes.c_int64
# name -> (restype, argtypes); the set of exported entry points
COLLECTIVE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int64, ctypes.c_void_p,
                                 ctypes.c_void_p)


class Collectives(ctypes.Structure):
    """mshqc_cd_collectives (include/mshqc_cd.h)."""
    _fields_ = [("allgather", COLLECTIVE_FN), ("reduce_scatter", COLLECTIVE_FN), ("user", ctypes.c_void_p)]


SIGNATURES = {
    "mshqc_cd_ctx_create": (_i32, [_i32, ctypes.POINTER(_vp)]),
    "mshqc_cd_ctx_destroy": (_i32, [_vp]),
    "mshqc_cd_last_error": (ctypes.c_char_p, []),
    "mshqc_cd_abi_version": (_i32, []),
    "mshqc_cd_set_stream": (_i32, [_vp, _vp]),
    "mshqc_cd_set_partition": (_i32, [_vp, _i32, _i32]),
    "mshqc_cd_device_bytes": (_i32, [_vp, ctypes.POINTER(_i64)]),
    "mshqc_cd_launch_count": (_i32, [_vp, ctypes.POINTER(_i64)]),
    "mshqc_cd_stage_times": (_i32, [_vp, ctypes.POINTER(ctypes.c_double), _i32]),
    "mshqc_cd_stage_counts": (_i32, [_vp, ctypes.POINTER(ctypes.c_int64), _i32]),
    "mshqc_cd_mixed_exact": (_i32, [_vp, ctypes.POINTER(_i32)]),
    "mshqc_cd_set_vectors": (_i32, [_vp, _vp, _i64, _i64, _i32, _i32]),
    "mshqc_cd_set_orbitals": (_i32, [_vp, _i32, _vp, _vp, _i64, _i32]),
    "mshqc_cd_transform": (_i32, [_vp, _i32, _i32, _vp, _i32]),
    "mshqc_cd_mp2_energy": (_i32, [_vp, _i32, _i32, ctypes.POINTER(Energy)]),
    "mshqc_cd_pair_energies": (_i32, [_vp, _i32, _vp, _i32]),
    "mshqc_cd_mp2_gradient": (_i32, [_vp, _i32, _i32, ctypes.POINTER(Energy), _vp, _vp, _vp,
                                     _vp, _i32]),
    "mshqc_cd_gen_vectors": (_i32, [_vp, _i64, _i64, ctypes.c_uint64, ctypes.c_double]),
    "mshqc_cd_cholesky_decompose": (_i32, [_vp, _vp, _i64, ctypes.c_double, _vp, _i64,
                                           ctypes.POINTER(_i64), ctypes.POINTER(_i32), _i32]),
    "mshqc_cd_set_core_hamiltonian": (_i32, [_vp, _vp, _i32]),
    "mshqc_cd_get_orbitals": (_i32, [_vp, _i32, _vp, _i32]),
    "mshqc_cd_omp2_pieces": (_i32, [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_double), _vp, _vp, _vp, _vp,
                                    _vp, _vp, _i32]),
    "mshqc_cd_omp2": (_i32, [_vp, ctypes.POINTER(Omp2Config), _vp, _vp, _i32, ctypes.POINTER(Omp2Result)]),
    "mshqc_cd_cholesky_fock": (_i32, [_vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp, _i32]),
    "mshqc_cd_rmp2_energy_noalloc": (_i32, [_vp, _vp, _i64, _i64, _i64, _vp, _vp]),
    "mshqc_cd_get_t2_block": (_i32, [_vp, _i32, _i64, _i64, _i64, _i64, _vp, _i32]),
    "mshqc_cd_set_collectives": (_i32, [_vp, ctypes.POINTER(Collectives)]),
    "mshqc_cd_cholesky_direct": (_i32, [_vp, _vp, ctypes.c_double, _vp, _i64, ctypes.POINTER(_i64),
                                        ctypes.POINTER(_i32), _i32]),
}

_lib = None


def library_available() -> bool:
    return os.path.exists(LIB_PATH)


def load_library():
    """Load libmshqc_cuda.so (fails loudly if it was not built)."""
    global _lib
    if _lib is None:
        if not library_available():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m mshqc_b200.build` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _check(rc: int):
    if rc != OK:
        raise CDError(rc, load_library().mshqc_cd_last_error().decode())


def _is_torch_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _host_f64(x, order="C"):
    a = np.asarray(x, dtype=np.float64)
    return np.asfortranarray(a) if order == "F" else np.ascontiguousarray(a)


def _ptr(a):
    if _is_torch_cuda(a):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Gradient:
    energy: dict
    dC_a: np.ndarray | None
    dC_b: np.ndarray | None
    deps_a: np.ndarray | None
    deps_b: np.ndarray | None


class Context:
    """One device context (stream + workspaces) of libmshqc_cuda."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        h = ctypes.c_void_p()
        _check(self._lib.mshqc_cd_ctx_create(device, ctypes.byref(h)))
        self._h = h
        self.device = device
        self.nbf = 0
        self.nvec = 0
        self.nocc = [0, 0]

    # -- lifecycle --------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.mshqc_cd_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_handle: int | None):
        _check(self._lib.mshqc_cd_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    def set_partition(self, rank: int, nranks: int):
        """Compute only share `rank` of `nranks` of the gradient's backward
        (sum the shares' energies and derivatives over the ranks)."""
        _check(self._lib.mshqc_cd_set_partition(self._h, int(rank), int(nranks)))
        return self

    def set_collectives(self, allgather, reduce_scatter):
        """Host collectives for a shared gradient (mshqc_cd_set_collectives):
        allgather(ptr, count, stream) and reduce_scatter(ptr, count, stream)
        act in place on `nranks * count` doubles of device memory at the
        integer address ptr, in the order of the CUDA stream handle `stream`.
        With a partition of more than one rank the half transforms and the
        transposed transforms are then shared too.  None clears them.  An
        exception in a callback fails the library call and is re-raised."""
        if allgather is None:
            self._coll = None
            _check(self._lib.mshqc_cd_set_collectives(self._h, None))
            return self
        self._coll_error = None

        def wrap(fn):
            def cb(buf, count, stream, user):
                try:
                    fn(ctypes.cast(buf, ctypes.c_void_p).value, int(count), stream or 0)
                    return 0
                except BaseException as ex:   # reported through the library's status
                    self._coll_error = ex
                    return 1
            return COLLECTIVE_FN(cb)

        cbs = (wrap(allgather), wrap(reduce_scatter))
        self._coll = (cbs, Collectives(cbs[0], cbs[1], None))
        _check(self._lib.mshqc_cd_set_collectives(self._h, ctypes.byref(self._coll[1])))
        return self

    def device_bytes(self) -> int:
        b = ctypes.c_int64(0)
        _check(self._lib.mshqc_cd_device_bytes(self._h, ctypes.byref(b)))
        return int(b.value)

    def launch_count(self) -> int:
        c = ctypes.c_int64(0)
        _check(self._lib.mshqc_cd_launch_count(self._h, ctypes.byref(c)))
        return int(c.value)

    STAGES = ("transform", "split", "pair_energy", "amplitude", "gamma", "transposed", "other",
              "amp_elem")

    def stage_times(self) -> dict:
        buf = (ctypes.c_double * 8)()
        _check(self._lib.mshqc_cd_stage_times(self._h, buf, 8))
        return {name: buf[k] for k, name in enumerate(self.STAGES)}

    def stage_counts(self) -> dict:
        """Timed intervals per stage of the last call (one per launch of the
        integral-tile and Gamma kernels of the mixed-precision backward)."""
        buf = (ctypes.c_int64 * 8)()
        _check(self._lib.mshqc_cd_stage_counts(self._h, buf, 8))
        return {name: int(buf[k]) for k, name in enumerate(self.STAGES)}

    def mixed_exact(self) -> bool:
        x = ctypes.c_int(0)
        _check(self._lib.mshqc_cd_mixed_exact(self._h, ctypes.byref(x)))
        return bool(x.value)

    # -- inputs -----------------------------------------------------------
    def set_vectors(self, L, nbf: int | None = None, layout: str = "full"):
        """L: (M, N*N) host array or CUDA tensor (or packed (M, N(N+1)/2))."""
        lay = LAYOUT_PACKED if layout == "packed" else LAYOUT_FULL
        if _is_torch_cuda(L):
            import torch
            L = L.to(torch.float64).contiguous()
            # the library copies on its own stream: the conversion (and the
            # caller's producer) on torch's current stream must be done first
            torch.cuda.current_stream(L.device).synchronize()
            where = DEVICE
        else:
            L = _host_f64(L)
            where = HOST
        M = L.shape[0]
        if nbf is None:
            per = L.shape[1] if L.ndim == 2 else int(np.prod(L.shape[1:]))
            nbf = int(round(per ** 0.5)) if lay == LAYOUT_FULL else int((np.sqrt(8 * per + 1) - 1) / 2)
        _check(self._lib.mshqc_cd_set_vectors(self._h, _ptr(L), int(nbf), int(M), lay, where))
        self.nbf, self.nvec = int(nbf), int(M)
        return self

    def cholesky_decompose(self, eri, threshold: float = 1e-6):
        """Pivoted Cholesky of eri[i, j, k, l] = (ij|kl) on the device; the
        vectors (M, N*N) are returned and become the context's vectors."""
        E = _host_f64(eri)
        N = E.shape[0]
        out = np.empty((N * N, N * N), dtype=np.float64)
        m = ctypes.c_int64(0)
        conv = ctypes.c_int(0)
        _check(self._lib.mshqc_cd_cholesky_decompose(self._h, _ptr(E), N, float(threshold), _ptr(out), N * N,
                                                      ctypes.byref(m), ctypes.byref(conv), HOST))
        self.nbf, self.nvec = N, int(m.value)
        self.decompose_converged = bool(conv.value)
        return out[:m.value].copy()

    def cholesky_direct(self, basis, threshold: float = 1e-6):
        """Integral-direct pivoted Cholesky over an ``ao.BasisSet``: the ERI
        diagonal and columns from the host AO engine, the decomposition on
        the device.  Returns the vectors (M, N*N); they become the
        context's vectors."""
        st, keep = basis._struct()
        N = basis.n_basis_functions()
        cap = N * N // 2 + 1
        out = np.empty((cap, N * N), dtype=np.float64)
        m = ctypes.c_int64(0)
        conv = ctypes.c_int(0)
        _check(self._lib.mshqc_cd_cholesky_direct(self._h, ctypes.addressof(st), float(threshold), _ptr(out), cap,
                                                  ctypes.byref(m), ctypes.byref(conv), HOST))
        self.nbf, self.nvec = N, int(m.value)
        self.decompose_converged = bool(conv.value)
        return out[:m.value].copy()

    def gen_vectors(self, nbf: int, nvec: int, seed: int, sigma: float = 1.0):
        """Synthetic vectors generated on the device (never stored); the
        numpy twin is synthetic.make_vectors_philox."""
        _check(self._lib.mshqc_cd_gen_vectors(self._h, int(nbf), int(nvec), int(seed), float(sigma)))
        self.nbf, self.nvec = int(nbf), int(nvec)
        return self

    def set_orbitals(self, spin: int, C, eps, nocc: int):
        """C[mu, p] (N x N), eps (N,), first nocc columns occupied."""
        if _is_torch_cuda(C):
            import torch
            Cc = C.to(torch.float64).t().contiguous()     # column-major bytes
            ec = eps.to(torch.float64).contiguous()
            # the transpose runs on torch's current stream, the library's copy
            # on its own: finish the transpose before handing over the pointer
            torch.cuda.current_stream(Cc.device).synchronize()
            where = DEVICE
        else:
            Cc = _host_f64(C, "F")
            ec = _host_f64(eps)
            where = HOST
        _check(self._lib.mshqc_cd_set_orbitals(self._h, spin, _ptr(Cc), _ptr(ec), int(nocc), where))
        self.nocc[spin] = int(nocc)
        return self

    # -- forward ----------------------------------------------------------
    def transform(self, spin: int = ALPHA, precision: int = FP64) -> np.ndarray:
        o = self.nocc[spin]
        v = self.nbf - o
        out = np.empty((o, v, self.nvec), dtype=np.float64)
        _check(self._lib.mshqc_cd_transform(self._h, spin, precision, _ptr(out), HOST))
        return out

    def mp2_energy(self, kind: int = RESTRICTED, precision: int = FP64) -> dict:
        e = Energy()
        _check(self._lib.mshqc_cd_mp2_energy(self._h, kind, precision, ctypes.byref(e)))
        return e.as_dict()

    def pair_energies(self, block: int = 0) -> np.ndarray:
        oa, ob = self.nocc
        rows, cols = {0: (oa, oa), 1: (ob, ob), 2: (oa, ob)}[block]
        out = np.empty((rows, cols), dtype=np.float64)
        _check(self._lib.mshqc_cd_pair_energies(self._h, block, _ptr(out), HOST))
        return out

    def t2_block(self, block: int = 0, i0: int = 0, ni: int | None = None, j0: int = 0,
                 nj: int | None = None) -> np.ndarray:
        """FP64 amplitudes t[i, j, a, b] = (ia|jb)/D of pairs i0 <= i < i0+ni,
        j0 <= j < j0+nj (block 0 alpha-alpha / restricted, 1 beta-beta,
        2 alpha-beta), as an (ni, nj, vx, vy) array."""
        oa, ob = self.nocc
        ox = ob if block == 1 else oa
        oy = oa if block == 0 else ob
        ni = ox - i0 if ni is None else ni
        nj = oy - j0 if nj is None else nj
        vx, vy = self.nbf - ox, self.nbf - oy
        out = np.empty((ni, nj, vx, vy), dtype=np.float64)
        _check(self._lib.mshqc_cd_get_t2_block(self._h, block, i0, ni, j0, nj, _ptr(out), HOST))
        return out

    # -- backward ---------------------------------------------------------
    def _grad_call(self, fn):
        self._coll_error = None
        rc = fn()
        err = getattr(self, "_coll_error", None)
        if err is not None:
            self._coll_error = None
            raise err
        _check(rc)

    def mp2_gradient(self, kind: int = RESTRICTED, precision: int = FP64) -> Gradient:
        N = self.nbf
        e = Energy()
        dCa = np.zeros((N, N), dtype=np.float64, order="F")
        dea = np.zeros(N, dtype=np.float64)
        if kind == UNRESTRICTED:
            dCb = np.zeros((N, N), dtype=np.float64, order="F")
            deb = np.zeros(N, dtype=np.float64)
        else:
            dCb = deb = None
        self._grad_call(lambda: self._lib.mshqc_cd_mp2_gradient(
            self._h, kind, precision, ctypes.byref(e), _ptr(dCa),
            _ptr(dCb) if dCb is not None else None, _ptr(dea),
            _ptr(deb) if deb is not None else None, HOST))
        return Gradient(e.as_dict(), dCa, dCb, dea, deb)

    def mp2_gradient_torch(self, kind: int = RESTRICTED, precision: int = FP64, device=None) -> Gradient:
        """mp2_gradient with the derivatives written straight into CUDA
        tensors on `device` (default: the context's GPU; dC as an (N, N)
        tensor dC[mu, p])."""
        import torch
        if device is None:
            device = torch.device("cuda", self.device)
        N = self.nbf
        e = Energy()
        nspin = 2 if kind == UNRESTRICTED else 1
        dCt = [torch.empty((N, N), dtype=torch.float64, device=device) for _ in range(nspin)]
        de = [torch.empty(N, dtype=torch.float64, device=device) for _ in range(nspin)]
        torch.cuda.current_stream(device).synchronize()
        self._grad_call(lambda: self._lib.mshqc_cd_mp2_gradient(
            self._h, kind, precision, ctypes.byref(e), _ptr(dCt[0]), _ptr(dCt[1]) if nspin == 2 else None,
            _ptr(de[0]), _ptr(de[1]) if nspin == 2 else None, DEVICE))
        # the library writes column-major dC: the tensor holds dC^T
        dC = [t.t() for t in dCt]
        return Gradient(e.as_dict(), dC[0], dC[1] if nspin == 2 else None, de[0],
                        de[1] if nspin == 2 else None)

    # -- CD-OMP2 ------------------------------------------------------------
    def set_core_hamiltonian(self, H):
        """Core Hamiltonian (N x N, symmetric) of the OMP2 generalized Fock."""
        Hc = _host_f64(H)
        _check(self._lib.mshqc_cd_set_core_hamiltonian(self._h, _ptr(Hc), HOST))
        return self

    def get_orbitals(self, spin: int = ALPHA) -> np.ndarray:
        N = self.nbf
        C = np.empty((N, N), dtype=np.float64, order="F")
        _check(self._lib.mshqc_cd_get_orbitals(self._h, spin, _ptr(C), HOST))
        return C

    def _densities(self, P_a, P_b):
        pa = _host_f64(P_a, "F") if P_a is not None else None
        pb = _host_f64(P_b, "F") if P_b is not None else None
        return pa, pb, (_ptr(pa) if pa is not None else None), (_ptr(pb) if pb is not None else None)

    def omp2_pieces(self, P_a=None, P_b=None) -> dict:
        """One CholeskyOMP2 gradient evaluation: e_mp2, G_oo / G_vv per spin,
        F_mo per spin (N x N) and w_ai = 2 F(o+a, i)."""
        N = self.nbf
        oa, ob = self.nocc
        out = {"Goo_a": np.empty((oa, oa)), "Gvv_a": np.empty((N - oa, N - oa)),
               "Goo_b": np.empty((ob, ob)), "Gvv_b": np.empty((N - ob, N - ob)),
               "F_a": np.empty((N, N), order="F"), "F_b": np.empty((N, N), order="F")}
        e = ctypes.c_double()
        pa, pb, ppa, ppb = self._densities(P_a, P_b)
        _check(self._lib.mshqc_cd_omp2_pieces(
            self._h, ppa, ppb, ctypes.byref(e), _ptr(out["Goo_a"]), _ptr(out["Gvv_a"]),
            _ptr(out["Goo_b"]), _ptr(out["Gvv_b"]), _ptr(out["F_a"]), _ptr(out["F_b"]), HOST))
        out["e_mp2"] = e.value
        out["w_a"] = 2.0 * out["F_a"][oa:, :oa]
        out["w_b"] = 2.0 * out["F_b"][ob:, :ob]
        return out

    def cholesky_fock(self, H, P_a, P_b=None, screen_exchange: bool = True) -> dict:
        """Cholesky Fock build on the context's vectors: with one density the
        CholeskyRHF build (P_a the total density, F = H + J - K/2), with two
        the CholeskyUHF build (F_s = H + J - K_s).  Returns J, K_a, F_a (and
        K_b, F_b), N x N column-major."""
        N = self.nbf
        f = lambda x: np.asfortranarray(x, dtype=np.float64)
        H, P_a = f(H), f(P_a)
        nspin = 1 if P_b is None else 2
        P_b = f(P_b) if P_b is not None else None
        out = {k: np.empty((N, N), order="F") for k in ("J", "K_a", "F_a")}
        if nspin == 2:
            out.update({k: np.empty((N, N), order="F") for k in ("K_b", "F_b")})
        _check(self._lib.mshqc_cd_cholesky_fock(
            self._h, nspin, _ptr(P_a), _ptr(P_b) if P_b is not None else None, _ptr(H),
            1 if screen_exchange else 0, _ptr(out["F_a"]), _ptr(out["F_b"]) if nspin == 2 else None,
            _ptr(out["J"]), _ptr(out["K_a"]), _ptr(out["K_b"]) if nspin == 2 else None, HOST))
        return out

    def omp2(self, max_iterations: int = 50, energy_threshold: float = 1e-6,
             gradient_threshold: float = 1e-5, e_scf: float = 0.0, P_a=None, P_b=None) -> dict:
        """CholeskyOMP2::compute; the rotated orbitals stay in the context."""
        cfg = Omp2Config(int(max_iterations), float(energy_threshold), float(gradient_threshold),
                         float(e_scf))
        res = Omp2Result()
        pa, pb, ppa, ppb = self._densities(P_a, P_b)
        _check(self._lib.mshqc_cd_omp2(self._h, ctypes.byref(cfg), ppa, ppb, HOST, ctypes.byref(res)))
        return {"energy_scf": res.energy_scf, "energy_mp2_corr": res.energy_mp2_corr,
                "energy_total": res.energy_total, "iterations": res.iterations,
                "converged": bool(res.converged), "ms_total": res.ms_total,
                "C_alpha": self.get_orbitals(ALPHA), "C_beta": self.get_orbitals(BETA)}


def noalloc_shape(nocc: int, nvir: int, nvec: int) -> tuple[int, int, int]:
    """Shape (nocc, vp, Mp) of the zero-padded MO vectors that
    mshqc_cd_rmp2_energy_noalloc reads."""
    return nocc, -(-nvir // 64) * 64, -(-nvec // 16) * 16


def rmp2_energy_noalloc(B, eps, nocc: int, nvir: int, nvec: int, energy, stream=None) -> None:
    """Queue the allocation-free FP64 closed-shell energy on CUDA tensors.

    B: float64 CUDA tensor of noalloc_shape(nocc, nvir, nvec), zero padded;
    eps: float64 CUDA tensor (nocc + nvir,); energy: float64 CUDA tensor (2,)
    receiving [E_corr, opposite-spin part] in stream order.  stream: a
    torch.cuda.Stream (default: the current stream).  Nothing is allocated
    by the call; synchronize the stream before reading energy."""
    import torch
    for name, t in (("B", B), ("eps", eps), ("energy", energy)):
        if not (_is_torch_cuda(t) and t.dtype == torch.float64 and t.is_contiguous()):
            raise ValueError(f"{name} must be a contiguous float64 CUDA tensor")
    if tuple(B.shape) != noalloc_shape(nocc, nvir, nvec):
        raise ValueError(f"B has shape {tuple(B.shape)}, expected {noalloc_shape(nocc, nvir, nvec)}")
    if stream is None:
        stream = torch.cuda.current_stream(B.device)
    with torch.cuda.device(B.device):
        _check(load_library().mshqc_cd_rmp2_energy_noalloc(
            B.data_ptr(), eps.data_ptr(), nocc, nvir, nvec, energy.data_ptr(), stream.cuda_stream))


def exported_symbols_from_header(path: str = HEADER) -> list[str]:
    """Function names declared with MSHQC_CD_API in include/mshqc_cd.h."""
    import re
    txt = open(path).read()
    return sorted(set(re.findall(r"MSHQC_CD_API\s+[\w\s\*]*?\b(mshqc_cd_\w+)\s*\(", txt)))
