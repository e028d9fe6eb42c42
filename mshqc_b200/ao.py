"""AO integrals on the host: the integral engine under the Cholesky-MP2 path.

The reference computes S, T, V and the ERI tensor with libint2 behind its
``IntegralEngine`` (include/mshqc/integrals.h:38-224, src/core/integrals.cc)
and reads basis sets from Gaussian94 files (src/core/basis.cc:114-245).  This
module gives the same pieces over the library's own engine
(``mshqc_ao_*`` in libmshqc_cuda.so, include/mshqc_ao.h; host code only):

* ``parse_g94(text)``    element -> list of (l, exponents, coefficients), the
                         reference's reader (``SP`` shells split into S and P);
* ``Molecule``           atoms (Z, position in bohr), built from Angstrom with
                         the reference's conversion 1.88972612457
                         (include/mshqc/molecule.h:192) unless told otherwise;
* ``BasisSet``           shells on the atoms, coefficients normalized like
                         the reference's Shell::normalize, all pure
                         (spherical) unless the file or caller says Cartesian;
* ``IntegralEngine``     compute_overlap / compute_kinetic / compute_nuclear /
                         compute_core_hamiltonian / compute_eri /
                         compute_eri_diagonal / compute_eri_column and
                         nuclear_repulsion_energy, numpy arrays in the
                         reference's layouts.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import capi

ANGSTROM_TO_BOHR = 1.88972612457          # reference include/mshqc/molecule.h:192
AM = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "I": 6}
ELEMENTS = ["X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl",
            "Ar"]


def parse_g94(text: str) -> tuple[dict, bool]:
    """Gaussian94 basis text -> ({element: [(l, exps, coefs), ...]}, spherical).

    A file whose header names "cartesian" is Cartesian, otherwise spherical
    (the reference's default).  Exponents may use a Fortran "D" exponent."""
    spherical = "cartesian" not in text.split("****")[0].lower()
    out: dict = {}
    lines = [ln.strip() for ln in text.splitlines()]
    i = 0
    while i < len(lines):
        ln = lines[i]
        parts = ln.split()
        if len(parts) == 2 and parts[0] in ELEMENTS and parts[1] == "0":
            el = parts[0]
            shells = []
            i += 1
            while i < len(lines) and not lines[i].startswith("****"):
                hdr = lines[i].split()
                if not hdr or hdr[0].startswith("!"):
                    i += 1
                    continue
                kind, nprim = hdr[0].upper(), int(hdr[1])
                rows = []
                for k in range(nprim):
                    rows.append([float(x.replace("D", "E").replace("d", "e")) for x in lines[i + 1 + k].split()])
                rows = np.asarray(rows)
                if kind == "SP":
                    shells.append((0, rows[:, 0].copy(), rows[:, 1].copy()))
                    shells.append((1, rows[:, 0].copy(), rows[:, 2].copy()))
                else:
                    shells.append((AM[kind], rows[:, 0].copy(), rows[:, 1].copy()))
                i += 1 + nprim
            out[el] = shells
        i += 1
    return out, spherical


@dataclass
class Molecule:
    Z: np.ndarray          # (natom,) nuclear charges
    xyz: np.ndarray        # (natom, 3) bohr
    symbols: list = field(default_factory=list)

    @classmethod
    def from_angstrom(cls, atoms, to_bohr: float = ANGSTROM_TO_BOHR) -> "Molecule":
        """atoms: [(symbol, x, y, z), ...] in Angstrom."""
        sym = [a[0] for a in atoms]
        Z = np.array([float(ELEMENTS.index(s)) for s in sym])
        xyz = np.array([[a[1], a[2], a[3]] for a in atoms], dtype=np.float64) * to_bohr
        return cls(Z, xyz, sym)

    def n_electrons(self, charge: int = 0) -> int:
        return int(round(self.Z.sum())) - charge

    def nuclei(self):
        return _Nuclei(self)


class _Nuclei(ctypes.Structure):
    _fields_ = [("natom", ctypes.c_int), ("Z", ctypes.POINTER(ctypes.c_double)),
                ("xyz", ctypes.POINTER(ctypes.c_double))]

    def __init__(self, mol: Molecule):
        self._Z = np.ascontiguousarray(mol.Z, dtype=np.float64)
        self._xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64).reshape(-1)
        super().__init__(len(self._Z), self._Z.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                         self._xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))


class _Basis(ctypes.Structure):
    _fields_ = [("nshell", ctypes.c_int), ("l", ctypes.POINTER(ctypes.c_int)),
                ("pure", ctypes.POINTER(ctypes.c_int)), ("nprim", ctypes.POINTER(ctypes.c_int)),
                ("center", ctypes.POINTER(ctypes.c_double)), ("exps", ctypes.POINTER(ctypes.c_double)),
                ("coefs", ctypes.POINTER(ctypes.c_double))]


def _lib():
    lib = capi.load_library()
    if not getattr(lib, "_ao_ready", False):
        B = ctypes.POINTER(_Basis)
        Nu = ctypes.POINTER(_Nuclei)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.mshqc_ao_last_error.restype = ctypes.c_char_p
        lib.mshqc_ao_normalize_shell.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
        lib.mshqc_ao_nbf.argtypes = [B, ctypes.POINTER(ctypes.c_int64)]
        lib.mshqc_ao_one_electron.argtypes = [B, Nu, dp, dp, dp]
        lib.mshqc_ao_eri.argtypes = [B, dp]
        lib.mshqc_ao_eri_diagonal.argtypes = [B, dp]
        lib.mshqc_ao_eri_column.argtypes = [B, ctypes.c_int64, dp]
        lib.mshqc_ao_nuclear_repulsion.argtypes = [Nu, dp]
        lib._ao_ready = True
    return lib


def _check(rc):
    if rc != 0:
        raise capi.CDError(rc, _lib().mshqc_ao_last_error().decode())


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def normalize_shell(l: int, exps, coefs) -> np.ndarray:
    """Coefficients scaled like the reference's Shell::normalize."""
    e = np.ascontiguousarray(exps, dtype=np.float64)
    c = np.array(coefs, dtype=np.float64)
    _check(_lib().mshqc_ao_normalize_shell(int(l), len(e), _p(e), _p(c)))
    return c


@dataclass
class Shell:
    l: int
    pure: bool
    center: np.ndarray
    exps: np.ndarray
    coefs: np.ndarray      # normalized
    atom: int = 0

    @property
    def nf(self) -> int:
        return 2 * self.l + 1 if self.pure else (self.l + 1) * (self.l + 2) // 2


class BasisSet:
    """Shells of a Gaussian94 basis on the atoms of a molecule, in atom order
    and file order (the reference's BasisSet, src/core/basis.cc:114-169)."""

    def __init__(self, library: dict, mol: Molecule, spherical: bool = True):
        self.shells: list[Shell] = []
        for k, sym in enumerate(mol.symbols):
            if sym not in library:
                raise KeyError(f"basis has no entry for {sym}")
            for (l, e, c) in library[sym]:
                self.shells.append(Shell(l, spherical, mol.xyz[k].copy(), np.asarray(e, dtype=np.float64),
                                         normalize_shell(l, e, c), k))

    @classmethod
    def from_g94(cls, text: str, mol: Molecule) -> "BasisSet":
        lib, spherical = parse_g94(text)
        return cls(lib, mol, spherical)

    def n_basis_functions(self) -> int:
        return sum(s.nf for s in self.shells)

    def _struct(self):
        ls = np.array([s.l for s in self.shells], dtype=np.int32)
        pure = np.array([1 if s.pure else 0 for s in self.shells], dtype=np.int32)
        npr = np.array([len(s.exps) for s in self.shells], dtype=np.int32)
        cen = np.ascontiguousarray(np.array([s.center for s in self.shells], dtype=np.float64).reshape(-1))
        ex = np.ascontiguousarray(np.concatenate([s.exps for s in self.shells]))
        co = np.ascontiguousarray(np.concatenate([s.coefs for s in self.shells]))
        keep = (ls, pure, npr, cen, ex, co)
        ip = ctypes.POINTER(ctypes.c_int)
        st = _Basis(len(ls), ls.ctypes.data_as(ip), pure.ctypes.data_as(ip), npr.ctypes.data_as(ip), _p(cen), _p(ex),
                    _p(co))
        return st, keep


class IntegralEngine:
    """The reference's IntegralEngine over the library's host AO engine."""

    def __init__(self, mol: Molecule, basis: BasisSet):
        self.mol = mol
        self.basis = basis
        self.nbasis = basis.n_basis_functions()

    def _one(self, which):
        N = self.nbasis
        st, keep = self.basis._struct()
        nu = self.mol.nuclei()
        M = np.zeros((N, N))
        args = [None, None, None]
        args[which] = _p(M)
        _check(_lib().mshqc_ao_one_electron(ctypes.byref(st), ctypes.byref(nu), *args))
        return M

    def compute_overlap(self) -> np.ndarray:
        return self._one(0)

    def compute_kinetic(self) -> np.ndarray:
        return self._one(1)

    def compute_nuclear(self) -> np.ndarray:
        return self._one(2)

    def compute_core_hamiltonian(self) -> np.ndarray:
        return self.compute_kinetic() + self.compute_nuclear()

    def compute_eri(self) -> np.ndarray:
        """(N, N, N, N) array eri[mu, nu, lam, sig] = (mu nu|lam sig)."""
        N = self.nbasis
        st, keep = self.basis._struct()
        out = np.zeros(N ** 4)
        _check(_lib().mshqc_ao_eri(ctypes.byref(st), _p(out)))
        return out.reshape(N, N, N, N)

    def compute_eri_diagonal(self) -> np.ndarray:
        """(mu nu|mu nu) at mu N + nu."""
        N = self.nbasis
        st, keep = self.basis._struct()
        out = np.zeros(N * N)
        _check(_lib().mshqc_ao_eri_diagonal(ctypes.byref(st), _p(out)))
        return out

    def compute_eri_column(self, pivot_index: int) -> np.ndarray:
        """(mu nu|r s) at mu N + nu for pivot_index = r N + s."""
        N = self.nbasis
        st, keep = self.basis._struct()
        out = np.zeros(N * N)
        _check(_lib().mshqc_ao_eri_column(ctypes.byref(st), int(pivot_index), _p(out)))
        return out

    def nuclear_repulsion_energy(self) -> float:
        nu = self.mol.nuclei()
        e = ctypes.c_double()
        _check(_lib().mshqc_ao_nuclear_repulsion(ctypes.byref(nu), ctypes.byref(e)))
        return e.value
