"""The pybind11 module mshqc_b200._mshqc (CPU side): the reference's Python
names, configuration defaults (include/mshqc/cholesky_omp2.h:28-34,
cholesky_rmp2.h:70-73, cholesky_ump2.h:40-46) and error behaviour."""
import numpy as np
import pytest

from mshqc_b200 import _mshqc as m


def test_names():
    for name in ("CholeskyERI", "CholeskyDecompositionResult", "SCFResult", "CholeskyRMP2Config", "CholeskyRMP2",
                 "CholeskyRMP2Result", "CholeskyUMP2Config", "CholeskyUMP2Result", "CholeskyUMP2",
                 "CholeskyOMP2Config", "CholeskyOMP2", "OMP2Result"):
        assert hasattr(m, name), name


def test_config_defaults():
    o = m.CholeskyOMP2Config()
    assert (o.max_iterations, o.energy_threshold, o.gradient_threshold, o.cholesky_threshold, o.print_level) == \
        (50, 1e-6, 1e-5, 1e-6, 1)
    r = m.CholeskyRMP2Config()
    assert (r.cholesky_threshold, r.print_level, r.precision) == (1e-6, 1, 0)
    u = m.CholeskyUMP2Config()
    assert (u.cholesky_threshold, u.use_on_the_fly, u.validate_energy, u.print_level) == (1e-6, False, False, 1)


def test_cholesky_eri_threshold_and_vectors():
    with pytest.raises(ValueError):
        m.CholeskyERI(0.0)
    c = m.CholeskyERI(1e-6)
    assert c.threshold() == 1e-6 and c.n_vectors() == 0
    L = np.arange(2 * 9, dtype=np.float64).reshape(2, 9)
    c.set_vectors(L)
    assert c.n_vectors() == 2 and c.n_basis() == 3
    assert c.reconstruct(0, 1, 2, 0) == L[0, 1] * L[0, 6] + L[1, 1] * L[1, 6]
    assert np.array_equal(np.array(c.get_L_vectors()), L)
    assert c.compression_ratio() == 81 / 18


def test_scf_result_round_trip():
    s = m.SCFResult()
    C = np.arange(12.0).reshape(3, 4)
    s.C_alpha = C
    s.orbital_energies_alpha = np.array([1.0, 2.0, 3.0])
    s.n_occ_alpha = 2
    assert np.array_equal(s.C_alpha, C)
    assert np.array_equal(s.orbital_energies_alpha, [1.0, 2.0, 3.0])
    assert s.n_occ_alpha == 2


def test_reconstruct_before_decompose_raises():
    with pytest.raises(RuntimeError):
        m.CholeskyERI().reconstruct(0, 0, 0, 0)
