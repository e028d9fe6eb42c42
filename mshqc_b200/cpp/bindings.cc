// pybind11 module mshqc_b200._mshqc: the Cholesky-MP2 part of mshqc's Python
// API (reference python/bindings.cc:160-173 CholeskyERI, :189-206 SCFResult,
// :311-331 OMP2Result, :431-456 CholeskyUMP2, :495-519 CholeskyOMP2,
// :561-592 CholeskyRMP2) with the same class, argument and attribute names,
// over the GPU classes of mshqc_b200.hpp.
//
// Where the reference takes a Molecule, a BasisSet and an IntegralEngine,
// any Python objects do: the molecule is not read, the basis needs
// n_basis_functions() (or is the basis size itself), and the integrals need
// compute_core_hamiltonian() -> (N, N) and, to decompose, compute_eri() ->
// (N, N, N, N) with [i, j, k, l] = (ij|kl).
#include <cmath>
#include <cstring>

#include <pybind11/pybind11.h>
#include <pybind11/numpy.h>
#include <pybind11/stl.h>

#include "mshqc_b200.hpp"

namespace py = pybind11;
using namespace mshqc_b200;

namespace {

using farray = py::array_t<double, py::array::f_style | py::array::forcecast>;
using carray = py::array_t<double, py::array::c_style | py::array::forcecast>;

py::array_t<double> to_numpy(const Matrix& m) {
    py::array_t<double> a({(py::ssize_t)m.rows(), (py::ssize_t)m.cols()},
                          {(py::ssize_t)sizeof(double), (py::ssize_t)(sizeof(double) * m.rows())});
    if (!m.empty()) std::memcpy(a.mutable_data(), m.data(), sizeof(double) * m.rows() * m.cols());
    return a;
}

Matrix to_matrix(const farray& a) {
    if (a.ndim() != 2) throw std::invalid_argument("expected a 2-D array");
    Matrix m((int)a.shape(0), (int)a.shape(1));
    std::memcpy(m.data(), a.data(), sizeof(double) * m.rows() * m.cols());
    return m;
}

// (i,j,a,b) column-major amplitudes as an (o1, o2, v1, v2) Fortran-ordered array
py::object t2_to_numpy(const std::vector<double>& t, int o1, int o2, int v1, int v2) {
    if (t.empty()) return py::none();
    py::array_t<double, py::array::f_style> a({(py::ssize_t)o1, (py::ssize_t)o2, (py::ssize_t)v1, (py::ssize_t)v2});
    std::memcpy(a.mutable_data(), t.data(), t.size() * sizeof(double));
    return std::move(a);
}

py::array_t<double> vec_to_numpy(const Vector& v) {
    py::array_t<double> a((py::ssize_t)v.size());
    if (!v.empty()) std::memcpy(a.mutable_data(), v.data(), sizeof(double) * v.size());
    return a;
}

Vector to_vector(const carray& a) {
    if (a.ndim() != 1) throw std::invalid_argument("expected a 1-D array");
    return Vector(a.data(), a.data() + a.size());
}

int basis_size(const py::object& basis) {
    if (py::hasattr(basis, "n_basis_functions")) return basis.attr("n_basis_functions")().cast<int>();
    return basis.cast<int>();
}

// A Python integral engine seen through IntegralSource.
class PyIntegrals : public IntegralSource {
public:
    explicit PyIntegrals(py::object obj) : obj_(std::move(obj)) {}
    Matrix compute_core_hamiltonian() override {
        return to_matrix(obj_.attr("compute_core_hamiltonian")().cast<farray>());
    }
    std::vector<double> compute_eri() override {
        const carray a = obj_.attr("compute_eri")().cast<carray>();
        if (a.ndim() != 4) throw std::invalid_argument("compute_eri must return an (N, N, N, N) array");
        return std::vector<double>(a.data(), a.data() + a.size());
    }

private:
    py::object obj_;
};

std::shared_ptr<IntegralSource> integrals_of(const py::object& obj) {
    if (obj.is_none()) return nullptr;
    return std::make_shared<PyIntegrals>(obj);
}

#define MATRIX_PROPERTY(cls, field)                                                               \
    def_property(                                                                                 \
        #field, [](const cls& s) { return to_numpy(s.field); },                                  \
        [](cls& s, const farray& a) { s.field = to_matrix(a); })
#define VECTOR_PROPERTY(cls, field)                                                               \
    def_property(                                                                                 \
        #field, [](const cls& s) { return vec_to_numpy(s.field); },                              \
        [](cls& s, const carray& a) { s.field = to_vector(a); })

}  // namespace

PYBIND11_MODULE(_mshqc, m) {
    m.doc() = "Cholesky-vector MP2 (CD-RMP2 / CD-UMP2 / CD-OMP2) on the GPU, mshqc's Python API";

    py::class_<CholeskyDecompositionResult>(m, "CholeskyDecompositionResult")
        .def_readonly("n_vectors", &CholeskyDecompositionResult::n_vectors)
        .def_readonly("n_basis", &CholeskyDecompositionResult::n_basis)
        .def_readonly("threshold", &CholeskyDecompositionResult::threshold)
        .def_readonly("compression_ratio", &CholeskyDecompositionResult::compression_ratio)
        .def_readonly("converged", &CholeskyDecompositionResult::converged);

    py::class_<CholeskyERI>(m, "CholeskyERI")
        .def(py::init<double>(), py::arg("threshold") = 1e-6)
        .def(
            "decompose",
            [](CholeskyERI& c, const carray& eri, int device) {
                if (eri.ndim() != 4) throw std::invalid_argument("eri must be an (N, N, N, N) array");
                return c.decompose(std::vector<double>(eri.data(), eri.data() + eri.size()), (int)eri.shape(0),
                                   device);
            },
            py::arg("eri"), py::arg("device") = 0)
        .def("get_L_vectors",
             [](const CholeskyERI& c) {
                 py::list out;
                 for (const auto& v : c.get_L_vectors()) out.append(vec_to_numpy(v));
                 return out;
             })
        .def(
            "set_vectors",
            [](CholeskyERI& c, const carray& L) {
                if (L.ndim() != 2) throw std::invalid_argument("L must be (n_vectors, N*N)");
                const int n = (int)std::lround(std::sqrt((double)L.shape(1)));
                if ((py::ssize_t)n * n != L.shape(1)) throw std::invalid_argument("vector length is not N*N");
                c.set_vectors(L.data(), n, (int)L.shape(0));
            },
            py::arg("L"))
        .def("reconstruct", &CholeskyERI::reconstruct)
        .def("n_vectors", &CholeskyERI::n_vectors)
        .def("n_basis", &CholeskyERI::n_basis)
        .def("threshold", &CholeskyERI::threshold)
        .def("is_decomposed", &CholeskyERI::is_decomposed)
        .def("compression_ratio", &CholeskyERI::compression_ratio);

    py::class_<SCFResult>(m, "SCFResult")
        .def(py::init<>())
        .def_readwrite("energy_electronic", &SCFResult::energy_electronic)
        .def_readwrite("energy_nuclear", &SCFResult::energy_nuclear)
        .def_readwrite("energy_total", &SCFResult::energy_total)
        .VECTOR_PROPERTY(SCFResult, orbital_energies_alpha)
        .VECTOR_PROPERTY(SCFResult, orbital_energies_beta)
        .MATRIX_PROPERTY(SCFResult, C_alpha)
        .MATRIX_PROPERTY(SCFResult, C_beta)
        .MATRIX_PROPERTY(SCFResult, P_alpha)
        .MATRIX_PROPERTY(SCFResult, P_beta)
        .MATRIX_PROPERTY(SCFResult, F_alpha)
        .MATRIX_PROPERTY(SCFResult, F_beta)
        .def_readwrite("iterations", &SCFResult::iterations)
        .def_readwrite("converged", &SCFResult::converged)
        .def_readwrite("gradient_norm", &SCFResult::gradient_norm)
        .def_readwrite("n_occ_alpha", &SCFResult::n_occ_alpha)
        .def_readwrite("n_occ_beta", &SCFResult::n_occ_beta);

    // ---- CD-RMP2
    py::class_<CholeskyRMP2Config>(m, "CholeskyRMP2Config")
        .def(py::init<>())
        .def_readwrite("cholesky_threshold", &CholeskyRMP2Config::cholesky_threshold)
        .def_readwrite("print_level", &CholeskyRMP2Config::print_level)
        .def_readwrite("precision", &CholeskyRMP2Config::precision)
        .def_readwrite("device", &CholeskyRMP2Config::device);

    py::class_<foundation::CholeskyRMP2Result>(m, "CholeskyRMP2Result")
        .def_readonly("e_rhf", &foundation::CholeskyRMP2Result::e_rhf)
        .def_readonly("e_corr", &foundation::CholeskyRMP2Result::e_corr)
        .def_readonly("e_total", &foundation::CholeskyRMP2Result::e_total)
        .def_readonly("n_chol_vectors", &foundation::CholeskyRMP2Result::n_chol_vectors)
        .def_readonly("n_occ", &foundation::CholeskyRMP2Result::n_occ)
        .def_readonly("n_virt", &foundation::CholeskyRMP2Result::n_virt)
        .def_property_readonly("t2", [](const foundation::CholeskyRMP2Result& r) {
            return t2_to_numpy(r.t2, r.n_occ, r.n_occ, r.n_virt, r.n_virt);
        })
        .def_property_readonly("chol_vectors", [](const foundation::CholeskyRMP2Result& r) {
            py::list out;
            for (const auto& v : r.chol_vectors) out.append(vec_to_numpy(v));
            return out;
        });

    py::class_<CholeskyRMP2>(m, "CholeskyRMP2")
        .def(py::init([](const py::object&, const py::object& basis, const py::object& integrals,
                         const SCFResult& rhf, const CholeskyRMP2Config& cfg) {
                 return std::make_unique<CholeskyRMP2>(basis_size(basis), integrals_of(integrals), rhf, cfg);
             }),
             py::arg("molecule"), py::arg("basis"), py::arg("integrals"), py::arg("rhf_result"),
             py::arg("config") = CholeskyRMP2Config())
        .def(py::init([](const py::object&, const py::object& basis, const py::object& integrals,
                         const SCFResult& rhf, const CholeskyRMP2Config& cfg, const CholeskyERI& chol) {
                 return std::make_unique<CholeskyRMP2>(basis_size(basis), integrals_of(integrals), rhf, cfg, chol);
             }),
             py::arg("molecule"), py::arg("basis"), py::arg("integrals"), py::arg("rhf_result"), py::arg("config"),
             py::arg("existing_cholesky"), py::keep_alive<1, 7>())
        .def("compute", &CholeskyRMP2::compute);

    // ---- CD-UMP2
    py::class_<CholeskyUMP2Config>(m, "CholeskyUMP2Config")
        .def(py::init<>())
        .def_readwrite("cholesky_threshold", &CholeskyUMP2Config::cholesky_threshold)
        .def_readwrite("use_on_the_fly", &CholeskyUMP2Config::use_on_the_fly)
        .def_readwrite("validate_energy", &CholeskyUMP2Config::validate_energy)
        .def_readwrite("print_level", &CholeskyUMP2Config::print_level)
        .def_readwrite("precision", &CholeskyUMP2Config::precision)
        .def_readwrite("device", &CholeskyUMP2Config::device);

    py::class_<CholeskyUMP2Result>(m, "CholeskyUMP2Result")
        .def_readonly("e_corr_ss_aa", &CholeskyUMP2Result::e_corr_ss_aa)
        .def_readonly("e_corr_ss_bb", &CholeskyUMP2Result::e_corr_ss_bb)
        .def_readonly("e_corr_os", &CholeskyUMP2Result::e_corr_os)
        .def_readonly("e_corr_total", &CholeskyUMP2Result::e_corr_total)
        .def_readonly("e_total", &CholeskyUMP2Result::e_total)
        .def_readonly("n_cholesky_vectors", &CholeskyUMP2Result::n_cholesky_vectors)
        .def_readonly("compression_ratio", &CholeskyUMP2Result::compression_ratio)
        .def_readonly("memory_mb", &CholeskyUMP2Result::memory_mb)
        .def_readonly("time_cholesky_s", &CholeskyUMP2Result::time_cholesky_s)
        .def_readonly("time_transform_s", &CholeskyUMP2Result::time_transform_s)
        .def_readonly("time_energy_s", &CholeskyUMP2Result::time_energy_s);

    py::class_<CholeskyUMP2>(m, "CholeskyUMP2")
        .def(py::init([](const SCFResult& scf, const py::object& basis, const py::object& integrals,
                         const CholeskyUMP2Config& cfg, const CholeskyERI& chol) {
            return std::make_unique<CholeskyUMP2>(scf, basis_size(basis), integrals_of(integrals), cfg, chol);
        }))
        .def("compute", &CholeskyUMP2::compute, "Compute UMP2 energy using Cholesky vectors")
        .def("compute_t2_amplitudes", &CholeskyUMP2::compute_t2_amplitudes)
        .def_property_readonly("L_ia_alpha", [](const CholeskyUMP2& u) {
            py::list out;
            for (const auto& m : u.L_ia_alpha()) out.append(to_numpy(m));
            return out;
        })
        .def_property_readonly("L_ia_beta", [](const CholeskyUMP2& u) {
            py::list out;
            for (const auto& m : u.L_ia_beta()) out.append(to_numpy(m));
            return out;
        })
        .def_property_readonly("t2_aa", [](const CholeskyUMP2& u) {
            const int a = u.n_occ_alpha(), va = u.n_basis() - a;
            return t2_to_numpy(u.t2_aa(), a, a, va, va);
        })
        .def_property_readonly("t2_bb", [](const CholeskyUMP2& u) {
            const int b = u.n_occ_beta(), vb = u.n_basis() - b;
            return t2_to_numpy(u.t2_bb(), b, b, vb, vb);
        })
        .def_property_readonly("t2_ab", [](const CholeskyUMP2& u) {
            const int a = u.n_occ_alpha(), b = u.n_occ_beta();
            return t2_to_numpy(u.t2_ab(), a, b, u.n_basis() - a, u.n_basis() - b);
        })
        .def("get_cholesky", &CholeskyUMP2::get_cholesky, py::return_value_policy::reference_internal);

    // ---- CD-OMP2
    py::class_<CholeskyOMP2Config>(m, "CholeskyOMP2Config")
        .def(py::init<>())
        .def_readwrite("max_iterations", &CholeskyOMP2Config::max_iterations)
        .def_readwrite("energy_threshold", &CholeskyOMP2Config::energy_threshold)
        .def_readwrite("gradient_threshold", &CholeskyOMP2Config::gradient_threshold)
        .def_readwrite("cholesky_threshold", &CholeskyOMP2Config::cholesky_threshold)
        .def_readwrite("print_level", &CholeskyOMP2Config::print_level)
        .def_readwrite("device", &CholeskyOMP2Config::device);

    py::class_<OMP2Result>(m, "OMP2Result")
        .def(py::init<>())
        .def_readwrite("energy_scf", &OMP2Result::energy_scf)
        .def_readwrite("energy_mp2_ss", &OMP2Result::energy_mp2_ss)
        .def_readwrite("energy_mp2_os", &OMP2Result::energy_mp2_os)
        .def_readwrite("energy_mp2_corr", &OMP2Result::energy_mp2_corr)
        .def_readwrite("energy_total", &OMP2Result::energy_total)
        .def_readwrite("converged", &OMP2Result::converged)
        .def_readwrite("iterations", &OMP2Result::iterations)
        .def_readwrite("n_occ_alpha", &OMP2Result::n_occ_alpha)
        .def_readwrite("n_occ_beta", &OMP2Result::n_occ_beta)
        .def_readwrite("n_virt_alpha", &OMP2Result::n_virt_alpha)
        .def_readwrite("n_virt_beta", &OMP2Result::n_virt_beta)
        .MATRIX_PROPERTY(OMP2Result, C_alpha)
        .MATRIX_PROPERTY(OMP2Result, C_beta)
        .VECTOR_PROPERTY(OMP2Result, orbital_energies_alpha)
        .VECTOR_PROPERTY(OMP2Result, orbital_energies_beta);

    py::class_<CholeskyOMP2>(m, "CholeskyOMP2")
        .def(py::init([](const py::object&, const py::object&, const py::object& integrals, const SCFResult& scf,
                         const CholeskyOMP2Config& cfg) {
                 return std::make_unique<CholeskyOMP2>(integrals_of(integrals), scf, cfg);
             }),
             py::arg("molecule"), py::arg("basis"), py::arg("integrals"), py::arg("scf_guess"),
             py::arg("config") = CholeskyOMP2Config())
        .def(py::init([](const py::object&, const py::object&, const py::object& integrals, const SCFResult& scf,
                         const CholeskyOMP2Config& cfg, const CholeskyERI& chol) {
                 return std::make_unique<CholeskyOMP2>(integrals_of(integrals), scf, cfg, chol);
             }),
             py::arg("molecule"), py::arg("basis"), py::arg("integrals"), py::arg("scf_guess"), py::arg("config"),
             py::arg("existing_cholesky"), py::keep_alive<1, 7>())
        .def("compute", &CholeskyOMP2::compute);
}
