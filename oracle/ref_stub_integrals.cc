// Oracle test infrastructure -- NOT part of the product.
//
// A repo-owned stand-in for mshqc's libint2-backed IntegralEngine
// (interface: include/mshqc/integrals.h:38-224 of the reference; the real
// implementation in src/core/integrals.cc needs libint2, which is absent).
// The Cholesky-MP2 sources of the reference only touch four members of the
// engine on the hot path (and its RHF, src/scf/rhf.cc:60-140, the overlap,
// kinetic and nuclear matrices and the ERI tensor):
//   compute_eri()               CholeskyRMP2/CholeskyOMP2 constructor 1
//                               (src/mp2/cholesky_rmp2.cc:38, cholesky_omp2.cc:37)
//   compute_core_hamiltonian()  CholeskyOMP2::build_gfock_from_density
//                               (src/mp2/cholesky_omp2.cc:336)
//   compute_eri_diagonal/column CholeskyUMP2::decompose_eri fallback
//                               (src/mp2/cholesky_ump2.cc:188, :206)
// This file serves them from matrices the harness installs beforehand
// (ref_set_core_hamiltonian / ref_set_eri in ref_harness.cc), so the
// reference's own MP2 code runs unchanged on synthetic inputs.
#include "mshqc/integrals.h"

#include <stdexcept>
#include <string>

namespace mshqc {

struct IntegralEngine::LibintShellData {};

namespace oracle_stub {
Eigen::MatrixXd g_core_hamiltonian;
Eigen::MatrixXd g_overlap, g_kinetic, g_nuclear;
Eigen::Tensor<double, 4> g_eri;
bool g_have_eri = false;
}  // namespace oracle_stub

IntegralEngine::IntegralEngine(const Molecule& mol, const BasisSet& basis)
    : mol_(mol), basis_(basis), nbasis_(basis.n_basis_functions()) {}

IntegralEngine::~IntegralEngine() = default;

namespace {
const Eigen::MatrixXd& installed(const Eigen::MatrixXd& m, size_t n, const char* what) {
    if (m.rows() != static_cast<long>(n)) throw std::runtime_error(std::string("oracle stub: ") + what + " not installed");
    return m;
}
}  // namespace

// S, T, V installed by the harness (the reference's RHF reads them,
// src/scf/rhf.cc:60-67)
Eigen::MatrixXd IntegralEngine::compute_overlap() { return installed(oracle_stub::g_overlap, nbasis_, "overlap"); }
Eigen::MatrixXd IntegralEngine::compute_kinetic() { return installed(oracle_stub::g_kinetic, nbasis_, "kinetic"); }
Eigen::MatrixXd IntegralEngine::compute_nuclear() { return installed(oracle_stub::g_nuclear, nbasis_, "nuclear"); }

Eigen::MatrixXd IntegralEngine::compute_core_hamiltonian() {
    if (oracle_stub::g_core_hamiltonian.rows() == static_cast<long>(nbasis_)) return oracle_stub::g_core_hamiltonian;
    return compute_kinetic() + compute_nuclear();
}

Eigen::Tensor<double, 4> IntegralEngine::compute_eri() {
    if (!oracle_stub::g_have_eri)
        throw std::runtime_error("oracle stub: ERI tensor not installed");
    return oracle_stub::g_eri;
}

Eigen::VectorXd IntegralEngine::compute_eri_diagonal() {
    throw std::runtime_error("oracle stub: compute_eri_diagonal not provided");
}

Eigen::VectorXd IntegralEngine::compute_eri_column(int) {
    throw std::runtime_error("oracle stub: compute_eri_column not provided");
}

}  // namespace mshqc
