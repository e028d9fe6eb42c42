// Oracle test infrastructure -- NOT part of the product.
//
// A repo-owned stand-in for mshqc's libint2-backed IntegralEngine
// (interface: include/mshqc/integrals.h:38-224 of the reference; the real
// implementation in src/core/integrals.cc needs libint2, which is absent).
// The Cholesky-MP2 sources of the reference only touch four members of the
// engine on the hot path:
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

namespace mshqc {

struct IntegralEngine::LibintShellData {};

namespace oracle_stub {
Eigen::MatrixXd g_core_hamiltonian;
Eigen::Tensor<double, 4> g_eri;
bool g_have_eri = false;
}  // namespace oracle_stub

IntegralEngine::IntegralEngine(const Molecule& mol, const BasisSet& basis)
    : mol_(mol), basis_(basis), nbasis_(basis.n_basis_functions()) {}

IntegralEngine::~IntegralEngine() = default;

Eigen::MatrixXd IntegralEngine::compute_core_hamiltonian() {
    if (oracle_stub::g_core_hamiltonian.rows() != static_cast<long>(nbasis_))
        throw std::runtime_error("oracle stub: core Hamiltonian not installed");
    return oracle_stub::g_core_hamiltonian;
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
