// The reference's IntegralEngine (include/mshqc/integrals.h:38-224;
// libint2-based in src/core/integrals.cc) on the library's host AO engine
// (include/mshqc_ao.h): the same member functions and layouts, the shells
// taken from the reference's BasisSet as it hands them to libint2
// (src/core/integrals.cc:96-145: coefficients already normalized by
// BasisSet, pure per Shell::is_spherical).  The density-fitting entries
// (compute_3center_eri, compute_2center_eri) are not on the Cholesky path
// and throw.
#include <cmath>
#include <iostream>
#include <stdexcept>
#include <vector>

#include "dropin_common.h"
#include "mshqc/integrals.h"

namespace mshqc {

struct IntegralEngine::LibintShellData {
    std::vector<int> l, pure, nprim;
    std::vector<double> center, exps, coefs, Z, xyz;
    mshqc_ao_basis basis{};
    mshqc_ao_nuclei nuclei{};
};

IntegralEngine::IntegralEngine(const Molecule& mol, const BasisSet& basis)
    : mol_(mol), basis_(basis), nbasis_(basis.n_basis_functions()) {
    initialize_libint();
}

IntegralEngine::~IntegralEngine() { finalize_libint(); }

void IntegralEngine::initialize_libint() {
    libint_shells_ = std::make_unique<LibintShellData>();
    convert_basis_to_libint();
}

void IntegralEngine::finalize_libint() {}

void IntegralEngine::convert_basis_to_libint() {
    LibintShellData& d = *libint_shells_;
    for (const Shell& s : basis_.shells()) {
        d.l.push_back(s.l());
        d.pure.push_back(s.is_spherical() ? 1 : 0);
        d.nprim.push_back((int)s.n_primitives());
        for (double x : s.position()) d.center.push_back(x);
        for (const auto& p : s.primitives()) {
            d.exps.push_back(p.exponent);
            d.coefs.push_back(p.coefficient);
        }
    }
    for (size_t a = 0; a < mol_.n_atoms(); ++a) {
        const Atom& at = mol_.atom(a);
        d.Z.push_back((double)at.atomic_number);
        d.xyz.push_back(at.x);
        d.xyz.push_back(at.y);
        d.xyz.push_back(at.z);
    }
    d.basis = mshqc_ao_basis{(int)d.l.size(), d.l.data(), d.pure.data(), d.nprim.data(),
                             d.center.data(), d.exps.data(), d.coefs.data()};
    d.nuclei = mshqc_ao_nuclei{(int)mol_.n_atoms(), d.Z.data(), d.xyz.data()};
}

namespace {
void ao_check(int rc) {
    if (rc != MSHQC_AO_OK) throw std::runtime_error(std::string("AO integrals: ") + mshqc_ao_last_error());
}
}  // namespace

Eigen::MatrixXd IntegralEngine::compute_overlap() {
    Eigen::MatrixXd S((long)nbasis_, (long)nbasis_);
    ao_check(mshqc_ao_one_electron(&libint_shells_->basis, &libint_shells_->nuclei, S.data(), nullptr, nullptr));
    return S;
}

Eigen::MatrixXd IntegralEngine::compute_kinetic() {
    Eigen::MatrixXd T((long)nbasis_, (long)nbasis_);
    ao_check(mshqc_ao_one_electron(&libint_shells_->basis, &libint_shells_->nuclei, nullptr, T.data(), nullptr));
    return T;
}

Eigen::MatrixXd IntegralEngine::compute_nuclear() {
    Eigen::MatrixXd V((long)nbasis_, (long)nbasis_);
    ao_check(mshqc_ao_one_electron(&libint_shells_->basis, &libint_shells_->nuclei, nullptr, nullptr, V.data()));
    return V;
}

Eigen::MatrixXd IntegralEngine::compute_core_hamiltonian() { return compute_kinetic() + compute_nuclear(); }

Eigen::Tensor<double, 4> IntegralEngine::compute_eri() {
    const long N = (long)nbasis_;
    Eigen::Tensor<double, 4> eri(N, N, N, N);
    // the eight-fold symmetry makes the row-major tensor of the engine the
    // same array as Eigen's column-major one
    ao_check(mshqc_ao_eri(&libint_shells_->basis, eri.data()));
    return eri;
}

Eigen::Tensor<double, 4> IntegralEngine::compute_eri_screened(double threshold) {
    Eigen::Tensor<double, 4> eri = compute_eri();
    const Eigen::VectorXd diag = compute_eri_diagonal();
    const long N = (long)nbasis_;
    for (long l = 0; l < N; ++l)
        for (long k = 0; k < N; ++k)
            for (long j = 0; j < N; ++j)
                for (long i = 0; i < N; ++i)
                    if (std::sqrt(std::fabs(diag(i * N + j) * diag(k * N + l))) < threshold) eri(i, j, k, l) = 0.0;
    return eri;
}

Eigen::VectorXd IntegralEngine::compute_eri_diagonal() {
    Eigen::VectorXd d((long)(nbasis_ * nbasis_));
    ao_check(mshqc_ao_eri_diagonal(&libint_shells_->basis, d.data()));
    return d;
}

Eigen::VectorXd IntegralEngine::compute_eri_column(int pivot_index) {
    Eigen::VectorXd c((long)(nbasis_ * nbasis_));
    ao_check(mshqc_ao_eri_column(&libint_shells_->basis, pivot_index, c.data()));
    return c;
}

double IntegralEngine::compute_single_eri(int mu, int nu, int lam, int sig) {
    const Eigen::VectorXd c = compute_eri_column(lam * (int)nbasis_ + sig);
    return c(mu * (long)nbasis_ + nu);
}

void IntegralEngine::print_statistics() const {
    std::cout << "AO integral engine (host, McMurchie-Davidson): " << nbasis_ << " basis functions, "
              << basis_.n_shells() << " shells\n";
}

Eigen::Tensor<double, 3> IntegralEngine::compute_3center_eri(const BasisSet&) {
    throw std::runtime_error("compute_3center_eri: density fitting is not part of the Cholesky-MP2 drop-in");
}

Eigen::MatrixXd IntegralEngine::compute_2center_eri(const BasisSet&) {
    throw std::runtime_error("compute_2center_eri: density fitting is not part of the Cholesky-MP2 drop-in");
}

}  // namespace mshqc
