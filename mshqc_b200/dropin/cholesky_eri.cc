// The reference's CholeskyERI (include/mshqc/integrals/cholesky_eri.h:37-99;
// src/integrals/cholesky_eri.cc) with decompose() on the GPU
// (mshqc_cd_cholesky_decompose: pivoted incomplete Cholesky with the FP64
// diagonal, first-index pivots and the clamped diagonal update of
// src/integrals/cholesky_eri.cc:40-203).  The other members behave as the
// reference's: same exceptions, same statistics.
#include <algorithm>
#include <cmath>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <vector>

#include "dropin_common.h"
#include "mshqc/integrals/cholesky_eri.h"

namespace mshqc {
namespace integrals {

CholeskyERI::CholeskyERI(double threshold) : threshold_(threshold) {
    if (threshold_ <= 0.0) throw std::invalid_argument("Cholesky threshold must be positive");
}

CholeskyDecompositionResult CholeskyERI::decompose(const Eigen::Tensor<double, 4>& eri_full) {
    reset();
    n_basis_ = (int)eri_full.dimension(0);
    const int64_t N = n_basis_, n2 = N * N;
    std::vector<double> L((size_t)(n2 * n2));
    int64_t m = 0;
    int converged = 0;
    // column-major (i,j,k,l) of Eigen and the row-major order of the C ABI
    // hold the same values for a symmetric ERI tensor
    mshqc_dropin::check(mshqc_cd_cholesky_decompose(mshqc_dropin::context(), eri_full.data(), N, threshold_,
                                                    L.data(), n2, &m, &converged, MSHQC_CD_HOST));
    L_vectors_.reserve((size_t)m);
    for (int64_t q = 0; q < m; ++q)
        L_vectors_.push_back(Eigen::Map<const Eigen::VectorXd>(L.data() + q * n2, (long)n2));
    n_vectors_ = (int)m;
    decomposed_ = true;
    CholeskyDecompositionResult r;
    r.n_vectors = n_vectors_;
    r.n_basis = n_basis_;
    r.threshold = threshold_;
    r.compression_ratio = compression_ratio();
    r.converged = converged != 0;
    return r;
}

double CholeskyERI::reconstruct(int i, int j, int a, int b) const {
    if (!decomposed_) throw std::runtime_error("Cannot reconstruct: decomposition not performed");
    const int ij = composite_index(i, j), ab = composite_index(a, b);
    double v = 0.0;
    for (int k = 0; k < n_vectors_; ++k) v += L_vectors_[k](ij) * L_vectors_[k](ab);
    return v;
}

Eigen::Tensor<double, 4> CholeskyERI::reconstruct_full() const {
    if (!decomposed_) throw std::runtime_error("Cannot reconstruct: decomposition not performed");
    Eigen::Tensor<double, 4> t(n_basis_, n_basis_, n_basis_, n_basis_);
    for (int i = 0; i < n_basis_; ++i)
        for (int j = 0; j < n_basis_; ++j)
            for (int a = 0; a < n_basis_; ++a)
                for (int b = 0; b < n_basis_; ++b) t(i, j, a, b) = reconstruct(i, j, a, b);
    return t;
}

double CholeskyERI::compression_ratio() const {
    if (n_vectors_ == 0 || n_basis_ == 0) return 0.0;
    const double full = std::pow((double)n_basis_, 4);
    return full / ((double)n_vectors_ * n_basis_ * n_basis_);
}

size_t CholeskyERI::storage_bytes() const { return (size_t)n_vectors_ * n_basis_ * n_basis_ * sizeof(double); }

std::pair<double, double> CholeskyERI::validate_reconstruction(const Eigen::Tensor<double, 4>& eri_exact) {
    if ((int)eri_exact.dimension(0) != n_basis_) throw std::invalid_argument("ERI dimensions mismatch");
    double mx = 0.0, ss = 0.0;
    long cnt = 0;
    for (int i = 0; i < n_basis_; ++i)
        for (int j = 0; j < n_basis_; ++j)
            for (int a = 0; a < n_basis_; ++a)
                for (int b = 0; b < n_basis_; ++b) {
                    const double e = std::fabs(eri_exact(i, j, a, b) - reconstruct(i, j, a, b));
                    mx = std::max(mx, e);
                    ss += e * e;
                    ++cnt;
                }
    max_error_ = mx;
    rms_error_ = cnt ? std::sqrt(ss / cnt) : 0.0;
    return {max_error_, rms_error_};
}

void CholeskyERI::print_statistics(bool) const {
    std::cout << "Cholesky vectors: " << n_vectors_ << " (basis " << n_basis_ << ", threshold " << std::scientific
              << threshold_ << ", decomposed on the GPU)\n";
}

void CholeskyERI::reset() {
    L_vectors_.clear();
    n_basis_ = 0;
    n_vectors_ = 0;
    decomposed_ = false;
    max_error_ = 0.0;
    rms_error_ = 0.0;
}

}  // namespace integrals
}  // namespace mshqc
