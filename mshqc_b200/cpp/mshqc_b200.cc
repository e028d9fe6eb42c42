// Implementation of the C++ mirror classes (mshqc_b200.hpp): every compute
// step is a call into libmshqc_cuda.so.
#include "mshqc_b200.hpp"

#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <iostream>

namespace mshqc_b200 {

void check(int rc) {
    if (rc != MSHQC_CD_OK) throw std::runtime_error(std::string("mshqc_cd: ") + mshqc_cd_last_error());
}

DeviceContext::DeviceContext(int device) { check(mshqc_cd_ctx_create(device, &ctx_)); }
DeviceContext::~DeviceContext() {
    if (ctx_) mshqc_cd_ctx_destroy(ctx_);
}

namespace {

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void require_orbitals(const Matrix& C, const Vector& eps, int nbf, int nocc, const char* what) {
    if (C.rows() != nbf || C.cols() != nbf)
        throw std::invalid_argument(std::string(what) + ": C must be nbf x nbf");
    if ((int)eps.size() != nbf) throw std::invalid_argument(std::string(what) + ": orbital energies must have nbf entries");
    if (nocc < 1 || nocc >= nbf) throw std::invalid_argument(std::string(what) + ": need 1 <= n_occ < nbf");
}

void set_vectors(const DeviceContext& ctx, const CholeskyERI& chol) {
    if (chol.n_vectors() == 0) throw std::runtime_error("no Cholesky vectors");
    check(mshqc_cd_set_vectors(ctx.get(), chol.vectors().data(), chol.n_basis(), chol.n_vectors(),
                               MSHQC_CD_LAYOUT_FULL, MSHQC_CD_HOST));
}

size_t t2_max_bytes() {
    const char* env = std::getenv("MSHQC_T2_MAX_BYTES");
    return env ? (size_t)std::strtoull(env, nullptr, 10) : (size_t(8) << 30);
}

// amplitudes of one spin block, (i,j,a,b) column-major; empty above the limit
std::vector<double> fetch_t2(const DeviceContext& ctx, int block, int ox, int oy, int vx, int vy) {
    if (8.0 * ox * oy * (double)vx * vy > (double)t2_max_bytes()) return {};
    std::vector<double> t2((size_t)ox * oy * vx * vy), row((size_t)oy * vx * vy);
    for (int i = 0; i < ox; ++i) {
        check(mshqc_cd_get_t2_block(ctx.get(), block, i, 1, 0, oy, row.data(), MSHQC_CD_HOST));
        for (int j = 0; j < oy; ++j)
            for (int a = 0; a < vx; ++a)
                for (int b = 0; b < vy; ++b)
                    t2[(size_t)i + (size_t)ox * (j + (size_t)oy * (a + (size_t)vx * b))] =
                        row[((size_t)j * vx + a) * vy + b];
    }
    return t2;
}

std::vector<Matrix> fetch_mo_vectors(const DeviceContext& ctx, int spin, int nocc, int nvir, int nvec) {
    std::vector<double> B((size_t)nocc * nvir * nvec);
    check(mshqc_cd_transform(ctx.get(), spin, MSHQC_CD_FP64, B.data(), MSHQC_CD_HOST));
    std::vector<Matrix> out(nvec, Matrix(nocc, nvir));
    for (int i = 0; i < nocc; ++i)
        for (int a = 0; a < nvir; ++a)
            for (int q = 0; q < nvec; ++q) out[q](i, a) = B[((size_t)i * nvir + a) * nvec + q];
    return out;
}

}  // namespace

// ---------------------------------------------------------------------------
// CholeskyERI
// ---------------------------------------------------------------------------
CholeskyERI::CholeskyERI(double threshold) : threshold_(threshold) {
    if (!(threshold > 0.0)) throw std::invalid_argument("Cholesky threshold must be positive");
}

void CholeskyERI::reset() {
    L_.clear();
    n_basis_ = n_vectors_ = 0;
    decomposed_ = false;
}

CholeskyDecompositionResult CholeskyERI::decompose(const std::vector<double>& eri_full, int n_basis, int device) {
    reset();
    const size_t n2 = (size_t)n_basis * n_basis;
    if (n_basis <= 0 || eri_full.size() != n2 * n2)
        throw std::invalid_argument("ERI tensor must hold n_basis^4 elements");
    DeviceContext ctx(device);
    std::vector<double> out(n2 * n2);
    int64_t m = 0;
    int conv = 0;
    check(mshqc_cd_cholesky_decompose(ctx.get(), eri_full.data(), n_basis, threshold_, out.data(), (int64_t)n2,
                                      &m, &conv, MSHQC_CD_HOST));
    L_.assign(out.begin(), out.begin() + (ptrdiff_t)(m * n2));
    n_basis_ = n_basis;
    n_vectors_ = (int)m;
    decomposed_ = true;
    CholeskyDecompositionResult r;
    r.n_vectors = n_vectors_;
    r.n_basis = n_basis_;
    r.threshold = threshold_;
    r.compression_ratio = compression_ratio();
    r.converged = conv != 0;
    return r;
}

void CholeskyERI::set_vectors(const double* L, int n_basis, int n_vectors) {
    if (n_basis <= 0 || n_vectors < 0 || (!L && n_vectors > 0)) throw std::invalid_argument("bad vectors");
    const size_t n = (size_t)n_vectors * n_basis * n_basis;
    L_.assign(L, L + n);
    n_basis_ = n_basis;
    n_vectors_ = n_vectors;
    decomposed_ = true;
}

double CholeskyERI::reconstruct(int i, int j, int a, int b) const {
    if (!decomposed_) throw std::runtime_error("Cannot reconstruct: decomposition not performed");
    const size_t n2 = (size_t)n_basis_ * n_basis_, ij = (size_t)i * n_basis_ + j, ab = (size_t)a * n_basis_ + b;
    double v = 0.0;
    for (int q = 0; q < n_vectors_; ++q) v += L_[q * n2 + ij] * L_[q * n2 + ab];
    return v;
}

double CholeskyERI::compression_ratio() const {
    if (n_basis_ == 0 || n_vectors_ == 0) return 0.0;
    return std::pow((double)n_basis_, 4) / ((double)n_vectors_ * n_basis_ * n_basis_);
}

std::vector<Vector> CholeskyERI::get_L_vectors() const {
    const size_t n2 = (size_t)n_basis_ * n_basis_;
    std::vector<Vector> out(n_vectors_);
    for (int q = 0; q < n_vectors_; ++q) out[q].assign(L_.begin() + q * n2, L_.begin() + (q + 1) * n2);
    return out;
}

// ---------------------------------------------------------------------------
// CholeskyRMP2
// ---------------------------------------------------------------------------
CholeskyRMP2::CholeskyRMP2(int n_basis, std::shared_ptr<IntegralSource> integrals, const SCFResult& rhf_result,
                           const CholeskyRMP2Config& config)
    : nbf_(n_basis), nocc_(rhf_result.n_occ_alpha), nvirt_(n_basis - rhf_result.n_occ_alpha),
      integrals_(std::move(integrals)), rhf_(rhf_result), config_(config) {
    if (!integrals_) throw std::invalid_argument("CholeskyRMP2: integrals are needed to decompose");
    if (config_.print_level > 0)
        std::cout << "\n[CholeskyRMP2] Decomposing integrals internally (Threshold=" << config_.cholesky_threshold
                  << ")...\n";
    internal_ = std::make_unique<CholeskyERI>(config_.cholesky_threshold);
    internal_->decompose(integrals_->compute_eri(), nbf_, config_.device);
    chol_ = internal_.get();
}

CholeskyRMP2::CholeskyRMP2(int n_basis, std::shared_ptr<IntegralSource> integrals, const SCFResult& rhf_result,
                           const CholeskyRMP2Config& config, const CholeskyERI& existing_cholesky)
    : nbf_(n_basis), nocc_(rhf_result.n_occ_alpha), nvirt_(n_basis - rhf_result.n_occ_alpha),
      integrals_(std::move(integrals)), rhf_(rhf_result), config_(config), chol_(&existing_cholesky) {
    if (config_.print_level > 0)
        std::cout << "\n[CholeskyRMP2] Initialized with reused vectors (" << chol_->n_vectors() << " vectors)\n";
}

foundation::CholeskyRMP2Result CholeskyRMP2::compute() {
    require_orbitals(rhf_.C_alpha, rhf_.orbital_energies_alpha, nbf_, nocc_, "CholeskyRMP2");
    if (chol_->n_basis() != nbf_) throw std::invalid_argument("CholeskyRMP2: vectors and basis differ in size");
    DeviceContext ctx(config_.device);
    set_vectors(ctx, *chol_);
    check(mshqc_cd_set_orbitals(ctx.get(), MSHQC_CD_ALPHA, rhf_.C_alpha.data(), rhf_.orbital_energies_alpha.data(),
                                nocc_, MSHQC_CD_HOST));
    mshqc_cd_energy e{};
    check(mshqc_cd_mp2_energy(ctx.get(), MSHQC_CD_RESTRICTED, config_.precision, &e));
    foundation::CholeskyRMP2Result r;
    r.e_rhf = rhf_.energy_total;
    r.e_corr = e.total;
    r.e_total = r.e_rhf + r.e_corr;
    r.t2 = fetch_t2(ctx, 0, nocc_, nocc_, nvirt_, nvirt_);
    r.chol_vectors = chol_->get_L_vectors();
    r.n_chol_vectors = chol_->n_vectors();
    r.n_occ = nocc_;
    r.n_virt = nvirt_;
    if (config_.print_level > 0)
        std::cout << "[CholeskyRMP2] E(corr) = " << e.total << " Eh  (" << e.ms_total << " ms on the GPU)\n";
    return r;
}

// ---------------------------------------------------------------------------
// CholeskyUMP2
// ---------------------------------------------------------------------------
CholeskyUMP2::CholeskyUMP2(const SCFResult& uhf_result, int n_basis, std::shared_ptr<IntegralSource> integrals,
                           const CholeskyUMP2Config& config, const CholeskyERI& cholesky)
    : uhf_(uhf_result), nbf_(n_basis), integrals_(std::move(integrals)), config_(config), chol_(cholesky) {
    if (config_.print_level > 0)
        std::cout << "\n[CholeskyUMP2] occupied (alpha/beta) " << uhf_.n_occ_alpha << " / " << uhf_.n_occ_beta
                  << ", reusing " << chol_.n_vectors() << " Cholesky vectors\n";
}

CholeskyUMP2Result CholeskyUMP2::compute() {
    const auto t0 = std::chrono::steady_clock::now();
    require_orbitals(uhf_.C_alpha, uhf_.orbital_energies_alpha, nbf_, uhf_.n_occ_alpha, "CholeskyUMP2 (alpha)");
    require_orbitals(uhf_.C_beta, uhf_.orbital_energies_beta, nbf_, uhf_.n_occ_beta, "CholeskyUMP2 (beta)");
    CholeskyUMP2Result r;
    const CholeskyERI* chol = &chol_;
    std::unique_ptr<CholeskyERI> own;
    if (chol_.n_vectors() == 0) {
        // no vectors: decompose the integrals (reference cholesky_ump2.cc:74-110)
        if (!integrals_) throw std::invalid_argument("CholeskyUMP2: no vectors and no integrals");
        own = std::make_unique<CholeskyERI>(config_.cholesky_threshold);
        own->decompose(integrals_->compute_eri(), nbf_, config_.device);
        chol = own.get();
        r.time_cholesky_s = seconds_since(t0);
    }
    DeviceContext ctx(config_.device);
    set_vectors(ctx, *chol);
    check(mshqc_cd_set_orbitals(ctx.get(), MSHQC_CD_ALPHA, uhf_.C_alpha.data(), uhf_.orbital_energies_alpha.data(),
                                uhf_.n_occ_alpha, MSHQC_CD_HOST));
    check(mshqc_cd_set_orbitals(ctx.get(), MSHQC_CD_BETA, uhf_.C_beta.data(), uhf_.orbital_energies_beta.data(),
                                uhf_.n_occ_beta, MSHQC_CD_HOST));
    mshqc_cd_energy e{};
    check(mshqc_cd_mp2_energy(ctx.get(), MSHQC_CD_UNRESTRICTED, config_.precision, &e));
    r.e_corr_ss_aa = e.ss_aa;
    r.e_corr_ss_bb = e.ss_bb;
    r.e_corr_os = e.os;
    r.e_corr_total = e.total;
    r.e_total = uhf_.energy_total + e.total;
    r.n_cholesky_vectors = chol->n_vectors();
    r.compression_ratio = chol->compression_ratio();
    r.memory_mb = chol->storage_bytes() / 1024.0 / 1024.0;
    r.time_transform_s = e.ms_transform / 1e3;
    r.time_energy_s = e.ms_energy / 1e3;
    const int nva = nbf_ - uhf_.n_occ_alpha, nvb = nbf_ - uhf_.n_occ_beta;
    L_ia_alpha_ = fetch_mo_vectors(ctx, MSHQC_CD_ALPHA, uhf_.n_occ_alpha, nva, chol->n_vectors());
    L_ia_beta_ = fetch_mo_vectors(ctx, MSHQC_CD_BETA, uhf_.n_occ_beta, nvb, chol->n_vectors());
    if (config_.print_level > 0)
        std::cout << "[CholeskyUMP2] E(corr) = " << e.total << " Eh (ss_aa " << e.ss_aa << ", ss_bb " << e.ss_bb
                  << ", os " << e.os << ")\n";
    return r;
}

void CholeskyUMP2::compute_t2_amplitudes() {
    const int na = uhf_.n_occ_alpha, nb = uhf_.n_occ_beta, va = nbf_ - na, vb = nbf_ - nb;
    require_orbitals(uhf_.C_alpha, uhf_.orbital_energies_alpha, nbf_, na, "CholeskyUMP2 (alpha)");
    require_orbitals(uhf_.C_beta, uhf_.orbital_energies_beta, nbf_, nb, "CholeskyUMP2 (beta)");
    DeviceContext ctx(config_.device);
    set_vectors(ctx, chol_);
    check(mshqc_cd_set_orbitals(ctx.get(), MSHQC_CD_ALPHA, uhf_.C_alpha.data(), uhf_.orbital_energies_alpha.data(),
                                na, MSHQC_CD_HOST));
    check(mshqc_cd_set_orbitals(ctx.get(), MSHQC_CD_BETA, uhf_.C_beta.data(), uhf_.orbital_energies_beta.data(),
                                nb, MSHQC_CD_HOST));
    t2_aa_ = fetch_t2(ctx, 0, na, na, va, va);
    t2_bb_ = fetch_t2(ctx, 1, nb, nb, vb, vb);
    t2_ab_ = fetch_t2(ctx, 2, na, nb, va, vb);
}

// ---------------------------------------------------------------------------
// CholeskyOMP2
// ---------------------------------------------------------------------------
CholeskyOMP2::CholeskyOMP2(std::shared_ptr<IntegralSource> integrals, const SCFResult& scf_guess,
                           const CholeskyOMP2Config& config)
    : integrals_(std::move(integrals)), scf_(scf_guess), config_(config) {
    if (!integrals_) throw std::invalid_argument("CholeskyOMP2: integrals are needed");
    if (config_.print_level > 0)
        std::cout << "[CholeskyOMP2] Decomposing integrals (Thresh=" << config_.cholesky_threshold << ")...\n";
    internal_ = std::make_unique<CholeskyERI>(config_.cholesky_threshold);
    internal_->decompose(integrals_->compute_eri(), scf_.C_alpha.rows(), config_.device);
    chol_ = internal_.get();
}

CholeskyOMP2::CholeskyOMP2(std::shared_ptr<IntegralSource> integrals, const SCFResult& scf_guess,
                           const CholeskyOMP2Config& config, const CholeskyERI& cholesky_vectors)
    : integrals_(std::move(integrals)), scf_(scf_guess), config_(config), chol_(&cholesky_vectors) {
    if (chol_->n_vectors() == 0)
        throw std::runtime_error("CholeskyOMP2 initialized with empty reused vectors");
}

OMP2Result CholeskyOMP2::compute() {
    const int nbf = scf_.C_alpha.rows(), na = scf_.n_occ_alpha, nb = scf_.n_occ_beta;
    require_orbitals(scf_.C_alpha, scf_.orbital_energies_alpha, nbf, na, "CholeskyOMP2 (alpha)");
    require_orbitals(scf_.C_beta, scf_.orbital_energies_beta, nbf, nb, "CholeskyOMP2 (beta)");
    if (!integrals_) throw std::invalid_argument("CholeskyOMP2: integrals are needed for the core Hamiltonian");
    const Matrix H = integrals_->compute_core_hamiltonian();
    if (H.rows() != nbf || H.cols() != nbf) throw std::invalid_argument("core Hamiltonian must be nbf x nbf");
    DeviceContext ctx(config_.device);
    set_vectors(ctx, *chol_);
    check(mshqc_cd_set_orbitals(ctx.get(), MSHQC_CD_ALPHA, scf_.C_alpha.data(), scf_.orbital_energies_alpha.data(),
                                na, MSHQC_CD_HOST));
    check(mshqc_cd_set_orbitals(ctx.get(), MSHQC_CD_BETA, scf_.C_beta.data(), scf_.orbital_energies_beta.data(),
                                nb, MSHQC_CD_HOST));
    check(mshqc_cd_set_core_hamiltonian(ctx.get(), H.data(), MSHQC_CD_HOST));
    mshqc_cd_omp2_config cfg{config_.max_iterations, config_.energy_threshold, config_.gradient_threshold,
                             scf_.energy_total};
    const bool have_p = scf_.P_alpha.rows() == nbf && scf_.P_beta.rows() == nbf;
    mshqc_cd_omp2_result res{};
    check(mshqc_cd_omp2(ctx.get(), &cfg, have_p ? scf_.P_alpha.data() : nullptr,
                        have_p ? scf_.P_beta.data() : nullptr, MSHQC_CD_HOST, &res));
    OMP2Result r;
    r.energy_scf = res.energy_scf;
    r.energy_mp2_corr = res.energy_mp2_corr;
    r.energy_total = res.energy_total;
    r.converged = res.converged != 0;
    r.iterations = res.iterations;
    r.n_occ_alpha = na;
    r.n_occ_beta = nb;
    r.n_virt_alpha = nbf - na;
    r.n_virt_beta = nbf - nb;
    r.C_alpha = Matrix(nbf, nbf);
    r.C_beta = Matrix(nbf, nbf);
    check(mshqc_cd_get_orbitals(ctx.get(), MSHQC_CD_ALPHA, r.C_alpha.data(), MSHQC_CD_HOST));
    check(mshqc_cd_get_orbitals(ctx.get(), MSHQC_CD_BETA, r.C_beta.data(), MSHQC_CD_HOST));
    r.orbital_energies_alpha = scf_.orbital_energies_alpha;   // never updated (reference :509)
    r.orbital_energies_beta = scf_.orbital_energies_beta;
    if (config_.print_level > 0)
        std::cout << "[CholeskyOMP2] " << (r.converged ? "converged" : "not converged") << " after "
                  << r.iterations << " iterations, E(corr) = " << r.energy_mp2_corr << " Eh\n";
    return r;
}

}  // namespace mshqc_b200
