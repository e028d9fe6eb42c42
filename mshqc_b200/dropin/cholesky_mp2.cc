// The reference's Cholesky-MP2 classes -- CholeskyRMP2
// (include/mshqc/cholesky_rmp2.h:52-117), CholeskyUMP2
// (include/mshqc/cholesky_ump2.h:40-200) and CholeskyOMP2
// (include/mshqc/cholesky_omp2.h:28-80) -- implemented on libmshqc_cuda.so:
// the same constructors, compute() results and error behaviour, with the
// half transforms, pair energies, amplitudes and the OMP2 loop on the GPU.
//
// What the reference stores for its consumers is filled the same way:
// CholeskyRMP2Result::t2 and ::chol_vectors (CholeskyRMP3), CholeskyUMP2's
// L_ia_alpha_/L_ia_beta_ after compute() and t2_aa_/t2_bb_/t2_ab_ after
// compute_t2_amplitudes() (CholeskyUMP3); amplitudes come from
// mshqc_cd_get_t2_block in FP64 and are left empty above
// MSHQC_T2_MAX_BYTES (default 8 GiB), where the reference would run out of
// host memory.  Where the reference calls exit(1) on empty reused vectors
// (src/mp2/cholesky_omp2.cc:62-65) this throws std::runtime_error.
#include <chrono>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <vector>

#include "dropin_common.h"
#include "mshqc/cholesky_omp2.h"
#include "mshqc/cholesky_rmp2.h"
#include "mshqc/cholesky_ump2.h"

namespace mshqc {

namespace {

using mshqc_dropin::check;
using mshqc_dropin::context;

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// the context's vectors := the CholeskyERI's (contiguous copy, vector Q at Q N^2)
void upload_vectors(mshqc_cd_ctx* ctx, const integrals::CholeskyERI& chol, int nbf) {
    const auto& L = chol.get_L_vectors();
    if (L.empty()) throw std::runtime_error("Cholesky vectors are empty");
    const size_t n2 = (size_t)nbf * nbf;
    std::vector<double> flat(L.size() * n2);
    for (size_t q = 0; q < L.size(); ++q) {
        if ((size_t)L[q].size() != n2) throw std::invalid_argument("Cholesky vectors and basis differ in size");
        std::memcpy(flat.data() + q * n2, L[q].data(), n2 * sizeof(double));
    }
    check(mshqc_cd_set_vectors(ctx, flat.data(), nbf, (int64_t)L.size(), MSHQC_CD_LAYOUT_FULL, MSHQC_CD_HOST));
}

void upload_orbitals(mshqc_cd_ctx* ctx, int spin, const Eigen::MatrixXd& C, const Eigen::VectorXd& eps, int nocc) {
    if (C.rows() != C.cols() || eps.size() != C.rows() || nocc < 1 || nocc >= C.rows())
        throw std::invalid_argument("orbitals: C must be N x N, eps of length N, 0 < nocc < N");
    check(mshqc_cd_set_orbitals(ctx, spin, C.data(), eps.data(), nocc, MSHQC_CD_HOST));
}

// t(i, j, a, b) of one spin block into an Eigen (o_x, o_y, v_x, v_y) tensor,
// one row of pairs per call
bool fetch_t2(mshqc_cd_ctx* ctx, int block, int ox, int oy, int vx, int vy, Eigen::Tensor<double, 4>& t2) {
    const double bytes = 8.0 * ox * oy * (double)vx * vy;
    if (bytes > (double)mshqc_dropin::t2_max_bytes()) {
        t2 = Eigen::Tensor<double, 4>();
        return false;
    }
    t2 = Eigen::Tensor<double, 4>(ox, oy, vx, vy);
    std::vector<double> row((size_t)oy * vx * vy);
    for (int i = 0; i < ox; ++i) {
        check(mshqc_cd_get_t2_block(ctx, block, i, 1, 0, oy, row.data(), MSHQC_CD_HOST));
        for (int j = 0; j < oy; ++j)
            for (int a = 0; a < vx; ++a)
                for (int b = 0; b < vy; ++b) t2(i, j, a, b) = row[((size_t)j * vx + a) * vy + b];
    }
    return true;
}

// B^Q_ia of one spin into the reference's vector<MatrixXd>[Q](i, a)
std::vector<Eigen::MatrixXd> fetch_mo_vectors(mshqc_cd_ctx* ctx, int spin, int nocc, int nvir, int nvec) {
    std::vector<double> B((size_t)nocc * nvir * nvec);
    check(mshqc_cd_transform(ctx, spin, MSHQC_CD_FP64, B.data(), MSHQC_CD_HOST));
    std::vector<Eigen::MatrixXd> out(nvec, Eigen::MatrixXd(nocc, nvir));
    for (int i = 0; i < nocc; ++i)
        for (int a = 0; a < nvir; ++a)
            for (int q = 0; q < nvec; ++q) out[q](i, a) = B[((size_t)i * nvir + a) * nvec + q];
    return out;
}

}  // namespace

// ---------------------------------------------------------------------------
// CholeskyRMP2 (reference src/mp2/cholesky_rmp2.cc)
// ---------------------------------------------------------------------------
CholeskyRMP2::CholeskyRMP2(const Molecule& mol, const BasisSet& basis, std::shared_ptr<IntegralEngine> integrals,
                           const SCFResult& rhf_result, const CholeskyRMP2Config& config)
    : mol_(mol), basis_(basis), integrals_(integrals), rhf_(rhf_result), config_(config), cholesky_ptr_(nullptr) {
    nbf_ = basis.n_basis_functions();
    nocc_ = rhf_.n_occ_alpha;
    nvirt_ = nbf_ - nocc_;
    if (config_.print_level > 0)
        std::cout << "\n[CholeskyRMP2] Decomposing integrals on the GPU (Threshold=" << config_.cholesky_threshold
                  << ")...\n";
    internal_cholesky_ = std::make_unique<integrals::CholeskyERI>(config_.cholesky_threshold);
    internal_cholesky_->decompose(integrals_->compute_eri());
    cholesky_ptr_ = internal_cholesky_.get();
}

CholeskyRMP2::CholeskyRMP2(const Molecule& mol, const BasisSet& basis, std::shared_ptr<IntegralEngine> integrals,
                           const SCFResult& rhf_result, const CholeskyRMP2Config& config,
                           const integrals::CholeskyERI& existing_cholesky)
    : mol_(mol), basis_(basis), integrals_(integrals), rhf_(rhf_result), config_(config),
      cholesky_ptr_(&existing_cholesky) {
    nbf_ = basis.n_basis_functions();
    nocc_ = rhf_.n_occ_alpha;
    nvirt_ = nbf_ - nocc_;
}

foundation::CholeskyRMP2Result CholeskyRMP2::compute() {
    mshqc_cd_ctx* ctx = context();
    upload_vectors(ctx, *cholesky_ptr_, nbf_);
    upload_orbitals(ctx, MSHQC_CD_ALPHA, rhf_.C_alpha, rhf_.orbital_energies_alpha, nocc_);
    mshqc_cd_energy e{};
    check(mshqc_cd_mp2_energy(ctx, MSHQC_CD_RESTRICTED, mshqc_dropin::precision(), &e));
    fetch_t2(ctx, 0, nocc_, nocc_, nvirt_, nvirt_, t2_);
    foundation::CholeskyRMP2Result r;
    r.e_rhf = rhf_.energy_total;
    r.e_corr = e.total;
    r.e_total = r.e_rhf + r.e_corr;
    r.t2 = t2_;
    r.n_occ = nocc_;
    r.n_virt = nvirt_;
    r.chol_vectors = cholesky_ptr_->get_L_vectors();
    r.n_chol_vectors = cholesky_ptr_->n_vectors();
    if (config_.print_level > 0) {
        std::cout << std::setprecision(8);
        std::cout << "  RHF Energy:      " << std::setw(14) << r.e_rhf << " Ha\n";
        std::cout << "  Cholesky RMP2:   " << std::setw(14) << r.e_corr << " Ha (" << e.ms_total
                  << " ms on the GPU)\n";
        std::cout << "  Total Energy:    " << std::setw(14) << r.e_total << " Ha\n";
    }
    return r;
}

std::vector<Eigen::MatrixXd> CholeskyRMP2::transform_vectors() {
    mshqc_cd_ctx* ctx = context();
    upload_vectors(ctx, *cholesky_ptr_, nbf_);
    upload_orbitals(ctx, MSHQC_CD_ALPHA, rhf_.C_alpha, rhf_.orbital_energies_alpha, nocc_);
    return fetch_mo_vectors(ctx, MSHQC_CD_ALPHA, nocc_, nvirt_, cholesky_ptr_->n_vectors());
}

// ---------------------------------------------------------------------------
// CholeskyUMP2 (reference src/mp2/cholesky_ump2.cc)
// ---------------------------------------------------------------------------
CholeskyUMP2::CholeskyUMP2(const SCFResult& uhf_result, const BasisSet& basis,
                           std::shared_ptr<IntegralEngine> integrals, const CholeskyUMP2Config& config,
                           const integrals::CholeskyERI& cholesky_from_uhf)
    : uhf_(uhf_result), basis_(basis), integrals_(integrals), config_(config) {
    nbf_ = basis.n_basis_functions();
    nocc_a_ = uhf_result.n_occ_alpha;
    nocc_b_ = uhf_result.n_occ_beta;
    nvir_a_ = nbf_ - nocc_a_;
    nvir_b_ = nbf_ - nocc_b_;
    cholesky_ = std::make_unique<integrals::CholeskyERI>(cholesky_from_uhf);   // a copy, as the reference
    n_cholesky_ = cholesky_->n_vectors();
}

void CholeskyUMP2::decompose_eri() {
    cholesky_ = std::make_unique<integrals::CholeskyERI>(config_.cholesky_threshold);
    cholesky_->decompose(integrals_->compute_eri());
    n_cholesky_ = cholesky_->n_vectors();
}

void CholeskyUMP2::transform_cholesky_vectors() {
    mshqc_cd_ctx* ctx = context();
    L_ia_alpha_ = fetch_mo_vectors(ctx, MSHQC_CD_ALPHA, nocc_a_, nvir_a_, n_cholesky_);
    L_ia_beta_ = fetch_mo_vectors(ctx, MSHQC_CD_BETA, nocc_b_, nvir_b_, n_cholesky_);
}

CholeskyUMP2Result CholeskyUMP2::compute() {
    const auto t_start = std::chrono::steady_clock::now();
    CholeskyUMP2Result result;
    if (n_cholesky_ == 0) {
        decompose_eri();
        result.time_cholesky_s = seconds_since(t_start);
    }
    mshqc_cd_ctx* ctx = context();
    upload_vectors(ctx, *cholesky_, nbf_);
    upload_orbitals(ctx, MSHQC_CD_ALPHA, uhf_.C_alpha, uhf_.orbital_energies_alpha, nocc_a_);
    upload_orbitals(ctx, MSHQC_CD_BETA, uhf_.C_beta, uhf_.orbital_energies_beta, nocc_b_);
    mshqc_cd_energy e{};
    check(mshqc_cd_mp2_energy(ctx, MSHQC_CD_UNRESTRICTED, mshqc_dropin::precision(), &e));
    const auto t1 = std::chrono::steady_clock::now();
    transform_cholesky_vectors();   // L_ia for CholeskyUMP3 (friend access)
    result.time_transform_s = seconds_since(t1) + e.ms_transform / 1e3;
    result.time_energy_s = e.ms_energy / 1e3;
    result.e_corr_ss_aa = e.ss_aa;
    result.e_corr_ss_bb = e.ss_bb;
    result.e_corr_os = e.os;
    result.e_corr_total = e.total;
    result.e_total = uhf_.energy_total + e.total;
    result.n_cholesky_vectors = n_cholesky_;
    result.compression_ratio = cholesky_->compression_ratio();
    size_t mem = 0;
    for (const auto& L : L_ia_alpha_) mem += L.size() * sizeof(double);
    for (const auto& L : L_ia_beta_) mem += L.size() * sizeof(double);
    result.memory_mb = mem / (1024.0 * 1024.0);
    if (config_.print_level > 0) {
        std::cout << std::fixed << std::setprecision(10);
        std::cout << "SS (aa):        " << std::setw(18) << result.e_corr_ss_aa << " Ha\n";
        std::cout << "SS (bb):        " << std::setw(18) << result.e_corr_ss_bb << " Ha\n";
        std::cout << "OS (ab):        " << std::setw(18) << result.e_corr_os << " Ha\n";
        std::cout << "Correlation:    " << std::setw(18) << result.e_corr_total << " Ha\n";
    }
    return result;
}

void CholeskyUMP2::compute_t2_amplitudes() {
    mshqc_cd_ctx* ctx = context();
    upload_vectors(ctx, *cholesky_, nbf_);
    upload_orbitals(ctx, MSHQC_CD_ALPHA, uhf_.C_alpha, uhf_.orbital_energies_alpha, nocc_a_);
    upload_orbitals(ctx, MSHQC_CD_BETA, uhf_.C_beta, uhf_.orbital_energies_beta, nocc_b_);
    fetch_t2(ctx, 0, nocc_a_, nocc_a_, nvir_a_, nvir_a_, t2_aa_);
    fetch_t2(ctx, 1, nocc_b_, nocc_b_, nvir_b_, nvir_b_, t2_bb_);
    fetch_t2(ctx, 2, nocc_a_, nocc_b_, nvir_a_, nvir_b_, t2_ab_);
}

// ---------------------------------------------------------------------------
// CholeskyOMP2 (reference src/mp2/cholesky_omp2.cc)
// ---------------------------------------------------------------------------
CholeskyOMP2::CholeskyOMP2(const Molecule& mol, const BasisSet& basis, std::shared_ptr<IntegralEngine> integrals,
                           const SCFResult& scf_guess, const CholeskyOMP2Config& config)
    : mol_(mol), basis_(basis), integrals_(integrals), scf_(scf_guess), config_(config) {
    nbf_ = (int)scf_.C_alpha.rows();
    na_ = scf_.n_occ_alpha;
    nb_ = scf_.n_occ_beta;
    va_ = nbf_ - na_;
    vb_ = nbf_ - nb_;
    internal_cholesky_ = std::make_unique<integrals::CholeskyERI>(config_.cholesky_threshold);
    internal_cholesky_->decompose(integrals_->compute_eri());
    cholesky_ptr_ = internal_cholesky_.get();
}

CholeskyOMP2::CholeskyOMP2(const Molecule& mol, const BasisSet& basis, std::shared_ptr<IntegralEngine> integrals,
                           const SCFResult& scf_guess, const CholeskyOMP2Config& config,
                           const integrals::CholeskyERI& cholesky_vectors)
    : mol_(mol), basis_(basis), integrals_(integrals), scf_(scf_guess), config_(config),
      cholesky_ptr_(&cholesky_vectors) {
    nbf_ = (int)scf_.C_alpha.rows();
    na_ = scf_.n_occ_alpha;
    nb_ = scf_.n_occ_beta;
    va_ = nbf_ - na_;
    vb_ = nbf_ - nb_;
    if (cholesky_ptr_->n_vectors() == 0)
        throw std::runtime_error("CholeskyOMP2 initialized with empty reused vectors");
}

OMP2Result CholeskyOMP2::compute() {
    mshqc_cd_ctx* ctx = context();
    upload_vectors(ctx, *cholesky_ptr_, nbf_);
    upload_orbitals(ctx, MSHQC_CD_ALPHA, scf_.C_alpha, scf_.orbital_energies_alpha, na_);
    upload_orbitals(ctx, MSHQC_CD_BETA, scf_.C_beta, scf_.orbital_energies_beta, nb_);
    const Eigen::MatrixXd H = integrals_->compute_core_hamiltonian();
    check(mshqc_cd_set_core_hamiltonian(ctx, H.data(), MSHQC_CD_HOST));
    mshqc_cd_omp2_config cfg{config_.max_iterations, config_.energy_threshold, config_.gradient_threshold,
                             scf_.energy_total};
    const bool have_p = scf_.P_alpha.rows() == nbf_ && scf_.P_beta.rows() == nbf_;
    mshqc_cd_omp2_result res{};
    check(mshqc_cd_omp2(ctx, &cfg, have_p ? scf_.P_alpha.data() : nullptr, have_p ? scf_.P_beta.data() : nullptr,
                        MSHQC_CD_HOST, &res));
    OMP2Result r;
    r.energy_scf = res.energy_scf;
    r.energy_total = res.energy_total;
    r.energy_mp2_corr = res.energy_mp2_corr;
    r.converged = res.converged != 0;
    r.iterations = res.iterations;
    r.n_occ_alpha = na_;
    r.n_occ_beta = nb_;
    r.n_virt_alpha = va_;
    r.n_virt_beta = vb_;
    r.C_alpha = Eigen::MatrixXd(nbf_, nbf_);
    r.C_beta = Eigen::MatrixXd(nbf_, nbf_);
    check(mshqc_cd_get_orbitals(ctx, MSHQC_CD_ALPHA, r.C_alpha.data(), MSHQC_CD_HOST));
    check(mshqc_cd_get_orbitals(ctx, MSHQC_CD_BETA, r.C_beta.data(), MSHQC_CD_HOST));
    scf_.C_alpha = r.C_alpha;
    scf_.C_beta = r.C_beta;
    r.orbital_energies_alpha = scf_.orbital_energies_alpha;   // never updated, as in the reference
    r.orbital_energies_beta = scf_.orbital_energies_beta;
    if (config_.print_level > 0)
        std::cout << "[CholeskyOMP2] " << (r.converged ? "converged" : "not converged") << " after "
                  << r.iterations << " iterations, E(corr) = " << r.energy_mp2_corr << " Eh\n";
    return r;
}

}  // namespace mshqc
