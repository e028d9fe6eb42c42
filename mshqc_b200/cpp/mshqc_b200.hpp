// C++ mirror of mshqc's Cholesky-vector MP2 classes over the C ABI of
// libmshqc_cuda.so (include/mshqc_cd.h).
//
// Same class names, constructor arguments, configuration fields, result
// fields and error behaviour as the reference's CholeskyERI
// (include/mshqc/integrals/cholesky_eri.h:37-99), CholeskyRMP2
// (include/mshqc/cholesky_rmp2.h:28-90), CholeskyUMP2
// (include/mshqc/cholesky_ump2.h:40-118) and CholeskyOMP2
// (include/mshqc/cholesky_omp2.h:28-55), with the compute on the GPU.
// The reference's Molecule / BasisSet / IntegralEngine are outside this
// path: the classes read only the basis size and, through IntegralSource,
// the core Hamiltonian and the ERI tensor.
//
// Deviations, all additive or safer:
//  * CholeskyERI::set_vectors injects vectors (the reference's add_vector
//    does not count them, cholesky_eri.h:76-83);
//  * CholeskyRMP2Config / CholeskyUMP2Config carry `precision` (0 = FP64,
//    1 = mixed FP16x3) and all configs carry `device`;
//  * the stored amplitudes (CholeskyRMP2Result::t2, CholeskyUMP2's t2 after
//    compute_t2_amplitudes, both (i,j,a,b) column-major as Eigen stores
//    them) come from mshqc_cd_get_t2_block in FP64 and stay empty above
//    MSHQC_T2_MAX_BYTES (default 8 GiB), where the reference would run out
//    of host memory;
//  * an empty set of reused vectors makes CholeskyOMP2 throw
//    std::runtime_error where the reference calls exit(1) (cholesky_omp2.cc:62-65).
#pragma once

#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mshqc_cd.h"

namespace mshqc_b200 {

// Dense matrix in column-major order (the storage of Eigen::MatrixXd).
class Matrix {
public:
    Matrix() = default;
    Matrix(int rows, int cols, double value = 0.0) : r_(rows), c_(cols), d_((size_t)rows * cols, value) {}
    int rows() const { return r_; }
    int cols() const { return c_; }
    double* data() { return d_.data(); }
    const double* data() const { return d_.data(); }
    double& operator()(int r, int c) { return d_[(size_t)c * r_ + r]; }
    double operator()(int r, int c) const { return d_[(size_t)c * r_ + r]; }
    bool empty() const { return d_.empty(); }

private:
    int r_ = 0, c_ = 0;
    std::vector<double> d_;
};
using Vector = std::vector<double>;

// What the MP2 classes need from the reference's IntegralEngine.
class IntegralSource {
public:
    virtual ~IntegralSource() = default;
    virtual Matrix compute_core_hamiltonian() = 0;
    // (ij|kl) at ((i N + j) N + k) N + l
    virtual std::vector<double> compute_eri() = 0;
};

// SCFResult (reference include/mshqc/scf.h:67-115), the fields read here.
struct SCFResult {
    double energy_electronic = 0.0, energy_nuclear = 0.0, energy_total = 0.0;
    Vector orbital_energies_alpha, orbital_energies_beta;
    Matrix C_alpha, C_beta, P_alpha, P_beta, F_alpha, F_beta;
    int iterations = 0;
    bool converged = false;
    double gradient_norm = 0.0;
    int n_occ_alpha = 0, n_occ_beta = 0;
};

struct CholeskyDecompositionResult {
    int n_vectors = 0;
    int n_basis = 0;
    double threshold = 0.0;
    double max_error = 0.0;
    double rms_error = 0.0;
    double compression_ratio = 0.0;
    bool converged = false;
};

// Owns one device context; every failure of the C ABI becomes a
// std::runtime_error with the library's message.
class DeviceContext {
public:
    explicit DeviceContext(int device = 0);
    ~DeviceContext();
    DeviceContext(const DeviceContext&) = delete;
    DeviceContext& operator=(const DeviceContext&) = delete;
    mshqc_cd_ctx* get() const { return ctx_; }

private:
    mshqc_cd_ctx* ctx_ = nullptr;
};
void check(int rc);

class CholeskyERI {
public:
    explicit CholeskyERI(double threshold = 1e-6);   // std::invalid_argument if threshold <= 0
    // eri_full: N^4, (ij|kl) at ((i N + j) N + k) N + l; decomposed on the GPU
    CholeskyDecompositionResult decompose(const std::vector<double>& eri_full, int n_basis, int device = 0);
    void set_vectors(const double* L, int n_basis, int n_vectors);
    double reconstruct(int i, int j, int a, int b) const;
    int n_vectors() const { return n_vectors_; }
    int n_basis() const { return n_basis_; }
    double threshold() const { return threshold_; }
    bool is_decomposed() const { return decomposed_; }
    double compression_ratio() const;
    size_t storage_bytes() const { return L_.size() * sizeof(double); }
    const std::vector<double>& vectors() const { return L_; }   // M * N * N, vector Q at Q N^2
    std::vector<Vector> get_L_vectors() const;
    void reset();

private:
    std::vector<double> L_;
    int n_basis_ = 0, n_vectors_ = 0;
    double threshold_ = 1e-6;
    bool decomposed_ = false;
};

namespace foundation {
struct CholeskyRMP2Result {
    double e_rhf = 0.0, e_corr = 0.0, e_total = 0.0;
    std::vector<double> t2;              // o*o*v*v, element (i,j,a,b) at i + o (j + o (a + v b))
    std::vector<Vector> chol_vectors;    // the AO vectors, for reuse by MP3
    int n_chol_vectors = 0, n_occ = 0, n_virt = 0;
};
}  // namespace foundation

struct CholeskyRMP2Config {
    double cholesky_threshold = 1e-6;
    int print_level = 1;
    int precision = MSHQC_CD_FP64;
    int device = 0;
};

class CholeskyRMP2 {
public:
    // decomposes integrals->compute_eri() (reference cholesky_rmp2.cc:20-41)
    CholeskyRMP2(int n_basis, std::shared_ptr<IntegralSource> integrals, const SCFResult& rhf_result,
                 const CholeskyRMP2Config& config = CholeskyRMP2Config());
    // reuses vectors without copying them (reference cholesky_rmp2.cc:46-66)
    CholeskyRMP2(int n_basis, std::shared_ptr<IntegralSource> integrals, const SCFResult& rhf_result,
                 const CholeskyRMP2Config& config, const CholeskyERI& existing_cholesky);
    foundation::CholeskyRMP2Result compute();

private:
    int nbf_, nocc_, nvirt_;
    std::shared_ptr<IntegralSource> integrals_;
    SCFResult rhf_;
    CholeskyRMP2Config config_;
    std::unique_ptr<CholeskyERI> internal_;
    const CholeskyERI* chol_ = nullptr;
};

struct CholeskyUMP2Config {
    double cholesky_threshold = 1e-6;
    bool use_on_the_fly = false;
    bool validate_energy = false;
    int print_level = 1;
    int precision = MSHQC_CD_FP64;
    int device = 0;
};

struct CholeskyUMP2Result {
    double e_corr_ss_aa = 0.0, e_corr_ss_bb = 0.0, e_corr_os = 0.0, e_corr_total = 0.0, e_total = 0.0;
    int n_cholesky_vectors = 0;
    double compression_ratio = 0.0, memory_mb = 0.0;
    double time_cholesky_s = 0.0, time_transform_s = 0.0, time_energy_s = 0.0;
};

class CholeskyUMP2 {
public:
    // reference cholesky_ump2.cc:30-62 (the vectors are copied, as there)
    CholeskyUMP2(const SCFResult& uhf_result, int n_basis, std::shared_ptr<IntegralSource> integrals,
                 const CholeskyUMP2Config& config, const CholeskyERI& cholesky);
    CholeskyUMP2Result compute();
    // t2_aa, t2_bb, t2_ab = (ia|jb)/D (reference cholesky_ump2.cc:471-556)
    void compute_t2_amplitudes();
    const CholeskyERI& get_cholesky() const { return chol_; }
    int n_occ_alpha() const { return uhf_.n_occ_alpha; }
    int n_occ_beta() const { return uhf_.n_occ_beta; }
    int n_basis() const { return nbf_; }
    const std::vector<double>& t2_aa() const { return t2_aa_; }   // (i,j,a,b) column-major
    const std::vector<double>& t2_bb() const { return t2_bb_; }
    const std::vector<double>& t2_ab() const { return t2_ab_; }
    // L^K_ia after compute(): [K](i, a) (the reference's L_ia_alpha_ / L_ia_beta_)
    const std::vector<Matrix>& L_ia_alpha() const { return L_ia_alpha_; }
    const std::vector<Matrix>& L_ia_beta() const { return L_ia_beta_; }

private:
    SCFResult uhf_;
    int nbf_;
    std::shared_ptr<IntegralSource> integrals_;
    CholeskyUMP2Config config_;
    CholeskyERI chol_;
    std::vector<double> t2_aa_, t2_bb_, t2_ab_;
    std::vector<Matrix> L_ia_alpha_, L_ia_beta_;
};

struct CholeskyOMP2Config {
    int max_iterations = 50;
    double energy_threshold = 1e-6;
    double gradient_threshold = 1e-5;
    double cholesky_threshold = 1e-6;
    int print_level = 1;
    int device = 0;
};

struct OMP2Result {
    double energy_scf = 0.0, energy_mp2_ss = 0.0, energy_mp2_os = 0.0, energy_mp2_corr = 0.0,
           energy_total = 0.0;
    int n_occ_alpha = 0, n_occ_beta = 0, n_virt_alpha = 0, n_virt_beta = 0;
    Vector orbital_energies_alpha, orbital_energies_beta;
    Matrix C_alpha, C_beta;
    bool converged = false;
    int iterations = 0;
};

class CholeskyOMP2 {
public:
    CholeskyOMP2(std::shared_ptr<IntegralSource> integrals, const SCFResult& scf_guess,
                 const CholeskyOMP2Config& config = CholeskyOMP2Config());
    CholeskyOMP2(std::shared_ptr<IntegralSource> integrals, const SCFResult& scf_guess,
                 const CholeskyOMP2Config& config, const CholeskyERI& cholesky_vectors);
    OMP2Result compute();

private:
    std::shared_ptr<IntegralSource> integrals_;
    SCFResult scf_;
    CholeskyOMP2Config config_;
    std::unique_ptr<CholeskyERI> internal_;
    const CholeskyERI* chol_ = nullptr;
};

}  // namespace mshqc_b200
