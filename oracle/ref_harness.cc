// Oracle test infrastructure -- NOT part of the product.
//
// A C-callable harness around the reference's OWN Cholesky-MP2 classes,
// compiled unchanged from the reference sources by oracle/Makefile:
//   CholeskyRMP2   src/mp2/cholesky_rmp2.cc
//   CholeskyUMP2   src/mp2/cholesky_ump2.cc
//   CholeskyOMP2   src/mp2/cholesky_omp2.cc
//   CholeskyERI    src/integrals/cholesky_eri.cc
//   CholeskyRHF / CholeskyUHF Fock builds  src/scf/cholesky_{rhf,uhf}.cc
// Tests and bench.py's reference arm call it through ctypes (oracle/ref.py)
// to pin the CPU restatement and to time the reference CPU path.
//
// Vector injection: CholeskyERI::add_vector (include/mshqc/integrals/
// cholesky_eri.h:76-78) does not bump the private n_vectors_ counter, so the
// only public route to a populated container is decompose() of a full N^4
// tensor.  The harness therefore opens the private members of the reference
// classes in THIS translation unit only (the #define below); the reference
// objects themselves are compiled untouched.
#include <Eigen/Dense>
#include <Eigen/Eigenvalues>
#include <unsupported/Eigen/CXX11/Tensor>
#include <unsupported/Eigen/MatrixFunctions>

#include <chrono>
#include <cstring>
#include <exception>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <omp.h>

#define private public
#define protected public
#include "mshqc/basis.h"
#include "mshqc/cholesky_omp2.h"
#include "mshqc/cholesky_rhf.h"
#include "mshqc/cholesky_rmp2.h"
#include "mshqc/cholesky_uhf.h"
#include "mshqc/cholesky_ump2.h"
#include "mshqc/integrals.h"
#include "mshqc/integrals/cholesky_eri.h"
#include "mshqc/molecule.h"
#include "mshqc/scf.h"
#undef private
#undef protected

namespace mshqc {
namespace oracle_stub {
extern Eigen::MatrixXd g_core_hamiltonian;
extern Eigen::MatrixXd g_overlap, g_kinetic, g_nuclear;
extern Eigen::Tensor<double, 4> g_eri;
extern bool g_have_eri;
}  // namespace oracle_stub
}  // namespace mshqc

using namespace mshqc;

namespace {

thread_local std::string g_err;

struct Quiet {
    std::streambuf* old;
    std::ostringstream sink;
    explicit Quiet(bool on) : old(nullptr) {
        if (on) old = std::cout.rdbuf(sink.rdbuf());
    }
    ~Quiet() {
        if (old) std::cout.rdbuf(old);
    }
};

// A basis of N s-shells: the reference classes only ask it for
// n_basis_functions() (src/core/basis.cc:252-256).
BasisSet make_basis(int N) {
    BasisSet b;
    for (int k = 0; k < N; ++k) {
        Shell s(AngularMomentum::S, 0, {0.0, 0.0, 0.0});
        s.add_primitive(1.0, 1.0);
        b.add_shell(s);
    }
    return b;
}

void fill_cholesky(integrals::CholeskyERI& chol, int N, int M, const double* L) {
    chol.L_vectors_.clear();
    chol.L_vectors_.reserve(M);
    const size_t nn = static_cast<size_t>(N) * N;
    for (int q = 0; q < M; ++q) {
        Eigen::VectorXd v(nn);
        std::memcpy(v.data(), L + q * nn, nn * sizeof(double));
        chol.L_vectors_.push_back(std::move(v));
    }
    chol.n_vectors_ = M;
    chol.n_basis_ = N;
    chol.decomposed_ = true;
}

SCFResult make_scf(int N, const double* Ca, const double* Cb, const double* ea,
                   const double* eb, int na, int nb, double e_scf) {
    SCFResult r{};
    r.C_alpha = Eigen::Map<const Eigen::MatrixXd>(Ca, N, N);
    r.C_beta = Eigen::Map<const Eigen::MatrixXd>(Cb ? Cb : Ca, N, N);
    r.orbital_energies_alpha = Eigen::Map<const Eigen::VectorXd>(ea, N);
    r.orbital_energies_beta = Eigen::Map<const Eigen::VectorXd>(eb ? eb : ea, N);
    r.n_occ_alpha = na;
    r.n_occ_beta = nb;
    r.P_alpha = r.C_alpha.leftCols(na) * r.C_alpha.leftCols(na).transpose();
    r.P_beta = r.C_beta.leftCols(nb) * r.C_beta.leftCols(nb).transpose();
    r.energy_total = e_scf;
    r.energy_electronic = e_scf;
    r.energy_nuclear = 0.0;
    r.iterations = 0;
    r.converged = true;
    r.gradient_norm = 0.0;
    return r;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

// CholeskyRMP2 (reuse-vector constructor, src/mp2/cholesky_rmp2.cc:46-66)
// then compute() (:97-179).  out[0]=e_corr, out[1]=e_total, out[2]=seconds
// spent in compute().  t2 (o*o*v*v, Eigen column-major (i,j,a,b)) is copied
// out when t2_out is non-null.
int ref_rmp2(int N, int M, const double* L, const double* C, const double* eps,
             int nocc, double e_scf, int nthreads, double* out, double* t2_out) {
    try {
        if (nthreads > 0) omp_set_num_threads(nthreads);
        Quiet q(true);
        Molecule mol;
        BasisSet basis = make_basis(N);
        auto ints = std::make_shared<IntegralEngine>(mol, basis);
        integrals::CholeskyERI chol(1e-6);
        fill_cholesky(chol, N, M, L);
        SCFResult scf = make_scf(N, C, nullptr, eps, nullptr, nocc, nocc, e_scf);
        CholeskyRMP2Config cfg;
        cfg.print_level = 0;
        CholeskyRMP2 rmp2(mol, basis, ints, scf, cfg, chol);
        auto t0 = std::chrono::steady_clock::now();
        auto res = rmp2.compute();
        out[2] = seconds_since(t0);
        out[0] = res.e_corr;
        out[1] = res.e_total;
        if (t2_out) std::memcpy(t2_out, res.t2.data(), res.t2.size() * sizeof(double));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// CholeskyUMP2 (src/mp2/cholesky_ump2.cc:30-62) then compute() (:68-174).
// out[0..4] = ss_aa, ss_bb, os, e_corr_total, e_total; out[5] = seconds.
int ref_ump2(int N, int M, const double* L, const double* Ca, const double* Cb,
             const double* ea, const double* eb, int na, int nb, double e_scf,
             int nthreads, double* out) {
    try {
        if (nthreads > 0) omp_set_num_threads(nthreads);
        Quiet q(true);
        Molecule mol;
        BasisSet basis = make_basis(N);
        auto ints = std::make_shared<IntegralEngine>(mol, basis);
        integrals::CholeskyERI chol(1e-6);
        fill_cholesky(chol, N, M, L);
        SCFResult scf = make_scf(N, Ca, Cb, ea, eb, na, nb, e_scf);
        CholeskyUMP2Config cfg;
        cfg.print_level = 0;
        CholeskyUMP2 ump2(scf, basis, ints, cfg, chol);
        auto t0 = std::chrono::steady_clock::now();
        auto res = ump2.compute();
        out[5] = seconds_since(t0);
        out[0] = res.e_corr_ss_aa;
        out[1] = res.e_corr_ss_bb;
        out[2] = res.e_corr_os;
        out[3] = res.e_corr_total;
        out[4] = res.e_total;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// One CholeskyOMP2 gradient evaluation, step by step as compute() does it
// (src/mp2/cholesky_omp2.cc:441-466): t2, energy, OPDM, relaxed densities,
// generalized Fock per spin, w_ai = 2 F_mo(vir, occ).
// Outputs (column-major): e[0]=E_mp2, e[1]=seconds;
// Goo_a (na*na), Gvv_a (va*va), Goo_b (nb*nb), Gvv_b (vb*vb),
// Fa, Fb (N*N MO-basis generalized Fock), wa (va*na), wb (vb*nb).
int ref_omp2_pieces(int N, int M, const double* L, const double* Ca,
                    const double* Cb, const double* ea, const double* eb, int na,
                    int nb, const double* H, int nthreads, double* e,
                    double* Goo_a, double* Gvv_a, double* Goo_b, double* Gvv_b,
                    double* Fa, double* Fb, double* wa, double* wb) {
    try {
        if (nthreads > 0) omp_set_num_threads(nthreads);
        Quiet q(true);
        oracle_stub::g_core_hamiltonian = Eigen::Map<const Eigen::MatrixXd>(H, N, N);
        Molecule mol;
        BasisSet basis = make_basis(N);
        auto ints = std::make_shared<IntegralEngine>(mol, basis);
        integrals::CholeskyERI chol(1e-6);
        fill_cholesky(chol, N, M, L);
        SCFResult scf = make_scf(N, Ca, Cb, ea, eb, na, nb, 0.0);
        CholeskyOMP2Config cfg;
        cfg.print_level = 0;
        CholeskyOMP2 omp2(mol, basis, ints, scf, cfg, chol);
        auto t0 = std::chrono::steady_clock::now();
        omp2.compute_t2_amplitudes();
        e[0] = omp2.compute_mp2_energy_from_t2();
        omp2.build_opdm_alpha();
        omp2.build_opdm_beta();
        const int va = N - na, vb = N - nb;
        Eigen::MatrixXd Gfa = Eigen::MatrixXd::Zero(N, N);
        Gfa.block(0, 0, na, na) = omp2.G_oo_alpha_;
        Gfa.block(na, na, va, va) = omp2.G_vv_alpha_;
        Eigen::MatrixXd Pa = omp2.scf_.P_alpha +
                             omp2.scf_.C_alpha * Gfa * omp2.scf_.C_alpha.transpose();
        Eigen::MatrixXd Gfb = Eigen::MatrixXd::Zero(N, N);
        Gfb.block(0, 0, nb, nb) = omp2.G_oo_beta_;
        Gfb.block(nb, nb, vb, vb) = omp2.G_vv_beta_;
        Eigen::MatrixXd Pb = omp2.scf_.P_beta +
                             omp2.scf_.C_beta * Gfb * omp2.scf_.C_beta.transpose();
        Eigen::MatrixXd FA = omp2.build_gfock_from_density(Pa, Pb, true);
        Eigen::MatrixXd FB = omp2.build_gfock_from_density(Pa, Pb, false);
        Eigen::MatrixXd WA = 2.0 * FA.block(na, 0, va, na);
        Eigen::MatrixXd WB = 2.0 * FB.block(nb, 0, vb, nb);
        e[1] = seconds_since(t0);
        std::memcpy(Goo_a, omp2.G_oo_alpha_.data(), sizeof(double) * na * na);
        std::memcpy(Gvv_a, omp2.G_vv_alpha_.data(), sizeof(double) * va * va);
        std::memcpy(Goo_b, omp2.G_oo_beta_.data(), sizeof(double) * nb * nb);
        std::memcpy(Gvv_b, omp2.G_vv_beta_.data(), sizeof(double) * vb * vb);
        std::memcpy(Fa, FA.data(), sizeof(double) * N * N);
        std::memcpy(Fb, FB.data(), sizeof(double) * N * N);
        std::memcpy(wa, WA.data(), sizeof(double) * va * na);
        std::memcpy(wb, WB.data(), sizeof(double) * vb * nb);
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// The MP2 part of one CholeskyOMP2 gradient evaluation, as compute() runs it
// (src/mp2/cholesky_omp2.cc:445-449): both spins' half transforms and t2
// (compute_t2_amplitudes :94-183), the energy from t2 (:189-230) and the
// OPDM blocks of both spins (:232-326); the generalized Fock builds that
// follow are not timed.  out[0] = E_mp2, out[1] = seconds.
int ref_omp2_mp2_part(int N, int M, const double* L, const double* Ca, const double* Cb,
                      const double* ea, const double* eb, int na, int nb, int nthreads,
                      double* out) {
    try {
        if (nthreads > 0) omp_set_num_threads(nthreads);
        Quiet q(true);
        Molecule mol;
        BasisSet basis = make_basis(N);
        auto ints = std::make_shared<IntegralEngine>(mol, basis);
        integrals::CholeskyERI chol(1e-6);
        fill_cholesky(chol, N, M, L);
        SCFResult scf = make_scf(N, Ca, Cb, ea, eb, na, nb, 0.0);
        CholeskyOMP2Config cfg;
        cfg.print_level = 0;
        CholeskyOMP2 omp2(mol, basis, ints, scf, cfg, chol);
        auto t0 = std::chrono::steady_clock::now();
        omp2.compute_t2_amplitudes();
        out[0] = omp2.compute_mp2_energy_from_t2();
        omp2.build_opdm_alpha();
        omp2.build_opdm_beta();
        out[1] = seconds_since(t0);
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// Full CholeskyOMP2::compute() (src/mp2/cholesky_omp2.cc:427-512).
// out[0..2] = energy_mp2_corr, energy_total, energy_scf; out[3] = seconds;
// iters[0] = iterations, iters[1] = converged.  Final C_alpha/C_beta are
// copied to Ca_out/Cb_out (column-major N*N).
int ref_omp2(int N, int M, const double* L, const double* Ca, const double* Cb,
             const double* ea, const double* eb, int na, int nb, const double* H,
             double e_scf, int max_iter, double e_thr, double g_thr, int nthreads,
             double* out, int* iters, double* Ca_out, double* Cb_out) {
    try {
        if (nthreads > 0) omp_set_num_threads(nthreads);
        Quiet q(true);
        oracle_stub::g_core_hamiltonian = Eigen::Map<const Eigen::MatrixXd>(H, N, N);
        Molecule mol;
        BasisSet basis = make_basis(N);
        auto ints = std::make_shared<IntegralEngine>(mol, basis);
        integrals::CholeskyERI chol(1e-6);
        fill_cholesky(chol, N, M, L);
        SCFResult scf = make_scf(N, Ca, Cb, ea, eb, na, nb, e_scf);
        CholeskyOMP2Config cfg;
        cfg.print_level = 0;
        cfg.max_iterations = max_iter;
        cfg.energy_threshold = e_thr;
        cfg.gradient_threshold = g_thr;
        CholeskyOMP2 omp2(mol, basis, ints, scf, cfg, chol);
        auto t0 = std::chrono::steady_clock::now();
        OMP2Result r = omp2.compute();
        out[3] = seconds_since(t0);
        out[0] = r.energy_mp2_corr;
        out[1] = r.energy_total;
        out[2] = r.energy_scf;
        iters[0] = r.iterations;
        iters[1] = r.converged ? 1 : 0;
        std::memcpy(Ca_out, r.C_alpha.data(), sizeof(double) * N * N);
        std::memcpy(Cb_out, r.C_beta.data(), sizeof(double) * N * N);
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// The reference's closed-shell pipeline on given AO integrals: RHF
// (src/scf/rhf.cc, DIIS src/scf/diis.cc) on S, T, V and the ERI tensor
// (N^4, element (ij|kl) at ((i N + j) N + k) N + l), then CholeskyRMP2 with
// constructor 1 (src/mp2/cholesky_rmp2.cc:20-41: decomposes the ERI tensor
// from the engine with cholesky_threshold) and compute().  Atoms: Z[natom],
// xyz[3 natom] in bohr.  out[0] = E_SCF (total), out[1] = E_corr,
// out[2] = number of Cholesky vectors, out[3] = SCF iterations,
// out[4] = converged; C_out (N*N column-major), eps_out (N), and nocc_out.
int ref_rhf_cdrmp2(int N, int natom, const double* Z, const double* xyz, const double* S, const double* T,
                   const double* V, const double* eri, double chol_thr, double e_thr, double d_thr, int nthreads,
                   double* out, double* C_out, double* eps_out, int* nocc_out) {
    try {
        if (nthreads > 0) omp_set_num_threads(nthreads);
        Quiet q(true);
        oracle_stub::g_core_hamiltonian.resize(0, 0);
        oracle_stub::g_overlap = Eigen::Map<const Eigen::MatrixXd>(S, N, N);
        oracle_stub::g_kinetic = Eigen::Map<const Eigen::MatrixXd>(T, N, N);
        oracle_stub::g_nuclear = Eigen::Map<const Eigen::MatrixXd>(V, N, N);
        oracle_stub::g_eri = Eigen::Tensor<double, 4>(N, N, N, N);
        std::memcpy(oracle_stub::g_eri.data(), eri, sizeof(double) * (size_t)N * N * N * N);
        oracle_stub::g_have_eri = true;
        Molecule mol;
        for (int a = 0; a < natom; ++a)
            mol.add_atom((int)std::lround(Z[a]), xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2]);
        BasisSet basis = make_basis(N);
        auto ints = std::make_shared<IntegralEngine>(mol, basis);
        SCFConfig scfg;
        scfg.print_level = 0;
        scfg.max_iterations = 200;
        scfg.energy_threshold = e_thr;
        scfg.density_threshold = d_thr;
        RHF rhf(mol, basis, ints, scfg);
        SCFResult r = rhf.compute();
        CholeskyRMP2Config cfg;
        cfg.cholesky_threshold = chol_thr;
        cfg.print_level = 0;
        CholeskyRMP2 rmp2(mol, basis, ints, r, cfg);
        auto res = rmp2.compute();
        out[0] = r.energy_total;
        out[1] = res.e_corr;
        out[2] = rmp2.cholesky_ptr_->n_vectors();
        out[3] = r.iterations;
        out[4] = r.converged ? 1.0 : 0.0;
        std::memcpy(C_out, r.C_alpha.data(), sizeof(double) * (size_t)N * N);
        std::memcpy(eps_out, r.orbital_energies_alpha.data(), sizeof(double) * (size_t)N);
        *nocc_out = r.n_occ_alpha;
        oracle_stub::g_have_eri = false;
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        oracle_stub::g_have_eri = false;
        return -1;
    }
}

// One Cholesky Fock build of the reference's SCF classes on given vectors,
// core Hamiltonian and densities (N x N, column-major):
//   nspin = 1: CholeskyRHF::build_fock (src/scf/cholesky_rhf.cc:99-137),
//              F = H + J - 0.5 K with P the total density, K screened when
//              screen != 0 (vectors of norm <= 1e-8 skipped);
//   nspin = 2: CholeskyUHF::build_fock_cholesky (src/scf/cholesky_uhf.cc:77-103),
//              F_s = H + J[P_a + P_b] - K[P_s].
int ref_cholesky_fock(int N, int M, const double* L, int nspin, const double* Pa, const double* Pb,
                      const double* H, int screen, double* Fa, double* Fb) {
    try {
        Quiet q(true);
        const Eigen::Map<const Eigen::MatrixXd> Hm(H, N, N);
        if (nspin == 1) {
            integrals::CholeskyERI chol(1e-6);
            fill_cholesky(chol, N, M, L);
            Molecule mol;
            mol.add_atom(2, 0.0, 0.0, 0.0);   // any closed shell: the Fock build reads no electron count
            BasisSet basis = make_basis(N);
            auto ints = std::make_shared<IntegralEngine>(mol, basis);
            CholeskyRHFConfig cfg;
            cfg.print_level = 0;
            cfg.screen_exchange = screen != 0;
            CholeskyRHF rhf(mol, basis, ints, cfg, chol);
            rhf.H_ = Hm;
            rhf.P_ = Eigen::Map<const Eigen::MatrixXd>(Pa, N, N);
            rhf.build_fock();
            std::memcpy(Fa, rhf.F_.data(), sizeof(double) * (size_t)N * N);
            return 0;
        }
        Molecule mol;
        mol.add_atom(2, 0.0, 0.0, 0.0);
        BasisSet basis = make_basis(N);
        auto ints = std::make_shared<IntegralEngine>(mol, basis);
        CholeskyUHFConfig cfg;
        cfg.print_level = 0;
        CholeskyUHF uhf(mol, basis, ints, 1, 1, cfg);
        const size_t nn = static_cast<size_t>(N) * N;
        std::vector<Eigen::VectorXd> vecs;
        vecs.reserve(M);
        for (int k = 0; k < M; ++k) vecs.push_back(Eigen::Map<const Eigen::VectorXd>(L + k * nn, nn));
        uhf.set_cholesky_vectors(vecs);
        uhf.H_ = Hm;
        uhf.P_a_ = Eigen::Map<const Eigen::MatrixXd>(Pa, N, N);
        uhf.P_b_ = Eigen::Map<const Eigen::MatrixXd>(Pb, N, N);
        uhf.build_fock_cholesky();
        std::memcpy(Fa, uhf.F_a_.data(), sizeof(double) * nn);
        std::memcpy(Fb, uhf.F_b_.data(), sizeof(double) * nn);
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

// CholeskyERI::decompose (src/integrals/cholesky_eri.cc:40-149) of a full
// ERI tensor given as Eigen's column-major (i,j,k,l) N^4 array.  Writes up to
// max_vec vectors of length N*N into L_out and the count into *M_out.
int ref_cholesky_decompose(int N, const double* eri, double threshold,
                           int max_vec, double* L_out, int* M_out) {
    try {
        Quiet q(true);
        Eigen::Tensor<double, 4> full(N, N, N, N);
        std::memcpy(full.data(), eri, sizeof(double) * full.size());
        integrals::CholeskyERI chol(threshold);
        chol.decompose(full);
        const int M = chol.n_vectors();
        *M_out = M;
        if (M > max_vec) {
            g_err = "ref_cholesky_decompose: output buffer too small";
            return -2;
        }
        const size_t nn = static_cast<size_t>(N) * N;
        for (int k = 0; k < M; ++k)
            std::memcpy(L_out + k * nn, chol.get_L_vectors()[k].data(), nn * sizeof(double));
        return 0;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return -1;
    }
}

}  // extern "C"
