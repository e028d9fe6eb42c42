// Test infrastructure: a program of the reference, written against its own
// public API (Molecule, BasisSet, IntegralEngine, RHF, CholeskyERI,
// CholeskyRMP2, CholeskyUMP2, CholeskyOMP2 from include/mshqc/*.h), linked
// with the reference's own molecule/basis/RHF sources and with the drop-in
// library in place of its integral, Cholesky and MP2 sources.  One entry
// point runs a closed-shell molecule through all of it for the Python test.
#include <cstring>
#include <exception>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>

#include "mshqc/basis.h"
#include "mshqc/cholesky_omp2.h"
#include "mshqc/cholesky_rmp2.h"
#include "mshqc/cholesky_ump2.h"
#include "mshqc/integrals.h"
#include "mshqc/integrals/cholesky_eri.h"
#include "mshqc/molecule.h"
#include "mshqc/scf.h"

using namespace mshqc;

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* dropin_last_error(void) { return g_err.c_str(); }

// Atoms Z[natom], xyz in Angstrom (converted with the reference's own
// ANGSTROM_TO_BOHR); basis `name` read by the reference's BasisSet from
// basis_dir/<name>.gbs.  out: [0] E_SCF, [1] RMP2 E_corr, [2] n vectors,
// [3] nocc, [4] nbf, [5] UMP2 ss_aa, [6] ss_bb, [7] os, [8] total,
// [9] OMP2 E_corr, [10] OMP2 iterations, [11] OMP2 converged,
// [12] number of alpha L_ia matrices, [13] t2 elements stored by UMP2 (aa).
// C_out (N*N), eps_out (N), L_out (room for max_vec * N*N), t2_out
// (o*o*v*v, the RMP2 result's t2 in Eigen's (i,j,a,b) column-major order).
int dropin_closed_shell(int natom, const int* Z, const double* xyz_ang, const char* basis_dir, const char* name,
                        double chol_thr, double* out, double* C_out, double* eps_out, double* L_out, int max_vec,
                        double* t2_out) {
    try {
        std::ostringstream sink;
        std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
        struct Restore {
            std::streambuf* o;
            ~Restore() { std::cout.rdbuf(o); }
        } restore{old};
        Molecule mol;
        for (int a = 0; a < natom; ++a)
            mol.add_atom(Z[a], xyz_ang[3 * a] * ANGSTROM_TO_BOHR, xyz_ang[3 * a + 1] * ANGSTROM_TO_BOHR,
                         xyz_ang[3 * a + 2] * ANGSTROM_TO_BOHR);
        BasisSet basis(name, mol, basis_dir);
        auto ints = std::make_shared<IntegralEngine>(mol, basis);
        SCFConfig scfg;
        scfg.print_level = 0;
        scfg.energy_threshold = 1e-12;
        scfg.density_threshold = 1e-10;
        scfg.max_iterations = 200;
        RHF rhf(mol, basis, ints, scfg);
        SCFResult scf = rhf.compute();
        const int N = basis.n_basis_functions(), o = scf.n_occ_alpha, v = N - o;

        CholeskyRMP2Config rcfg;
        rcfg.cholesky_threshold = chol_thr;
        rcfg.print_level = 0;
        CholeskyRMP2 rmp2(mol, basis, ints, scf, rcfg);           // decomposes on the GPU
        auto rr = rmp2.compute();

        integrals::CholeskyERI chol(chol_thr);
        chol.decompose(ints->compute_eri());
        CholeskyUMP2Config ucfg;
        ucfg.print_level = 0;
        CholeskyUMP2 ump2(scf, basis, ints, ucfg, chol);
        auto ur = ump2.compute();
        ump2.compute_t2_amplitudes();

        CholeskyOMP2Config ocfg;
        ocfg.print_level = 0;
        ocfg.max_iterations = 3;
        CholeskyOMP2 omp2(mol, basis, ints, scf, ocfg, chol);
        auto orr = omp2.compute();

        out[0] = scf.energy_total;
        out[1] = rr.e_corr;
        out[2] = rr.n_chol_vectors;
        out[3] = o;
        out[4] = N;
        out[5] = ur.e_corr_ss_aa;
        out[6] = ur.e_corr_ss_bb;
        out[7] = ur.e_corr_os;
        out[8] = ur.e_corr_total;
        out[9] = orr.energy_mp2_corr;
        out[10] = orr.iterations;
        out[11] = orr.converged ? 1.0 : 0.0;
        out[12] = 0.0;
        out[13] = 0.0;
        std::memcpy(C_out, scf.C_alpha.data(), sizeof(double) * N * N);
        std::memcpy(eps_out, scf.orbital_energies_alpha.data(), sizeof(double) * N);
        const auto& L = rr.chol_vectors;
        if ((int)L.size() > max_vec) {
            g_err = "L_out too small";
            return -2;
        }
        for (size_t q = 0; q < L.size(); ++q)
            std::memcpy(L_out + q * (size_t)N * N, L[q].data(), sizeof(double) * N * N);
        if (rr.t2.size() != (long)o * o * v * v) {
            g_err = "RMP2 result holds no t2";
            return -3;
        }
        std::memcpy(t2_out, rr.t2.data(), sizeof(double) * rr.t2.size());
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
