/*
 * mshqc_ao.h -- C ABI of the host-side AO integral engine (in
 * libmshqc_cuda.so, CPU only: no function here touches a GPU).
 *
 * Replaces the integral engine the reference builds on libint2: its
 * IntegralEngine (reference include/mshqc/integrals.h:38-224;
 * compute_overlap / compute_kinetic / compute_nuclear / compute_eri /
 * compute_eri_diagonal / compute_eri_column, implemented in
 * src/core/integrals.cc:96-459), whose ERI tensor feeds
 * CholeskyERI::decompose (src/integrals/cholesky_eri.cc:40-149) and whose
 * diagonal and columns feed the integral-direct decomposition
 * (src/integrals/cholesky_direct.cc:32-187).
 *
 * Shells follow what the reference hands to libint2 (src/core/basis.cc,
 * src/core/integrals.cc:96-145): coefficients as mshqc_ao_normalize_shell
 * leaves them (the reference's Shell::normalize; they multiply the raw
 * primitives, as in libint2 without renormalization, so functions are not
 * unit-norm in general), every Cartesian component of a shell with that same
 * coefficient, Cartesian order x^l, x^(l-1) y, ..., z^l, pure shells as real
 * solid harmonics m = -l .. l, each with the norm of the shell's x^l
 * component.  Coordinates in bohr.  Matrices N x N (symmetric);
 * the ERI tensor N^4 with (mu nu|lam sig) at ((mu N + nu) N + lam) N + sig
 * (by symmetry also Eigen's column-major (mu, nu, lam, sig), the reference's
 * ERITensor).  Every function returns 0 or a negative MSHQC_AO_ERR_*;
 * mshqc_ao_last_error() gives the message.
 */
#ifndef MSHQC_AO_H
#define MSHQC_AO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define MSHQC_AO_API __attribute__((visibility("default")))
#else
#define MSHQC_AO_API
#endif

enum mshqc_ao_status { MSHQC_AO_OK = 0, MSHQC_AO_ERR_ARG = -1, MSHQC_AO_ERR_INTERNAL = -2 };

/* A basis: nshell shells; shell s has angular momentum l[s] (0..6), pure[s]
 * (1: solid harmonics, 0: Cartesian; pure may be NULL for all Cartesian),
 * nprim[s] primitives whose exponents and normalized coefficients follow
 * those of the shells before it in exps / coefs, and its centre at
 * center[3 s .. 3 s + 2]. */
typedef struct {
    int nshell;
    const int* l;
    const int* pure;
    const int* nprim;
    const double* center;
    const double* exps;
    const double* coefs;
} mshqc_ao_basis;

/* Point nuclei: charges Z[natom], positions xyz[3 natom] (bohr). */
typedef struct {
    int natom;
    const double* Z;
    const double* xyz;
} mshqc_ao_nuclei;

MSHQC_AO_API const char* mshqc_ao_last_error(void);

/* In place, the reference's Shell::normalize (src/core/basis.cc:53-110):
 * coefs *= primitive norms of the x^l component, then coefs /=
 * sqrt(sum_ij coefs_i coefs_j (2 sqrt(a_i a_j) / (a_i + a_j))^(l + 3/2)). */
MSHQC_AO_API int mshqc_ao_normalize_shell(int l, int nprim, const double* exps, double* coefs);

/* Number of basis functions. */
MSHQC_AO_API int mshqc_ao_nbf(const mshqc_ao_basis* basis, int64_t* nbf);

/* Overlap, kinetic and nuclear-attraction matrices (any may be NULL):
 * IntegralEngine::compute_overlap / compute_kinetic / compute_nuclear. */
MSHQC_AO_API int mshqc_ao_one_electron(const mshqc_ao_basis* basis, const mshqc_ao_nuclei* nuclei, double* S,
                                       double* T, double* V);

/* The full ERI tensor (N^4 doubles): IntegralEngine::compute_eri. */
MSHQC_AO_API int mshqc_ao_eri(const mshqc_ao_basis* basis, double* eri);

/* (mu nu|mu nu) for every (mu, nu), N^2 doubles at mu N + nu:
 * IntegralEngine::compute_eri_diagonal. */
MSHQC_AO_API int mshqc_ao_eri_diagonal(const mshqc_ao_basis* basis, double* diag);

/* (mu nu|r s) for every (mu, nu) with pivot = r N + s, N^2 doubles:
 * IntegralEngine::compute_eri_column. */
MSHQC_AO_API int mshqc_ao_eri_column(const mshqc_ao_basis* basis, int64_t pivot, double* col);

/* sum_{A<B} Z_A Z_B / R_AB (Molecule::nuclear_repulsion_energy). */
MSHQC_AO_API int mshqc_ao_nuclear_repulsion(const mshqc_ao_nuclei* nuclei, double* e);

#ifdef __cplusplus
}
#endif

#endif /* MSHQC_AO_H */
