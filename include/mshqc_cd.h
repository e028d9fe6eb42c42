/*
 * mshqc_cd.h -- C ABI of the B200 Cholesky-vector MP2 library
 * (libmshqc_cuda.so).
 *
 * The library replaces the compute inside mshqc's CD-RMP2 / CD-UMP2 /
 * CD-OMP2 classes.  Every function returns an int status (0 = ok, negative =
 * error, see MSHQC_CD_ERR_*); the message of the last failure on the calling
 * thread is available from mshqc_cd_last_error().  No function calls exit()
 * or throws.  A context is single-threaded and stream-ordered: calls on one
 * context must not overlap; results are complete when a call returns.
 *
 * Array conventions (the reference's own, so its data can be passed as-is):
 *   L     AO Cholesky vectors, M vectors of N*N doubles, vector Q element
 *         mu*N+nu (CholeskyERI::L_vectors_, reference
 *         include/mshqc/integrals/cholesky_eri.h:67,81,89-91).  Packed layout:
 *         N(N+1)/2 doubles per vector, the upper triangle mu<=nu row by row.
 *   C     N*N MO coefficients, column-major (Eigen::MatrixXd, reference
 *         SCFResult::C_alpha include/mshqc/scf.h:83); the first nocc columns
 *         are occupied (leftCols(nocc)).
 *   eps   N orbital energies (SCFResult::orbital_energies_alpha, scf.h:77).
 *   B     MO vectors B^Q_ia, o*v*M doubles, element (i*v + a)*M + Q.
 *   dC    N*N column-major, dE/dC[mu, p].
 *   grad  v*o column-major orbital gradient g[a, i] = dE/dkappa_ai for
 *         C -> C exp(-kappa), kappa_ai = -kappa_ia (rotation of reference
 *         src/mp2/cholesky_omp2.cc:385-396), orbital energies held fixed.
 */
#ifndef MSHQC_CD_H
#define MSHQC_CD_H

#include <stdint.h>

#include "mshqc_ao.h"

#ifdef __cplusplus
extern "C" {
#endif

#define MSHQC_CD_ABI_VERSION 1

#if defined(__GNUC__)
#define MSHQC_CD_API __attribute__((visibility("default")))
#else
#define MSHQC_CD_API
#endif

enum mshqc_cd_status {
    MSHQC_CD_OK = 0,
    MSHQC_CD_ERR_ARG = -1,         /* invalid argument or shape              */
    MSHQC_CD_ERR_STATE = -2,       /* call order (e.g. energy before inputs) */
    MSHQC_CD_ERR_CUDA = -3,        /* CUDA runtime / driver error            */
    MSHQC_CD_ERR_ALLOC = -4,       /* device allocation failed               */
    MSHQC_CD_ERR_NUMERIC = -5,     /* NaN / Inf in the inputs                */
    MSHQC_CD_ERR_UNSUPPORTED = -6, /* no such device / not sm_100            */
    MSHQC_CD_ERR_TIMEOUT = -7      /* a device-side bounded wait gave up     */
};

enum mshqc_cd_precision {
    MSHQC_CD_FP64 = 0,    /* FP64 contractions (DMMA)                       */
    MSHQC_CD_FP16X3 = 1   /* scaled FP16 x3: every MO row in fixed point with
                             one power-of-two scale, integer hi/lo carried in
                             FP16, three products per pair, exact FP32
                             accumulation on the tensor cores; FP64
                             denominators, diagonal integrals and energies;
                             the half transforms (from nbf = 512 on;
                             below, FP64 DMMA) and the backward's
                             transposed transforms as FP64 products of
                             int8 slices (5 x 7 bits per operand row) on
                             the tensor cores, about 2^-32 of the row
                             maxima per term (MSHQC_CD_TRANSFORM=f64 in the
                             environment: FP64 DMMA for both, =i8: int8
                             slices for both at every size)              */
};

enum mshqc_cd_kind {
    MSHQC_CD_RESTRICTED = 0,   /* closed shell, one set of orbitals (RMP2) */
    MSHQC_CD_UNRESTRICTED = 1  /* alpha and beta orbitals (UMP2 / OMP2)    */
};

enum mshqc_cd_layout { MSHQC_CD_LAYOUT_FULL = 0, MSHQC_CD_LAYOUT_PACKED = 1 };
/* Where a pointer argument lives.  MSHQC_CD_DEVICE buffers are read and
 * written in the order of the context's stream (its own non-blocking stream,
 * or the one given to mshqc_cd_set_stream): work of another stream that
 * produces an input must be complete (synchronize it, or give the context
 * that stream) before the call.  Every call returns only after its device
 * outputs are written. */
enum mshqc_cd_where { MSHQC_CD_HOST = 0, MSHQC_CD_DEVICE = 1 };
enum mshqc_cd_spin { MSHQC_CD_ALPHA = 0, MSHQC_CD_BETA = 1 };

typedef struct mshqc_cd_ctx mshqc_cd_ctx;

/* Energy components (Eh).  Restricted: total = e_corr of CholeskyRMP2;
 * ss_aa = ss_bb and os are its same-/opposite-spin parts.  Unrestricted:
 * the CholeskyUMP2Result fields e_corr_ss_aa/_ss_bb/_os/_total
 * (reference include/mshqc/cholesky_ump2.h:51-68).  Stage times in ms,
 * measured with CUDA events on the context stream. */
typedef struct {
    double ss_aa, ss_bb, os, total;
    double ms_transform, ms_energy, ms_total;
} mshqc_cd_energy;

/* --- context ---------------------------------------------------------- */
/* Replaces: nothing in the reference (it keeps no device state); owns the
 * device, the stream and the grow-only workspaces. */
MSHQC_CD_API int mshqc_cd_ctx_create(int device, mshqc_cd_ctx** out);
MSHQC_CD_API int mshqc_cd_ctx_destroy(mshqc_cd_ctx* ctx);
MSHQC_CD_API const char* mshqc_cd_last_error(void);
MSHQC_CD_API int mshqc_cd_abi_version(void);
/* Run on a caller stream (cudaStream_t) instead of the context's own. */
MSHQC_CD_API int mshqc_cd_set_stream(mshqc_cd_ctx* ctx, void* stream);
/* Share one gradient among nranks contexts, one per GPU (no counterpart in
 * the reference, which runs on one node): mshqc_cd_mp2_gradient of this
 * context then computes its share of the backward's units (block pairs of
 * occupied orbitals, on the mixed and the FP64 path) and returns that
 * share's energy, dE/dC and dE/deps.  Their sums over the ranks (one
 * all-reduce of 3 + 2 N^2 + 2 N doubles at most) are the full result.
 * The shares: with nranks > 1 the occupied block sizes depend only on the
 * orbital counts, the number of vectors and nranks (never on the free device
 * memory, which differs between GPUs), giving about 32 block pairs per rank;
 * each unit is weighed by its integral-tile and Gamma work and the units are
 * dealt out longest first to the least-loaded rank.  All ranks compute the
 * same plan, so every unit is computed exactly once.  The half transforms
 * and the transposed transforms run in full on every rank;
 * mshqc_cd_mp2_energy and the OMP2 entry points are not partitioned.
 * (0, 1) is the default: everything on this context. */
MSHQC_CD_API int mshqc_cd_set_partition(mshqc_cd_ctx* ctx, int rank, int nranks);
/* Collective operations for a shared gradient, supplied by the host (no
 * counterpart in the reference).  Both run on the calling thread and act on
 * device memory in the order of `stream` (the context's stream; the host may
 * also synchronize it): `buf` holds nranks chunks of `count` doubles.
 *   allgather       chunk `rank` of every rank's buf to all ranks (in place);
 *   reduce_scatter  the sum over ranks of chunk r of buf lands in chunk r of
 *                   rank r's buf (in place; other chunks may be overwritten).
 * NCCL's in-place ncclAllGather / ncclReduceScatter on buf match these
 * (recvbuff = buf, sendbuff = buf + rank * count).  Return 0, or nonzero to
 * fail the call (MSHQC_CD_ERR_STATE). */
typedef struct {
    int (*allgather)(double* buf, int64_t count, void* stream, void* user);
    int (*reduce_scatter)(double* buf, int64_t count, void* stream, void* user);
    void* user;
} mshqc_cd_collectives;
/* With collectives set and a partition of nranks > 1, mshqc_cd_mp2_gradient
 * also shares the half transforms and the transposed transforms: rank r
 * transforms the occupied orbitals [r p, (r + 1) p) of each spin
 * (p = ceil(nocc / nranks)) and allgather completes the MO vectors B on every
 * rank; after the backward, reduce_scatter gives rank r the complete Gamma
 * of its orbitals and its transposed transforms the columns of dE/dC they
 * reach.  The returned shares still add up to the full result.  NULL
 * clears them (the transforms then run in full on every rank). */
MSHQC_CD_API int mshqc_cd_set_collectives(mshqc_cd_ctx* ctx, const mshqc_cd_collectives* ops);
/* Bytes of device memory the context holds. */
MSHQC_CD_API int mshqc_cd_device_bytes(mshqc_cd_ctx* ctx, int64_t* bytes);
/* Number of kernels this context has launched so far. */
MSHQC_CD_API int mshqc_cd_launch_count(mshqc_cd_ctx* ctx, int64_t* count);
/* Device time (ms, CUDA events) of the stages of the last energy or gradient
 * call: [0] half transforms, [1] fixed-point split, [2] pair-energy kernels,
 * [3] integral tiles of the backward, [4] Gamma GEMM, [5] transposed
 * transforms, [6] other, [7] element-wise amplitude pass.  n_out entries are
 * written (at most 8). */
MSHQC_CD_API int mshqc_cd_stage_times(mshqc_cd_ctx* ctx, double* ms_out, int n_out);
/* Timed intervals per stage of the last call, in the order of
 * mshqc_cd_stage_times.  In the mixed-precision backward each integral-tile
 * and each Gamma interval is one kernel launch, so stage_times / stage_counts
 * is the average launch duration of those kernels. */
MSHQC_CD_API int mshqc_cd_stage_counts(mshqc_cd_ctx* ctx, int64_t* n_out, int n);
/* 1 when every tensor-core accumulation of the last mixed-precision call was
 * provably exact (Cauchy-Schwarz bound of the integer accumulators below
 * 2^24 and no accumulator seen at 2^24), else 0. */
MSHQC_CD_API int mshqc_cd_mixed_exact(mshqc_cd_ctx* ctx, int* exact);

/* --- inputs ----------------------------------------------------------- */
/* AO Cholesky vectors.  Replaces the CholeskyERI container read by the
 * transforms (reference src/mp2/cholesky_rmp2.cc:69-71,
 * src/mp2/cholesky_ump2.cc:250, src/mp2/cholesky_omp2.cc:77). */
MSHQC_CD_API int mshqc_cd_set_vectors(mshqc_cd_ctx* ctx, const double* L, int64_t nbf,
                         int64_t nvec, int layout, int where);
/* Pivoted incomplete Cholesky decomposition of the ERI matrix, FP64 on the
 * device: CholeskyERI::decompose (reference src/integrals/cholesky_eri.cc:40-149;
 * first-index pivot :155-167, new vector :169-203, clamped diagonal update
 * :108-109).  eri: N^4 doubles, element (ij|kl) at ((i N + j) N + k) N + l.
 * Stops when the largest remaining diagonal is below threshold (or after N^2
 * vectors; *converged tells which).  The vectors become the context's
 * vectors (as after mshqc_cd_set_vectors) and, when L_out is not NULL, are
 * copied there (max_vectors * N^2 doubles of room, vector Q at Q N^2). */
MSHQC_CD_API int mshqc_cd_cholesky_decompose(mshqc_cd_ctx* ctx, const double* eri, int64_t nbf,
                                             double threshold, double* L_out, int64_t max_vectors,
                                             int64_t* n_vectors, int* converged, int where);
/* Integral-direct pivoted Cholesky: DirectCholesky::compute (reference
 * src/integrals/cholesky_direct.cc:32-187), without the N^4 ERI tensor.  The
 * ERI diagonal and one ERI column per vector come from the host AO engine
 * (include/mshqc_ao.h; `basis` as there), the pivot search (first index of
 * the largest diagonal), the column reduction and the diagonal update
 * (negatives above -1e-10 set to zero) run on the device.  Stops below the
 * threshold, at a negative largest diagonal (*converged = 0 when it is
 * below -1e-10) or after N^2 / 2 vectors.  The vectors become the context's
 * (as after mshqc_cd_set_vectors) and, when L_out is not NULL, are copied
 * there (max_vectors * N^2 doubles of room). */
MSHQC_CD_API int mshqc_cd_cholesky_direct(mshqc_cd_ctx* ctx, const mshqc_ao_basis* basis,
                                          double threshold, double* L_out, int64_t max_vectors,
                                          int64_t* n_vectors, int* converged, int where);
/* Synthetic Cholesky vectors generated on the device instead of uploaded
 * (no counterpart in the reference, which takes them as data): L^Q = sigma
 * 10^(-6 Q / nvec) (X^Q + X^Q^T)/2, X^Q standard normal: for mu <= nu one
 * block of the counter-based Philox4x32-10 generator (key = seed, counter =
 * (Q nbf + mu) nbf + nu) gives the Box-Muller pair (X^Q_{mu nu}, X^Q_{nu mu})
 * (the cosine member on the diagonal).  The vectors are never stored: the
 * consumers regenerate the chunks they read, so sizes whose FP64 vectors
 * exceed device memory run (nbf = 2000, nvec = 8000: 256 GB).  The OMP2
 * entry points need stored vectors. */
MSHQC_CD_API int mshqc_cd_gen_vectors(mshqc_cd_ctx* ctx, int64_t nbf, int64_t nvec, uint64_t seed,
                                      double sigma);
/* Orbitals of one spin.  Replaces the SCFResult fields C_alpha/C_beta,
 * orbital_energies_alpha/beta, n_occ_alpha/beta read by the MP2 classes
 * (reference src/mp2/cholesky_rmp2.cc:27-29,77-78,106;
 * src/mp2/cholesky_ump2.cc:41-44,255-258). */
MSHQC_CD_API int mshqc_cd_set_orbitals(mshqc_cd_ctx* ctx, int spin, const double* C,
                          const double* eps, int64_t nocc, int where);

/* --- forward ---------------------------------------------------------- */
/* AO->MO half transform B^Q_ia = sum C_mu,i L^Q_mu,nu C_nu,a of one spin.
 * Replaces CholeskyRMP2::transform_vectors (src/mp2/cholesky_rmp2.cc:68-93),
 * CholeskyUMP2::transform_cholesky_vectors (src/mp2/cholesky_ump2.cc:244-293)
 * and CholeskyOMP2::transform_vectors (src/mp2/cholesky_omp2.cc:71-92).
 * B_out (o*v*M, see header) may be NULL to keep the result on the device
 * only.  MSHQC_CD_FP64 returns FP64 DMMA products; MSHQC_CD_FP16X3 may
 * return the int8-slice products (or reuse FP64 ones already computed). */
MSHQC_CD_API int mshqc_cd_transform(mshqc_cd_ctx* ctx, int spin, int precision,
                       double* B_out, int where);
/* MP2 correlation energy.  Replaces the pair loop of CholeskyRMP2::compute
 * (src/mp2/cholesky_rmp2.cc:118-153) for kind RESTRICTED and
 * CholeskyUMP2::compute_ss_alpha/compute_ss_beta/compute_os
 * (src/mp2/cholesky_ump2.cc:299-465) for kind UNRESTRICTED; runs the
 * transforms first when the orbitals changed. */
MSHQC_CD_API int mshqc_cd_mp2_energy(mshqc_cd_ctx* ctx, int kind, int precision,
                        mshqc_cd_energy* out);
/* Pair energies of the last mp2_energy call: restricted o*o (e_ij, all
 * ordered pairs, symmetric); unrestricted block 0 = aa (oa*oa), 1 = bb,
 * 2 = ab (oa*ob).  Row-major [i][j]. */
MSHQC_CD_API int mshqc_cd_pair_energies(mshqc_cd_ctx* ctx, int block, double* out, int where);

/* Amplitudes of a block of pairs for the consumers of the reference's stored
 * t2: CholeskyRMP2Result::t2 (reference include/mshqc/cholesky_rmp2.h:32-49,
 * filled in src/mp2/cholesky_rmp2.cc:118-153, read by CholeskyRMP3) and
 * CholeskyUMP2::compute_t2_amplitudes (src/mp2/cholesky_ump2.cc:471-556).
 * FP64, the reference's convention in every block:
 *   t_ij^ab = (ia|jb) / (e_i + e_j - e_a - e_b), 0 where |D| < 1e-12.
 * block 0: alpha-alpha (the restricted amplitudes), 1: beta-beta,
 * 2: alpha-beta.  Pairs i0 <= i < i0 + ni, j0 <= j < j0 + nj; out holds
 * ni * nj * vx * vy doubles, element ((i - i0) nj + (j - j0)) vx vy + a vy + b
 * (vx, vy: virtual counts of the two spins).  Runs the FP64 transforms
 * first when needed. */
MSHQC_CD_API int mshqc_cd_get_t2_block(mshqc_cd_ctx* ctx, int block, int64_t i0, int64_t ni, int64_t j0,
                                       int64_t nj, double* out, int where);

/* --- backward (exact differentiation; no reference counterpart) ------- */
/* Energy and its exact derivatives with respect to the orbitals and the
 * orbital energies.  dC_a/dC_b: N*N column-major; deps_a/deps_b: N; any
 * output may be NULL.  For RESTRICTED only the _a outputs are written and
 * they are the derivatives of the closed-shell energy with respect to the
 * one shared C and eps.  e_out may be NULL. */
MSHQC_CD_API int mshqc_cd_mp2_gradient(mshqc_cd_ctx* ctx, int kind, int precision,
                          mshqc_cd_energy* e_out, double* dC_a, double* dC_b,
                          double* deps_a, double* deps_b, int where);

/* --- CD-OMP2 (FP64; reference src/mp2/cholesky_omp2.cc) ---------------- */
/* Core Hamiltonian H (N*N, symmetric) of the OMP2 generalized Fock matrix:
 * IntegralEngine::compute_core_hamiltonian as read by
 * CholeskyOMP2::build_gfock_from_density (src/mp2/cholesky_omp2.cc:336). */
MSHQC_CD_API int mshqc_cd_set_core_hamiltonian(mshqc_cd_ctx* ctx, const double* H, int where);

/* Current orbitals of one spin (N*N column-major); after mshqc_cd_omp2 these
 * are the rotated orbitals (OMP2Result::C_alpha / C_beta). */
MSHQC_CD_API int mshqc_cd_get_orbitals(mshqc_cd_ctx* ctx, int spin, double* C, int where);

/* Cholesky Fock build of the SCF classes on the context's vectors (stored or
 * generated), FP64: J = sum_Q <L^Q, P_tot> L^Q and K_s = sum_Q L^Q P_s L^Q.
 *  nspin = 1 replaces CholeskyRHF::build_fock (src/scf/cholesky_rhf.cc:99-137):
 *    P_a is the total density 2 C_occ C_occ^T, F_a = H + J - K_a / 2, and with
 *    screen_exchange != 0 vectors of Frobenius norm <= 1e-8 are left out of K
 *    (CholeskyRHFConfig::screen_exchange, default on in the reference);
 *  nspin = 2 replaces CholeskyUHF::build_fock_cholesky
 *    (src/scf/cholesky_uhf.cc:77-103): J from P_a + P_b, F_s = H + J - K_s
 *    (never screened).
 * All matrices N*N (symmetric, so either storage order).  Every output may be
 * NULL; a Fock matrix needs H. */
MSHQC_CD_API int mshqc_cd_cholesky_fock(mshqc_cd_ctx* ctx, int nspin, const double* P_a, const double* P_b,
                                        const double* H, int screen_exchange, double* F_a, double* F_b,
                                        double* J, double* K_a, double* K_b, int where);

/* One gradient evaluation of CholeskyOMP2::compute at the context's current
 * alpha and beta orbitals (src/mp2/cholesky_omp2.cc:442-466): amplitudes
 * (:94-183), MP2 energy (:189-230), the one-particle density blocks G_oo
 * (o*o) and G_vv (v*v) per spin (:232-326, row-major), and the generalized
 * Fock matrices F = C^T (H + J - K) C (:331-369, N*N column-major); the
 * reference gradient is w_ai = 2 F(o+a, i) (:465-466).  P_a / P_b: the
 * reference densities SCFResult::P_alpha / P_beta (N*N), or NULL for
 * C_occ C_occ^T.  Any output may be NULL.  Both spins must be set (the same
 * orbitals twice for a closed shell) and the core Hamiltonian given. */
MSHQC_CD_API int mshqc_cd_omp2_pieces(mshqc_cd_ctx* ctx, const double* P_a, const double* P_b,
                                      double* e_mp2, double* Goo_a, double* Gvv_a, double* Goo_b,
                                      double* Gvv_b, double* F_a, double* F_b, int where);

/* CholeskyOMP2Config (reference include/mshqc/cholesky_omp2.h:28-34) plus
 * the SCF energy the reference reads from SCFResult::energy_total. */
typedef struct {
    int max_iterations;        /* 50 */
    double energy_threshold;   /* 1e-6 */
    double gradient_threshold; /* 1e-5 */
    double e_scf;
} mshqc_cd_omp2_config;

/* The energies and counters of OMP2Result (reference include/mshqc/mp2.h:52-72). */
typedef struct {
    double energy_scf;
    double energy_mp2_corr;
    double energy_total;       /* E_SCF + E_MP2 of the last iteration before the final one */
    int iterations;
    int converged;
    double ms_total;
} mshqc_cd_omp2_result;

/* CholeskyOMP2::compute (src/mp2/cholesky_omp2.cc:427-512): repeat the
 * gradient evaluation, stop when |w| < gradient_threshold and |dE| <
 * energy_threshold, else rotate C <- C exp(-kappa) with kappa_ai =
 * 0.5 w_ai / (F_aa - F_ii + 0.2) (|denominator| >= 1e-2; :375-424); when
 * nocc_alpha == nocc_beta beta takes alpha's orbitals after each step.
 * Orbital energies and E_SCF are never updated, as in the reference.  The
 * final orbitals replace the context's (mshqc_cd_get_orbitals). */
MSHQC_CD_API int mshqc_cd_omp2(mshqc_cd_ctx* ctx, const mshqc_cd_omp2_config* cfg, const double* P_a,
                               const double* P_b, int where, mshqc_cd_omp2_result* res);

/* --- allocation-free energy (no counterpart in the reference) --------- */
/* Size of the static device scratch of mshqc_cd_rmp2_energy_noalloc. */
#define MSHQC_CD_NOALLOC_SCRATCH_BYTES (16u << 20)

/* The FP64 closed-shell MP2 energy of mshqc_cd_mp2_energy(RESTRICTED, FP64)
 * from MO vectors already on the device, allocating nothing: no context, no
 * cudaMalloc / cudaFree, no allocating library call.  It is meant for callers
 * that cannot allocate at that point: code inside a framework or memory pool
 * that owns the whole device budget, and code on a latency-critical stream
 * (cudaMalloc and cudaFree synchronize the device and stall other streams).
 *
 * Scratch: one static device array of MSHQC_CD_NOALLOC_SCRATCH_BYTES
 * (16 MiB) per device.  A call needs
 *     roundup(8 (P + K), 256) + 16 P K + 16 P  bytes,
 *     P = nocc (nocc + 1) / 2,  K = nb (nb + 1) / 2,  nb = ceil(nvir / 64)
 * (nocc = 100, nvir = 900 needs 9.8 MB); larger sizes are rejected with
 * MSHQC_CD_ERR_ARG and a message, before the device is touched.
 *
 * B       device, nocc * vp * Mp doubles, element (i * vp + a) * Mp + Q with
 *         vp = ceil(nvir / 64) * 64, Mp = ceil(nvec / 16) * 16; the padding
 *         (a >= nvir or Q >= nvec) must be zero.
 * eps     device, nocc + nvir orbital energies, occupied first.
 * energy  device, 2 doubles, written in stream order: [0] E_corr,
 *         [1] its opposite-spin part.
 * stream  a cudaStream_t, or NULL for the legacy default stream.  The call
 *         returns once its kernels are queued; synchronize the stream before
 *         reading energy.
 *
 * Set-up happens on the first call with each device current, and again on
 * the first call in a new CUDA context of that device (after cudaDeviceReset):
 * it looks up the scratch address and the kernel attributes.  Make that first
 * call outside any stream capture.  No scratch word needs to start at zero: a call writes
 * all the scratch it reads before reading it.  All calls on one device share
 * the scratch, so calls that overlap in time (different streams or host
 * threads) race on it: order them (one stream, or events).  Inputs are not
 * checked for NaN/Inf. */
MSHQC_CD_API int mshqc_cd_rmp2_energy_noalloc(const double* B, const double* eps, int64_t nocc,
                                              int64_t nvir, int64_t nvec, double* energy,
                                              void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MSHQC_CD_H */
