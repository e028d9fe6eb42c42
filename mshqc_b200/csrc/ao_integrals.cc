// AO integrals over contracted Gaussian shells on the host: overlap S,
// kinetic T, nuclear attraction V and electron repulsion (mu nu|lam sig), plus
// the ERI diagonal and single ERI columns for integral-direct Cholesky.
//
// This is the integral engine the reference gets from libint2 (its
// IntegralEngine, include/mshqc/integrals.h:38-224, implemented on libint2 in
// src/core/integrals.cc:351-459), rebuilt from the published McMurchie-
// Davidson scheme (L. E. McMurchie and E. R. Davidson, J. Comput. Phys. 26,
// 218 (1978); the recurrences as written in Helgaker, Jorgensen and Olsen,
// "Molecular Electronic-Structure Theory", sections 9.5-9.9):
//   * the product of two 1-D Gaussians expanded in Hermite Gaussians,
//     coefficients E^{ij}_t by the two-term recurrences (eq. 9.5.6-9.5.7);
//   * overlap from E^{ij}_0, kinetic energy from overlaps with the ket
//     power raised and lowered by two;
//   * Coulomb integrals from the Hermite integrals R_{tuv} (eq. 9.9.18-9.9.20)
//     over the Boys function F_n (series plus downward recursion for small
//     arguments, the asymptotic form plus upward recursion for large ones,
//     eq. 9.8.12-9.8.14).
// Conventions follow what the reference passes to libint2
// (src/core/integrals.cc:96-145, src/core/basis.cc:53-110):
//   * contraction coefficients arrive as the reference's Shell::normalize
//     leaves them (mshqc_ao_normalize_shell does the same) and multiply the
//     raw primitives, as they do in libint2 when the reference builds its
//     shells without renormalization; every Cartesian component of a shell
//     carries the same coefficient;
//   * Cartesian components in the order x^l, x^(l-1) y, x^(l-1) z, ...,
//     z^l; pure shells as real solid harmonics m = -l .. l ("standard"
//     ordering), each of unit norm -- for p that is (y, z, x);
//   * ERI element (mu nu|lam sig) at ((mu N + nu) N + lam) N + sig, which by
//     the eight-fold symmetry is also Eigen's column-major (mu,nu,lam,sig).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mshqc_ao.h"

namespace mshqc_ao_impl {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxL = 6;

thread_local std::string g_err;

double dfact(int n) {  // (n)!! with (-1)!! = 0!! = 1
    double r = 1.0;
    for (int k = n; k > 1; k -= 2) r *= k;
    return r;
}
double fact(int n) {
    double r = 1.0;
    for (int k = 2; k <= n; ++k) r *= k;
    return r;
}
double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    return fact(n) / (fact(k) * fact(n - k));
}

// Cartesian components of angular momentum l in the order x^l, x^(l-1)y, ...
std::vector<std::array<int, 3>> cart_components(int l) {
    std::vector<std::array<int, 3>> c;
    for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) c.push_back({i, j, l - i - j});
    return c;
}

// <x^a y^b z^c | x^a' y^b' z^c'> of same-centre, same-exponent Gaussians
// relative to <x^l | x^l> (l = a + b + c = a' + b' + c')
double mono_overlap(const std::array<int, 3>& p, const std::array<int, 3>& q, int l) {
    double r = 1.0;
    for (int k = 0; k < 3; ++k) {
        const int s = p[k] + q[k];
        if (s & 1) return 0.0;
        r *= dfact(s - 1);
    }
    return r / dfact(2 * l - 1);
}

// Real solid harmonics of degree l as combinations of the x^l-normalized
// Cartesian components: rows m = -l .. l, columns in cart_components order.
// The unnormalized expansion is that of Helgaker et al. eq. 6.4.47-6.4.50:
//   S_lm ~ sum_{t,u,v} (-1)^(t+v-vm) (1/4)^t C(l,t) C(l-t,|m|+t) C(t,u) C(|m|,2v)
//          x^(2t+|m|-2(u+v)) y^(2(u+v)) z^(l-2t-|m|),
// vm = 0 (m >= 0) or 1/2 (m < 0); each row is then scaled to unit norm with
// the monomial overlaps above (which fixes the normalization convention).
std::vector<double> solid_harmonics(int l) {
    const auto cc = cart_components(l);
    const int nc = (int)cc.size(), ns = 2 * l + 1;
    std::vector<double> T((size_t)ns * nc, 0.0);
    for (int m = -l; m <= l; ++m) {
        const int am = std::abs(m);
        std::vector<double> row(nc, 0.0);
        // 2v runs over even values for m >= 0, odd values for m < 0
        for (int t = 0; t <= (l - am) / 2; ++t)
            for (int u = 0; u <= t; ++u)
                for (int v2 = (m < 0 ? 1 : 0); v2 <= am; v2 += 2) {
                    const double vv = 0.5 * v2, vm = m < 0 ? 0.5 : 0.0;
                    const double sgn = ((int)std::lround(t + vv - vm) & 1) ? -1.0 : 1.0;
                    const double coef = sgn * std::pow(0.25, t) * binom(l, t) * binom(l - t, am + t) *
                                        binom(t, u) * binom(am, v2);
                    const int px = 2 * t + am - 2 * u - v2, py = 2 * u + v2, pz = l - 2 * t - am;
                    if (px < 0 || py < 0 || pz < 0) continue;
                    // every Cartesian component carries the same x^l factor,
                    // so the monomial coefficients carry over unchanged
                    for (int k = 0; k < nc; ++k)
                        if (cc[k][0] == px && cc[k][1] == py && cc[k][2] == pz) row[k] += coef;
                }
        double n2 = 0.0;
        for (int a = 0; a < nc; ++a)
            for (int b = 0; b < nc; ++b) n2 += row[a] * row[b] * mono_overlap(cc[a], cc[b], l);
        const double s = 1.0 / std::sqrt(n2);
        for (int a = 0; a < nc; ++a) T[(size_t)(m + l) * nc + a] = row[a] * s;
    }
    return T;
}

struct Shell {
    int l = 0;
    bool pure = false;
    double O[3] = {0, 0, 0};
    std::vector<double> a, c;   // exponents, normalized coefficients
    int nc = 1, nf = 1, off = 0;
    const std::vector<double>* T = nullptr;   // solid harmonics (pure)
};

struct Basis {
    std::vector<Shell> sh;
    int nbf = 0;
    std::vector<double> sph[kMaxL + 1];
};

int build_basis(const mshqc_ao_basis* b, Basis& out) {
    if (!b || b->nshell < 0) {
        g_err = "basis is null";
        return MSHQC_AO_ERR_ARG;
    }
    out.sh.resize(b->nshell);
    int64_t p = 0, off = 0;
    for (int s = 0; s < b->nshell; ++s) {
        Shell& S = out.sh[s];
        S.l = b->l[s];
        S.pure = b->pure && b->pure[s] != 0;
        if (S.l < 0 || S.l > kMaxL || b->nprim[s] < 1) {
            g_err = "shell " + std::to_string(s) + ": angular momentum 0.." + std::to_string(kMaxL) +
                    " and at least one primitive required";
            return MSHQC_AO_ERR_ARG;
        }
        for (int k = 0; k < 3; ++k) S.O[k] = b->center[3 * s + k];
        S.a.assign(b->exps + p, b->exps + p + b->nprim[s]);
        S.c.assign(b->coefs + p, b->coefs + p + b->nprim[s]);
        for (double x : S.a)
            if (!(x > 0.0)) {
                g_err = "shell " + std::to_string(s) + ": exponents must be positive";
                return MSHQC_AO_ERR_ARG;
            }
        p += b->nprim[s];
        S.nc = (S.l + 1) * (S.l + 2) / 2;
        S.nf = S.pure ? 2 * S.l + 1 : S.nc;
        S.off = (int)off;
        off += S.nf;
        if (S.pure) {
            if (out.sph[S.l].empty()) out.sph[S.l] = solid_harmonics(S.l);
            S.T = &out.sph[S.l];
        }
    }
    out.nbf = (int)off;
    return MSHQC_AO_OK;
}

// ---------------------------------------------------------------------------
// Boys function F_n(T), n = 0 .. nmax
// ---------------------------------------------------------------------------
void boys(int nmax, double T, double* F) {
    if (T < 1e-14) {
        for (int n = 0; n <= nmax; ++n) F[n] = 1.0 / (2 * n + 1);
        return;
    }
    const double eT = std::exp(-T);
    if (T < 45.0) {
        // F_nmax(T) = e^-T sum_k (2T)^k / ((2nmax+1)(2nmax+3)...(2nmax+2k+1))
        double term = 1.0 / (2 * nmax + 1), sum = term;
        for (int k = 1; k < 400; ++k) {
            term *= 2.0 * T / (2 * nmax + 2 * k + 1);
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        F[nmax] = eT * sum;
        for (int n = nmax - 1; n >= 0; --n) F[n] = (2.0 * T * F[n + 1] + eT) / (2 * n + 1);
    } else {
        // F_0 = sqrt(pi/T)/2 (1 - erfc(sqrt T)), erfc below 1e-20 here
        F[0] = 0.5 * std::sqrt(kPi / T);
        for (int n = 0; n < nmax; ++n) F[n + 1] = ((2 * n + 1) * F[n] - eT) / (2.0 * T);
    }
}

// ---------------------------------------------------------------------------
// Hermite expansion coefficients E^{ij}_t of one Cartesian direction:
// E[(i * (lb + 1) + j) * (la + lb + 1) + t]
// ---------------------------------------------------------------------------
void hermite_E(int la, int lb, double a, double b, double XAB, std::vector<double>& E) {
    const double p = a + b, mu = a * b / p;
    const double XPA = -b / p * XAB, XPB = a / p * XAB, i2p = 0.5 / p;
    const int nt = la + lb + 1;
    E.assign((size_t)(la + 1) * (lb + 1) * nt, 0.0);
    auto at = [&](int i, int j, int t) -> double& { return E[((size_t)i * (lb + 1) + j) * nt + t]; };
    auto get = [&](int i, int j, int t) -> double {
        if (t < 0 || t > i + j) return 0.0;
        return E[((size_t)i * (lb + 1) + j) * nt + t];
    };
    at(0, 0, 0) = std::exp(-mu * XAB * XAB);
    for (int i = 0; i <= la; ++i)
        for (int j = 0; j <= lb; ++j) {
            if (i == 0 && j == 0) continue;
            for (int t = 0; t <= i + j; ++t) {
                double v;
                if (i > 0)
                    v = i2p * get(i - 1, j, t - 1) + XPA * get(i - 1, j, t) + (t + 1) * get(i - 1, j, t + 1);
                else
                    v = i2p * get(i, j - 1, t - 1) + XPB * get(i, j - 1, t) + (t + 1) * get(i, j - 1, t + 1);
                at(i, j, t) = v;
            }
        }
}

// Hermite Coulomb integrals R_{tuv}(alpha, PC) for t + u + v <= L into
// R[(t * (L + 1) + u) * (L + 1) + v]
void hermite_R(int L, double alpha, const double PC[3], std::vector<double>& R, std::vector<double>& work) {
    const int n1 = L + 1;
    const size_t per = (size_t)n1 * n1 * n1;
    work.assign(per * n1, 0.0);
    double F[4 * kMaxL + 2];
    const double T = alpha * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
    boys(L, T, F);
    auto W = [&](int n, int t, int u, int v) -> double& { return work[(size_t)n * per + ((size_t)t * n1 + u) * n1 + v]; };
    double m2a = 1.0;
    for (int n = 0; n <= L; ++n) {
        W(n, 0, 0, 0) = m2a * F[n];
        m2a *= -2.0 * alpha;
    }
    // R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X R^{n+1}_{t,u,v}, likewise for u and v
    for (int n = L - 1; n >= 0; --n) {
        const int top = L - n;
        for (int t = 0; t <= top; ++t)
            for (int u = 0; u + t <= top; ++u)
                for (int v = 0; v + u + t <= top; ++v) {
                    if (t + u + v == 0) continue;
                    double r;
                    if (t > 0)
                        r = (t > 1 ? (t - 1) * W(n + 1, t - 2, u, v) : 0.0) + PC[0] * W(n + 1, t - 1, u, v);
                    else if (u > 0)
                        r = (u > 1 ? (u - 1) * W(n + 1, t, u - 2, v) : 0.0) + PC[1] * W(n + 1, t, u - 1, v);
                    else
                        r = (v > 1 ? (v - 1) * W(n + 1, t, u, v - 2) : 0.0) + PC[2] * W(n + 1, t, u, v - 1);
                    W(n, t, u, v) = r;
                }
    }
    R.assign(per, 0.0);
    std::memcpy(R.data(), work.data(), per * sizeof(double));
}

// Cartesian block of a one-electron operator between shells A and B:
// out[ia * ncB + ib]
enum OneKind { OVERLAP, KINETIC, NUCLEAR };

void one_electron_cart(const Shell& A, const Shell& B, OneKind kind, const mshqc_ao_nuclei* nuc,
                       std::vector<double>& out) {
    const auto ca = cart_components(A.l), cb = cart_components(B.l);
    out.assign((size_t)A.nc * B.nc, 0.0);
    const double AB[3] = {A.O[0] - B.O[0], A.O[1] - B.O[1], A.O[2] - B.O[2]};
    const int lbk = B.l + (kind == KINETIC ? 2 : 0);
    std::vector<double> Ex, Ey, Ez, R, work;
    for (size_t pa = 0; pa < A.a.size(); ++pa)
        for (size_t pb = 0; pb < B.a.size(); ++pb) {
            const double a = A.a[pa], b = B.a[pb], p = a + b;
            const double cab = A.c[pa] * B.c[pb];
            hermite_E(A.l, lbk, a, b, AB[0], Ex);
            hermite_E(A.l, lbk, a, b, AB[1], Ey);
            hermite_E(A.l, lbk, a, b, AB[2], Ez);
            const int nt = A.l + lbk + 1;
            auto e = [&](const std::vector<double>& E, int i, int j, int t) {
                return E[((size_t)i * (lbk + 1) + j) * nt + t];
            };
            if (kind == OVERLAP || kind == KINETIC) {
                const double pre = std::pow(kPi / p, 1.5);
                auto s1 = [&](const std::vector<double>& E, int i, int j) { return j < 0 ? 0.0 : e(E, i, j, 0); };
                // -1/2 d^2/dx^2 of x^j e^{-b x^2}: 1-D kinetic factor
                auto t1 = [&](const std::vector<double>& E, int i, int j) {
                    return -0.5 * (4.0 * b * b * s1(E, i, j + 2) - 2.0 * b * (2 * j + 1) * s1(E, i, j) +
                                   (double)j * (j - 1) * s1(E, i, j - 2));
                };
                for (int ia = 0; ia < A.nc; ++ia)
                    for (int ib = 0; ib < B.nc; ++ib) {
                        const auto& I = ca[ia];
                        const auto& J = cb[ib];
                        const double sx = s1(Ex, I[0], J[0]), sy = s1(Ey, I[1], J[1]), sz = s1(Ez, I[2], J[2]);
                        double v;
                        if (kind == OVERLAP)
                            v = sx * sy * sz;
                        else
                            v = t1(Ex, I[0], J[0]) * sy * sz + sx * t1(Ey, I[1], J[1]) * sz +
                                sx * sy * t1(Ez, I[2], J[2]);
                        out[(size_t)ia * B.nc + ib] += cab * pre * v;
                    }
            } else {
                const double P[3] = {(a * A.O[0] + b * B.O[0]) / p, (a * A.O[1] + b * B.O[1]) / p,
                                     (a * A.O[2] + b * B.O[2]) / p};
                const int L = A.l + B.l, n1 = L + 1;
                for (int k = 0; k < nuc->natom; ++k) {
                    const double PC[3] = {P[0] - nuc->xyz[3 * k], P[1] - nuc->xyz[3 * k + 1],
                                          P[2] - nuc->xyz[3 * k + 2]};
                    hermite_R(L, p, PC, R, work);
                    const double pre = -nuc->Z[k] * 2.0 * kPi / p * cab;
                    for (int ia = 0; ia < A.nc; ++ia)
                        for (int ib = 0; ib < B.nc; ++ib) {
                            const auto& I = ca[ia];
                            const auto& J = cb[ib];
                            double v = 0.0;
                            for (int t = 0; t <= I[0] + J[0]; ++t) {
                                const double et = e(Ex, I[0], J[0], t);
                                if (et == 0.0) continue;
                                for (int u = 0; u <= I[1] + J[1]; ++u) {
                                    const double eu = e(Ey, I[1], J[1], u);
                                    if (eu == 0.0) continue;
                                    for (int w = 0; w <= I[2] + J[2]; ++w)
                                        v += et * eu * e(Ez, I[2], J[2], w) * R[((size_t)t * n1 + u) * n1 + w];
                                }
                            }
                            out[(size_t)ia * B.nc + ib] += pre * v;
                        }
                }
            }
        }
}

// Cartesian block -> the shells' functions (solid harmonics where pure):
// out[fa * nfB + fb] = sum TA[fa][ia] cart[ia][ib] TB[fb][ib]
void to_functions(const Shell& A, const Shell& B, const std::vector<double>& cart, std::vector<double>& out) {
    std::vector<double> tmp((size_t)A.nf * B.nc, 0.0);
    for (int fa = 0; fa < A.nf; ++fa)
        for (int ib = 0; ib < B.nc; ++ib) {
            double s = 0.0;
            if (A.pure)
                for (int ia = 0; ia < A.nc; ++ia) s += (*A.T)[(size_t)fa * A.nc + ia] * cart[(size_t)ia * B.nc + ib];
            else
                s = cart[(size_t)fa * B.nc + ib];
            tmp[(size_t)fa * B.nc + ib] = s;
        }
    out.assign((size_t)A.nf * B.nf, 0.0);
    for (int fa = 0; fa < A.nf; ++fa)
        for (int fb = 0; fb < B.nf; ++fb) {
            double s = 0.0;
            if (B.pure)
                for (int ib = 0; ib < B.nc; ++ib) s += tmp[(size_t)fa * B.nc + ib] * (*B.T)[(size_t)fb * B.nc + ib];
            else
                s = tmp[(size_t)fa * B.nc + fb];
            out[(size_t)fa * B.nf + fb] = s;
        }
}

void one_electron(const Basis& bs, OneKind kind, const mshqc_ao_nuclei* nuc, double* M) {
    const int N = bs.nbf;
    const int ns = (int)bs.sh.size();
#pragma omp parallel for schedule(dynamic)
    for (int s1 = 0; s1 < ns; ++s1) {
        std::vector<double> cart, f;
        for (int s2 = 0; s2 <= s1; ++s2) {
            const Shell& A = bs.sh[s1];
            const Shell& B = bs.sh[s2];
            one_electron_cart(A, B, kind, nuc, cart);
            to_functions(A, B, cart, f);
            for (int fa = 0; fa < A.nf; ++fa)
                for (int fb = 0; fb < B.nf; ++fb) {
                    const double v = f[(size_t)fa * B.nf + fb];
                    M[(size_t)(A.off + fa) * N + (B.off + fb)] = v;
                    M[(size_t)(B.off + fb) * N + (A.off + fa)] = v;
                }
        }
    }
}

// ---------------------------------------------------------------------------
// two-electron integrals
// ---------------------------------------------------------------------------
// Hermite expansion of a shell pair's Cartesian products, one primitive pair:
// for each component pair (ia, ib) the nonzero E^x_t E^y_u E^z_v
struct PairPrim {
    double p, P[3], c;
    // coefficient tables [ia * ncB + ib] -> list of (t, u, v, value)
    std::vector<std::vector<std::pair<int, double>>> terms;   // index (t * n1 + u) * n1 + v
};

struct PairData {
    int L = 0;
    std::vector<PairPrim> prims;
};

void make_pair(const Shell& A, const Shell& B, PairData& pd) {
    const auto ca = cart_components(A.l), cb = cart_components(B.l);
    const double AB[3] = {A.O[0] - B.O[0], A.O[1] - B.O[1], A.O[2] - B.O[2]};
    pd.L = A.l + B.l;
    const int n1 = pd.L + 1, nt = pd.L + 1;
    pd.prims.clear();
    std::vector<double> Ex, Ey, Ez;
    for (size_t pa = 0; pa < A.a.size(); ++pa)
        for (size_t pb = 0; pb < B.a.size(); ++pb) {
            PairPrim pp;
            const double a = A.a[pa], b = B.a[pb];
            pp.p = a + b;
            for (int k = 0; k < 3; ++k) pp.P[k] = (a * A.O[k] + b * B.O[k]) / pp.p;
            pp.c = A.c[pa] * B.c[pb];
            hermite_E(A.l, B.l, a, b, AB[0], Ex);
            hermite_E(A.l, B.l, a, b, AB[1], Ey);
            hermite_E(A.l, B.l, a, b, AB[2], Ez);
            auto e = [&](const std::vector<double>& E, int i, int j, int t) {
                return E[((size_t)i * (B.l + 1) + j) * nt + t];
            };
            pp.terms.resize((size_t)A.nc * B.nc);
            for (int ia = 0; ia < A.nc; ++ia)
                for (int ib = 0; ib < B.nc; ++ib) {
                    auto& lst = pp.terms[(size_t)ia * B.nc + ib];
                    const auto& I = ca[ia];
                    const auto& J = cb[ib];
                    for (int t = 0; t <= I[0] + J[0]; ++t)
                        for (int u = 0; u <= I[1] + J[1]; ++u)
                            for (int v = 0; v <= I[2] + J[2]; ++v) {
                                const double val = e(Ex, I[0], J[0], t) * e(Ey, I[1], J[1], u) * e(Ez, I[2], J[2], v);
                                if (val != 0.0) lst.push_back({(t * n1 + u) * n1 + v, val});
                            }
                }
            pd.prims.push_back(std::move(pp));
        }
}

// (AB|CD) over Cartesian components: out[((ia * ncB + ib) * ncC + ic) * ncD + id]
void eri_cart(const Shell& A, const Shell& B, const Shell& C, const Shell& D, const PairData& bra,
              const PairData& ket, std::vector<double>& out, std::vector<double>& R, std::vector<double>& work,
              std::vector<double>& Wk) {
    const int L = bra.L + ket.L, n1 = L + 1;
    const int nb1 = bra.L + 1, nk1 = ket.L + 1;
    const size_t nab = (size_t)A.nc * B.nc, ncd = (size_t)C.nc * D.nc;
    out.assign(nab * ncd, 0.0);
    const size_t nbh = (size_t)nb1 * nb1 * nb1;
    Wk.assign(nbh * ncd, 0.0);
    for (const auto& pk : ket.prims)
        for (const auto& pb : bra.prims) {
            const double p = pb.p, q = pk.p, alpha = p * q / (p + q);
            const double PQ[3] = {pb.P[0] - pk.P[0], pb.P[1] - pk.P[1], pb.P[2] - pk.P[2]};
            hermite_R(L, alpha, PQ, R, work);
            const double pre = 2.0 * std::pow(kPi, 2.5) / (p * q * std::sqrt(p + q)) * pb.c * pk.c;
            // W[tuv_bra][cd] = sum_{tau nu phi} (-1)^(tau+nu+phi) E^cd R_{t+tau, u+nu, v+phi}
            std::fill(Wk.begin(), Wk.end(), 0.0);
            for (size_t cd = 0; cd < ncd; ++cd)
                for (const auto& kt : pk.terms[cd]) {
                    const int tk = kt.first / (nk1 * nk1), uk = (kt.first / nk1) % nk1, vk = kt.first % nk1;
                    const double s = ((tk + uk + vk) & 1) ? -kt.second : kt.second;
                    for (int t = 0; t <= bra.L; ++t)
                        for (int u = 0; u + t <= bra.L; ++u)
                            for (int v = 0; v + u + t <= bra.L; ++v)
                                Wk[(((size_t)t * nb1 + u) * nb1 + v) * ncd + cd] +=
                                    s * R[((size_t)(t + tk) * n1 + (u + uk)) * n1 + (v + vk)];
                }
            for (size_t ab = 0; ab < nab; ++ab)
                for (const auto& bt : pb.terms[ab]) {
                    const int tb = bt.first / (nb1 * nb1), ub = (bt.first / nb1) % nb1, vb = bt.first % nb1;
                    const double* w = &Wk[(((size_t)tb * nb1 + ub) * nb1 + vb) * ncd];
                    const double f = pre * bt.second;
                    double* o = &out[ab * ncd];
                    for (size_t cd = 0; cd < ncd; ++cd) o[cd] += f * w[cd];
                }
        }
}

// Cartesian quartet -> functions: out[((fa * nfB + fb) * nfC + fc) * nfD + fd]
void quartet_to_functions(const Shell* S[4], const std::vector<double>& cart, std::vector<double>& out) {
    // transform one index at a time; dims[k] = current extent of index k
    std::vector<double> cur = cart, nxt;
    int dims[4] = {S[0]->nc, S[1]->nc, S[2]->nc, S[3]->nc};
    for (int k = 0; k < 4; ++k) {
        if (!S[k]->pure) continue;
        const int nf = S[k]->nf, nc = S[k]->nc;
        size_t pre = 1, post = 1;
        for (int j = 0; j < k; ++j) pre *= dims[j];
        for (int j = k + 1; j < 4; ++j) post *= dims[j];
        nxt.assign(pre * nf * post, 0.0);
        const auto& T = *S[k]->T;
        for (size_t a = 0; a < pre; ++a)
            for (int f = 0; f < nf; ++f)
                for (int c = 0; c < nc; ++c) {
                    const double t = T[(size_t)f * nc + c];
                    if (t == 0.0) continue;
                    const double* src = &cur[(a * nc + c) * post];
                    double* dst = &nxt[(a * nf + f) * post];
                    for (size_t b = 0; b < post; ++b) dst[b] += t * src[b];
                }
        cur.swap(nxt);
        dims[k] = nf;
    }
    out.swap(cur);
}

void compute_eri_all(const Basis& bs, double* eri) {
    const int N = bs.nbf, ns = (int)bs.sh.size();
    std::vector<PairData> pairs((size_t)ns * ns);
    for (int a = 0; a < ns; ++a)
        for (int b = 0; b < ns; ++b) make_pair(bs.sh[a], bs.sh[b], pairs[(size_t)a * ns + b]);
    std::vector<std::array<int, 2>> sp;
    for (int a = 0; a < ns; ++a)
        for (int b = 0; b <= a; ++b) sp.push_back({a, b});
    const int64_t nsp = (int64_t)sp.size();
#pragma omp parallel for schedule(dynamic)
    for (int64_t x = 0; x < nsp; ++x) {
        std::vector<double> cart, f, R, work, Wk;
        for (int64_t y = 0; y <= x; ++y) {
            const int a = sp[x][0], b = sp[x][1], c = sp[y][0], d = sp[y][1];
            const Shell* S[4] = {&bs.sh[a], &bs.sh[b], &bs.sh[c], &bs.sh[d]};
            eri_cart(*S[0], *S[1], *S[2], *S[3], pairs[(size_t)a * ns + b], pairs[(size_t)c * ns + d], cart, R, work,
                     Wk);
            quartet_to_functions(S, cart, f);
            const int na = S[0]->nf, nb = S[1]->nf, nc = S[2]->nf, nd = S[3]->nf;
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j)
                    for (int k = 0; k < nc; ++k)
                        for (int l = 0; l < nd; ++l) {
                            const double v = f[(((size_t)i * nb + j) * nc + k) * nd + l];
                            const int64_t I = S[0]->off + i, J = S[1]->off + j, K = S[2]->off + k,
                                          Lx = S[3]->off + l;
                            const int64_t idx[8][4] = {{I, J, K, Lx}, {J, I, K, Lx}, {I, J, Lx, K}, {J, I, Lx, K},
                                                       {K, Lx, I, J}, {Lx, K, I, J}, {K, Lx, J, I}, {Lx, K, J, I}};
                            for (const auto& q : idx) eri[((q[0] * N + q[1]) * N + q[2]) * N + q[3]] = v;
                        }
        }
    }
}

// (mu nu | lam sig) for every (lam, sig) of the shell pair (c, d) and every
// (mu, nu) of shell pairs (a, b): used for the diagonal and single columns
void pair_block(const Basis& bs, int a, int b, int c, int d, std::vector<double>& f) {
    PairData bra, ket;
    make_pair(bs.sh[a], bs.sh[b], bra);
    make_pair(bs.sh[c], bs.sh[d], ket);
    std::vector<double> cart, R, work, Wk;
    const Shell* S[4] = {&bs.sh[a], &bs.sh[b], &bs.sh[c], &bs.sh[d]};
    eri_cart(*S[0], *S[1], *S[2], *S[3], bra, ket, cart, R, work, Wk);
    quartet_to_functions(S, cart, f);
}

int shell_of(const Basis& bs, int fn) {
    for (int s = 0; s < (int)bs.sh.size(); ++s)
        if (fn >= bs.sh[s].off && fn < bs.sh[s].off + bs.sh[s].nf) return s;
    return -1;
}

}  // namespace mshqc_ao_impl

using namespace mshqc_ao_impl;

extern "C" {

MSHQC_AO_API const char* mshqc_ao_last_error(void) { return g_err.c_str(); }

// The reference's Shell::normalize (src/core/basis.cc:82-104): the
// coefficients times the primitive norms of the x^l component, then divided
// by sqrt(sum c_i c_j (2 sqrt(a_i a_j) / (a_i + a_j))^(l + 3/2)) of those
// products.  (That sum is the norm of the contraction over normalized
// primitives only before the first step, so the resulting functions are not
// unit-norm in general -- a one-primitive shell keeps coefficient 1 on the raw
// Gaussian; energies do not depend on the scale of the basis functions.)
MSHQC_AO_API int mshqc_ao_normalize_shell(int l, int nprim, const double* exps, double* coefs) {
    if (l < 0 || l > kMaxL || nprim < 1 || !exps || !coefs) {
        g_err = "normalize_shell: bad arguments";
        return MSHQC_AO_ERR_ARG;
    }
    // primitive norm of the x^l component: (2a/pi)^(3/4) (4a)^(l/2) / sqrt((2l-1)!!)
    for (int k = 0; k < nprim; ++k)
        coefs[k] *= std::pow(2.0 * exps[k] / kPi, 0.75) * std::pow(4.0 * exps[k], 0.5 * l) /
                    std::sqrt(dfact(2 * l - 1));
    double s = 0.0;
    for (int i = 0; i < nprim; ++i)
        for (int j = 0; j < nprim; ++j) {
            const double r = 2.0 * std::sqrt(exps[i] * exps[j]) / (exps[i] + exps[j]);
            s += coefs[i] * coefs[j] * std::pow(r, l + 1.5);
        }
    if (s > 1e-14) {
        const double f = 1.0 / std::sqrt(s);
        for (int k = 0; k < nprim; ++k) coefs[k] *= f;
    }
    return MSHQC_AO_OK;
}

MSHQC_AO_API int mshqc_ao_nbf(const mshqc_ao_basis* basis, int64_t* nbf) {
    Basis bs;
    const int rc = build_basis(basis, bs);
    if (rc) return rc;
    if (!nbf) return MSHQC_AO_ERR_ARG;
    *nbf = bs.nbf;
    return MSHQC_AO_OK;
}

MSHQC_AO_API int mshqc_ao_one_electron(const mshqc_ao_basis* basis, const mshqc_ao_nuclei* nuclei, double* S,
                                       double* T, double* V) {
    try {
        Basis bs;
        const int rc = build_basis(basis, bs);
        if (rc) return rc;
        if (V && (!nuclei || nuclei->natom < 0)) {
            g_err = "nuclear attraction needs the nuclei";
            return MSHQC_AO_ERR_ARG;
        }
        if (S) one_electron(bs, OVERLAP, nuclei, S);
        if (T) one_electron(bs, KINETIC, nuclei, T);
        if (V) one_electron(bs, NUCLEAR, nuclei, V);
        return MSHQC_AO_OK;
    } catch (const std::exception& e) {
        g_err = e.what();
        return MSHQC_AO_ERR_INTERNAL;
    }
}

MSHQC_AO_API int mshqc_ao_eri(const mshqc_ao_basis* basis, double* eri) {
    try {
        Basis bs;
        const int rc = build_basis(basis, bs);
        if (rc) return rc;
        if (!eri) return MSHQC_AO_ERR_ARG;
        compute_eri_all(bs, eri);
        return MSHQC_AO_OK;
    } catch (const std::exception& e) {
        g_err = e.what();
        return MSHQC_AO_ERR_INTERNAL;
    }
}

MSHQC_AO_API int mshqc_ao_eri_diagonal(const mshqc_ao_basis* basis, double* diag) {
    try {
        Basis bs;
        const int rc = build_basis(basis, bs);
        if (rc) return rc;
        if (!diag) return MSHQC_AO_ERR_ARG;
        const int N = bs.nbf, ns = (int)bs.sh.size();
        for (int a = 0; a < ns; ++a)
            for (int b = 0; b < ns; ++b) {
                std::vector<double> f;
                pair_block(bs, a, b, a, b, f);
                const Shell& A = bs.sh[a];
                const Shell& B = bs.sh[b];
                for (int i = 0; i < A.nf; ++i)
                    for (int j = 0; j < B.nf; ++j)
                        diag[(size_t)(A.off + i) * N + (B.off + j)] =
                            f[(((size_t)i * B.nf + j) * A.nf + i) * B.nf + j];
            }
        return MSHQC_AO_OK;
    } catch (const std::exception& e) {
        g_err = e.what();
        return MSHQC_AO_ERR_INTERNAL;
    }
}

MSHQC_AO_API int mshqc_ao_eri_column(const mshqc_ao_basis* basis, int64_t pivot, double* col) {
    try {
        Basis bs;
        const int rc = build_basis(basis, bs);
        if (rc) return rc;
        const int N = bs.nbf;
        if (!col || pivot < 0 || pivot >= (int64_t)N * N) {
            g_err = "eri_column: pivot out of range";
            return MSHQC_AO_ERR_ARG;
        }
        const int r = (int)(pivot / N), s = (int)(pivot % N);
        const int c = shell_of(bs, r), d = shell_of(bs, s);
        const Shell& C = bs.sh[c];
        const Shell& D = bs.sh[d];
        const int ns = (int)bs.sh.size();
        for (int a = 0; a < ns; ++a)
            for (int b = 0; b < ns; ++b) {
                std::vector<double> f;
                pair_block(bs, a, b, c, d, f);
                const Shell& A = bs.sh[a];
                const Shell& B = bs.sh[b];
                for (int i = 0; i < A.nf; ++i)
                    for (int j = 0; j < B.nf; ++j)
                        col[(size_t)(A.off + i) * N + (B.off + j)] =
                            f[(((size_t)i * B.nf + j) * C.nf + (r - C.off)) * D.nf + (s - D.off)];
            }
        return MSHQC_AO_OK;
    } catch (const std::exception& e) {
        g_err = e.what();
        return MSHQC_AO_ERR_INTERNAL;
    }
}

MSHQC_AO_API int mshqc_ao_nuclear_repulsion(const mshqc_ao_nuclei* nuclei, double* e) {
    if (!nuclei || !e) return MSHQC_AO_ERR_ARG;
    double s = 0.0;
    for (int i = 0; i < nuclei->natom; ++i)
        for (int j = 0; j < i; ++j) {
            const double dx = nuclei->xyz[3 * i] - nuclei->xyz[3 * j], dy = nuclei->xyz[3 * i + 1] - nuclei->xyz[3 * j + 1],
                         dz = nuclei->xyz[3 * i + 2] - nuclei->xyz[3 * j + 2];
            s += nuclei->Z[i] * nuclei->Z[j] / std::sqrt(dx * dx + dy * dy + dz * dz);
        }
    *e = s;
    return MSHQC_AO_OK;
}

}  // extern "C"
