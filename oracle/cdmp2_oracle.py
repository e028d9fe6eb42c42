"""Oracle test infrastructure -- NOT part of the product.

A CPU (numpy, float64) restatement of the reference's Cholesky-vector MP2
algorithms, used only as the checker in tests/, in the smoke check and in
bench.py's cpu_baseline leg.  Each function cites the reference lines it
follows.  It is pinned against the reference itself (oracle/_ref, compiled
from the reference sources) by tests/test_oracle_golden.py through golden
fixtures in tests/golden/.

Array conventions
-----------------
* ``L``: (M, N*N) AO Cholesky vectors, index mu*N+nu (CholeskyERI storage,
  reference include/mshqc/integrals/cholesky_eri.h:81).
* ``C``: (N, N) MO coefficients C[mu, p]; ``eps``: (N,) orbital energies.
* ``B``: (o, v, M) MO vectors B[i, a, Q] = B^Q_ia.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg

DENOM_SKIP = 1e-12  # |D| < 1e-12 terms are skipped (src/mp2/cholesky_rmp2.cc:139)


# ---------------------------------------------------------------------------
# AO -> MO half transform (A3)
# ---------------------------------------------------------------------------
def transform(L, C, nocc, convention="rmp2"):
    """B^Q_ia = sum_{mu nu} C_{mu i} Lmap^Q_{mu nu} C_{nu a}.

    convention "rmp2": Lmap is the column-major map of the stored vector
      (src/mp2/cholesky_rmp2.cc:84-88, src/mp2/cholesky_omp2.cc:84-86), i.e.
      Lmap[mu, nu] = L[nu*N + mu].
    convention "ump2": row-major reshape Lmap[mu, nu] = L[mu*N + nu]
      (src/mp2/cholesky_ump2.cc:265-281).
    The two agree for symmetric vectors.  Returns B as (o, v, M).
    """
    M = L.shape[0]
    N = C.shape[0]
    L3 = L.reshape(M, N, N)
    Co = C[:, :nocc]
    Cv = C[:, nocc:]
    if convention == "rmp2":
        # Lmap[Q] = L3[Q].T ; B = Co^T L3[Q]^T Cv
        Y = np.einsum("Qnm,mi->Qin", L3, Co, optimize=True)   # (Co^T Lmap)[i, nu]
    else:
        Y = np.einsum("Qmn,mi->Qin", L3, Co, optimize=True)
    B = np.einsum("Qin,na->iaQ", Y, Cv, optimize=True)
    return np.ascontiguousarray(B)


def denominators_block(e_i, e_j, e_a, e_b):
    return (e_i + e_j) - e_a[:, None] - e_b[None, :]


# ---------------------------------------------------------------------------
# CD-RMP2 energy (A4): src/mp2/cholesky_rmp2.cc:118-153
# ---------------------------------------------------------------------------
def rmp2_energy(B, eps, nocc):
    """E = sum_{ij} sum_{ab} (ia|jb) (2 (ia|jb) - (ib|ja)) / D_ijab.

    Returns (E, pair) with pair[i, j] the (i,j) pair energy (all ordered
    pairs, as the reference loop visits them)."""
    o, v, M = B.shape
    eo, ev = eps[:nocc], eps[nocc:]
    Bf = B.reshape(o * v, M)
    pair = np.zeros((o, o))
    for i in range(o):
        V = (B[i] @ Bf.T).reshape(v, o, v).transpose(1, 0, 2)     # [j, a, b]
        D = eo[i] + eo[:, None, None] - ev[None, :, None] - ev[None, None, :]
        ok = np.abs(D) >= DENOM_SKIP
        num = V * (2.0 * V - V.transpose(0, 2, 1))
        pair[i] = np.where(ok, num / np.where(ok, D, 1.0), 0.0).sum(axis=(1, 2))
    return float(pair.sum()), pair


def rmp2_t2(B, eps, nocc):
    """t_ij^ab = (ia|jb)/D (src/mp2/cholesky_rmp2.cc:142-148), (o,o,v,v)."""
    o, v, M = B.shape
    eo, ev = eps[:nocc], eps[nocc:]
    V = np.einsum("iaQ,jbQ->ijab", B, B, optimize=True)
    D = eo[:, None, None, None] + eo[None, :, None, None] - ev[None, None, :, None] - ev
    return np.where(np.abs(D) >= DENOM_SKIP, V / D, 0.0)


# ---------------------------------------------------------------------------
# CD-UMP2 energies (A5): src/mp2/cholesky_ump2.cc:299-465
# ---------------------------------------------------------------------------
def ump2_energies(Ba, Bb, ea, eb, na, nb):
    """Returns dict(ss_aa, ss_bb, os, e_corr)."""
    def same_spin(B, eps, n):
        o, v, M = B.shape
        eo, ev = eps[:n], eps[n:]
        Bf = B.reshape(o * v, M)
        e = 0.0
        for i in range(o):
            V = (B[i] @ Bf.T).reshape(v, o, v).transpose(1, 0, 2)
            g = V - V.transpose(0, 2, 1)
            D = eo[i] + eo[:, None, None] - ev[None, :, None] - ev[None, None, :]
            ok = np.abs(D) >= DENOM_SKIP
            e += 0.25 * np.where(ok, g * g / np.where(ok, D, 1.0), 0.0).sum()
        return float(e)

    def opposite_spin():
        oa, va, M = Ba.shape
        ob, vb, _ = Bb.shape
        Bbf = Bb.reshape(ob * vb, M)
        e = 0.0
        for i in range(oa):
            V = (Ba[i] @ Bbf.T).reshape(va, ob, vb).transpose(1, 0, 2)   # [j, a, b]
            D = ea[i] + eb[:nb, None, None] - ea[na:][None, :, None] - eb[nb:][None, None, :]
            ok = np.abs(D) >= DENOM_SKIP
            e += np.where(ok, V * V / np.where(ok, D, 1.0), 0.0).sum()
        return float(e)

    ss_aa = same_spin(Ba, ea, na)
    ss_bb = same_spin(Bb, eb, nb)
    os_ = opposite_spin()
    return dict(ss_aa=ss_aa, ss_bb=ss_bb, os=os_, e_corr=ss_aa + ss_bb + os_)


# ---------------------------------------------------------------------------
# Exact gradient (north-star backward; no reference counterpart)
# ---------------------------------------------------------------------------
def _dE_dC(L, C, nocc, G):
    """Chain rule through B^Q_ia = sum C_{mu i} Lmap^Q_{mu nu} C_{nu a} with
    the rmp2 (column-major) map.  G = dE/dB as (o, v, M).  Returns (N, N)."""
    M = L.shape[0]
    N = C.shape[0]
    L3 = L.reshape(M, N, N)
    Co, Cv = C[:, :nocc], C[:, nocc:]
    Z = np.einsum("Qnm,na->Qma", L3, Cv, optimize=True)     # (Lmap Cv)[mu, a]
    W = np.einsum("Qnm,mi->Qni", L3, Co, optimize=True)     # (Lmap^T Co)[nu, i]
    dC = np.zeros((N, N))
    dC[:, :nocc] = np.einsum("iaQ,Qma->mi", G, Z, optimize=True)
    dC[:, nocc:] = np.einsum("iaQ,Qni->na", G, W, optimize=True)
    return dC


def restricted_gradient(L, C, eps, nocc):
    """E_RMP2 and its exact derivatives with respect to B, C and eps.

    E = sum_{ijab} V (2V - V^T)/D, V^{ij}_ab = sum_Q B^Q_ia B^Q_jb.
    dE/dV^{ij}_ab = 2 tt_ab with tt = 2t - t^T, t = V/D.
    Gamma^Q_ia = sum_{jb} tt^{ij}_ab B^Q_jb ; dE/dB = 4 Gamma.
    dE/deps_k = -2 sum_{jab} t^{kj}_ab tt^{kj}_ab (occupied),
    dE/deps_c = +2 sum_{ijb} t^{ij}_cb tt^{ij}_cb (virtual).
    """
    B = transform(L, C, nocc)
    o, v, M = B.shape
    eo, ev = eps[:nocc], eps[nocc:]
    Bf = B.reshape(o * v, M)
    E = 0.0
    Gam = np.zeros_like(B)
    deps = np.zeros(len(eps))
    for i in range(o):
        V = (B[i] @ Bf.T).reshape(v, o, v).transpose(1, 0, 2)
        D = eo[i] + eo[:, None, None] - ev[None, :, None] - ev[None, None, :]
        t = V / D
        tt = 2.0 * t - t.transpose(0, 2, 1)
        E += float((V * tt).sum())
        Gam[i] = np.einsum("jab,jbQ->aQ", tt, B, optimize=True)
        r = t * tt
        deps[i] += -2.0 * r.sum()
        deps[nocc:] += 2.0 * r.sum(axis=(0, 2))
    dB = 4.0 * Gam
    dC = _dE_dC(L, C, nocc, dB)
    return dict(E=E, B=B, Gamma=Gam, dB=dB, dC=dC, deps=deps)


def unrestricted_gradient(L, Ca, Cb, ea, eb, na, nb):
    """E_UMP2 = E_ss(aa) + E_ss(bb) + E_os and its exact derivatives.

    Same spin: E = 1/4 sum g^2/D, g = V - V^T; dE/dV = t = g/D (antisymmetric).
    Opposite spin: E = sum V^2/D; dE/dV = 2 t, t = V/D.
    Gamma_a = sum_jb (t_ss^a B_a + t_os B_b) ; dE/dB_a = 2 Gamma_a (likewise b).
    """
    Ba = transform(L, Ca, na)
    Bb = transform(L, Cb, nb)
    oa, va, M = Ba.shape
    ob, vb, _ = Bb.shape
    res = {}
    Ga = np.zeros_like(Ba)
    Gb = np.zeros_like(Bb)
    da = np.zeros(len(ea))
    db = np.zeros(len(eb))

    def same(B, eps, n, Gam, deps):
        o, v, _ = B.shape
        eo, ev = eps[:n], eps[n:]
        Bf = B.reshape(o * v, M)
        e = 0.0
        for i in range(o):
            V = (B[i] @ Bf.T).reshape(v, o, v).transpose(1, 0, 2)
            D = eo[i] + eo[:, None, None] - ev[None, :, None] - ev[None, None, :]
            t = (V - V.transpose(0, 2, 1)) / D
            e += 0.25 * float((t * t * D).sum())
            Gam[i] += np.einsum("jab,jbQ->aQ", t, B, optimize=True)
            deps[i] += -0.5 * (t * t).sum()
            deps[n:] += 0.5 * (t * t).sum(axis=(0, 2))
        return e

    res["ss_aa"] = same(Ba, ea, na, Ga, da)
    res["ss_bb"] = same(Bb, eb, nb, Gb, db)
    Bbf = Bb.reshape(ob * vb, M)
    e_os = 0.0
    for i in range(oa):
        V = (Ba[i] @ Bbf.T).reshape(va, ob, vb).transpose(1, 0, 2)   # [j, a, b]
        D = ea[i] + eb[:nb, None, None] - ea[na:][None, :, None] - eb[nb:][None, None, :]
        t = V / D
        e_os += float((V * t).sum())
        Ga[i] += np.einsum("jab,jbQ->aQ", t, Bb, optimize=True)
        Gb += np.einsum("jab,aQ->jbQ", t, Ba[i], optimize=True)
        tt = t * t
        da[i] += -tt.sum()
        db[:nb] += -tt.sum(axis=(1, 2))
        da[na:] += tt.sum(axis=(0, 2))
        db[nb:] += tt.sum(axis=(0, 1))
    res["os"] = e_os
    res["E"] = res["ss_aa"] + res["ss_bb"] + e_os
    res.update(Ba=Ba, Bb=Bb, Gamma_a=Ga, Gamma_b=Gb, dB_a=2 * Ga, dB_b=2 * Gb,
               dC_a=_dE_dC(L, Ca, na, 2 * Ga), dC_b=_dE_dC(L, Cb, nb, 2 * Gb),
               deps_a=da, deps_b=db)
    return res


def orbital_gradient(C, dC, nocc):
    """g[a, i] = dE/dkappa_ai for C -> C exp(-kappa), kappa_ai = -kappa_ia
    (the rotation of src/mp2/cholesky_omp2.cc:385-396), eps held fixed:
    g = (C^T dE/dC)[i, a] - (C^T dE/dC)[a, i]."""
    X = C.T @ dC
    return X[:nocc, nocc:].T - X[nocc:, :nocc]


# ---------------------------------------------------------------------------
# CD-OMP2 (A6-A11): src/mp2/cholesky_omp2.cc
# ---------------------------------------------------------------------------
def omp2_t2(Ba, Bb, ea, eb, na, nb):
    """t2_aa, t2_bb (antisymmetrised, i<j, a<b filled 4 ways) and t2_ab
    (src/mp2/cholesky_omp2.cc:94-183)."""
    def ss(B, eps, n):
        eo, ev = eps[:n], eps[n:]
        V = np.einsum("iaQ,jbQ->ijab", B, B, optimize=True)
        D = eo[:, None, None, None] + eo[None, :, None, None] - ev[None, None, :, None] - ev
        g = V - V.transpose(0, 1, 3, 2)
        t = np.where(np.abs(D) >= DENOM_SKIP, g / np.where(np.abs(D) >= DENOM_SKIP, D, 1.0), 0.0)
        o, v = len(eo), len(ev)
        mask = (np.arange(o)[:, None] < np.arange(o)[None, :])[:, :, None, None] & \
               (np.arange(v)[:, None] < np.arange(v)[None, :])[None, None, :, :]
        tu = np.where(mask, t, 0.0)
        return tu - tu.transpose(1, 0, 2, 3) - tu.transpose(0, 1, 3, 2) + tu.transpose(1, 0, 3, 2)

    taa = ss(Ba, ea, na)
    tbb = ss(Bb, eb, nb)
    V = np.einsum("iaQ,jbQ->ijab", Ba, Bb, optimize=True)
    D = ea[:na, None, None, None] + eb[None, :nb, None, None] - ea[na:][None, None, :, None] - eb[nb:]
    ok = np.abs(D) >= DENOM_SKIP
    tab = np.where(ok, V / np.where(ok, D, 1.0), 0.0)
    return taa, tbb, tab


def omp2_energy(taa, tbb, tab, ea, eb, na, nb):
    """E = sum t^2 D over i<j,a<b (aa, bb) and all (ab)
    (src/mp2/cholesky_omp2.cc:189-230)."""
    def ss(t, eps, n):
        eo, ev = eps[:n], eps[n:]
        D = eo[:, None, None, None] + eo[None, :, None, None] - ev[None, None, :, None] - ev
        o, v = len(eo), len(ev)
        mask = (np.arange(o)[:, None] < np.arange(o)[None, :])[:, :, None, None] & \
               (np.arange(v)[:, None] < np.arange(v)[None, :])[None, None, :, :]
        return float((np.where(mask, t * t * D, 0.0)).sum())
    D = ea[:na, None, None, None] + eb[None, :nb, None, None] - ea[na:][None, None, :, None] - eb[nb:]
    return ss(taa, ea, na) + ss(tbb, eb, nb) + float((tab * tab * D).sum())


def omp2_opdm(taa, tbb, tab):
    """G_oo, G_vv per spin (src/mp2/cholesky_omp2.cc:232-326)."""
    Goo_a = -(0.5 * np.einsum("ikab,jkab->ij", taa, taa, optimize=True)
              + np.einsum("ikab,jkab->ij", tab, tab, optimize=True))
    Gvv_a = (0.5 * np.einsum("ijac,ijbc->ab", taa, taa, optimize=True)
             + np.einsum("ijac,ijbc->ab", tab, tab, optimize=True))
    Goo_b = -(0.5 * np.einsum("ikab,jkab->ij", tbb, tbb, optimize=True)
              + np.einsum("kiab,kjab->ij", tab, tab, optimize=True))
    Gvv_b = (0.5 * np.einsum("ijac,ijbc->ab", tbb, tbb, optimize=True)
             + np.einsum("ijca,ijcb->ab", tab, tab, optimize=True))
    return Goo_a, Gvv_a, Goo_b, Gvv_b


def cholesky_jk(L, P_tot, P_spin):
    """J = sum_Q <Lmap^Q, P_tot> Lmap^Q, K = sum_Q Lmap^Q P_spin Lmap^Q
    (src/mp2/cholesky_omp2.cc:347-358), Lmap the column-major map."""
    M = L.shape[0]
    N = P_tot.shape[0]
    Lm = L.reshape(M, N, N).transpose(0, 2, 1)
    coef = np.einsum("Qmn,mn->Q", Lm, P_tot, optimize=True)
    J = np.einsum("Q,Qmn->mn", coef, Lm, optimize=True)
    K = np.einsum("Qml,ls,Qsn->mn", Lm, P_spin, Lm, optimize=True)
    return J, K


def gfock_mo(L, H, C, P_tot_a, P_tot_b, alpha):
    """F_mo = C^T (H + J[P_a+P_b] - K[P_spin]) C (src/mp2/cholesky_omp2.cc:331-369)."""
    J, K = cholesky_jk(L, P_tot_a + P_tot_b, P_tot_a if alpha else P_tot_b)
    return C.T @ (H + J - K) @ C


def omp2_rotate(C, w, F, nocc):
    """kappa_ai = 0.5 w_ai / (F_aa - F_ii + 0.2) with |denominator| >= 1e-2,
    C <- C exp(-kappa) (src/mp2/cholesky_omp2.cc:375-400)."""
    N = C.shape[0]
    v = N - nocc
    diff = np.diag(F)[nocc:][:, None] - np.diag(F)[:nocc][None, :] + 0.2
    small = np.abs(diff) < 1e-2
    diff = np.where(small, np.where(diff >= 0, 1e-2, -1e-2), diff)
    val = (w / diff) * 0.5
    kap = np.zeros((N, N))
    kap[nocc:, :nocc] = val
    kap[:nocc, nocc:] = -val.T
    return C @ scipy.linalg.expm(-kap)


def omp2_pieces(L, H, Ca, Cb, ea, eb, na, nb):
    """One gradient evaluation of CholeskyOMP2::compute (src/mp2/cholesky_omp2.cc:442-466)."""
    N = Ca.shape[0]
    Ba = transform(L, Ca, na)
    Bb = transform(L, Cb, nb)
    taa, tbb, tab = omp2_t2(Ba, Bb, ea, eb, na, nb)
    E = omp2_energy(taa, tbb, tab, ea, eb, na, nb)
    Goo_a, Gvv_a, Goo_b, Gvv_b = omp2_opdm(taa, tbb, tab)
    Ga = np.zeros((N, N)); Ga[:na, :na] = Goo_a; Ga[na:, na:] = Gvv_a
    Gb = np.zeros((N, N)); Gb[:nb, :nb] = Goo_b; Gb[nb:, nb:] = Gvv_b
    Pa = Ca[:, :na] @ Ca[:, :na].T + Ca @ Ga @ Ca.T
    Pb = Cb[:, :nb] @ Cb[:, :nb].T + Cb @ Gb @ Cb.T
    Fa = gfock_mo(L, H, Ca, Pa, Pb, True)
    Fb = gfock_mo(L, H, Cb, Pa, Pb, False)
    return dict(e_mp2=E, Goo_a=Goo_a, Gvv_a=Gvv_a, Goo_b=Goo_b, Gvv_b=Gvv_b,
                F_a=Fa, F_b=Fb, w_a=2.0 * Fa[na:, :na], w_b=2.0 * Fb[nb:, :nb])


def omp2(L, H, Ca, Cb, ea, eb, na, nb, e_scf=0.0, max_iter=50, e_thr=1e-6, g_thr=1e-5):
    """CholeskyOMP2::compute (src/mp2/cholesky_omp2.cc:427-512), including its
    stale orbital energies / SCF energy and the beta copy when na == nb."""
    Ca = Ca.copy(); Cb = Cb.copy()
    e_prev = e_scf
    e_corr = 0.0
    converged = False
    it = 0
    while it < max_iter:
        it += 1
        p = omp2_pieces(L, H, Ca, Cb, ea, eb, na, nb)
        e_corr = p["e_mp2"]
        e_cur = e_scf + e_corr
        g = np.sqrt(np.sum(p["w_a"] ** 2) + np.sum(p["w_b"] ** 2))
        if g < g_thr and abs(e_cur - e_prev) < e_thr:
            converged = True
            break
        Ca = omp2_rotate(Ca, p["w_a"], p["F_a"], na)
        if na != nb:
            Cb = omp2_rotate(Cb, p["w_b"], p["F_b"], nb)
        else:
            Cb = Ca.copy()
        e_prev = e_cur
    return dict(e_corr=e_corr, e_total=e_prev, e_scf=e_scf, iterations=it,
                converged=converged, C_alpha=Ca, C_beta=Cb)


# ---------------------------------------------------------------------------
# Pivoted Cholesky of the ERI matrix (A2): src/integrals/cholesky_eri.cc:40-203
# ---------------------------------------------------------------------------
def cholesky_decompose(eri, threshold):
    """eri[i,j,k,l] = (ij|kl).  Composite index ij = i*N + j.  First-argmax
    pivot, column minus previous vectors, divide by sqrt(D_p) when > 1e-12,
    FP64 diagonal update clamped at 0, stop when max D < threshold."""
    N = eri.shape[0]
    n2 = N * N
    Emat = eri.reshape(n2, n2)         # row (i,j), col (k,l)
    D = np.array([eri[i, j, i, j] for i in range(N) for j in range(N)], dtype=np.float64)
    vecs = []
    if D.max() < threshold:
        return np.zeros((0, n2))
    while len(vecs) < n2:
        p = int(np.argmax(D))           # first maximum
        if D[p] < threshold:
            break
        col = Emat[:, p].copy()
        for Lk in vecs:
            col -= Lk * Lk[p]
        nf = np.sqrt(D[p])
        if nf > 1e-12:
            col /= nf
        D -= col * col
        D[D < 0.0] = 0.0
        vecs.append(col)
    return np.array(vecs) if vecs else np.zeros((0, n2))
