"""A gradient shared among ranks (mshqc_cd_set_partition), the ranks run one
after another on one GPU: the shares' energies and derivatives add up to the
unpartitioned gradient (FP64 path: to rounding, 1e-12 of the largest entry;
mixed path: 1e-8, since its transposed transforms slice each share's Gamma
with its own row scales, ~2^-32 relative per term), restricted and
unrestricted, with small occupied blocks so that there are many block pairs
to share.  A share that owns no unit returns zeros."""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def twin(N, o, M, seed, nocc_beta=None):
    base = syn.make_inputs(N, o, M, seed=seed, nocc_beta=nocc_beta)
    sig = syn.twin_sigma(N, o, M, base.alpha.eps)
    return syn.make_inputs(N, o, M, seed=seed, sigma=sig, nocc_beta=nocc_beta)


def setup(ctx, inp, unres):
    ctx.set_vectors(inp.L)
    ctx.set_orbitals(capi.ALPHA, inp.alpha.C, inp.alpha.eps, inp.alpha.nocc)
    if unres:
        ctx.set_orbitals(capi.BETA, inp.beta.C, inp.beta.eps, inp.beta.nocc)


def close(x, y, tol):
    return np.max(np.abs(x - y)) <= tol * np.max(np.abs(y))


@pytest.mark.parametrize("unres", [False, True])
@pytest.mark.parametrize("precision", [capi.FP16X3, capi.FP64])
@pytest.mark.parametrize("nranks", [2, 3])
def test_shares_add_up(monkeypatch, unres, precision, nranks):
    monkeypatch.setenv("MSHQC_CD_BWD_BLOCK", "3")
    inp = twin(110, 11, 260, seed=17, nocc_beta=9 if unres else None)
    kind = capi.UNRESTRICTED if unres else capi.RESTRICTED
    with capi.Context(0) as ctx:
        setup(ctx, inp, unres)
        full = ctx.mp2_gradient(kind, precision)
        shares = []
        for r in range(nranks):
            ctx.set_partition(r, nranks)
            setup(ctx, inp, unres)
            shares.append(ctx.mp2_gradient(kind, precision))
        ctx.set_partition(0, 1)
        again = ctx.mp2_gradient(kind, precision)      # back to the whole gradient
    tot = lambda f: sum(f(g) for g in shares)
    tol = 1e-12 if precision == capi.FP64 else 1e-8
    for k in ("ss_aa", "ss_bb", "os", "total"):
        assert abs(tot(lambda g: g.energy[k]) - full.energy[k]) <= 1e-12 * abs(full.energy["total"]), k
    assert close(tot(lambda g: g.dC_a), full.dC_a, tol)
    assert close(tot(lambda g: g.deps_a), full.deps_a, tol)
    if unres:
        assert close(tot(lambda g: g.dC_b), full.dC_b, tol)
        assert close(tot(lambda g: g.deps_b), full.deps_b, tol)
    assert abs(again.energy["total"] - full.energy["total"]) <= 1e-12 * abs(full.energy["total"])


def test_partition_arguments_are_checked():
    with capi.Context(0) as ctx:
        for bad in ((1, 1), (-1, 2), (0, 0)):
            with pytest.raises(capi.CDError):
                ctx.set_partition(*bad)
