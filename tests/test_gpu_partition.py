"""A gradient shared among ranks (mshqc_cd_set_partition), the ranks run one
after another on one GPU: the shares' energies and derivatives add up to the
unpartitioned gradient (FP64 path: to rounding, 1e-12 of the largest entry;
mixed path: the energies to 1e-12 -- its integral tiles are exact -- and the
derivatives to 2e-6 of the largest entry: the shares run smaller occupied
blocks than the whole gradient, and Gamma, accumulated as BF16x3 products in
FP32 chunks per block pair, rounds differently at ~1e-7 relative, 1e-10
absolute here against the 1e-6 the mixed path states), restricted and
unrestricted.  With a partition the block sizes come from the dimensions and
the rank count alone (about 32 block pairs per rank), so every share gets
work (a nonzero energy) and the shares do not change when a GPU has less
free memory."""
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


def shares_of(ctx, inp, unres, kind, precision, nranks):
    out = []
    for r in range(nranks):
        ctx.set_partition(r, nranks)
        setup(ctx, inp, unres)
        out.append(ctx.mp2_gradient(kind, precision))
    ctx.set_partition(0, 1)
    return out


def check_sum(shares, full, unres, precision):
    tot = lambda f: sum(f(g) for g in shares)
    tol = 1e-12 if precision == capi.FP64 else 2e-6
    for k in ("ss_aa", "ss_bb", "os", "total"):
        assert abs(tot(lambda g: g.energy[k]) - full.energy[k]) <= 1e-12 * abs(full.energy["total"]), k
    assert close(tot(lambda g: g.dC_a), full.dC_a, tol)
    assert close(tot(lambda g: g.deps_a), full.deps_a, tol)
    if unres:
        assert close(tot(lambda g: g.dC_b), full.dC_b, tol)
        assert close(tot(lambda g: g.deps_b), full.deps_b, tol)


@pytest.mark.parametrize("unres", [False, True])
@pytest.mark.parametrize("precision", [capi.FP16X3, capi.FP64])
@pytest.mark.parametrize("nranks", [2, 3])
def test_shares_add_up(monkeypatch, unres, precision, nranks):
    monkeypatch.delenv("MSHQC_CD_BWD_BLOCK", raising=False)
    inp = twin(110, 13, 260, seed=17, nocc_beta=11 if unres else None)
    kind = capi.UNRESTRICTED if unres else capi.RESTRICTED
    with capi.Context(0) as ctx:
        setup(ctx, inp, unres)
        full = ctx.mp2_gradient(kind, precision)
        shares = shares_of(ctx, inp, unres, kind, precision, nranks)
        again = ctx.mp2_gradient(kind, precision)      # back to the whole gradient
    check_sum(shares, full, unres, precision)
    # every rank got units (13 occupied orbitals give at least 4 per rank)
    for g in shares:
        assert g.energy["total"] != 0.0
        assert np.max(np.abs(g.dC_a)) > 0.0
    assert abs(again.energy["total"] - full.energy["total"]) <= 1e-12 * abs(full.energy["total"])


@pytest.mark.parametrize("precision", [capi.FP16X3, capi.FP64])
def test_block_override_applies_to_every_pass(monkeypatch, precision):
    """MSHQC_CD_BWD_BLOCK sets the occupied block of the FP64 passes too: with
    blocks of 2 of 9 orbitals every one of 3 ranks owns units."""
    monkeypatch.setenv("MSHQC_CD_BWD_BLOCK", "2")
    inp = twin(90, 9, 200, seed=5, nocc_beta=8)
    with capi.Context(0) as ctx:
        for unres in (False, True):
            kind = capi.UNRESTRICTED if unres else capi.RESTRICTED
            setup(ctx, inp, unres)
            full = ctx.mp2_gradient(kind, precision)
            shares = shares_of(ctx, inp, unres, kind, precision, 3)
            check_sum(shares, full, unres, precision)
            assert all(g.energy["total"] != 0.0 for g in shares)


def test_shares_do_not_depend_on_free_memory(monkeypatch):
    """The shares are the same when the GPU has most of its memory taken by
    another allocation (a rank on a busier GPU, 24 GB left free) as when it
    is free."""
    import torch
    monkeypatch.delenv("MSHQC_CD_BWD_BLOCK", raising=False)
    inp = twin(400, 40, 1600, seed=23)
    with capi.Context(0) as ctx:
        setup(ctx, inp, False)
        free_run = shares_of(ctx, inp, False, capi.RESTRICTED, capi.FP16X3, 2)
    free_b, _ = torch.cuda.mem_get_info(0)
    ballast = torch.empty(max(0, free_b - (24 << 30)), dtype=torch.uint8, device="cuda:0")
    try:
        with capi.Context(0) as ctx:
            setup(ctx, inp, False)
            busy_run = shares_of(ctx, inp, False, capi.RESTRICTED, capi.FP16X3, 2)
    finally:
        del ballast
        torch.cuda.empty_cache()
    for a, b in zip(free_run, busy_run):
        assert a.energy["total"] == b.energy["total"]
        assert np.array_equal(a.dC_a, b.dC_a)


def test_partition_arguments_are_checked():
    with capi.Context(0) as ctx:
        for bad in ((1, 1), (-1, 2), (0, 0)):
            with pytest.raises(capi.CDError):
                ctx.set_partition(*bad)
