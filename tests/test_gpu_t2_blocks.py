"""Amplitude blocks for t2 consumers (mshqc_cd_get_t2_block): the restricted
block against the t2 the reference's own CholeskyRMP2 stores
(CholeskyRMP2Result::t2, oracle/_ref, src/mp2/cholesky_rmp2.cc:118-153), and
the alpha-alpha, beta-beta, alpha-beta blocks against (ia|jb)/D of the numpy
oracle (the convention of CholeskyUMP2::compute_t2_amplitudes,
src/mp2/cholesky_ump2.cc:471-556); sub-blocks of pairs agree with the full
array; 1e-12 of the largest amplitude."""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn
from oracle import cdmp2_oracle as orc
from oracle import ref

pytestmark = pytest.mark.gpu


def close(x, y):
    return np.max(np.abs(x - y)) <= 1e-12 * np.max(np.abs(y))


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_restricted_block_matches_reference_t2():
    N, o, M = 60, 7, 150
    inp = syn.make_inputs(N, o, M, seed=31)
    a = inp.alpha
    r = ref.rmp2(inp.L, a.C, a.eps, o, want_t2=True)
    with capi.Context(0) as ctx:
        ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
        t = ctx.t2_block(0)
        sub = ctx.t2_block(0, 2, 3, 1, 4)
    assert t.shape == (o, o, N - o, N - o)
    assert close(t, r["t2"])
    assert close(sub, t[2:5, 1:5])


def test_unrestricted_blocks_match_oracle():
    N, oa, ob, M = 50, 6, 4, 120
    inp = syn.make_inputs(N, oa, M, seed=33, nocc_beta=ob)
    A, B = inp.alpha, inp.beta
    Ba = orc.transform(inp.L, A.C, oa)
    Bb = orc.transform(inp.L, B.C, ob)
    with capi.Context(0) as ctx:
        ctx.set_vectors(inp.L)
        ctx.set_orbitals(capi.ALPHA, A.C, A.eps, oa)
        ctx.set_orbitals(capi.BETA, B.C, B.eps, ob)
        blocks = [ctx.t2_block(k) for k in range(3)]
    for k, (X, Y, ex, ey, ox, oy) in enumerate([(Ba, Ba, A.eps, A.eps, oa, oa), (Bb, Bb, B.eps, B.eps, ob, ob),
                                               (Ba, Bb, A.eps, B.eps, oa, ob)]):
        g = np.einsum("iaQ,jbQ->ijab", X, Y)
        D = ex[:ox, None, None, None] + ey[None, :oy, None, None] - ex[None, None, ox:, None] - ey[None, None, None, oy:]
        assert close(blocks[k], g / D), k
