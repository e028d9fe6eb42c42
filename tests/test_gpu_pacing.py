"""Wave pacing and the Γ tile order decide only when and where each tile is
computed, never how: the mixed gradient is bit-identical with pacing off,
with the integral tiles paced as well, with other epoch lengths, and with
row-block-major or wider Γ tile groups (MSHQC_CD_PACE, MSHQC_CD_PACE_TILES,
MSHQC_CD_GAMMA_GROUP are read at every launch)."""
import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

N, O, M = 300, 30, 1200

VARIANTS = [
    {},
    {"MSHQC_CD_PACE": "off"},
    {"MSHQC_CD_PACE": "4,1", "MSHQC_CD_PACE_TILES": "16,2"},
    {"MSHQC_CD_GAMMA_GROUP": "1"},
    {"MSHQC_CD_GAMMA_GROUP": "7", "MSHQC_CD_BWD_BLOCK": "9"},
]


def test_pacing_and_tile_order_do_not_change_results(monkeypatch):
    inp = syn.make_inputs(N, O, M, seed=31)
    results = []
    with capi.Context(0) as ctx:
        ctx.set_vectors(inp.L)
        for env in VARIANTS:
            for k in ("MSHQC_CD_PACE", "MSHQC_CD_PACE_TILES", "MSHQC_CD_GAMMA_GROUP", "MSHQC_CD_BWD_BLOCK"):
                monkeypatch.delenv(k, raising=False)
            for k, v in env.items():
                monkeypatch.setenv(k, v)
            ctx.set_orbitals(capi.ALPHA, inp.alpha.C, inp.alpha.eps, O)
            results.append(ctx.mp2_gradient(capi.RESTRICTED, capi.FP16X3))
    base = results[0]
    for env, g in zip(VARIANTS[1:4], results[1:4]):
        assert g.energy["total"] == base.energy["total"], env
        assert np.array_equal(g.dC_a, base.dC_a), env
        assert np.array_equal(g.deps_a, base.deps_a), env
    # other occupied blocks change the block pairs, hence the order of the
    # FP32 chunk sums of Gamma: the energy stays exact, dC within 2e-6
    g = results[4]
    assert abs(g.energy["total"] - base.energy["total"]) <= 1e-12 * abs(base.energy["total"])
    assert np.max(np.abs(g.dC_a - base.dC_a)) <= 2e-6 * np.max(np.abs(base.dC_a))
