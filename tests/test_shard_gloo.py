"""Host side of a gradient shared among ranks (mshqc_b200.shard): two gloo
ranks on 127.0.0.1 add their partial energies, dE/dC and dE/deps, restricted
(alpha only) and unrestricted, and both end with the sums in the input's
layout (Fortran-ordered numpy dC stays Fortran-ordered)."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = 7


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _partial(rank, unres):
    from mshqc_b200 import capi
    rng = np.random.default_rng(10 + rank)
    e = {"ss_aa": 0.1 * (rank + 1), "ss_bb": 0.2 * (rank + 1), "os": 0.3 * (rank + 1), "total": 0.6 * (rank + 1),
         "ms_total": 5.0 + rank}
    dCa = np.asfortranarray(rng.standard_normal((N, N)))
    dea = rng.standard_normal(N)
    dCb = np.asfortranarray(rng.standard_normal((N, N))) if unres else None
    deb = rng.standard_normal(N) if unres else None
    return capi.Gradient(e, dCa, dCb, dea, deb)


def _rank(rank, world, port, unres, out):
    sys.path.insert(0, ROOT)
    from mshqc_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = shard.allreduce_gradient(_partial(rank, unres))
        out[rank] = (g.energy, g.dC_a, g.deps_a, g.dC_b, g.deps_b, bool(g.dC_a.flags.f_contiguous))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("unres", [False, True])
def test_allreduce_gradient_two_gloo_ranks(unres):
    sys.path.insert(0, ROOT)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, unres, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
            assert p.exitcode == 0
        res = dict(out)
    want = [_partial(r, unres) for r in range(2)]
    for r in range(2):
        energy, dCa, dea, dCb, deb, fortran = res[r]
        for k in ("ss_aa", "ss_bb", "os", "total"):
            assert abs(energy[k] - (want[0].energy[k] + want[1].energy[k])) < 1e-15
        assert energy["ms_total"] == want[r].energy["ms_total"]       # timings stay local
        assert np.array_equal(dCa, want[0].dC_a + want[1].dC_a) and fortran
        assert np.array_equal(dea, want[0].deps_a + want[1].deps_a)
        if unres:
            assert np.array_equal(dCb, want[0].dC_b + want[1].dC_b)
            assert np.array_equal(deb, want[0].deps_b + want[1].deps_b)
        else:
            assert dCb is None and deb is None
