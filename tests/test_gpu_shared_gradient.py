"""A gradient shared by two ranks end to end (the library's partition, the
transforms shared over occupied orbitals through host collectives, the
shares summed by shard.allreduce_gradient): two gloo processes on one GPU
(their kernels never wait on each other; the collectives are staged through
host memory), restricted and unrestricted, mixed precision and FP64.  The
all-reduced energy and derivatives equal the unpartitioned gradient of the
same process (1e-12 of the largest entry on the FP64 path; 2e-6 on the mixed
path, whose shares run smaller occupied blocks than the whole gradient: Gamma,
BF16x3 products accumulated in FP32 chunks per block pair, then rounds
differently at ~1e-7 relative, and the int8-slice transforms scale each
share's operands by its own row maxima).  A one-rank NCCL group drives the NCCL callbacks of
shard.nccl_collectives on a library-sized buffer in place."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CASES = [("restricted", 1), ("restricted", 0), ("unrestricted", 1), ("unrestricted", 0)]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime
    from mshqc_b200 import capi, shard
    from mshqc_b200 import synthetic as syn
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        base = syn.make_inputs(130, 13, 300, seed=41, nocc_beta=11)
        sig = syn.twin_sigma(130, 13, 300, base.alpha.eps)
        inp = syn.make_inputs(130, 13, 300, seed=41, sigma=sig, nocc_beta=11)
        res = {}
        with capi.Context(0) as ctx:
            ctx.set_collectives(*shard.staged_collectives(torch.device("cuda", 0)))
            for kind_name, prec in CASES:
                unres = kind_name == "unrestricted"
                kind = capi.UNRESTRICTED if unres else capi.RESTRICTED
                ctx.set_vectors(inp.L)
                ctx.set_orbitals(capi.ALPHA, inp.alpha.C, inp.alpha.eps, inp.alpha.nocc)
                if unres:
                    ctx.set_orbitals(capi.BETA, inp.beta.C, inp.beta.eps, inp.beta.nocc)
                ctx.set_partition(rank, world)
                share = ctx.mp2_gradient(kind, prec)
                total = shard.allreduce_gradient(share)
                ctx.set_partition(0, 1)
                ctx.set_orbitals(capi.ALPHA, inp.alpha.C, inp.alpha.eps, inp.alpha.nocc)
                if unres:
                    ctx.set_orbitals(capi.BETA, inp.beta.C, inp.beta.eps, inp.beta.nocc)
                full = ctx.mp2_gradient(kind, prec)
                res[(kind_name, prec)] = (total, full, share.energy["total"])
        if rank == 0:
            out.put({k: (t.energy["total"], f.energy["total"], t.dC_a, f.dC_a, t.deps_a, f.deps_a,
                         t.dC_b, f.dC_b, e) for k, (t, f, e) in res.items()})
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_transforms_and_backward():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for (kind_name, prec), (et, ef, ta, fa, tda, fda, tb, fb, eshare) in res.items():
        tol = 1e-12 if prec == 0 else 2e-6
        assert eshare != 0.0
        assert abs(et - ef) <= 1e-12 * abs(ef), (kind_name, prec)
        assert np.max(np.abs(ta - fa)) <= tol * np.max(np.abs(fa)), (kind_name, prec)
        assert np.max(np.abs(tda - fda)) <= tol * np.max(np.abs(fda)), (kind_name, prec)
        if kind_name == "unrestricted":
            assert np.max(np.abs(tb - fb)) <= tol * np.max(np.abs(fb)), (kind_name, prec)


def _nccl_rank(port, out):
    sys.path.insert(0, ROOT)
    import datetime
    from mshqc_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120))
    try:
        dev = torch.device("cuda", 0)
        ag, rs = shard.nccl_collectives(dev)
        buf = torch.arange(1000, dtype=torch.float64, device=dev)
        ref = buf.clone()
        st = torch.cuda.Stream(device=dev)
        ag(buf.data_ptr(), 1000, st.cuda_stream)
        rs(buf.data_ptr(), 1000, st.cuda_stream)
        st.synchronize()
        out.put(bool(torch.equal(buf, ref)))
    finally:
        dist.destroy_process_group()


def test_nccl_callbacks_in_place_one_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_rank, args=(_free_port(), q))
    p.start()
    ok = q.get(timeout=300)
    p.join(timeout=120)
    assert p.exitcode == 0 and ok
