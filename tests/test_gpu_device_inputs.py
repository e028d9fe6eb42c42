"""Inputs handed over as CUDA tensors while the context runs on a stream of
its own (the bench's arrangement): the wrapper converts C to column-major
bytes on torch's current stream, and the library copies it on the context's
stream.  The copy must see the finished conversion; alternating alpha and
beta orbitals (whose temporaries torch's allocator hands out from the same
blocks) must give the results of host inputs on every call."""
import numpy as np
import pytest
import torch

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def test_unrestricted_device_orbitals_on_a_side_stream():
    N, oa, ob, M, seed = 320, 30, 27, 960, 41
    dev = torch.device("cuda", 0)
    orb_a = syn.make_orbitals(N, oa, seed)
    orb_b = syn.make_orbitals(N, ob, seed + 1)
    sigma = syn.twin_sigma(N, oa, M, orb_a.eps)
    L = syn.make_vectors_device(N, M, seed, sigma, dev)
    with capi.Context(0) as ref:
        ref.set_vectors(L)
        ref.set_orbitals(capi.ALPHA, orb_a.C, orb_a.eps, oa)
        ref.set_orbitals(capi.BETA, orb_b.C, orb_b.eps, ob)
        g_ref = ref.mp2_gradient(capi.UNRESTRICTED, capi.FP16X3)
        e_ref = ref.mp2_energy(capi.UNRESTRICTED, capi.FP64)
    Ca, ea = torch.from_numpy(orb_a.C).to(dev), torch.from_numpy(orb_a.eps).to(dev)
    Cb, eb = torch.from_numpy(orb_b.C).to(dev), torch.from_numpy(orb_b.eps).to(dev)
    stream = torch.cuda.Stream(device=dev)
    with capi.Context(0) as c:
        c.set_stream(stream.cuda_stream)
        c.set_vectors(L)
        for _ in range(4):
            c.set_orbitals(capi.ALPHA, Ca, ea, oa)
            c.set_orbitals(capi.BETA, Cb, eb, ob)
            g = c.mp2_gradient(capi.UNRESTRICTED, capi.FP16X3)
            assert abs(g.energy["total"] - g_ref.energy["total"]) <= 1e-9 * abs(g_ref.energy["total"])
            assert np.max(np.abs(g.dC_a - g_ref.dC_a)) <= 1e-9
            assert np.max(np.abs(g.dC_b - g_ref.dC_b)) <= 1e-9
            c.set_orbitals(capi.ALPHA, Ca, ea, oa)
            c.set_orbitals(capi.BETA, Cb, eb, ob)
            e = c.mp2_energy(capi.UNRESTRICTED, capi.FP64)
            assert abs(e["total"] - e_ref["total"]) <= 1e-12 * abs(e_ref["total"])
