"""The allocation-free entry point mshqc_cd_rmp2_energy_noalloc.

GPU: two calls in a row on the same buffers agree with the context entry
point mshqc_cd_mp2_energy(RESTRICTED, FP64) on the same MO vectors to 1e-12
relative (same kernel, same unit order; only the scratch differs).
CPU: an oversized request is refused with a clear message before the device
is touched.  This file is named to be collected last, so it also runs after
every other GPU test has used the library in the same process.
"""
import ctypes

import numpy as np
import pytest

from mshqc_b200 import capi
from mshqc_b200 import synthetic as syn

REL = 1e-12


def test_oversized_request_is_refused():
    lib = capi.load_library()
    # nocc = 400, nvir = 1600: 80,200 pairs x 325 blocks of partials >> 16 MiB
    rc = lib.mshqc_cd_rmp2_energy_noalloc(ctypes.c_void_p(16), ctypes.c_void_p(16), 400, 1600, 100,
                                          ctypes.c_void_p(16), None)
    assert rc == capi.ERR_ARG
    msg = lib.mshqc_cd_last_error().decode()
    assert "static scratch holds" in msg and str(16 << 20) in msg, msg


def test_null_pointers_are_refused():
    lib = capi.load_library()
    rc = lib.mshqc_cd_rmp2_energy_noalloc(None, None, 4, 10, 20, None, None)
    assert rc == capi.ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("N,o,M", [(160, 16, 400), (121, 9, 203)])
def test_noalloc_matches_context_energy_twice(N, o, M):
    torch = pytest.importorskip("torch")
    base = syn.make_inputs(N, o, M, seed=31)
    sigma = syn.twin_sigma(N, o, M, base.alpha.eps)
    inp = syn.make_inputs(N, o, M, seed=31, sigma=sigma)
    a = inp.alpha
    v = N - o
    with capi.Context(0) as ctx:
        ctx.set_vectors(inp.L).set_orbitals(capi.ALPHA, a.C, a.eps, o)
        ref = ctx.mp2_energy(capi.RESTRICTED, capi.FP64)
        B = ctx.transform(capi.ALPHA, capi.FP64)            # (o, v, M)
    shape = capi.noalloc_shape(o, v, M)
    Bp = torch.zeros(shape, dtype=torch.float64, device="cuda:0")
    Bp[:, :v, :M] = torch.from_numpy(np.ascontiguousarray(B)).to("cuda:0")
    eps = torch.from_numpy(a.eps).to("cuda:0")
    energy = torch.empty(2, dtype=torch.float64, device="cuda:0")
    for _ in range(2):
        energy.fill_(float("nan"))
        capi.rmp2_energy_noalloc(Bp, eps, o, v, M, energy)
        torch.cuda.synchronize()
        e_tot, e_os = energy.cpu().tolist()
        assert abs(e_tot - ref["total"]) <= REL * abs(ref["total"]), (e_tot, ref["total"])
        assert abs(e_os - ref["os"]) <= REL * abs(ref["os"]), (e_os, ref["os"])
