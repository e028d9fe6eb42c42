"""C-ABI checks that need no GPU: the library loads, exports every entry
point declared in include/mshqc_cd.h, and reports a missing device as an
error status instead of crashing."""
import ctypes

import pytest

from mshqc_b200 import capi


def test_library_built():
    assert capi.library_available(), "run `python -m mshqc_b200.build`"


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(capi.LIB_PATH)
    declared = capi.exported_symbols_from_header()
    assert declared, "no MSHQC_CD_API declarations found"
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared) == set(capi.SIGNATURES), "capi.SIGNATURES out of sync with the header"


def test_abi_version():
    assert capi.load_library().mshqc_cd_abi_version() == 1


def test_error_paths_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = capi.load_library()
    h = ctypes.c_void_p()
    rc = lib.mshqc_cd_ctx_create(0, ctypes.byref(h))
    assert rc == capi.ERR_UNSUPPORTED
    assert b"device" in lib.mshqc_cd_last_error()
    # null context and null outputs are argument errors, not crashes
    assert lib.mshqc_cd_mp2_energy(None, 0, 0, None) == capi.ERR_ARG
    assert lib.mshqc_cd_set_vectors(None, None, 4, 4, 0, 0) == capi.ERR_ARG
    assert lib.mshqc_cd_ctx_destroy(None) == capi.OK
