"""CPU-side checks of the C-ABI library: it loads, exports every function
include/gsofa.h declares, and reports (never aborts) when there is no GPU."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "gsofa.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gsofa_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    from gsofatpds_b200 import _lib
    L = _lib.load()
    declared = header_functions()
    assert len(declared) >= 20
    missing = [f for f in declared if not hasattr(L, f)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == declared


def test_status_strings_and_defaults():
    from gsofatpds_b200 import _lib
    L = _lib.load()
    for code in range(0, 10):
        assert L.gsofa_status_string(code)
    o = _lib.Opts()
    assert L.gsofa_opts_default(ctypes.byref(o)) == 0
    assert o.max_supernode_size == 128 and o.flags == (_lib.SUPERNODES | _lib.DIGESTS)


def test_no_gpu_is_an_error_code_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from gsofatpds_b200 import Context, GsofaError, _lib
    with pytest.raises(GsofaError) as e:
        Context(0)
    assert e.value.status == _lib.ERR_CUDA
    L = _lib.load()
    assert L.gsofa_factor_symbolic_noalloc(None, None, None, None, None, None, None, None,
                                           None) == _lib.ERR_ARG
    argv = (ctypes.c_char_p * 3)(b"x", b"y", b"z")
    assert L.gsofa_symbfact_min_id(3, argv, 0, None, None, None, None) == _lib.ERR_ARG


def test_server_calls_reject_null_handles():
    """The serving entry points check their handles before touching a device."""
    from gsofatpds_b200 import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    t = ctypes.c_uint64()
    assert L.gsofa_server_create(None, None, 1000, 0, ctypes.byref(h)) == _lib.ERR_ARG
    assert L.gsofa_server_submit(None, 10, 10, None, None, None, ctypes.byref(t)) == _lib.ERR_ARG
    assert L.gsofa_server_poll(None, 1, None) == _lib.ERR_ARG
    assert L.gsofa_server_wait(None, 1, 0.0, None) == _lib.ERR_ARG
    assert L.gsofa_server_ticket_info(None, 1, None) == _lib.ERR_ARG
    assert L.gsofa_server_get_stats(None, None) == _lib.ERR_ARG
    assert L.gsofa_server_destroy(None) == _lib.ERR_ARG
    assert L.gsofa_server_last_error(None) == b"null server"


def test_order_and_permute_reject_null_handles():
    from gsofatpds_b200 import _lib
    L = _lib.load()
    st = _lib.OrderStats()
    h = ctypes.c_void_p()
    assert L.gsofa_order_nd(None, None, 0, 0, None, ctypes.byref(st)) == _lib.ERR_ARG
    assert L.gsofa_matrix_permute(None, None, None, ctypes.byref(h)) == _lib.ERR_ARG
    assert L.gsofa_order_wait_selftest(None, 50.0) == _lib.ERR_ARG
    nb = ctypes.c_int64()
    assert L.gsofa_result_supernodal(None, ctypes.byref(nb), None, None, None, None, None, None,
                                     None) == _lib.ERR_ARG


def test_cli_usage_without_arguments():
    from gsofatpds_b200 import _lib
    out = subprocess.run([_lib.CLI_PATH], capture_output=True, text=True, timeout=60)
    assert out.returncode == 1 and "usage" in out.stderr
