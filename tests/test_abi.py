"""The C-ABI libraries load and export every function their headers declare;
status handling without a GPU.  CPU only (no compute calls)."""
import ctypes as C
import pytest

import bmb200 as bm


def _gpu_present():
    L = bm.cuda_lib()
    h = C.c_void_p()
    st = L.bm_ctx_create(0, C.byref(h))
    if st == bm.BM_OK:
        L.bm_ctx_destroy(h)
        return True
    return False


def test_cuda_lib_exports_header():
    L = bm.cuda_lib()
    names = bm.header_functions("bm_cuda.h")
    assert len(names) >= 35
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_host_lib_exports_header():
    L = bm.host_lib()
    names = bm.header_functions("bm_host.h")
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    L = bm.cuda_lib()
    for s in range(8):
        assert L.bm_status_str(s)
    assert L.bm_status_str(bm.BM_OK) == b"ok"


def test_create_without_gpu_reports_no_device():
    if _gpu_present():
        pytest.skip("a GPU is present")
    L = bm.cuda_lib()
    h = C.c_void_p()
    assert L.bm_ctx_create(0, C.byref(h)) == bm.BM_NO_DEVICE
    with pytest.raises(bm.BMError) as ei:
        bm.Engine(0)
    assert ei.value.status == bm.BM_NO_DEVICE


def test_null_context_is_rejected():
    L = bm.cuda_lib()
    assert L.bm_sync(None) == bm.BM_INVALID_ARG
    assert L.bm_set_mapping(None, None) == bm.BM_INVALID_ARG
    assert L.bm_score(None, None) == bm.BM_INVALID_ARG
    assert L.bm_launch_count(None) == 0
    m = C.c_int32(-1)
    assert L.bm_set_semantics(None, 1) == bm.BM_INVALID_ARG
    assert L.bm_get_semantics(None, C.byref(m)) == bm.BM_INVALID_ARG and m.value == -1
    assert L.bm_set_row_split(None, 0) == bm.BM_INVALID_ARG
    assert L.bm_set_row_tiers(None, 0) == bm.BM_INVALID_ARG
    assert L.bm_get_row_tiers(None, C.byref(m)) == bm.BM_INVALID_ARG
