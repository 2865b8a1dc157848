"""bm_sa_run_noalloc, the allocation-free variant of the annealing chains, for
callers that cannot call cudaMalloc/cudaFree while they run (device memory
owned by their own pool under a fixed budget, or a serving path that must not
take cudaFree's device-wide synchronisation).  Called through the C ABI, its
results must equal those of the allocating entry point bm_sa_run exactly (the
chains are integer and deterministic), on two calls in a row that share its
static scratch.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import bmb200 as bm

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    L = bm.cuda_lib()
    f = L.bm_sa_run_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(bm.SaParams), C.c_void_p,
                  C.c_void_p, C.c_void_p]
    return f


def test_noalloc_matches_allocating_entry_point():
    eng = bm.Engine(0)
    batch = bm.Batch(eng)
    try:
        pairs = []
        for seed, n, m in ((41, 260, 2600), (42, 500, 5000), (43, 180, 1400)):
            A, B, truth, init = bm.gen_pair(1, n=n, m_target=m, seed=seed)
            batch.add_pair(A, B)
            pairs.append((A, B, init))
        chain_pair = np.array([0, 1, 2, 1, 0, 2], np.int32)
        keys = np.array([101, 102, 103, 104, 105, 106], np.uint64)
        inits = [pairs[p][2] for p in chain_pair]
        steps, cand, chunk = 5000, 4, 1200
        ref_pis, ref_scores, ref_acc, _ = batch.sa_run(chain_pair, keys, inits, steps, 5.0, 0.01, cand, chunk)

        f = _noalloc_fn()
        flat = np.ascontiguousarray(np.concatenate([np.asarray(p, np.int32) for p in inits]))
        prm = bm.SaParams(steps, 5.0, 0.01, cand, chunk)
        for call in range(2):
            out = np.zeros_like(flat)
            scores = np.zeros(len(chain_pair), np.int64)
            acc = np.zeros(len(chain_pair), np.int64)
            st = f(batch.h, len(chain_pair), chain_pair.ctypes.data, keys.ctypes.data, flat.ctypes.data,
                   C.byref(prm), out.ctypes.data, scores.ctypes.data, acc.ctypes.data)
            assert st == bm.BM_OK, eng.L.bm_ctx_last_error(eng.h).decode()
            np.testing.assert_array_equal(scores, ref_scores)
            np.testing.assert_array_equal(acc, ref_acc)
            np.testing.assert_array_equal(out, np.concatenate(ref_pis))

        # sizes beyond the static scratch are rejected with a clear error
        many = np.zeros(1025, np.int32)
        st = f(batch.h, 1025, many.ctypes.data, np.zeros(1025, np.uint64).ctypes.data, flat.ctypes.data,
               C.byref(prm), None, None, None)
        assert st == bm.BM_INVALID_ARG
        assert b"at most 1024" in eng.L.bm_ctx_last_error(eng.h)
    finally:
        batch.close()
        eng.close()
