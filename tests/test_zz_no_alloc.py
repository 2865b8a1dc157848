"""bm_sa_run_noalloc, the allocation-free variant of the annealing chains.

It serves callers that cannot call cudaMalloc/cudaFree while they run: a
process whose device memory is owned by its own pool allocator under a fixed
budget, or a serving path that must not take cudaFree's device-wide
synchronisation while other streams are busy.  Called through the C ABI, its
results must equal those of the allocating entry point bm_sa_run exactly (the
chains are integer and deterministic), on two calls in a row that share its
static scratch, and neither call may allocate: the library's count of its own
allocation calls and the device's free memory stay where they were.  The
first call on a fresh context in a fresh process, before any other chain entry
point has run, allocates nothing either (the context reserved the scratch).
This file is collected last on purpose."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

import bmb200 as bm

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _noalloc_fn():
    L = bm.cuda_lib()
    f = L.bm_sa_run_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(bm.SaParams), C.c_void_p,
                  C.c_void_p, C.c_void_p]
    return f


def _free_bytes(eng):
    free, total = C.c_uint64(), C.c_uint64()
    assert eng.L.bm_device_memory(eng.h, C.byref(free), C.byref(total)) == bm.BM_OK
    return free.value


def _batch(eng):
    batch = bm.Batch(eng)
    pairs = []
    for seed, n, m in ((41, 260, 2600), (42, 500, 5000), (43, 180, 1400)):
        A, B, truth, init = bm.gen_pair(1, n=n, m_target=m, seed=seed)
        batch.add_pair(A, B)
        pairs.append(init)
    chain_pair = np.array([0, 1, 2, 1, 0, 2], np.int32)
    keys = np.array([101, 102, 103, 104, 105, 106], np.uint64)
    inits = [pairs[p] for p in chain_pair]
    return batch, chain_pair, keys, inits


STEPS, CAND, CHUNK = 5000, 4, 1200


def _call_noalloc(eng, batch, chain_pair, keys, flat):
    """One call through the C ABI; returns (mappings, scores, accepts,
    allocation calls made, change of the device's free bytes)."""
    f = _noalloc_fn()
    prm = bm.SaParams(STEPS, 5.0, 0.01, CAND, CHUNK)
    out = np.zeros_like(flat)
    scores = np.zeros(len(chain_pair), np.int64)
    acc = np.zeros(len(chain_pair), np.int64)
    eng.sync()
    a0, f0 = eng.L.bm_alloc_count(), _free_bytes(eng)
    st = f(batch.h, len(chain_pair), chain_pair.ctypes.data, keys.ctypes.data, flat.ctypes.data, C.byref(prm),
           out.ctypes.data, scores.ctypes.data, acc.ctypes.data)
    assert st == bm.BM_OK, eng.L.bm_ctx_last_error(eng.h).decode()
    a1, f1 = eng.L.bm_alloc_count(), _free_bytes(eng)
    return out, scores, acc, a1 - a0, f0 - f1


def test_noalloc_matches_allocating_entry_point():
    eng = bm.Engine(0)
    batch, chain_pair, keys, inits = _batch(eng)
    try:
        ref_pis, ref_scores, ref_acc, _ = batch.sa_run(chain_pair, keys, inits, STEPS, 5.0, 0.01, CAND, CHUNK)
        flat = np.ascontiguousarray(np.concatenate([np.asarray(p, np.int32) for p in inits]))
        for call in range(2):
            out, scores, acc, allocs, mem = _call_noalloc(eng, batch, chain_pair, keys, flat)
            np.testing.assert_array_equal(scores, ref_scores)
            np.testing.assert_array_equal(acc, ref_acc)
            np.testing.assert_array_equal(out, np.concatenate(ref_pis))
            assert allocs == 0, f"call {call} made {allocs} allocation calls"
            assert mem == 0, f"call {call} changed the device's free memory by {mem} bytes"

        # sizes beyond the static scratch are rejected with a clear error
        f = _noalloc_fn()
        prm = bm.SaParams(STEPS, 5.0, 0.01, CAND, CHUNK)
        many = np.zeros(1025, np.int32)
        st = f(batch.h, 1025, many.ctypes.data, np.zeros(1025, np.uint64).ctypes.data, flat.ctypes.data,
               C.byref(prm), None, None, None)
        assert st == bm.BM_INVALID_ARG
        assert b"at most 1024" in eng.L.bm_ctx_last_error(eng.h)
    finally:
        batch.close()
        eng.close()


_FRESH = r"""
import sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[2])
import numpy as np
import bmb200 as bm
import test_zz_no_alloc as t
eng = bm.Engine(0)
batch, chain_pair, keys, inits = t._batch(eng)
flat = np.ascontiguousarray(np.concatenate([np.asarray(p, np.int32) for p in inits]))
out, scores, acc, allocs, mem = t._call_noalloc(eng, batch, chain_pair, keys, flat)
ref_pis, ref_scores, ref_acc, _ = batch.sa_run(chain_pair, keys, inits, t.STEPS, 5.0, 0.01, t.CAND, t.CHUNK)
assert allocs == 0, f"first call made {allocs} allocation calls"
assert mem == 0, f"first call changed the device's free memory by {mem} bytes"
np.testing.assert_array_equal(scores, ref_scores)
np.testing.assert_array_equal(acc, ref_acc)
np.testing.assert_array_equal(out, np.concatenate(ref_pis))
batch.close()
eng.close()
print("fresh ok")
"""


def test_noalloc_first_call_in_fresh_process():
    """The first chain call of a new process is the allocation-free one, with
    the runtime's lazy module loading on: it must find the scratch reserved."""
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    py = os.path.join(os.path.dirname(HERE), "brain-match_b200", "python")
    r = subprocess.run([sys.executable, "-c", _FRESH, py, HERE], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "fresh ok" in r.stdout, r.stdout + r.stderr
