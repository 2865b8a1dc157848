"""The engine against the reference's own GPU kernel calculateSwapDeltasKernelQuick
(src/graph-re-alignment-gpu.cu:139-248, compiled for sm_100a into
oracle/_ref/librefgpu.so): identical deltas on the same pairs, and both timed
on the same device.  Set BM_RESULTS_DIR to keep the timings as JSON."""
import ctypes as C
import json
import os
import time

import numpy as np
import pytest

import bmb200 as bm
from oracle_bind import REPO

pytestmark = pytest.mark.gpu

REFGPU = os.path.join(REPO, "oracle", "_ref", "librefgpu.so")


def refgpu():
    L = C.CDLL(REFGPU)
    vp = C.c_void_p
    L.refgpu_quick.restype = C.c_int
    L.refgpu_quick.argtypes = [C.c_int, C.c_longlong, vp, vp, vp, C.c_longlong, vp, vp, vp, vp, vp, C.c_int, C.c_int,
                               C.POINTER(C.c_float), vp, vp]
    L.refgpu_total_pairs.restype = C.c_longlong
    L.refgpu_total_pairs.argtypes = [C.c_int, C.c_int]
    return L


@pytest.mark.skipif(not os.path.exists(REFGPU), reason="oracle/_ref/librefgpu.so not built")
@pytest.mark.parametrize("config,nrows", [(1, 16), (2, 57)])
def test_deltas_equal_reference_gpu_kernel(config, nrows):
    A, B, truth, init = bm.gen_pair(config, init_mode=0) if config == 2 else bm.gen_pair(config)
    n = A.n
    order = bm.rows_from_ordering(bm.ordering_by_weighted_degree(A))
    rows = np.ascontiguousarray(order[n // 3:n // 3 + nrows]).astype(np.int32)
    L = refgpu()
    total = L.refgpu_total_pairs(n, nrows)
    d_ref = np.zeros(total, np.int32)
    p_ref = np.zeros(2 * total, np.int32)
    ms = C.c_float()
    iters = 1 if config == 2 else 3
    st = L.refgpu_quick(n, A.m, A.src.ctypes.data, A.dst.ctypes.data, A.w.ctypes.data, B.m, B.src.ctypes.data,
                        B.dst.ctypes.data, B.w.ctypes.data, init.ctypes.data, rows.ctypes.data, nrows, iters,
                        C.byref(ms), d_ref.ctypes.data, p_ref.ctypes.data)
    assert st == 0, f"reference kernel failed with CUDA error {st}"
    pairs = p_ref.reshape(-1, 2)
    eng = bm.Engine(0)
    eng.set_graphs(A, B)
    eng.set_mapping(init)
    np.testing.assert_array_equal(eng.delta_pairs(pairs), d_ref.astype(np.int64))
    # the same deltas from whole rows: every pair has one endpoint in `rows`
    full = eng.delta_rows(rows)
    pos = {int(u): i for i, u in enumerate(rows)}
    r_idx = np.array([pos.get(int(a), -1) for a in pairs[:, 0]])
    assert (r_idx >= 0).all()
    np.testing.assert_array_equal(full[r_idx, pairs[:, 1]], d_ref.astype(np.int64))
    # timing of the engine's whole-row kernel on the same rows (materialised
    # rows and fused reduction), events on the engine stream
    d_rows = eng.dev_alloc(rows.nbytes)
    eng.h2d(d_rows, rows)
    d_res = eng.dev_alloc(bm.ROW_DTYPE.itemsize * nrows)
    e0, e1 = eng.event(), eng.event()
    eng.rows_best_dev(d_rows, None, nrows, d_res)
    eng.record(e0)
    for _ in range(20):
        eng.rows_best_dev(d_rows, None, nrows, d_res)
    eng.record(e1)
    ours_ms = eng.elapsed_ms(e0, e1) / 20
    eng.close()
    res = {"config": config, "n": n, "rows": nrows, "pairs": int(total), "reference_kernel_ms": ms.value,
           "reference_deltas_per_s": total / (ms.value / 1e3), "engine_rows_kernel_ms": ours_ms,
           "engine_deltas_per_s": nrows * (n - 1) / (ours_ms / 1e3)}
    print(json.dumps(res))
    out = os.environ.get("BM_RESULTS_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, f"refkernel_cfg{config}.json"), "w") as f:
            json.dump(res, f)


REFGPU3 = os.path.join(REPO, "oracle", "_ref", "librefgpu3.so")


def refgpu3():
    L = C.CDLL(REFGPU3)
    vp = C.c_void_p
    L.refgpu3_triplets.restype = C.c_int
    L.refgpu3_triplets.argtypes = [C.c_int, C.c_longlong, vp, vp, vp, C.c_longlong, vp, vp, vp, vp, vp, C.c_int,
                                   C.c_int, C.c_int, C.POINTER(C.c_float), vp, vp]
    return L


def run_refgpu3(A, B, pi, changed, batch, iters=1):
    """The reference's calculateThreeNodeSwapKernel on the first `batch`
    triplets of its enumeration around the vertices `changed`; returns
    (triplets (batch x 3), best deltas, ms per launch)."""
    L = refgpu3()
    changed = np.ascontiguousarray(changed, np.int32)
    deltas = np.zeros(batch, np.int32)
    trip = np.zeros(4 * batch, np.int32)
    ms = C.c_float()
    st = L.refgpu3_triplets(A.n, A.m, A.src.ctypes.data, A.dst.ctypes.data, A.w.ctypes.data, B.m, B.src.ctypes.data,
                            B.dst.ctypes.data, B.w.ctypes.data, pi.ctypes.data, changed.ctypes.data, len(changed),
                            batch, iters, C.byref(ms), deltas.ctypes.data, trip.ctypes.data)
    assert st == 0, f"reference 3-vertex kernel failed with CUDA error {st}"
    return trip.reshape(-1, 4)[:, :3].copy(), deltas.astype(np.int64), ms.value


@pytest.mark.skipif(not os.path.exists(REFGPU3), reason="oracle/_ref/librefgpu3.so not built")
@pytest.mark.parametrize("config,batch", [(1, 2048), (2, 1024)])
def test_3sets_equal_reference_gpu3_kernel(config, batch):
    """The best-permutation delta of every triplet the reference's 3-vertex
    GPU kernel (src/graph-re-alignment-gpu-3-swap.cu:43-305) evaluates, among
    its enumeration around six rows of the ordering, equals the engine's
    3-sets (all six permutations; the reference's identity permutation scores
    0, so both report max(0, best move))."""
    A, B, truth, init = bm.gen_pair(config)
    n = A.n
    order = bm.rows_from_ordering(bm.ordering_by_weighted_degree(A))
    changed = order[n // 4:n // 4 + 6]
    trip, d_ref, ms = run_refgpu3(A, B, init, changed, batch)
    assert (trip > 0).all() and (np.sort(trip, 1)[:, :2] != np.sort(trip, 1)[:, 1:]).all()
    with bm.Engine(0) as eng:
        eng.set_graphs(A, B)
        eng.set_mapping(init)
        best, perm = eng.kset_eval(3, trip)
    np.testing.assert_array_equal(np.maximum(best, 0), d_ref)
    print(json.dumps({"config": config, "triplets": batch, "reference_kernel_ms": ms,
                      "reference_triplets_per_s": batch / (ms / 1e3), "improving": int((d_ref > 0).sum())}))
