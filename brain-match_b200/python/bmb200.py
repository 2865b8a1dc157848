"""ctypes binding of the engine's C ABI (include/bm_cuda.h, include/bm_host.h).

The engine is C/CUDA; this module only marshals numpy arrays across the ABI for
tests and benchmarks.  It never computes deltas itself and has no CPU path:
if libbmcuda.so is missing or no GPU is present, the calls fail loudly.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import weakref
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_DIR = os.path.join(PKG_DIR, "lib")
BIN_DIR = os.path.join(PKG_DIR, "bin")
INCLUDE_DIR = os.path.join(REPO_DIR, "include")

BM_OK, BM_INVALID_ARG, BM_OOM, BM_CUDA_ERROR, BM_TIMEOUT, BM_PARITY_FAIL, BM_UNSUPPORTED, BM_NO_DEVICE = range(8)
STATUS_NAMES = ["OK", "INVALID_ARG", "OOM", "CUDA_ERROR", "TIMEOUT", "PARITY_FAIL", "UNSUPPORTED", "NO_DEVICE"]
SIDE_A, SIDE_B = 0, 1


def build(jobs: int = 8) -> None:
    """Compile libbmcuda.so (sm_100a), libbmhost.so and the CLIs in-tree."""
    subprocess.run(["make", "-C", PKG_DIR, f"-j{jobs}"], check=True, stdout=subprocess.DEVNULL)


def _lib(name: str) -> C.CDLL:
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        build()
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing and could not be built")
    return C.CDLL(path)


class RowResult(C.Structure):
    _fields_ = [("row", C.c_int32), ("first_pos", C.c_int32), ("best", C.c_int32), ("npos", C.c_int32),
                ("first_delta", C.c_int64), ("best_delta", C.c_int64)]


ROW_DTYPE = np.dtype([("row", np.int32), ("first_pos", np.int32), ("best", np.int32), ("npos", np.int32),
                      ("first_delta", np.int64), ("best_delta", np.int64)])
assert ROW_DTYPE.itemsize == C.sizeof(RowResult)


class Progress(C.Structure):
    _fields_ = [("rows_done", C.c_int64), ("evaluated", C.c_int64), ("accepts", C.c_int64), ("score", C.c_int64),
                ("launches", C.c_int64), ("next_row_pos", C.c_int32), ("next_col", C.c_int32),
                ("sweeps", C.c_int32), ("converged", C.c_int32), ("seconds", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SaParams(C.Structure):
    _fields_ = [("steps", C.c_int64), ("t0", C.c_double), ("t_end", C.c_double), ("candidates", C.c_int32),
                ("chunk", C.c_int64), ("threads_per_cta", C.c_int32)]


class SaStats(C.Structure):
    _fields_ = [("candidates", C.c_int32), ("ctas_per_chain", C.c_int32), ("launches", C.c_int64),
                ("seconds", C.c_double), ("threads_per_cta", C.c_int32)]


class LearnedParams(C.Structure):
    _fields_ = [("topk", C.c_int32), ("rows_per_batch", C.c_int32), ("refresh_batches", C.c_int32),
                ("uniform", C.c_int32), ("exact_fallback", C.c_int32), ("fallback_accepts", C.c_int32),
                ("train_every", C.c_int32),
                ("train_batch", C.c_int32), ("lr", C.c_float), ("weight_decay", C.c_float), ("seed", C.c_uint64),
                ("max_accepts", C.c_int64), ("max_sweeps", C.c_int32), ("time_budget_s", C.c_double),
                ("target_score", C.c_int64), ("sample", C.c_int32)]


class LearnedStats(C.Structure):
    _fields_ = [("proposals", C.c_int64), ("hits", C.c_int64), ("exact_passes", C.c_int64),
                ("train_steps", C.c_int64), ("t_propose", C.c_double), ("t_exact", C.c_double),
                ("t_train", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GenParams(C.Structure):
    _fields_ = [("n", C.c_int32), ("m_target", C.c_int64), ("degree_model", C.c_int32), ("alpha", C.c_double),
                ("max_degree", C.c_int32), ("weight_model", C.c_int32), ("geo_p", C.c_double),
                ("tail_frac", C.c_double), ("tail_max", C.c_int32), ("del_frac", C.c_double),
                ("add_frac", C.c_double), ("jitter", C.c_int32), ("shuffle_frac", C.c_double),
                ("init_mode", C.c_int32), ("seed", C.c_uint64)]


class Edges(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int64), ("src", C.POINTER(C.c_int32)), ("dst", C.POINTER(C.c_int32)),
                ("w", C.POINTER(C.c_int32))]


I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
I64P = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")

_cuda = None
_host = None


def cuda_lib() -> C.CDLL:
    global _cuda
    if _cuda is None:
        L = _lib("libbmcuda.so")
        vp = C.c_void_p
        sig = {
            "bm_ctx_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
            "bm_ctx_destroy": (None, [vp]),
            "bm_status_str": (C.c_char_p, [C.c_int]),
            "bm_ctx_last_error": (C.c_char_p, [vp]),
            "bm_ctx_stream": (vp, [vp]),
            "bm_sync": (C.c_int, [vp]),
            "bm_set_graph": (C.c_int, [vp, C.c_int, C.c_int32, C.c_int64, vp, vp, vp]),
            "bm_graph_info": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
            "bm_set_mapping": (C.c_int, [vp, vp]),
            "bm_get_mapping": (C.c_int, [vp, vp]),
            "bm_score": (C.c_int, [vp, C.POINTER(C.c_int64)]),
            "bm_tracked_score": (C.c_int, [vp, C.POINTER(C.c_int64)]),
            "bm_get_overlap": (C.c_int, [vp, vp]),
            "bm_delta_pairs": (C.c_int, [vp, vp, C.c_int64, vp]),
            "bm_delta_pairs_dev": (C.c_int, [vp, vp, C.c_int64, vp]),
            "bm_delta_rows": (C.c_int, [vp, vp, C.c_int32, vp]),
            "bm_delta_rows_dev": (C.c_int, [vp, vp, C.c_int32, vp]),
            "bm_rows_best": (C.c_int, [vp, vp, vp, C.c_int32, vp]),
            "bm_rows_best_dev": (C.c_int, [vp, vp, vp, C.c_int32, vp]),
            "bm_apply_swaps": (C.c_int, [vp, vp, vp, C.c_int32]),
            "bm_sweep_parity": (C.c_int, [vp, vp, C.c_int32, C.c_int64, C.c_int32, C.c_double, C.POINTER(Progress)]),
            "bm_search_batched": (C.c_int, [vp, vp, C.c_int32, C.c_int32, C.c_int64, C.c_int32, C.c_double,
                                            C.c_int64, C.POINTER(Progress)]),
            "bm_dev_alloc": (C.c_int, [vp, C.c_int64, C.POINTER(vp)]),
            "bm_dev_free": (C.c_int, [vp, vp]),
            "bm_memcpy_h2d": (C.c_int, [vp, vp, vp, C.c_int64]),
            "bm_memcpy_d2h": (C.c_int, [vp, vp, vp, C.c_int64]),
            "bm_host_alloc_pinned": (C.c_int, [C.c_int64, C.POINTER(vp)]),
            "bm_host_free_pinned": (C.c_int, [vp]),
            "bm_l2_flush": (C.c_int, [vp]),
            "bm_alloc_count": (C.c_uint64, []),
            "bm_comm_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_char_p, C.c_double, vp,
                                         C.POINTER(vp)]),
            "bm_comm_destroy": (None, [vp]),
            "bm_comm_last_error": (C.c_char_p, [vp]),
            "bm_comm_barrier": (C.c_int, [vp]),
            "bm_comm_allreduce_sum": (C.c_int, [vp, C.c_int64, C.POINTER(C.c_int64)]),
            "bm_comm_allgather_swaps": (C.c_int, [vp, vp, vp, C.c_int32, C.c_int32, vp, vp, C.POINTER(C.c_int32)]),
            "bm_comm_island_best": (C.c_int, [vp, C.c_int64, vp, C.c_int32, C.POINTER(C.c_int64),
                                              C.POINTER(C.c_int32)]),
            "bm_search_sharded": (C.c_int, [vp, vp, vp, C.c_int32, C.c_int32, C.c_int64, C.c_double,
                                            C.POINTER(Progress)]),
            "bm_select_independent": (C.c_int, [vp, vp, vp, C.c_int32, vp, C.POINTER(C.c_int32)]),
            "bm_sweep_similarity": (C.c_int, [vp, vp, C.c_int32, vp, vp, C.c_int64, C.c_double, C.POINTER(Progress)]),
            "bm_set_wait_limit": (C.c_int, [vp, C.c_int64]),
            "bm_probe_l2_bandwidth": (C.c_int, [vp, C.c_int64, C.c_int32, C.POINTER(C.c_double)]),
            "bm_device_memory": (C.c_int, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "bm_event_create": (C.c_int, [vp, C.POINTER(vp)]),
            "bm_event_destroy": (C.c_int, [vp, vp]),
            "bm_event_record": (C.c_int, [vp, vp]),
            "bm_event_elapsed_ms": (C.c_int, [vp, vp, vp, C.POINTER(C.c_float)]),
            "bm_launch_count": (C.c_int64, [vp]),
            "bm_device_pci_bus_id": (C.c_int, [vp, C.c_char_p, C.c_int32]),
            "bm_rows_max_active_clusters": (C.c_int, [vp, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
            "bm_set_row_tiling": (C.c_int, [vp, C.c_int32, C.c_int32]),
            "bm_set_row_split": (C.c_int, [vp, C.c_int32]),
            "bm_set_row_tiers": (C.c_int, [vp, C.c_int32]),
            "bm_get_row_tiers": (C.c_int, [vp, C.POINTER(C.c_int32)]),
            "bm_set_semantics": (C.c_int, [vp, C.c_int32]),
            "bm_get_semantics": (C.c_int, [vp, C.POINTER(C.c_int32)]),
            "bm_get_row_split": (C.c_int, [vp, C.POINTER(C.c_int32)]),
            "bm_kset_eval": (C.c_int, [vp, C.c_int32, vp, C.c_int64, vp, vp, vp]),
            "bm_kset_eval_dev": (C.c_int, [vp, C.c_int32, vp, C.c_int64, vp, vp, vp]),
            "bm_apply_sets": (C.c_int, [vp, C.c_int32, vp, vp, vp, C.c_int32]),
            "bm_search_ksets": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int64, C.c_double,
                                          C.POINTER(Progress)]),
            "bm_perturb": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_uint64, C.c_uint64, vp, C.POINTER(C.c_int64)]),
            "bm_search_restarts": (C.c_int, [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                             C.c_int32, C.c_double, C.POINTER(Progress), C.POINTER(C.c_int64)]),
            "bm_batch_create": (C.c_int, [vp, C.POINTER(vp)]),
            "bm_batch_destroy": (None, [vp]),
            "bm_batch_add_pair": (C.c_int, [vp, C.c_int32, C.c_int64, vp, vp, vp, C.c_int64, vp, vp, vp,
                                            C.POINTER(C.c_int32)]),
            "bm_sa_run": (C.c_int, [vp, C.c_int32, vp, vp, vp, C.POINTER(SaParams), vp, vp, vp, C.POINTER(SaStats)]),
            "bm_sa_layout_size": (C.c_int64, [vp, C.c_int32, vp]),
            "bm_get_row_tiling": (C.c_int, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "bm_greedy_match_dev": (C.c_int, [vp, C.c_int32, C.c_int64, vp, vp, C.c_int64, vp, vp, vp]),
            "bm_delta_table_dev": (C.c_int, [vp, vp, C.c_int64]),
            "bm_lap_solve": (C.c_int, [vp, vp, C.c_int32, vp, C.POINTER(C.c_int64)]),
            "bm_subset_assign": (C.c_int, [vp, vp, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
            "bm_search_hungarian": (C.c_int, [vp, C.c_int32, C.c_uint64, C.c_int32, C.c_double, C.POINTER(Progress)]),
            "bm_table_refresh_dev": (C.c_int, [vp, vp, C.c_int64, vp, C.c_int32]),
            "bm_table_topk": (C.c_int, [vp, vp, C.c_int64, C.c_int32, vp, vp, C.POINTER(C.c_int32)]),
            "bm_table_topk_dev": (C.c_int, [vp, vp, C.c_int64, C.c_int32, vp, vp, vp]),
            "bm_search_table": (C.c_int, [vp, vp, C.c_int64, C.c_int32, C.c_int64, C.c_int32, C.c_double,
                                          C.POINTER(Progress)]),
            "bm_mlp_create": (C.c_int, [vp, C.c_uint64, C.POINTER(vp)]),
            "bm_mlp_destroy": (None, [vp]),
            "bm_mlp_num_params": (C.c_int32, []),
            "bm_mlp_get_params": (C.c_int, [vp, vp]),
            "bm_mlp_set_params": (C.c_int, [vp, vp]),
            "bm_mlp_set_backend": (C.c_int, [vp, C.c_int32]),
            "bm_mlp_refresh_features": (C.c_int, [vp]),
            "bm_mlp_get_features": (C.c_int, [vp, vp]),
            "bm_mlp_pair_features": (C.c_int, [vp, vp, C.c_int64, vp]),
            "bm_mlp_score_pairs": (C.c_int, [vp, vp, C.c_int64, vp]),
            "bm_mlp_score_features": (C.c_int, [vp, vp, C.c_int64, vp]),
            "bm_mlp_score_rows": (C.c_int, [vp, vp, C.c_int32, vp]),
            "bm_mlp_rows_topk": (C.c_int, [vp, vp, C.c_int32, C.c_int32, vp, vp]),
            "bm_mlp_score_rows_dev": (C.c_int, [vp, vp, C.c_int32, vp]),
            "bm_mlp_score_candidates": (C.c_int, [vp, vp, C.c_int32, vp, C.c_int32, vp]),
            "bm_mlp_status": (C.c_int, [vp]),
            "bm_mlp_gradients": (C.c_int, [vp, vp, vp, C.c_int64, vp, C.POINTER(C.c_float)]),
            "bm_mlp_adamw_step": (C.c_int, [vp, vp, vp, C.c_int64, C.c_float, C.c_float, C.POINTER(C.c_float)]),
            "bm_mlp_reserve_records": (C.c_int, [vp, C.c_int64]),
            "bm_mlp_collect_rows": (C.c_int, [vp, vp, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_int64)]),
            "bm_mlp_clear_records": (C.c_int, [vp]),
            "bm_mlp_fit": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_uint64,
                                     C.POINTER(C.c_float)]),
            "bm_search_learned": (C.c_int, [vp, vp, vp, C.c_int32, C.POINTER(LearnedParams), C.POINTER(Progress),
                                            C.POINTER(LearnedStats)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _cuda = L
    return _cuda


def host_lib() -> C.CDLL:
    global _host
    if _host is None:
        L = _lib("libbmhost.so")
        vp = C.c_void_p
        sig = {
            "bm_edges_free": (None, [C.POINTER(Edges)]),
            "bm_read_graph_csv": (C.c_int, [C.c_char_p, C.POINTER(Edges), C.POINTER(C.c_int64)]),
            "bm_write_graph_csv": (C.c_int, [C.c_char_p, C.POINTER(Edges)]),
            "bm_read_ordering": (C.c_int, [C.c_char_p, C.c_int32, vp]),
            "bm_write_ordering": (C.c_int, [C.c_char_p, C.c_int32, vp]),
            "bm_read_mapping": (C.c_int, [C.c_char_p, C.c_int32, vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
            "bm_write_mapping": (C.c_int, [C.c_char_p, C.c_int32, vp]),
            "bm_scan_mapping_max_id": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32)]),
            "bm_gen_defaults": (C.c_int, [C.c_int, C.POINTER(GenParams)]),
            "bm_gen_pair": (C.c_int, [C.POINTER(GenParams), C.POINTER(Edges), C.POINTER(Edges), vp, vp]),
            "bm_ordering_by_weighted_degree": (None, [C.POINTER(Edges), vp]),
            "bm_rows_from_ordering": (None, [C.c_int32, vp, vp]),
            "bm_greedy_match": (C.c_int, [C.POINTER(Edges), C.POINTER(Edges), vp]),
            "bm_first_appearance": (C.c_int, [C.POINTER(Edges), vp, C.POINTER(C.c_int32)]),
            "bm_node_metrics": (C.c_int, [C.POINTER(Edges), vp, vp]),
            "bm_host_score": (C.c_int64, [C.POINTER(Edges), C.POINTER(Edges), vp]),
            "bm_check_bijection": (C.c_int32, [C.c_int32, vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _host = L
    return _host


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


# ---------------------------------------------------------------- host side

class Graph:
    """An edge list with ids 1..n (numpy int32 arrays)."""

    def __init__(self, n: int, src, dst, w):
        self.n = int(n)
        self.src, self.dst, self.w = _i32(src), _i32(dst), _i32(w)

    @property
    def m(self) -> int:
        return int(self.src.shape[0])

    def edges_struct(self) -> Edges:
        e = Edges()
        e.n, e.m = self.n, self.m
        e.src = self.src.ctypes.data_as(C.POINTER(C.c_int32))
        e.dst = self.dst.ctypes.data_as(C.POINTER(C.c_int32))
        e.w = self.w.ctypes.data_as(C.POINTER(C.c_int32))
        return e


def _take_edges(e: Edges) -> Graph:
    m = int(e.m)
    g = Graph(e.n, np.ctypeslib.as_array(e.src, (m,)).copy() if m else np.zeros(0, np.int32),
              np.ctypeslib.as_array(e.dst, (m,)).copy() if m else np.zeros(0, np.int32),
              np.ctypeslib.as_array(e.w, (m,)).copy() if m else np.zeros(0, np.int32))
    host_lib().bm_edges_free(C.byref(e))
    return g


def gen_params(config: int, **overrides) -> GenParams:
    p = GenParams()
    if host_lib().bm_gen_defaults(int(config), C.byref(p)) != 0:
        raise ValueError(f"unknown workload config {config}")
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def gen_pair(config: int, **overrides):
    """Synthetic pair: returns (A, B, pi_true, pi_init)."""
    p = gen_params(config, **overrides)
    a, b = Edges(), Edges()
    truth = np.zeros(p.n + 1, np.int32)
    init = np.zeros(p.n + 1, np.int32)
    if host_lib().bm_gen_pair(C.byref(p), C.byref(a), C.byref(b), _ptr(truth), _ptr(init)) != 0:
        raise RuntimeError("bm_gen_pair failed")
    return _take_edges(a), _take_edges(b), truth, init


def read_graph_csv(path: str):
    e = Edges()
    bad = C.c_int64(0)
    if host_lib().bm_read_graph_csv(path.encode(), C.byref(e), C.byref(bad)) != 0:
        raise OSError(f"cannot read {path}")
    return _take_edges(e), int(bad.value)


def write_graph_csv(path: str, g: Graph) -> None:
    e = g.edges_struct()
    if host_lib().bm_write_graph_csv(path.encode(), C.byref(e)) != 0:
        raise OSError(f"cannot write {path}")


def read_mapping(path: str, n: int):
    pi = np.zeros(n + 1, np.int32)
    cnt, mx = C.c_int64(0), C.c_int32(0)
    if host_lib().bm_read_mapping(path.encode(), n, _ptr(pi), C.byref(cnt), C.byref(mx)) != 0:
        raise OSError(f"cannot read {path}")
    return pi, int(cnt.value), int(mx.value)


def write_mapping(path: str, pi: np.ndarray) -> None:
    pi = _i32(pi)
    if host_lib().bm_write_mapping(path.encode(), pi.shape[0] - 1, _ptr(pi)) != 0:
        raise OSError(f"cannot write {path}")


def read_ordering(path: str, n: int) -> np.ndarray:
    o = np.zeros(n + 1, np.int32)
    if host_lib().bm_read_ordering(path.encode(), n, _ptr(o)) != 0:
        raise OSError(f"cannot read {path}")
    return o


def write_ordering(path: str, order: np.ndarray) -> None:
    order = _i32(order)
    if host_lib().bm_write_ordering(path.encode(), order.shape[0] - 1, _ptr(order)) != 0:
        raise OSError(f"cannot write {path}")


def ordering_by_weighted_degree(g: Graph) -> np.ndarray:
    o = np.zeros(g.n + 1, np.int32)
    e = g.edges_struct()
    host_lib().bm_ordering_by_weighted_degree(C.byref(e), _ptr(o))
    return o


def rows_from_ordering(order: np.ndarray) -> np.ndarray:
    order = _i32(order)
    n = order.shape[0] - 1
    rows = np.zeros(n, np.int32)
    host_lib().bm_rows_from_ordering(n, _ptr(order), _ptr(rows))
    return rows


def first_appearance(g: Graph) -> np.ndarray:
    """bm_first_appearance: vertices in order of first appearance in g's edges."""
    out = np.zeros(max(1, g.n), np.int32)
    cnt = C.c_int32()
    e = g.edges_struct()
    if host_lib().bm_first_appearance(C.byref(e), _ptr(out), C.byref(cnt)) != 0:
        raise RuntimeError("bm_first_appearance failed")
    return out[:cnt.value].copy()


def node_metrics(g: Graph, rank=None) -> np.ndarray:
    """bm_node_metrics: (n+1) x 5 doubles (in, out, avg in, avg out, rank)."""
    out = np.zeros((g.n + 1) * 5, np.float64)
    r = None if rank is None else _i32(rank)
    e = g.edges_struct()
    if host_lib().bm_node_metrics(C.byref(e), None if r is None else _ptr(r), _ptr(out)) != 0:
        raise RuntimeError("bm_node_metrics failed")
    return out.reshape(g.n + 1, 5)


def greedy_match(A: Graph, B: Graph) -> np.ndarray:
    n = max(A.n, B.n)
    pi = np.zeros(n + 1, np.int32)
    a, b = A.edges_struct(), B.edges_struct()
    if host_lib().bm_greedy_match(C.byref(a), C.byref(b), _ptr(pi)) != 0:
        raise RuntimeError("bm_greedy_match failed")
    return pi


def host_score(A: Graph, B: Graph, pi: np.ndarray) -> int:
    a, b = A.edges_struct(), B.edges_struct()
    return int(host_lib().bm_host_score(C.byref(a), C.byref(b), _ptr(_i32(pi))))


def check_bijection(pi: np.ndarray) -> int:
    pi = _i32(pi)
    return int(host_lib().bm_check_bijection(pi.shape[0] - 1, _ptr(pi)))


# -------------------------------------------------------------- device side

class BMError(RuntimeError):
    def __init__(self, status: int, msg: str):
        self.status = status
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {msg}")


_live_engines = weakref.WeakSet()


@atexit.register
def _close_live_engines() -> None:
    """Close every engine still open when the interpreter exits, each with its
    batches and models first, before the CUDA runtime is torn down."""
    for eng in list(_live_engines):
        try:
            eng.close()
        except Exception:
            pass


class Engine:
    """One device context: graphs, mapping and the search state."""

    def __init__(self, device: int = 0):
        self.L = cuda_lib()
        h = C.c_void_p()
        st = self.L.bm_ctx_create(device, C.byref(h))
        if st != BM_OK:
            raise BMError(st, f"bm_ctx_create({device})")
        self.h = h
        self.n = 0
        self._children = []  # weak references to batches and models, closed before the context
        _live_engines.add(self)

    def _chk(self, st: int, what: str, ok=(BM_OK,)) -> int:
        if st not in ok:
            raise BMError(st, f"{what}: {self.L.bm_ctx_last_error(self.h).decode()}")
        return st

    def close(self) -> None:
        for ref in self._children:
            child = ref()
            if child is not None:
                child.close()
        self._children = []
        if self.h:
            self.L.bm_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # graphs and mapping
    def set_graph(self, side: int, g: Graph) -> None:
        self._chk(self.L.bm_set_graph(self.h, side, g.n, g.m, _ptr(g.src), _ptr(g.dst), _ptr(g.w)), "bm_set_graph")
        self.n = g.n

    def set_graphs(self, A: Graph, B: Graph) -> None:
        self.set_graph(SIDE_A, A)
        self.set_graph(SIDE_B, B)

    def graph_info(self, side: int) -> dict:
        n, m, d, wd = C.c_int32(), C.c_int64(), C.c_int32(), C.c_int64()
        self._chk(self.L.bm_graph_info(self.h, side, C.byref(n), C.byref(m), C.byref(d), C.byref(wd)), "bm_graph_info")
        return {"n": n.value, "m": m.value, "max_degree": d.value, "max_weighted_degree": wd.value}

    def set_mapping(self, pi) -> None:
        pi = _i32(pi)
        self._chk(self.L.bm_set_mapping(self.h, _ptr(pi)), "bm_set_mapping")

    def get_mapping(self) -> np.ndarray:
        pi = np.zeros(self.n + 1, np.int32)
        self._chk(self.L.bm_get_mapping(self.h, _ptr(pi)), "bm_get_mapping")
        return pi

    def score(self) -> int:
        s = C.c_int64()
        self._chk(self.L.bm_score(self.h, C.byref(s)), "bm_score")
        return s.value

    def tracked_score(self) -> int:
        s = C.c_int64()
        self._chk(self.L.bm_tracked_score(self.h, C.byref(s)), "bm_tracked_score")
        return s.value

    def overlap(self) -> np.ndarray:
        o = np.zeros(self.n + 1, np.int32)
        self._chk(self.L.bm_get_overlap(self.h, _ptr(o)), "bm_get_overlap")
        return o

    # deltas
    def delta_pairs(self, pairs) -> np.ndarray:
        pairs = _i32(pairs).reshape(-1)
        k = pairs.shape[0] // 2
        out = np.zeros(k, np.int64)
        self._chk(self.L.bm_delta_pairs(self.h, _ptr(pairs), k, _ptr(out)), "bm_delta_pairs")
        return out

    def delta_rows(self, rows) -> np.ndarray:
        rows = _i32(rows).reshape(-1)
        out = np.zeros((rows.shape[0], self.n + 1), np.int64)
        self._chk(self.L.bm_delta_rows(self.h, _ptr(rows), rows.shape[0], _ptr(out)), "bm_delta_rows")
        return out

    def rows_best(self, rows, col_lo=None) -> np.ndarray:
        rows = _i32(rows).reshape(-1)
        out = np.zeros(rows.shape[0], ROW_DTYPE)
        cl = None if col_lo is None else _i32(col_lo).reshape(-1)
        self._chk(self.L.bm_rows_best(self.h, _ptr(rows), None if cl is None else _ptr(cl), rows.shape[0], _ptr(out)),
                  "bm_rows_best")
        return out

    def sweep_similarity(self, nodes, metrics_a, metrics_b, max_accepts=-1, time_budget=0.0, prog=None):
        """bm_sweep_similarity: one similarity-filtered pass; returns (Progress, status)."""
        prog = prog or Progress()
        nd = _i32(nodes)
        ma = np.ascontiguousarray(np.asarray(metrics_a, np.float64))
        mb = np.ascontiguousarray(np.asarray(metrics_b, np.float64))
        st = self.L.bm_sweep_similarity(self.h, _ptr(nd), nd.shape[0], _ptr(ma), _ptr(mb), max_accepts, time_budget,
                                        C.byref(prog))
        self._chk(st, "bm_sweep_similarity", ok=(BM_OK, BM_TIMEOUT))
        return prog, st

    def select_independent(self, pairs, deltas) -> np.ndarray:
        """bm_select_independent: indices of the chosen candidates."""
        p = _i32(np.asarray(pairs).reshape(-1))
        d = np.ascontiguousarray(np.asarray(deltas, np.int64).reshape(-1))
        chosen = np.zeros(max(1, d.shape[0]), np.int32)
        nc = C.c_int32()
        self._chk(self.L.bm_select_independent(self.h, _ptr(p), _ptr(d), d.shape[0], _ptr(chosen), C.byref(nc)),
                  "bm_select_independent")
        return chosen[:nc.value].copy()

    def apply_swaps(self, pairs, deltas=None) -> None:
        pairs = _i32(pairs).reshape(-1)
        d = None if deltas is None else np.ascontiguousarray(np.asarray(deltas, np.int64))
        self._chk(self.L.bm_apply_swaps(self.h, _ptr(pairs), None if d is None else _ptr(d), pairs.shape[0] // 2),
                  "bm_apply_swaps")

    # schedules
    def sweep_parity(self, rows=None, max_accepts=-1, max_sweeps=-1, time_budget=0.0, prog=None):
        prog = prog or Progress()
        r = None if rows is None else _i32(rows)
        st = self.L.bm_sweep_parity(self.h, None if r is None else _ptr(r), 0 if r is None else r.shape[0],
                                    max_accepts, max_sweeps, time_budget, C.byref(prog))
        self._chk(st, "bm_sweep_parity", ok=(BM_OK, BM_TIMEOUT))
        return prog, st

    def search_batched(self, rows=None, rows_per_batch=0, max_accepts=-1, max_sweeps=-1, time_budget=0.0,
                       target_score=0, prog=None):
        prog = prog or Progress()
        r = None if rows is None else _i32(rows)
        st = self.L.bm_search_batched(self.h, None if r is None else _ptr(r), 0 if r is None else r.shape[0],
                                      rows_per_batch, max_accepts, max_sweeps, time_budget, target_score,
                                      C.byref(prog))
        self._chk(st, "bm_search_batched", ok=(BM_OK, BM_TIMEOUT))
        return prog, st

    def kset_eval(self, k: int, sets, all_deltas: bool = False):
        """Best permutation of each k-set: returns (best_delta, best_perm[, all])."""
        sets = _i32(sets).reshape(-1)
        ns = sets.shape[0] // k
        best = np.zeros(ns, np.int64)
        perm = np.zeros(ns * k, np.int32)
        import math
        alld = np.zeros(ns * math.factorial(k), np.int64) if all_deltas else None
        self._chk(self.L.bm_kset_eval(self.h, k, _ptr(sets), ns, _ptr(best), _ptr(perm),
                                      None if alld is None else _ptr(alld)), "bm_kset_eval")
        perm = perm.reshape(ns, k)
        if all_deltas:
            return best, perm, alld.reshape(ns, -1)
        return best, perm

    def apply_sets(self, k: int, sets, perms, deltas=None) -> None:
        sets, perms = _i32(sets).reshape(-1), _i32(perms).reshape(-1)
        d = None if deltas is None else np.ascontiguousarray(np.asarray(deltas, np.int64))
        self._chk(self.L.bm_apply_sets(self.h, k, _ptr(sets), _ptr(perms), None if d is None else _ptr(d),
                                       sets.shape[0] // k), "bm_apply_sets")

    def search_ksets(self, k: int, sets_per_launch: int, mode: int = 0, seed: int = 1, max_launches: int = -1,
                     time_budget: float = 0.0, prog=None):
        prog = prog or Progress()
        st = self.L.bm_search_ksets(self.h, k, sets_per_launch, mode, seed, max_launches, time_budget,
                                    C.byref(prog))
        self._chk(st, "bm_search_ksets", ok=(BM_OK, BM_TIMEOUT))
        return prog, st

    def perturb(self, k: int, mode: int = 0, seed: int = 1, counter: int = 0):
        """k disjoint random swaps; returns (changed vertices (2k), total delta)."""
        ch = np.zeros(2 * k, np.int32)
        d = C.c_int64()
        self._chk(self.L.bm_perturb(self.h, k, mode, seed, counter, _ptr(ch), C.byref(d)), "bm_perturb")
        return ch, d.value

    def search_restarts(self, rows=None, rows_per_batch=0, k_perturb=5, mode=0, seed=1, max_restarts=3,
                        time_budget=0.0, prog=None):
        prog = prog or Progress()
        best = C.c_int64()
        r = None if rows is None else _i32(rows)
        st = self.L.bm_search_restarts(self.h, None if r is None else _ptr(r), 0 if r is None else r.shape[0],
                                       rows_per_batch, k_perturb, mode, seed, max_restarts, time_budget,
                                       C.byref(prog), C.byref(best))
        self._chk(st, "bm_search_restarts", ok=(BM_OK, BM_TIMEOUT))
        return prog, best.value, st

    # delta table (device array owned by the caller; see bm_delta_table_dev)
    def table_alloc(self):
        """A device int32 table for this context's n: returns (pointer, ld)."""
        ld = (self.n + 1 + 3) & ~3
        return self.dev_alloc(4 * (self.n + 1) * ld), ld

    def delta_table_dev(self, d_tab: int, ld: int) -> None:
        self._chk(self.L.bm_delta_table_dev(self.h, d_tab, ld), "bm_delta_table_dev")

    def table_refresh_dev(self, d_tab: int, ld: int, rows) -> None:
        r = _i32(rows)
        d_r = self.dev_alloc(max(4, r.nbytes))
        try:
            self.h2d(d_r, r)
            self._chk(self.L.bm_table_refresh_dev(self.h, d_tab, ld, d_r, r.shape[0]), "bm_table_refresh_dev")
            self.sync()
        finally:
            self.dev_free(d_r)

    def table_download(self, d_tab: int, ld: int) -> np.ndarray:
        out = np.zeros((self.n + 1, ld), np.int32)
        self.sync()
        self.d2h(out, d_tab)
        return out

    def table_topk(self, d_tab: int, ld: int, k: int):
        pairs = np.zeros((k, 2), np.int32)
        deltas = np.zeros(k, np.int64)
        cnt = C.c_int32()
        self._chk(self.L.bm_table_topk(self.h, d_tab, ld, k, _ptr(pairs), _ptr(deltas), C.byref(cnt)),
                  "bm_table_topk")
        return pairs[:cnt.value], deltas[:cnt.value]

    def search_table(self, d_tab: int, ld: int, k: int = 1024, max_accepts: int = -1, max_rounds: int = -1,
                     time_budget: float = 0.0, prog=None):
        prog = prog or Progress()
        st = self.L.bm_search_table(self.h, d_tab, ld, k, max_accepts, max_rounds, time_budget, C.byref(prog))
        self._chk(st, "bm_search_table", ok=(BM_OK, BM_TIMEOUT))
        return prog, st

    def lap_solve(self, benefit):
        a = np.ascontiguousarray(np.asarray(benefit, dtype=np.int32))
        k = a.shape[0]
        assign = np.zeros(k, np.int32)
        tot = C.c_int64()
        self._chk(self.L.bm_lap_solve(self.h, _ptr(a), k, _ptr(assign), C.byref(tot)), "bm_lap_solve")
        return assign, tot.value

    def subset_assign(self, subset):
        s = _i32(subset)
        d = C.c_int64()
        ch = C.c_int32()
        self._chk(self.L.bm_subset_assign(self.h, _ptr(s), s.shape[0], C.byref(d), C.byref(ch)), "bm_subset_assign")
        return d.value, ch.value

    def search_hungarian(self, k=1024, seed=1, iterations=10, time_budget=0.0, prog=None):
        prog = prog or Progress()
        st = self.L.bm_search_hungarian(self.h, k, seed, iterations, time_budget, C.byref(prog))
        self._chk(st, "bm_search_hungarian", ok=(BM_OK, BM_TIMEOUT))
        return prog, st

    def greedy_match(self, A: Graph, B: Graph) -> np.ndarray:
        """Greedy-similarity initial matching on the device (n+1 ints)."""
        n = max(A.n, B.n)
        pi = np.zeros(n + 1, np.int32)
        self._chk(self.L.bm_greedy_match_dev(self.h, n, A.m, _ptr(A.src), _ptr(A.dst), B.m, _ptr(B.src),
                                             _ptr(B.dst), _ptr(pi)), "bm_greedy_match_dev")
        return pi

    def set_row_tiling(self, ctas_per_row: int = 0, threads: int = 0) -> None:
        self._chk(self.L.bm_set_row_tiling(self.h, ctas_per_row, threads), "bm_set_row_tiling")

    def set_row_split(self, slots: int = 0) -> None:
        """Cluster slots of a row launch: 0 automatic, -1 off, k > 0 k slots."""
        self._chk(self.L.bm_set_row_split(self.h, slots), "bm_set_row_split")

    def row_split(self) -> int:
        v = C.c_int32()
        self._chk(self.L.bm_get_row_split(self.h, C.byref(v)), "bm_get_row_split")
        return v.value

    def set_row_tiers(self, heavy_rows: int = 0) -> None:
        """Rows of a launch run in twice-wider clusters: 0 automatic, -1 off, k > 0 at most k."""
        self._chk(self.L.bm_set_row_tiers(self.h, heavy_rows), "bm_set_row_tiers")

    def row_tiers(self) -> int:
        v = C.c_int32()
        self._chk(self.L.bm_get_row_tiers(self.h, C.byref(v)), "bm_get_row_tiers")
        return v.value

    SEMANTICS = {"exact": 0, "ref-cpu": 1}

    def set_semantics(self, mode: str = "exact") -> None:
        """Pairwise swap deltas as score differences ("exact") or as the
        reference's calculate_swap_delta computes them ("ref-cpu")."""
        if mode not in self.SEMANTICS:
            raise ValueError(f"semantics must be one of {sorted(self.SEMANTICS)}")
        self._chk(self.L.bm_set_semantics(self.h, self.SEMANTICS[mode]), "bm_set_semantics")

    def semantics(self) -> str:
        v = C.c_int32()
        self._chk(self.L.bm_get_semantics(self.h, C.byref(v)), "bm_get_semantics")
        return {i: k for k, i in self.SEMANTICS.items()}[v.value]

    def launch_count(self) -> int:
        return int(self.L.bm_launch_count(self.h))

    def pci_bus_id(self) -> str:
        buf = C.create_string_buffer(64)
        self._chk(self.L.bm_device_pci_bus_id(self.h, buf, 64), "bm_device_pci_bus_id")
        return buf.value.decode()

    def max_active_clusters(self, ctas_per_row: int, threads: int) -> int:
        v = C.c_int32()
        self._chk(self.L.bm_rows_max_active_clusters(self.h, ctas_per_row, threads, C.byref(v)),
                  "bm_rows_max_active_clusters")
        return v.value

    # device utilities
    def dev_alloc(self, nbytes: int) -> int:
        p = C.c_void_p()
        self._chk(self.L.bm_dev_alloc(self.h, nbytes, C.byref(p)), "bm_dev_alloc")
        return p.value

    def dev_free(self, p: int) -> None:
        self._chk(self.L.bm_dev_free(self.h, p), "bm_dev_free")

    def h2d(self, dptr: int, a: np.ndarray) -> None:
        self._chk(self.L.bm_memcpy_h2d(self.h, dptr, _ptr(a), a.nbytes), "bm_memcpy_h2d")

    def d2h(self, a: np.ndarray, dptr: int) -> None:
        self._chk(self.L.bm_memcpy_d2h(self.h, _ptr(a), dptr, a.nbytes), "bm_memcpy_d2h")

    def sync(self) -> None:
        self._chk(self.L.bm_sync(self.h), "bm_sync")

    def l2_flush(self) -> None:
        self._chk(self.L.bm_l2_flush(self.h), "bm_l2_flush")

    def event(self) -> int:
        e = C.c_void_p()
        self._chk(self.L.bm_event_create(self.h, C.byref(e)), "bm_event_create")
        return e.value

    def record(self, ev: int) -> None:
        self._chk(self.L.bm_event_record(self.h, ev), "bm_event_record")

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_float()
        self._chk(self.L.bm_event_elapsed_ms(self.h, a, b, C.byref(ms)), "bm_event_elapsed_ms")
        return ms.value

    def rows_best_dev(self, d_rows: int, d_col: int | None, nrows: int, d_out: int) -> None:
        self._chk(self.L.bm_rows_best_dev(self.h, d_rows, d_col, nrows, d_out), "bm_rows_best_dev")

    def kset_eval_dev(self, k: int, d_sets: int, nsets: int, d_best: int, d_perm: int, d_status: int) -> None:
        self._chk(self.L.bm_kset_eval_dev(self.h, k, d_sets, nsets, d_best, d_perm, d_status), "bm_kset_eval_dev")

    def delta_rows_dev(self, d_rows: int, nrows: int, d_out: int) -> None:
        self._chk(self.L.bm_delta_rows_dev(self.h, d_rows, nrows, d_out), "bm_delta_rows_dev")

    def delta_pairs_dev(self, d_pairs: int, k: int, d_out: int) -> None:
        self._chk(self.L.bm_delta_pairs_dev(self.h, d_pairs, k, d_out), "bm_delta_pairs_dev")


BM_COMM_TCP = 0
BM_COMM_NCCL = 1


class Comm:
    """One rank of a sharded search (bm_comm): TCP sockets around rank 0, or
    NCCL on an Engine's device.  Every method is collective."""

    def __init__(self, kind: int, rank: int, world: int, addr: str | None = None, timeout: float = 60.0,
                 eng: "Engine | None" = None):
        self.L = cuda_lib()
        h = C.c_void_p()
        st = self.L.bm_comm_create(kind, rank, world, addr.encode() if addr else None, timeout,
                                   eng.h if eng is not None else None, C.byref(h))
        if st != BM_OK:
            msg = self.L.bm_ctx_last_error(eng.h).decode() if eng is not None else ""
            raise BMError(st, f"bm_comm_create: {msg}")
        self.h, self.rank, self.world, self.eng = h, rank, world, eng

    def _chk(self, st: int, what: str, ok=(BM_OK,)) -> int:
        if st not in ok:
            raise BMError(st, f"{what}: {self.L.bm_comm_last_error(self.h).decode()}")
        return st

    def barrier(self) -> None:
        self._chk(self.L.bm_comm_barrier(self.h), "bm_comm_barrier")

    def allreduce_sum(self, v: int) -> int:
        t = C.c_int64()
        self._chk(self.L.bm_comm_allreduce_sum(self.h, int(v), C.byref(t)), "bm_comm_allreduce_sum")
        return t.value

    def allgather_swaps(self, pairs, deltas, cap: int):
        p = _i32(np.asarray(pairs).reshape(-1))
        d = np.ascontiguousarray(np.asarray(deltas, np.int64).reshape(-1))
        ap = np.zeros(2 * max(cap, 1), np.int32)
        ad = np.zeros(max(cap, 1), np.int64)
        tot = C.c_int32()
        self._chk(self.L.bm_comm_allgather_swaps(self.h, _ptr(p), _ptr(d), d.shape[0], cap, _ptr(ap), _ptr(ad),
                                                 C.byref(tot)), "bm_comm_allgather_swaps")
        k = tot.value
        return ap[:2 * k].reshape(-1, 2).copy(), ad[:k].copy()

    def island_best(self, score: int, pi):
        q = _i32(pi).copy()
        bs, br = C.c_int64(), C.c_int32()
        self._chk(self.L.bm_comm_island_best(self.h, int(score), _ptr(q), q.shape[0] - 1, C.byref(bs), C.byref(br)),
                  "bm_comm_island_best")
        return bs.value, br.value, q

    def search_sharded(self, rows=None, rows_per_rank=0, max_rounds=-1, time_budget=0.0, prog=None):
        prog = prog or Progress()
        r = None if rows is None else _i32(rows)
        st = self.L.bm_search_sharded(self.eng.h, self.h, None if r is None else _ptr(r),
                                      0 if r is None else r.shape[0], rows_per_rank, max_rounds, time_budget,
                                      C.byref(prog))
        self.eng._chk(st, "bm_search_sharded", ok=(BM_OK, BM_TIMEOUT))
        return prog, st

    def close(self) -> None:
        if self.h:
            self.L.bm_comm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Graph pairs of uneven size for batched annealing chains (bm_batch)."""

    def __init__(self, eng: Engine):
        self.eng = eng
        self.L = eng.L
        h = C.c_void_p()
        eng._chk(self.L.bm_batch_create(eng.h, C.byref(h)), "bm_batch_create")
        self.h = h
        self.ns = []
        eng._children.append(weakref.ref(self))

    def add_pair(self, A: Graph, B: Graph) -> int:
        idx = C.c_int32()
        n = max(A.n, B.n)
        self.eng._chk(self.L.bm_batch_add_pair(self.h, n, A.m, _ptr(A.src), _ptr(A.dst), _ptr(A.w), B.m, _ptr(B.src),
                                               _ptr(B.dst), _ptr(B.w), C.byref(idx)), "bm_batch_add_pair")
        self.ns.append(n)
        return idx.value

    def sa_run(self, chain_pair, keys, init_pis, steps, t0=5.0, t_end=0.01, candidates=0, chunk=0, threads=0):
        """Run chains; init_pis is a list of n+1 arrays.  Returns (final_pis,
        scores, accepts, stats)."""
        cp = _i32(chain_pair)
        k = np.ascontiguousarray(np.asarray(keys, dtype=np.uint64))
        flat = np.ascontiguousarray(np.concatenate([_i32(p) for p in init_pis]))
        out = np.zeros_like(flat)
        nch = cp.shape[0]
        scores = np.zeros(nch, np.int64)
        acc = np.zeros(nch, np.int64)
        prm = SaParams(steps, t0, t_end, candidates, chunk, threads)
        st = SaStats()
        self.eng._chk(self.L.bm_sa_run(self.h, nch, _ptr(cp), _ptr(k), _ptr(flat), C.byref(prm), _ptr(out),
                                       _ptr(scores), _ptr(acc), C.byref(st)), "bm_sa_run")
        pis, o = [], 0
        for c in range(nch):
            n = self.ns[int(cp[c])]
            pis.append(out[o:o + n + 1].copy())
            o += n + 1
        return pis, scores, acc, st

    def close(self):
        if self.h:
            self.L.bm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


MLP_IN = 24
MLP_FEATURES = 12


class Mlp:
    """Learned partner proposals (bm_mlp) bound to an Engine's graphs."""

    def __init__(self, eng: Engine, seed: int = 1):
        self.eng = eng
        self.L = eng.L
        h = C.c_void_p()
        eng._chk(self.L.bm_mlp_create(eng.h, seed, C.byref(h)), "bm_mlp_create")
        self.h = h
        self.n = eng.n
        self.nparams = int(self.L.bm_mlp_num_params())
        eng._children.append(weakref.ref(self))

    def _chk(self, st, what, ok=(BM_OK,)):
        return self.eng._chk(st, what, ok)

    def params(self) -> np.ndarray:
        w = np.zeros(self.nparams, np.float32)
        self._chk(self.L.bm_mlp_get_params(self.h, _ptr(w)), "bm_mlp_get_params")
        return w

    def set_params(self, w) -> None:
        w = np.ascontiguousarray(np.asarray(w, dtype=np.float32))
        assert w.shape == (self.nparams,)
        self._chk(self.L.bm_mlp_set_params(self.h, _ptr(w)), "bm_mlp_set_params")

    def set_backend(self, backend: int) -> None:
        self._chk(self.L.bm_mlp_set_backend(self.h, backend), "bm_mlp_set_backend")

    def refresh_features(self) -> None:
        self._chk(self.L.bm_mlp_refresh_features(self.h), "bm_mlp_refresh_features")

    def features(self) -> np.ndarray:
        t = np.zeros((self.n + 1, MLP_FEATURES), np.float32)
        self._chk(self.L.bm_mlp_get_features(self.h, _ptr(t)), "bm_mlp_get_features")
        return t

    def pair_features(self, pairs) -> np.ndarray:
        p = _i32(pairs).reshape(-1, 2)
        out = np.zeros((p.shape[0], MLP_IN), np.float32)
        self._chk(self.L.bm_mlp_pair_features(self.h, _ptr(p), p.shape[0], _ptr(out)), "bm_mlp_pair_features")
        return out

    def score_pairs(self, pairs) -> np.ndarray:
        p = _i32(pairs).reshape(-1, 2)
        out = np.zeros(p.shape[0], np.float32)
        self._chk(self.L.bm_mlp_score_pairs(self.h, _ptr(p), p.shape[0], _ptr(out)), "bm_mlp_score_pairs")
        return out

    def score_features(self, x) -> np.ndarray:
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float32).reshape(-1, MLP_IN))
        out = np.zeros(x.shape[0], np.float32)
        self._chk(self.L.bm_mlp_score_features(self.h, _ptr(x), x.shape[0], _ptr(out)), "bm_mlp_score_features")
        return out

    def score_rows(self, rows) -> np.ndarray:
        r = _i32(rows)
        out = np.zeros((r.shape[0], self.n), np.float32)
        self._chk(self.L.bm_mlp_score_rows(self.h, _ptr(r), r.shape[0], _ptr(out)), "bm_mlp_score_rows")
        return out

    def score_candidates(self, rows, cands) -> np.ndarray:
        """bm_mlp_score_candidates: scores (nrows x S) of the listed partners."""
        r = _i32(rows).reshape(-1)
        c = _i32(cands).reshape(r.shape[0], -1)
        out = np.zeros(c.shape, np.float32)
        self._chk(self.L.bm_mlp_score_candidates(self.h, _ptr(r), r.shape[0], _ptr(c), c.shape[1], _ptr(out)),
                  "bm_mlp_score_candidates")
        return out

    def score_rows_dev(self, d_rows: int, nrows: int, d_scores: int) -> None:
        self._chk(self.L.bm_mlp_score_rows_dev(self.h, d_rows, nrows, d_scores), "bm_mlp_score_rows_dev")

    def status(self) -> None:
        self._chk(self.L.bm_mlp_status(self.h), "bm_mlp_status")

    def rows_topk(self, rows, K: int = 64):
        r = _i32(rows)
        v = np.zeros((r.shape[0], K), np.int32)
        sc = np.zeros((r.shape[0], K), np.float32)
        self._chk(self.L.bm_mlp_rows_topk(self.h, _ptr(r), r.shape[0], K, _ptr(v), _ptr(sc)), "bm_mlp_rows_topk")
        return v, sc

    def gradients(self, x, y):
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float32).reshape(-1, MLP_IN))
        y = np.ascontiguousarray(np.asarray(y, dtype=np.float32))
        g = np.zeros(self.nparams, np.float32)
        loss = C.c_float()
        self._chk(self.L.bm_mlp_gradients(self.h, _ptr(x), _ptr(y), x.shape[0], _ptr(g), C.byref(loss)),
                  "bm_mlp_gradients")
        return g, loss.value

    def adamw_step(self, x, y, lr=1e-3, weight_decay=0.0) -> float:
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float32).reshape(-1, MLP_IN))
        y = np.ascontiguousarray(np.asarray(y, dtype=np.float32))
        loss = C.c_float()
        self._chk(self.L.bm_mlp_adamw_step(self.h, _ptr(x), _ptr(y), x.shape[0], lr, weight_decay, C.byref(loss)),
                  "bm_mlp_adamw_step")
        return loss.value

    def reserve_records(self, capacity: int) -> None:
        self._chk(self.L.bm_mlp_reserve_records(self.h, capacity), "bm_mlp_reserve_records")

    def collect_rows(self, rows, per_row: int = 64, seed: int = 1) -> int:
        r = _i32(rows)
        nrec = C.c_int64()
        self._chk(self.L.bm_mlp_collect_rows(self.h, _ptr(r), r.shape[0], per_row, seed, C.byref(nrec)),
                  "bm_mlp_collect_rows")
        return nrec.value

    def clear_records(self) -> None:
        self._chk(self.L.bm_mlp_clear_records(self.h), "bm_mlp_clear_records")

    def fit(self, steps: int, batch: int = 4096, lr: float = 1e-3, weight_decay: float = 0.0, seed: int = 1) -> float:
        loss = C.c_float()
        self._chk(self.L.bm_mlp_fit(self.h, steps, batch, lr, weight_decay, seed, C.byref(loss)), "bm_mlp_fit")
        return loss.value

    def search(self, rows=None, topk=64, rows_per_batch=0, refresh_batches=1, uniform=False, exact_fallback=True,
               fallback_accepts=0, train_every=0, train_batch=4096, lr=1e-3, weight_decay=0.0, seed=1,
               max_accepts=-1, max_sweeps=-1, time_budget=0.0, target_score=0, prog=None, stats=None, sample=0):
        """bm_search_learned; returns (status, Progress, LearnedStats)."""
        prm = LearnedParams(topk, rows_per_batch, refresh_batches, int(bool(uniform)), int(bool(exact_fallback)),
                            fallback_accepts, train_every, train_batch, lr, weight_decay, seed, max_accepts,
                            max_sweeps, time_budget, target_score, sample)
        prog = prog or Progress()
        stats = stats or LearnedStats()
        r = None if rows is None else _i32(rows)
        st = self.L.bm_search_learned(self.eng.h, self.h, None if r is None else _ptr(r),
                                      0 if r is None else r.shape[0], C.byref(prm), C.byref(prog), C.byref(stats))
        self._chk(st, "bm_search_learned", ok=(BM_OK, BM_TIMEOUT))
        return st, prog, stats

    def close(self):
        if self.h:
            self.L.bm_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def header_functions(header: str = "bm_cuda.h") -> list[str]:
    """Names of the functions declared in include/<header>."""
    import re
    txt = open(os.path.join(INCLUDE_DIR, header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b(bm_[a-z0-9_]+)\s*\(", txt)
    seen, out = set(), []
    for nme in names:
        if nme not in seen:
            seen.add(nme)
            out.append(nme)
    return out
