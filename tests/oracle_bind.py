"""ctypes binding of the oracle (oracle/liboracle.so) and of the reference's
own functions compiled from its sources (oracle/_ref/libref.so).

Test infrastructure: used by tests, __graft_entry__.smoke() and the CPU
baseline of bench.py only, always as the checker of the engine.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libref.so")
REF_GA_SO = os.path.join(ORACLE_DIR, "_ref", "libref_ga.so")

vp = C.c_void_p
_orc = None
_ref = None
_ref_ga = None


def _p(a):
    return None if a is None else a.ctypes.data


def oracle_lib() -> C.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True, stdout=subprocess.DEVNULL)
        L = C.CDLL(ORACLE_SO)
        L.orc_graph_new.restype = vp
        L.orc_graph_new.argtypes = [C.c_int32, C.c_int64, vp, vp, vp]
        L.orc_graph_free.argtypes = [vp]
        L.orc_graph_free.restype = None
        L.orc_score.restype = C.c_int64
        L.orc_score.argtypes = [vp, vp, vp]
        L.orc_swap_delta.restype = C.c_int64
        L.orc_swap_delta.argtypes = [vp, vp, vp, C.c_int32, C.c_int32]
        L.orc_exact_delta.restype = C.c_int64
        L.orc_exact_delta.argtypes = [vp, vp, vp, C.c_int32, C.c_int32]
        L.orc_serial.restype = C.c_int64
        L.orc_serial.argtypes = [vp, vp, vp, vp, C.c_int32, C.c_int64, C.c_int32, C.POINTER(C.c_int64), vp, vp, vp,
                                 C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.orc_rows_omp.restype = None
        L.orc_rows_omp.argtypes = [vp, vp, vp, vp, C.c_int32, vp, C.c_int32]
        L.orc_pairs.restype = None
        L.orc_pairs.argtypes = [vp, vp, vp, vp, C.c_int64, vp]
        L.orc_sim_sweep.restype = C.c_int64
        L.orc_sim_sweep.argtypes = [vp, vp, vp, vp, vp]
        L.orc_perm_delta.restype = C.c_int64
        L.orc_perm_delta.argtypes = [vp, vp, vp, vp, C.c_int32, vp]
        L.orc_sa_run.restype = C.c_int64
        L.orc_sa_run.argtypes = [vp, vp, vp, C.c_uint64, C.c_int64, C.c_double, C.c_double, C.POINTER(C.c_int64)]
        _orc = L
    return _orc


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_ga_available() -> bool:
    return os.path.exists(REF_GA_SO)


def ref_ga_lib() -> C.CDLL:
    global _ref_ga
    if _ref_ga is None:
        L = C.CDLL(REF_GA_SO)
        L.refga_build.restype = C.c_int
        L.refga_build.argtypes = [C.c_int, C.c_longlong, vp, vp, vp]
        L.refga_free.restype = None
        L.refga_max_node.restype = C.c_int
        L.refga_max_node.argtypes = [C.c_int]
        L.refga_score.restype = C.c_int
        L.refga_score.argtypes = [vp]
        L.refga_sweep.restype = C.c_int
        L.refga_sweep.argtypes = [vp, C.c_int, C.c_char_p, C.c_char_p, C.c_char_p, vp]
        _ref_ga = L
    return _ref_ga


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(REF_SO)
        L.ref_num_nodes.restype = C.c_int
        L.ref_build.restype = C.c_int
        L.ref_build.argtypes = [C.c_int, C.c_int, C.c_longlong, vp, vp, vp]
        L.ref_free.restype = None
        L.ref_score.restype = C.c_int
        L.ref_score.argtypes = [vp]
        L.ref_pairs.restype = None
        L.ref_pairs.argtypes = [vp, vp, C.c_longlong, vp]
        L.ref_serial.restype = C.c_longlong
        L.ref_serial.argtypes = [vp, vp, C.c_int, C.c_longlong, C.c_int, C.c_int, C.POINTER(C.c_longlong), vp, vp, vp,
                                 C.c_longlong, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_rows_omp.restype = None
        L.ref_rows_omp.argtypes = [vp, vp, C.c_int, vp, C.c_int]
        _ref = L
    return _ref


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class Oracle:
    """The CPU restatement over one graph pair (edge arrays as numpy int32)."""

    def __init__(self, n, A, B):
        L = oracle_lib()
        self.L, self.n = L, int(n)
        self._keep = [_i32(x) for x in (*A, *B)]
        a_s, a_d, a_w, b_s, b_d, b_w = self._keep
        self.gm = L.orc_graph_new(self.n, a_s.shape[0], _p(a_s), _p(a_d), _p(a_w))
        self.gf = L.orc_graph_new(self.n, b_s.shape[0], _p(b_s), _p(b_d), _p(b_w))
        if not self.gm or not self.gf:
            raise MemoryError("orc_graph_new failed")

    def close(self):
        if self.gm:
            self.L.orc_graph_free(self.gm)
            self.L.orc_graph_free(self.gf)
            self.gm = self.gf = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def score(self, pi) -> int:
        pi = _i32(pi)
        return int(self.L.orc_score(self.gm, self.gf, _p(pi)))

    def delta(self, pi, u, v) -> int:
        pi = _i32(pi)
        return int(self.L.orc_swap_delta(self.gm, self.gf, _p(pi), int(u), int(v)))

    def exact_delta(self, pi, u, v) -> int:
        pi = _i32(pi).copy()
        return int(self.L.orc_exact_delta(self.gm, self.gf, _p(pi), int(u), int(v)))

    def pairs(self, pi, pairs) -> np.ndarray:
        pi, pairs = _i32(pi), _i32(pairs).reshape(-1)
        out = np.zeros(pairs.shape[0] // 2, np.int64)
        self.L.orc_pairs(self.gm, self.gf, _p(pi), _p(pairs), out.shape[0], _p(out))
        return out

    def rows(self, pi, rows, threads=0) -> np.ndarray:
        pi, rows = _i32(pi), _i32(rows).reshape(-1)
        out = np.zeros((rows.shape[0], self.n + 1), np.int64)
        self.L.orc_rows_omp(self.gm, self.gf, _p(pi), _p(rows), rows.shape[0], _p(out), threads)
        return out

    def sim_sweep(self, pi, rank_m, rank_f):
        """The similarity-filtered pass of the graph-alignment variant;
        returns (pi after the pass, accepts)."""
        pi = _i32(pi).copy()
        rm, rf = _i32(rank_m), _i32(rank_f)
        acc = self.L.orc_sim_sweep(self.gm, self.gf, _p(pi), _p(rm), _p(rf))
        if acc < 0:
            raise MemoryError("orc_sim_sweep failed")
        return pi, int(acc)

    def perm_delta(self, pi, verts, perm) -> int:
        pi, verts, perm = _i32(pi), _i32(verts), _i32(perm)
        return int(self.L.orc_perm_delta(self.gm, self.gf, _p(pi), _p(verts), verts.shape[0], _p(perm)))

    def sa(self, pi, key, steps, t0=5.0, t_end=0.01):
        """Replay of one annealing chain; returns (pi, score, accepts)."""
        pi = _i32(pi).copy()
        score = C.c_int64(self.score(pi))
        acc = self.L.orc_sa_run(self.gm, self.gf, _p(pi), int(key), int(steps), float(t0), float(t_end),
                                C.byref(score))
        return pi, int(score.value), int(acc)

    def serial(self, pi, rows=None, max_accepts=-1, max_sweeps=-1, log_cap=1 << 20):
        """Bounded serial first-improvement loop; returns (pi, score, log, sweeps, converged)."""
        pi = _i32(pi).copy()
        r = None if rows is None else _i32(rows)
        score = C.c_int64(self.score(pi))
        l1 = np.zeros(log_cap, np.int32)
        l2 = np.zeros(log_cap, np.int32)
        ld = np.zeros(log_cap, np.int64)
        sw, cv = C.c_int32(), C.c_int32()
        nrows = self.n if r is None else r.shape[0]
        acc = self.L.orc_serial(self.gm, self.gf, _p(pi), _p(r), nrows, max_accepts, max_sweeps, C.byref(score),
                                _p(l1), _p(l2), _p(ld), log_cap, C.byref(sw), C.byref(cv))
        k = min(acc, log_cap)
        log = np.stack([l1[:k].astype(np.int64), l2[:k].astype(np.int64), ld[:k]], axis=1)
        return pi, int(score.value), log, int(sw.value), int(cv.value)


class Reference:
    """The reference's own functions (oracle/_ref/libref.so), one pair at a time."""

    def __init__(self, n, A, B):
        L = ref_lib()
        if n > L.ref_num_nodes():
            raise ValueError(f"the reference holds at most {L.ref_num_nodes()} vertices")
        self.L, self.n = L, int(n)
        for which, g in ((0, A), (1, B)):
            s, d, w = (_i32(x) for x in g)
            if L.ref_build(which, self.n, s.shape[0], _p(s), _p(d), _p(w)) != 0:
                raise RuntimeError("ref_build failed")

    def close(self):
        self.L.ref_free()

    def score(self, pi) -> int:
        return int(self.L.ref_score(_p(_i32(pi))))

    def pairs(self, pi, pairs) -> np.ndarray:
        pi, pairs = _i32(pi), _i32(pairs).reshape(-1)
        out = np.zeros(pairs.shape[0] // 2, np.int32)
        self.L.ref_pairs(_p(pi), _p(pairs), out.shape[0], _p(out))
        return out.astype(np.int64)

    def rows(self, pi, rows, threads=0) -> np.ndarray:
        pi, rows = _i32(pi), _i32(rows).reshape(-1)
        out = np.zeros((rows.shape[0], self.n + 1), np.int32)
        self.L.ref_rows_omp(_p(pi), _p(rows), rows.shape[0], _p(out), threads)
        return out.astype(np.int64)

    def serial(self, pi, rows=None, max_accepts=-1, max_sweeps=-1, verify=False, log_cap=1 << 20):
        pi = _i32(pi).copy()
        r = None if rows is None else _i32(rows)
        score = C.c_longlong()
        l1 = np.zeros(log_cap, np.int32)
        l2 = np.zeros(log_cap, np.int32)
        ld = np.zeros(log_cap, np.int32)
        sw, cv = C.c_int(), C.c_int()
        nrows = self.n if r is None else r.shape[0]
        acc = self.L.ref_serial(_p(pi), _p(r), nrows, max_accepts, max_sweeps, int(verify), C.byref(score),
                                _p(l1), _p(l2), _p(ld), log_cap, C.byref(sw), C.byref(cv))
        k = min(acc, log_cap)
        log = np.stack([l1[:k].astype(np.int64), l2[:k].astype(np.int64), ld[:k].astype(np.int64)], axis=1)
        return pi, int(score.value), log, int(sw.value), int(cv.value)


MLP_IN = 24


def mlp_oracle(w, x, y=None, rounding=True):
    """FP64 replica of the learned-proposal MLP: (out[k], grads or None, loss).
    w: packed float32 parameters; x: k x 24 float32 features; y: targets."""
    L = oracle_lib()
    L.orc_mlp.restype = C.c_int
    L.orc_mlp.argtypes = [vp, vp, vp, C.c_int64, C.c_int, vp, vp, C.POINTER(C.c_double)]
    w = np.ascontiguousarray(np.asarray(w, dtype=np.float32))
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float32).reshape(-1, MLP_IN))
    k = x.shape[0]
    out = np.zeros(k, np.float64)
    grads = None
    yy = None
    if y is not None:
        yy = np.ascontiguousarray(np.asarray(y, dtype=np.float32))
        grads = np.zeros(w.shape[0], np.float64)
    loss = C.c_double()
    mode = 2 if rounding == 2 else int(bool(rounding))  # 2: also the backward signals in BF16
    st = L.orc_mlp(_p(w), _p(x), _p(yy), k, mode, _p(out), _p(grads), C.byref(loss))
    if st != 0:
        raise MemoryError("orc_mlp failed")
    return out, grads, loss.value


class ReferenceGA:
    """The reference's similarity-filtered variant (src/graph-alignment.c,
    oracle/_ref/libref_ga.so): graphs built by its add_edge, one pass of its
    optimize_mapping.  Its orderings are read from CSV files by the variant."""

    def __init__(self, A, B):
        L = ref_ga_lib()
        self.L = L
        for which, g in ((0, A), (1, B)):
            s, d, w = (_i32(x) for x in g)
            if L.refga_build(which, s.shape[0], _p(s), _p(d), _p(w)) != 0:
                raise RuntimeError("refga_build failed")

    def close(self):
        self.L.refga_free()

    def max_node(self, which: int) -> int:
        return int(self.L.refga_max_node(which))

    def score(self, pi) -> int:
        return int(self.L.refga_score(_p(_i32(pi))))

    def sweep(self, pi, ord_m: str, ord_f: str, out_path: str) -> np.ndarray:
        pi = _i32(pi)
        out = np.zeros_like(pi)
        if self.L.refga_sweep(_p(pi), pi.shape[0], ord_m.encode(), ord_f.encode(), out_path.encode(), _p(out)) != 0:
            raise RuntimeError("refga_sweep failed")
        return out
