"""ctypes binding of the CPU oracle (oracle/lib/liboracle.so) -- the checker.

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it."""
import ctypes as C
import pathlib

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
_lib = C.CDLL(str(ROOT / "oracle" / "lib" / "liboracle.so"))
_P = C.c_void_p
_lib.orc_sum_i32.restype = C.c_int64
_lib.orc_sum_i32.argtypes = [_P, C.c_size_t]
_lib.orc_sum_i32_mt.restype = C.c_int64
_lib.orc_sum_i32_mt.argtypes = [_P, C.c_size_t, C.c_int]
_lib.orc_scan_u32.argtypes = [_P, _P, C.c_size_t]
_lib.orc_scan_u32_mt.argtypes = [_P, _P, C.c_size_t, C.c_int]
_lib.orc_scan_f32_f64.argtypes = [_P, _P, C.c_size_t]
_lib.orc_max_rel_err_f32_f64.restype = C.c_double
_lib.orc_max_rel_err_f32_f64.argtypes = [_P, _P, C.c_size_t, C.c_double]
_lib.orc_bfs.argtypes = [C.c_uint32, _P, _P, C.c_uint32, _P]
_lib.orc_dijkstra.argtypes = [C.c_uint32, _P, _P, _P, C.c_uint32, _P]
_lib.orc_pagerank_pull.argtypes = [C.c_uint32, _P, _P, C.c_double, C.c_int, _P]
_lib.orc_pagerank_push.argtypes = [C.c_uint32, _P, _P, C.c_double, C.c_int, _P]
_lib.orc_bfs_mt.argtypes = [C.c_uint32, _P, _P, C.c_uint32, _P, C.c_int]
_lib.orc_pagerank_pull_mt.argtypes = [C.c_uint32, _P, _P, C.c_double, C.c_int, _P, C.c_int]
_lib.orc_normalized_l1.restype = C.c_double
_lib.orc_normalized_l1.argtypes = [_P, _P, C.c_uint32]
_lib.orc_traversed_edges.restype = C.c_uint64
_lib.orc_traversed_edges.argtypes = [C.c_uint32, _P, _P]
_lib.orc_gr_read.restype = C.c_int
_lib.orc_gr_read.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                             C.POINTER(C.POINTER(C.c_uint32)), C.POINTER(C.POINTER(C.c_uint32)),
                             C.POINTER(C.POINTER(C.c_int32))]
_lib.orc_free.argtypes = [_P]
_lib.orc_mlp_forward.argtypes = [_P, _P, C.c_int, _P]
_lib.orc_heterosync_golden.argtypes = [C.c_int] * 7 + [_P, C.c_int]
_lib.orc_heterosync_storage_locs.restype = C.c_int
_lib.orc_heterosync_storage_locs.argtypes = [C.c_int] * 5
_lib.orc_cpu_srb_barrier.restype = C.c_double
_lib.orc_cpu_srb_barrier.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64)]
_lib.orc_cpu_semaphore.restype = C.c_double
_lib.orc_cpu_semaphore.argtypes = [C.c_int] * 5 + [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                                   C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
_lib.orc_cpu_srb_barrier_stalls.restype = C.c_double
_lib.orc_cpu_srb_barrier_stalls.argtypes = [C.c_int] * 4 + [C.c_uint64, C.POINTER(C.c_uint64),
                                                            C.POINTER(C.c_uint64)]
_lib.orc_cpu_srb_barrier_vcta.restype = C.c_double
_lib.orc_cpu_srb_barrier_vcta.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_uint64)]
_lib.orc_cpu_srb_barrier_kill.restype = C.c_double
_lib.orc_cpu_srb_barrier_kill.argtypes = [C.c_int] * 6 + [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
_lib.orc_cpu_semaphore_stalls.restype = C.c_double
_lib.orc_cpu_semaphore_stalls.argtypes = [C.c_int] * 6 + [C.c_uint64, C.POINTER(C.c_uint64),
                                                          C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                                          C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]

INF = 2**31 - 1


def _p(a):
    return a.ctypes.data


def sum_i32(a, threads=1):
    a = np.ascontiguousarray(a, dtype=np.int32)
    if threads > 1:
        return int(_lib.orc_sum_i32_mt(_p(a), a.size, threads))
    return int(_lib.orc_sum_i32(_p(a), a.size))


def scan_u32(a, threads=1):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    out = np.empty_like(a)
    if threads > 1:
        _lib.orc_scan_u32_mt(_p(a), _p(out), a.size, threads)
    else:
        _lib.orc_scan_u32(_p(a), _p(out), a.size)
    return out


_ref_scan = None


def ref_cpu_sum_scan(a):
    """The reference's own cpu_sum_scan (scan/main.cu:11-21), compiled from the
    reference sources into oracle/_ref/libref_scan.so by oracle/ref_build.sh;
    None when that library was not built."""
    global _ref_scan
    if _ref_scan is None:
        path = ROOT / "oracle" / "_ref" / "libref_scan.so"
        if not path.exists():
            return None
        lib = C.CDLL(str(path))
        fn = getattr(lib, "_Z12cpu_sum_scanPjPKjm")  # cpu_sum_scan(unsigned*, const unsigned*, size_t)
        fn.restype = None
        fn.argtypes = [_P, _P, C.c_size_t]
        _ref_scan = fn
    a = np.ascontiguousarray(a, dtype=np.uint32)
    out = np.empty_like(a)
    _ref_scan(_p(out), _p(a), a.size)
    return out


def scan_f32_f64(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    out = np.empty(a.size, dtype=np.float64)
    _lib.orc_scan_f32_f64(_p(a), _p(out), a.size)
    return out


def max_rel_err(gpu, ref, floor=1e-30):
    gpu = np.ascontiguousarray(gpu, dtype=np.float32)
    ref = np.ascontiguousarray(ref, dtype=np.float64)
    return float(_lib.orc_max_rel_err_f32_f64(_p(gpu), _p(ref), gpu.size, floor))


def mlp_forward(params, X):
    """FP64 forward pass of the policy network: X[B][12] -> [B][4]."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    out = np.zeros((X.shape[0], 4), np.float64)
    _lib.orc_mlp_forward(_p(p), _p(X), X.shape[0], _p(out))
    return out


def bfs(g, src=0, threads=1):
    out = np.empty(g.nnodes, dtype=np.int32)
    if threads > 1:
        _lib.orc_bfs_mt(g.nnodes, _p(g.row_start), _p(g.edge_dst), src, _p(out), threads)
    else:
        _lib.orc_bfs(g.nnodes, _p(g.row_start), _p(g.edge_dst), src, _p(out))
    return out


def dijkstra(g, src=0):
    out = np.empty(g.nnodes, dtype=np.int32)
    _lib.orc_dijkstra(g.nnodes, _p(g.row_start), _p(g.edge_dst), _p(g.edge_data), src, _p(out))
    return out


def pagerank(g, alpha=0.85, iters=50, threads=1):
    out = np.empty(g.nnodes, dtype=np.float64)
    if threads > 1:
        _lib.orc_pagerank_pull_mt(g.nnodes, _p(g.row_start), _p(g.edge_dst), alpha, iters, _p(out), threads)
    else:
        _lib.orc_pagerank_pull(g.nnodes, _p(g.row_start), _p(g.edge_dst), alpha, iters, _p(out))
    return out


def pagerank_push(g, alpha=0.85, iters=200):
    """The PageRank fixed point over out-edges, for any graph (see orc_pagerank_push)."""
    out = np.empty(g.nnodes, dtype=np.float64)
    _lib.orc_pagerank_push(g.nnodes, _p(g.row_start), _p(g.edge_dst), alpha, iters, _p(out))
    return out


def normalized_l1(a32, b64):
    a32 = np.ascontiguousarray(a32, dtype=np.float32)
    b64 = np.ascontiguousarray(b64, dtype=np.float64)
    return float(_lib.orc_normalized_l1(_p(a32), _p(b64), a32.size))


def traversed_edges(g, values):
    values = np.ascontiguousarray(values, dtype=np.int32)
    return int(_lib.orc_traversed_edges(g.nnodes, _p(g.row_start), _p(values)))


def gr_read(path):
    n = C.c_uint32()
    m = C.c_uint64()
    row = C.POINTER(C.c_uint32)()
    dst = C.POINTER(C.c_uint32)()
    w = C.POINTER(C.c_int32)()
    rc = _lib.orc_gr_read(str(path).encode(), C.byref(n), C.byref(m), C.byref(row), C.byref(dst), C.byref(w))
    if rc:
        raise IOError(f"orc_gr_read failed {rc}")
    nn, mm = n.value, m.value
    r = np.ctypeslib.as_array(row, shape=(nn + 1,)).copy()
    d = np.ctypeslib.as_array(dst, shape=(max(mm, 1),))[:mm].copy()
    ww = np.ctypeslib.as_array(w, shape=(max(mm, 1),))[:mm].copy()
    for p in (row, dst, w):
        _lib.orc_free(C.cast(p, C.c_void_p))
    return r, d, ww


def heterosync_storage_locs(prim, ldst, ntbs, nsm, tpb):
    return int(_lib.orc_heterosync_storage_locs(prim, ldst, ntbs, nsm, tpb))


def heterosync_golden(prim, ldst, ntbs, iters, repeats, nsm, tpb):
    n = heterosync_storage_locs(prim, ldst, ntbs, nsm, tpb)
    s = np.arange(n, dtype=np.float32)
    _lib.orc_heterosync_golden(prim, ldst, ntbs, iters, repeats, nsm, tpb, _p(s), n)
    return s


def cpu_srb_barrier(nthreads, ngroups, episodes):
    stale = C.c_uint64()
    ns = _lib.orc_cpu_srb_barrier(nthreads, ngroups, episodes, C.byref(stale))
    return float(ns), int(stale.value)


def cpu_srb_barrier_stalls(nthreads, ngroups, episodes, permille, seed):
    stale, stalls = C.c_uint64(), C.c_uint64()
    ns = _lib.orc_cpu_srb_barrier_stalls(nthreads, ngroups, episodes, permille, seed, C.byref(stale),
                                         C.byref(stalls))
    return float(ns), int(stale.value), int(stalls.value)


def cpu_srb_barrier_vcta(nthreads, nctas, ngroups, episodes):
    stale = C.c_uint64()
    ns = _lib.orc_cpu_srb_barrier_vcta(nthreads, nctas, ngroups, episodes, C.byref(stale))
    return float(ns), int(stale.value)


def cpu_srb_barrier_kill(nthreads, ngroups, episodes, kill_id, kill_episode, deadline_ms):
    stale, timeouts = C.c_uint64(), C.c_uint64()
    _lib.orc_cpu_srb_barrier_kill(nthreads, ngroups, episodes, kill_id, kill_episode, deadline_ms,
                                  C.byref(stale), C.byref(timeouts))
    return int(stale.value), int(timeouts.value)


def cpu_semaphore_stalls(nthreads, capacity, writer_every, iters, incs, permille, seed):
    W, R, stalls = C.c_uint64(), C.c_uint64(), C.c_uint64()
    mr, viol = C.c_uint32(), C.c_uint32()
    rate = _lib.orc_cpu_semaphore_stalls(nthreads, capacity, writer_every, iters, incs, permille, seed,
                                         C.byref(W), C.byref(R), C.byref(mr), C.byref(viol), C.byref(stalls))
    return float(rate), int(W.value), int(R.value), int(mr.value), int(viol.value), int(stalls.value)


def cpu_semaphore(nthreads, capacity, writer_every, iters, incs):
    W = C.c_uint64()
    R = C.c_uint64()
    mr = C.c_uint32()
    viol = C.c_uint32()
    rate = _lib.orc_cpu_semaphore(nthreads, capacity, writer_every, iters, incs, C.byref(W), C.byref(R),
                                  C.byref(mr), C.byref(viol))
    return float(rate), int(W.value), int(R.value), int(mr.value), int(viol.value)
