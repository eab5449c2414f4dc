"""ctypes binding of libgsrb (the C ABI declared in include/gsrb.h).

This is the Python face of the library used by the tests and by bench.py.  It
loads the in-tree ``lib/libgsrb.so`` and fails loudly when it is missing: there
is no CPU fallback for any operation.

The Python names mirror the reference entry points where one exists:
``reduce`` (Reduce/reduce.cuh:47), ``sum_scan_blelloch``
(scan/scan.h:16-18), ``cudaLocksInit`` / ``cudaLocksDestroy``
(Heterosync/cudaLocks.h:24-27) and the Lonestar ``gg_main`` applications
(LONESTAR/apps/{bfs,sssp,pr}/kernel_gsrb.cu).
"""
from __future__ import annotations

import ctypes as C
import weakref
import os
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libgsrb.so"

# status codes (include/gsrb.h)
OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_NOT_CORESIDENT = -3
ERR_TIMEOUT = -4
ERR_NOMEM = -5
ERR_STATE = -6
ERR_UNSUPPORTED = -7
ERR_OVERFLOW = -8
ERR_LOCK_TIMEOUT = -9
ERR_INVARIANT = -10

# barrier variants
BAR_CLUSTER = 0
BAR_CLUSTER_ALLPOLL = 1
BAR_DSMEM = 2
BAR_SOFT2 = 3
BAR_FLAT = 4
BAR_TREE = 5
BAR_CCG = 6
BAR_CLUSTER_RED = 7
BAR_FLIP = 8
BAR_FANOUT = 9
BAR_CLUSTER_FANOUT = 10
BAR_HIER = 11
BAR_LOCKFREE = 12
BAR_NONE = 99
FORM_AUTO = 0
FORM_L2 = 1
FORM_L1 = 2
FORM_REG = 3
SSSP_DELTA_LEARNED = 0
VARIANT_NAMES = {
    BAR_CLUSTER: "gsrb_cluster",
    BAR_CLUSTER_ALLPOLL: "gsrb_cluster_allpoll",
    BAR_DSMEM: "gsrb_dsmem",
    BAR_SOFT2: "gsrb_soft2",
    BAR_FLAT: "gcpusrb_flat",
    BAR_TREE: "atomic_tree",
    BAR_CCG: "ccg_grid_sync",
    BAR_CLUSTER_RED: "gsrb_cluster_red",
    BAR_FLIP: "gsrb_flip",
    BAR_FANOUT: "gsrb_fanout",
    BAR_CLUSTER_FANOUT: "gsrb_cluster_fanout",
    BAR_HIER: "gsrb_hier",
    BAR_LOCKFREE: "lockfree_tree",
    BAR_NONE: "none",
}


class GsrbError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = _lib().gsrb_status_string(status).decode() if _LIB is not None else str(status)
        super().__init__(f"{what}: {msg} ({status})" if what else f"{msg} ({status})")


class Cfg(C.Structure):
    _fields_ = [
        ("variant", C.c_int32),
        ("cluster", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("threads", C.c_int32),
        ("fanin_groups", C.c_int32),
        ("spin_ns", C.c_int32),
        ("timeout_ms", C.c_uint32),
        ("tile", C.c_int32),
        ("grid_override", C.c_int32),
        ("launch_mode", C.c_int32),
        ("wake_lines", C.c_int32),
        ("form", C.c_int32),
        ("overlap", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class HostCSR(C.Structure):
    _fields_ = [
        ("nnodes", C.c_uint32),
        ("_pad", C.c_uint32),
        ("nedges", C.c_uint64),
        ("row_start", C.POINTER(C.c_uint32)),
        ("edge_dst", C.POINTER(C.c_uint32)),
        ("edge_data", C.POINTER(C.c_int32)),
    ]


_LIB = None

_P = C.c_void_p
_SIGS = {
    "gsrb_cfg_default": (None, [C.POINTER(Cfg)]),
    "gsrb_status_string": (C.c_char_p, [C.c_int32]),
    "gsrb_ctx_create": (C.c_int32, [C.c_int, C.POINTER(_P)]),
    "gsrb_ctx_destroy": (C.c_int32, [_P]),
    "gsrb_ctx_set_stream": (C.c_int32, [_P, _P]),
    "gsrb_ctx_info": (C.c_int32, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "gsrb_ctx_status": (C.c_int32, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "gsrb_ctx_synchronize": (C.c_int32, [_P]),
    "gsrb_max_coresident": (C.c_int32, [_P, C.POINTER(Cfg), C.c_int32, C.POINTER(C.c_int32)]),
    "gsrb_malloc": (C.c_int32, [C.POINTER(_P), C.c_size_t]),
    "gsrb_free": (C.c_int32, [_P]),
    "gsrb_host_alloc": (C.c_int32, [C.POINTER(_P), C.c_size_t]),
    "gsrb_host_free": (C.c_int32, [_P]),
    "gsrb_memcpy_h2d": (C.c_int32, [_P, _P, _P, C.c_size_t]),
    "gsrb_memcpy_d2h": (C.c_int32, [_P, _P, _P, C.c_size_t]),
    "gsrb_memset": (C.c_int32, [_P, _P, C.c_int, C.c_size_t]),
    "gsrb_event_record": (C.c_int32, [_P, C.c_int32]),
    "gsrb_event_elapsed_ms": (C.c_int32, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_float)]),
    "gsrb_l2_flush": (C.c_int32, [_P]),
    "gsrb_launch_count": (C.c_uint64, []),
    "gsrb_barrier_bench": (C.c_int32, [_P, C.POINTER(Cfg), C.c_int32, C.c_int32, _P, _P]),
    "gsrb_barrier_litmus": (C.c_int32, [_P, C.POINTER(Cfg), C.c_int32, _P, _P]),
    "gsrb_barrier_fault_short_grid": (C.c_int32, [_P, C.POINTER(Cfg)]),
    "gsrb_reduce_i32": (C.c_int32, [_P, _P, C.c_size_t, _P, C.POINTER(Cfg)]),
    "gsrb_probe_l2_atomics": (C.c_int32, [_P, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_float)]),
    "gsrb_host_csr_free": (None, [C.POINTER(HostCSR)]),
    "gsrb_gen_uniform_i32": (C.c_int32, [C.c_uint64, C.c_size_t, C.c_int32, C.c_int32, _P]),
    "gsrb_gen_uniform_f32": (C.c_int32, [C.c_uint64, C.c_size_t, _P]),
    "gsrb_edge_weight": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint64, C.c_int32, C.c_int32]),
    "gsrb_csr_from_edges": (C.c_int32, [C.c_uint32, C.c_uint64, _P, _P, C.c_int, C.c_uint64, C.c_int32,
                                        C.c_int32, C.POINTER(HostCSR)]),
    "gsrb_gen_rmat": (C.c_int32, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                  C.c_int32, C.c_int32, C.POINTER(HostCSR)]),
    "gsrb_gen_grid2d": (C.c_int32, [C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.c_int32,
                                    C.POINTER(HostCSR)]),
    "gsrb_gr_read": (C.c_int32, [C.c_char_p, C.POINTER(HostCSR)]),
    "gsrb_gr_write": (C.c_int32, [C.c_char_p, C.POINTER(HostCSR), C.c_int32]),
    "gsrb_scan_u32": (C.c_int32, [_P, _P, _P, C.c_size_t, C.POINTER(Cfg)]),
    "gsrb_scan_f32": (C.c_int32, [_P, _P, _P, C.c_size_t, C.POINTER(Cfg)]),
    "gsrb_reduce_i32_segments": (C.c_int32, [_P, _P, _P, C.c_int32, _P, C.POINTER(Cfg)]),
    "gsrb_scan_u32_segments": (C.c_int32, [_P, _P, _P, _P, C.c_int32, C.POINTER(Cfg)]),
    "gsrb_scan_f32_segments": (C.c_int32, [_P, _P, _P, _P, C.c_int32, C.POINTER(Cfg)]),
    "gsrb_segments_layout": (C.c_int32, [_P, C.c_int32, C.c_int32, _P, _P]),
    "gsrb_semaphore_bench": (C.c_int32, [_P, C.POINTER(Cfg), C.c_int32, C.c_uint32, C.c_int32, C.c_int32,
                                         C.c_int32, _P]),
    "gsrb_mutex_bench": (C.c_int32, [_P, C.POINTER(Cfg), C.c_int32, C.c_int32, C.c_int32, _P]),
    "gsrb_semaphore_fault_overpost": (C.c_int32, [_P, C.c_uint32, _P]),
    "gsrb_semaphore_fault_writer_timeout": (C.c_int32, [_P, C.c_uint32, _P]),
    "gsrb_graph_upload": (C.c_int32, [_P, C.POINTER(HostCSR), C.POINTER(_P)]),
    "gsrb_graph_free": (C.c_int32, [_P]),
    "gsrb_graph_info": (C.c_int32, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "gsrb_graph_is_symmetric": (C.c_int32, [_P, C.POINTER(C.c_int32)]),
    "gsrb_graph_set_policy": (C.c_int32, [_P, _P, C.c_size_t]),
    "gsrb_graph_set_sssp_policy": (C.c_int32, [_P, _P, C.c_size_t]),
    "gsrb_probe_gather": (C.c_int32, [_P, _P, C.c_int32, C.POINTER(C.c_float)]),
    "gsrb_graph_sssp_plan": (C.c_int32, [_P, C.c_uint32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _P]),
    "gsrb_graph_sssp_features": (C.c_int32, [_P, C.c_uint32, _P]),
    "gsrb_sssp_features": (None, [C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_double, C.c_int32,
                                  C.c_int32, C.c_int32, _P]),
    "gsrb_graph_set_launch_choices": (C.c_int32, [_P, C.POINTER(Cfg), C.POINTER(Cfg)]),
    "gsrb_graph_policy_launch": (C.c_int32, [_P, C.c_uint32, C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "gsrb_graph_trace": (C.c_int32, [_P, _P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "gsrb_bfs": (C.c_int32, [_P, _P, C.c_uint32, _P, C.c_int32, C.POINTER(Cfg), C.c_void_p]),
    "gsrb_sssp": (C.c_int32, [_P, _P, C.c_uint32, _P, C.c_int32, C.POINTER(Cfg), C.c_void_p]),
    "gsrb_pagerank": (C.c_int32, [_P, _P, C.c_float, C.c_int32, _P, C.POINTER(Cfg), C.c_void_p]),
    "gsrb_pagerank_residual": (C.c_int32, [_P, _P, C.c_float, C.c_float, C.c_int32, _P, C.POINTER(Cfg), C.c_void_p]),
    "gsrb_batch_create": (C.c_int32, [_P, _P, C.c_int32, C.POINTER(Cfg), C.POINTER(_P)]),
    "gsrb_batch_free": (C.c_int32, [_P]),
    "gsrb_batch_layout": (C.c_int32, [_P, _P, _P]),
    "gsrb_batch_bfs": (C.c_int32, [_P, _P, _P, C.c_int32]),
    "gsrb_batch_sssp": (C.c_int32, [_P, _P, _P, C.c_int32]),
    "gsrb_batch_stats": (C.c_int32, [_P, _P]),
    "gsrb_capture_begin": (C.c_int32, [_P]),
    "gsrb_capture_end": (C.c_int32, [_P, C.POINTER(_P)]),
    "gsrb_exec_launch": (C.c_int32, [_P, _P]),
    "gsrb_exec_free": (C.c_int32, [_P]),
    "gsrb_mlp_param_count": (C.c_size_t, []),
    "gsrb_mlp_init": (C.c_int32, [C.c_uint64, _P]),
    "gsrb_level_features": (None, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint32,
                                   C.c_uint64, C.c_uint32, C.c_uint32, _P]),
    "gsrb_mlp_forward": (C.c_int32, [_P, _P, _P, C.c_int32, _P]),
    "gsrb_mlp_loss_grad": (C.c_int32, [_P, _P, _P, _P, _P, C.c_int32, _P, _P]),
    "gsrb_mlp_train": (C.c_int32, [_P, _P, _P, _P, _P, C.c_int32, C.c_int32, C.c_float, _P]),
}

# semaphore / mutex kinds, BFS modes
SEM_REF_SPIN, SEM_REF_EBO, SEM_REF_PRIORITY, SEM_REF_PRIORITY_EBO, SEM_PRIORITY, SEM_NONE = range(6)
MUTEX_SPIN, MUTEX_EBO, MUTEX_FA, MUTEX_SLEEP = range(4)
BFS_PUSH, BFS_HEURISTIC, BFS_LEARNED, BFS_PULL, BFS_TOPO = range(5)
BFS_FLAG_LB = 0x100  # OR-ed into a mode: load-balanced expansion of large push levels


class TraversalStats(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("aux", C.c_uint32), ("decisions", C.c_uint32),
                ("trace_records", C.c_uint32), ("edges", C.c_uint64), ("kernel_ms", C.c_float),
                ("launch", C.c_uint32), ("delta", C.c_int32)]


TRACE_DTYPE = np.dtype([("level", "<u4"), ("dir", "<u4"), ("nf", "<u4"), ("nu", "<u4"), ("mf", "<u8"),
                        ("mu", "<u8"), ("t_ns", "<u8"), ("pred", "<f4"), ("fallback", "<u4")])
assert TRACE_DTYPE.itemsize == 48


def _lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"libgsrb.so not built ({LIB_PATH}); run `make -C tpds22-artifact_b200` "
                "or __graft_entry__.build() -- there is no CPU fallback")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def register(name, restype, argtypes):
    """Declare an additional entry point's signature (used by later modules)."""
    _SIGS[name] = (restype, argtypes)
    if _LIB is not None:
        fn = getattr(_LIB, name)
        fn.restype = restype
        fn.argtypes = argtypes


class _Checked:
    """Exposes only entry points with a declared signature: calling a C function
    through ctypes without argtypes would silently truncate 64-bit pointers."""

    def __init__(self, raw):
        self._raw = raw

    def __getattr__(self, name):
        if name not in _SIGS:
            raise AttributeError(f"{name}: no ctypes signature declared in gsrb.py")
        return getattr(self._raw, name)


def lib():
    return _Checked(_lib())


def check(st: int, what: str = ""):
    if st != OK:
        raise GsrbError(st, what)


def cfg(**kw) -> Cfg:
    c = Cfg()
    _lib().gsrb_cfg_default(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class ElementRef:
    """A device address inside a DeviceArray (not an allocation of its own)."""

    def __init__(self, ptr: int, dtype):
        self.ptr, self.dtype = ptr, np.dtype(dtype)


class DeviceArray:
    """A device allocation with a numpy dtype and shape (plumbing only)."""

    def __init__(self, ctx: "Context", shape, dtype):
        self.ctx = ctx
        self.dtype = np.dtype(dtype)
        self.shape = (shape,) if np.isscalar(shape) else tuple(shape)
        self.size = int(np.prod(self.shape)) if self.shape else 1
        self.nbytes = self.size * self.dtype.itemsize
        p = C.c_void_p()
        check(_lib().gsrb_malloc(C.byref(p), max(self.nbytes, 1)), "gsrb_malloc")
        self.ptr = p.value

    def upload(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        assert a.nbytes <= self.nbytes
        check(_lib().gsrb_memcpy_h2d(self.ctx.h, self.ptr, _ptr(a), a.nbytes), "h2d")
        self.ctx.sync()
        return self

    def download(self, n=None) -> np.ndarray:
        n = self.size if n is None else n
        out = np.empty(n, dtype=self.dtype)
        check(_lib().gsrb_memcpy_d2h(self.ctx.h, _ptr(out), self.ptr, out.nbytes), "d2h")
        self.ctx.sync()
        return out

    def zero(self):
        check(_lib().gsrb_memset(self.ctx.h, self.ptr, 0, self.nbytes), "memset")
        return self

    def at(self, i: int) -> "ElementRef":
        """The device address of element i (for entry points that take a pointer)."""
        assert 0 <= i < self.size
        return ElementRef(self.ptr + i * self.dtype.itemsize, self.dtype)

    def free(self):
        if self.ptr:
            _lib().gsrb_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """One device context (stream, barrier state, scratch)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(_lib().gsrb_ctx_create(device, C.byref(h)), "gsrb_ctx_create")
        self.h = h.value
        n = C.c_int32()
        l2 = C.c_int64()
        d = C.c_int32()
        check(_lib().gsrb_ctx_info(self.h, C.byref(n), C.byref(l2), C.byref(d)))
        self.num_sms = n.value
        self.l2_bytes = l2.value
        self.device = d.value
        # graphs and batches refer to the context's stream: they are released
        # before the context (gsrb_graph_free / gsrb_batch_free need it alive)
        self._owned = weakref.WeakSet()

    def close(self):
        if self.h:
            for obj in [o for o in self._owned if isinstance(o, Batch)]:
                obj.free()
            for obj in list(self._owned):
                obj.free()
            _lib().gsrb_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- plumbing ---------------------------------------------------------
    def array(self, shape, dtype) -> DeviceArray:
        return DeviceArray(self, shape, dtype)

    def to_device(self, a: np.ndarray) -> DeviceArray:
        d = DeviceArray(self, a.shape, a.dtype)
        return d.upload(a)

    def sync(self):
        check(_lib().gsrb_ctx_synchronize(self.h), "synchronize")

    def status(self):
        code = C.c_uint32()
        where = C.c_uint32()
        who = C.c_uint32()
        st = _lib().gsrb_ctx_status(self.h, C.byref(code), C.byref(where), C.byref(who))
        return st, code.value, where.value, who.value

    def check_status(self, what=""):
        st, code, where, who = self.status()
        if st != OK:
            raise GsrbError(st, f"{what} (device code {code}, episode {where}, block {who})")

    def record(self, slot: int):
        check(_lib().gsrb_event_record(self.h, slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_float()
        check(_lib().gsrb_event_elapsed_ms(self.h, a, b, C.byref(ms)))
        return ms.value

    def l2_flush(self):
        check(_lib().gsrb_l2_flush(self.h), "l2_flush")

    def max_coresident(self, c: Cfg, family: int) -> int:
        n = C.c_int32()
        st = _lib().gsrb_max_coresident(self.h, C.byref(c), family, C.byref(n))
        check(st, "max_coresident")
        return n.value

    # -- barrier ------------------------------------------------------------
    def barrier_bench(self, c: Cfg, episodes: int, fma: int, sink: DeviceArray, count: DeviceArray) -> int:
        return _lib().gsrb_barrier_bench(self.h, C.byref(c), episodes, fma, sink.ptr, count.ptr)

    def barrier_litmus(self, c: Cfg, episodes: int, buf: DeviceArray, stale: DeviceArray) -> int:
        return _lib().gsrb_barrier_litmus(self.h, C.byref(c), episodes, buf.ptr, stale.ptr)

    def barrier_fault_short_grid(self, c: Cfg) -> int:
        return _lib().gsrb_barrier_fault_short_grid(self.h, C.byref(c))

    def probe_l2_atomics(self, ctas: int, iters: int, mode: int) -> float:
        ms = C.c_float()
        check(_lib().gsrb_probe_l2_atomics(self.h, ctas, iters, mode, C.byref(ms)), "probe")
        return ms.value

    # -- reduce ----------------------------------------------------------------
    def reduce_i32(self, d_in: DeviceArray, n: int, d_out: DeviceArray, c: Cfg | None = None) -> int:
        return _lib().gsrb_reduce_i32(self.h, d_in.ptr, n, d_out.ptr, C.byref(c) if c is not None else None)


    # -- scan ------------------------------------------------------------------
    def scan(self, d_in: DeviceArray, d_out: DeviceArray, n: int, c: Cfg | None = None) -> int:
        fn = _lib().gsrb_scan_f32 if d_in.dtype == np.float32 else _lib().gsrb_scan_u32
        return fn(self.h, d_in.ptr, d_out.ptr, n, C.byref(c) if c is not None else None)

    # -- batched segments ----------------------------------------------------------
    def reduce_i32_segments(self, d_in: DeviceArray, offsets, d_out: DeviceArray, c: Cfg | None = None) -> int:
        """int64 sums of the segments [offsets[i], offsets[i+1]) of d_in, one launch."""
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        return _lib().gsrb_reduce_i32_segments(self.h, d_in.ptr, off.ctypes.data, len(off) - 1, d_out.ptr,
                                               C.byref(c) if c is not None else None)

    def scan_u32_segments(self, d_in: DeviceArray, d_out: DeviceArray, offsets, c: Cfg | None = None) -> int:
        """Exclusive prefix sums within each segment, one launch (uint32, or
        FP32 when d_in is float32)."""
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        fn = _lib().gsrb_scan_f32_segments if d_in.dtype == np.float32 else _lib().gsrb_scan_u32_segments
        return fn(self.h, d_in.ptr, d_out.ptr, off.ctypes.data, len(off) - 1, C.byref(c) if c is not None else None)

    scan_segments = scan_u32_segments

    # -- locks ------------------------------------------------------------------
    def semaphore_bench(self, c: Cfg, kind: int, capacity: int, writer_every: int, iters: int, incs: int,
                        counters: DeviceArray) -> int:
        return _lib().gsrb_semaphore_bench(self.h, C.byref(c), kind, capacity, writer_every, iters, incs,
                                           counters.ptr)

    def semaphore_fault_overpost(self, capacity: int, out: DeviceArray) -> int:
        return _lib().gsrb_semaphore_fault_overpost(self.h, capacity, out.ptr)

    def semaphore_fault_writer_timeout(self, capacity: int, out: DeviceArray) -> int:
        return _lib().gsrb_semaphore_fault_writer_timeout(self.h, capacity, out.ptr)

    def mutex_bench(self, c: Cfg, kind: int, iters: int, incs: int, counters: DeviceArray) -> int:
        return _lib().gsrb_mutex_bench(self.h, C.byref(c), kind, iters, incs, counters.ptr)

    # -- graphs -----------------------------------------------------------------
    def graph(self, g: "Graph") -> "DeviceGraph":
        return DeviceGraph(self, g)


class DeviceGraph:
    """A graph resident on the device with its traversal scratch."""

    def __init__(self, ctx: Context, g: "Graph"):
        self.ctx = ctx
        self.host = g
        h = g._as_host()
        p = C.c_void_p()
        check(_lib().gsrb_graph_upload(ctx.h, C.byref(h), C.byref(p)), "graph_upload")
        self.h = p.value
        ctx._owned.add(self)
        self.n = g.nnodes
        self.m = g.nedges

    def free(self):
        if self.h:
            _lib().gsrb_graph_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @property
    def symmetric(self) -> bool:
        v = C.c_int32()
        check(_lib().gsrb_graph_is_symmetric(self.h, C.byref(v)), "graph_is_symmetric")
        return bool(v.value)

    def set_policy(self, weights: np.ndarray):
        w = np.ascontiguousarray(weights, dtype=np.float32)
        check(_lib().gsrb_graph_set_policy(self.h, w.ctypes.data, w.size), "set_policy")

    def set_launch_choices(self, c0: Cfg | None, c1: Cfg | None):
        """The two launch configurations head 3 of the policy chooses between
        for learned traversals run without a cfg (None, None: forget them)."""
        check(_lib().gsrb_graph_set_launch_choices(self.h, C.byref(c0) if c0 is not None else None,
                                                   C.byref(c1) if c1 is not None else None), "set_launch_choices")

    def set_sssp_policy(self, weights: np.ndarray | None):
        """Weights of the SSSP policy (None: forget it); gsrb_sssp with delta
        SSSP_DELTA_LEARNED then runs the width (and launch) it plans."""
        if weights is None:
            check(_lib().gsrb_graph_set_sssp_policy(self.h, None, 0), "set_sssp_policy")
            return
        w = np.ascontiguousarray(weights, dtype=np.float32)
        check(_lib().gsrb_graph_set_sssp_policy(self.h, w.ctypes.data, w.size), "set_sssp_policy")

    def sssp_plan(self, src: int = 0):
        """(bucket width, launch choice, head 2, head 3) of the SSSP policy for a traversal from src."""
        d, k = C.c_int32(), C.c_int32()
        sc = np.zeros(2, np.float32)
        check(_lib().gsrb_graph_sssp_plan(self.h, src, C.byref(d), C.byref(k), sc.ctypes.data), "sssp_plan")
        return int(d.value), int(k.value), float(sc[0]), float(sc[1])

    def probe_gather(self, l1: bool = True) -> float:
        """ms of one edge-parallel pass gathering an FP32 value per edge (the
        pull PageRank's gather floor on this graph)."""
        t = C.c_float()
        check(_lib().gsrb_probe_gather(self.ctx.h, self.h, 1 if l1 else 0, C.byref(t)), "probe_gather")
        return float(t.value)

    def sssp_features(self, src: int = 0) -> np.ndarray:
        out = np.zeros(12, np.float32)
        check(_lib().gsrb_graph_sssp_features(self.h, src, out.ctypes.data), "sssp_features")
        return out

    def policy_launch(self, src: int = 0):
        """(choice, head 3) of the policy for a BFS from src."""
        k, z = C.c_int32(), C.c_float()
        check(_lib().gsrb_graph_policy_launch(self.h, src, C.byref(k), C.byref(z)), "policy_launch")
        return int(k.value), float(z.value)

    def trace(self, max_records=1 << 16) -> np.ndarray:
        out = np.zeros(max_records, dtype=TRACE_DTYPE)
        r = C.c_uint32()
        check(_lib().gsrb_graph_trace(self.h, out.ctypes.data, max_records, C.byref(r)), "trace")
        return out[:r.value]

    def bfs(self, src: int, out: DeviceArray, mode: int = BFS_HEURISTIC, c: Cfg | None = None):
        st = TraversalStats()
        rc = _lib().gsrb_bfs(self.ctx.h, self.h, src, out.ptr, mode, C.byref(c) if c is not None else None,
                             C.addressof(st))
        return rc, st

    def sssp(self, src: int, out: DeviceArray, delta: int, c: Cfg | None = None):
        st = TraversalStats()
        rc = _lib().gsrb_sssp(self.ctx.h, self.h, src, out.ptr, delta, C.byref(c) if c is not None else None,
                              C.addressof(st))
        return rc, st

    def pagerank(self, out: DeviceArray, alpha: float = 0.85, iters: int = 50, c: Cfg | None = None):
        st = TraversalStats()
        rc = _lib().gsrb_pagerank(self.ctx.h, self.h, alpha, iters, out.ptr,
                                  C.byref(c) if c is not None else None, C.addressof(st))
        return rc, st

    def pagerank_residual(self, out: DeviceArray, alpha: float = 0.85, epsilon: float = 1e-6,
                          max_iters: int = 2**31 - 1, c: Cfg | None = None):
        st = TraversalStats()
        rc = _lib().gsrb_pagerank_residual(self.ctx.h, self.h, alpha, epsilon, max_iters, out.ptr,
                                           C.byref(c) if c is not None else None, C.addressof(st))
        return rc, st


def launch_count() -> int:
    return int(_lib().gsrb_launch_count())


# ---- batches and CUDA graphs -----------------------------------------------------
class Batch:
    """Many device graphs traversed in one persistent launch (sub-grid barriers)."""

    def __init__(self, ctx: Context, graphs, c: Cfg | None = None):
        self.ctx = ctx
        self.graphs = list(graphs)
        hs = (C.c_void_p * len(self.graphs))(*[g.h for g in self.graphs])
        self._hs = hs
        p = C.c_void_p()
        check(_lib().gsrb_batch_create(ctx.h, hs, len(self.graphs), C.byref(c) if c is not None else None,
                                       C.byref(p)), "batch_create")
        self.h = p.value
        ctx._owned.add(self)
        self.k = len(self.graphs)

    def free(self):
        if self.h:
            _lib().gsrb_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def layout(self):
        f = np.zeros(self.k, np.uint32)
        n = np.zeros(self.k, np.uint32)
        check(_lib().gsrb_batch_layout(self.h, f.ctypes.data, n.ctypes.data))
        return f, n

    def _ptrs(self, srcs, outs):
        s = np.ascontiguousarray(srcs, dtype=np.uint32)
        o = (C.c_void_p * self.k)(*[a.ptr for a in outs])
        self._keep = (s, o)
        return s, o

    def bfs(self, srcs, outs, mode=BFS_HEURISTIC) -> int:
        s, o = self._ptrs(srcs, outs)
        return _lib().gsrb_batch_bfs(self.h, s.ctypes.data, o, mode)

    def sssp(self, srcs, outs, delta) -> int:
        s, o = self._ptrs(srcs, outs)
        return _lib().gsrb_batch_sssp(self.h, s.ctypes.data, o, delta)

    def stats(self):
        st = (TraversalStats * self.k)()
        rc = _lib().gsrb_batch_stats(self.h, st)
        return rc, list(st)


class CudaGraph:
    """Capture asynchronous library calls on the context stream; replay them."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.h = None

    def __enter__(self):
        check(_lib().gsrb_capture_begin(self.ctx.h), "capture_begin")
        return self

    def __exit__(self, et, ev, tb):
        p = C.c_void_p()
        rc = _lib().gsrb_capture_end(self.ctx.h, C.byref(p))
        if et is None:
            check(rc, "capture_end")
            self.h = p.value

    def launch(self):
        check(_lib().gsrb_exec_launch(self.ctx.h, self.h), "exec_launch")

    def free(self):
        if self.h:
            _lib().gsrb_exec_free(self.h)
            self.h = None


# ---- the learned policy --------------------------------------------------------
def mlp_param_count() -> int:
    return int(_lib().gsrb_mlp_param_count())


def mlp_init(seed: int) -> np.ndarray:
    p = np.zeros(mlp_param_count(), dtype=np.float32)
    check(_lib().gsrb_mlp_init(seed, p.ctypes.data), "mlp_init")
    return p


def segments_layout(offsets, grid: int):
    """(first, count) CTAs of each segment for a batched segment launch of `grid` CTAs."""
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    k = len(off) - 1
    first = np.zeros(max(k, 1), np.uint32)
    count = np.zeros(max(k, 1), np.uint32)
    check(_lib().gsrb_segments_layout(off.ctypes.data, k, grid, first.ctypes.data, count.ctypes.data),
          "segments_layout")
    return first[:k], count[:k]


def level_features(n, m, level, nf, mf, nu, mu, prev_nf, prev_dir) -> np.ndarray:
    out = np.zeros(12, dtype=np.float32)
    _lib().gsrb_level_features(n, m, level, nf, mf, nu, mu, prev_nf, prev_dir, out.ctypes.data)
    return out


def mlp_forward(ctx: Context, params: np.ndarray, X: np.ndarray) -> np.ndarray:
    X = np.ascontiguousarray(X, dtype=np.float32)
    B = X.shape[0]
    dp, dx, do = ctx.to_device(params), ctx.to_device(X), ctx.array(B * 4, np.float32)
    check(_lib().gsrb_mlp_forward(ctx.h, dp.ptr, dx.ptr, B, do.ptr), "mlp_forward")
    return do.download().reshape(B, 4)


def mlp_loss_grad(ctx: Context, params, X, Y, M):
    X, Y, M = (np.ascontiguousarray(a, dtype=np.float32) for a in (X, Y, M))
    B = X.shape[0]
    dp, dx, dy, dm = (ctx.to_device(a) for a in (params, X, Y, M))
    dg, dl = ctx.array(mlp_param_count(), np.float32), ctx.array(1, np.float32)
    check(_lib().gsrb_mlp_loss_grad(ctx.h, dp.ptr, dx.ptr, dy.ptr, dm.ptr, B, dg.ptr, dl.ptr), "mlp_loss_grad")
    return dg.download(), float(dl.download()[0])


def mlp_train(ctx: Context, params, X, Y, M, steps=2000, lr=3e-3):
    X, Y, M = (np.ascontiguousarray(a, dtype=np.float32) for a in (X, Y, M))
    B = X.shape[0]
    dp = ctx.to_device(np.ascontiguousarray(params, dtype=np.float32))
    dx, dy, dm = (ctx.to_device(a) for a in (X, Y, M))
    dh = ctx.array(max(steps, 1), np.float32)
    check(_lib().gsrb_mlp_train(ctx.h, dp.ptr, dx.ptr, dy.ptr, dm.ptr, B, steps, lr, dh.ptr), "mlp_train")
    ctx.check_status("mlp_train")
    return dp.download(), dh.download()[:steps]


# ---- host-side inputs -------------------------------------------------------
def uniform_i32(seed: int, n: int, lo: int, hi: int) -> np.ndarray:
    out = np.empty(n, dtype=np.int32)
    check(_lib().gsrb_gen_uniform_i32(seed, n, lo, hi, _ptr(out)), "gen_uniform_i32")
    return out


def uniform_f32(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.float32)
    check(_lib().gsrb_gen_uniform_f32(seed, n, _ptr(out)), "gen_uniform_f32")
    return out


class Graph:
    """Host CSR graph (numpy copies of the library-owned arrays)."""

    def __init__(self, row_start: np.ndarray, edge_dst: np.ndarray, edge_data: np.ndarray):
        self.row_start = np.ascontiguousarray(row_start, dtype=np.uint32)
        self.edge_dst = np.ascontiguousarray(edge_dst, dtype=np.uint32)
        self.edge_data = np.ascontiguousarray(edge_data, dtype=np.int32)
        self.nnodes = len(self.row_start) - 1
        self.nedges = len(self.edge_dst)

    @staticmethod
    def _from_host(h: HostCSR) -> "Graph":
        n, m = h.nnodes, h.nedges
        row = np.ctypeslib.as_array(h.row_start, shape=(n + 1,)).copy()
        dst = np.ctypeslib.as_array(h.edge_dst, shape=(max(m, 1),))[:m].copy()
        w = np.ctypeslib.as_array(h.edge_data, shape=(max(m, 1),))[:m].copy()
        _lib().gsrb_host_csr_free(C.byref(h))
        return Graph(row, dst, w)

    def _as_host(self) -> HostCSR:
        h = HostCSR()
        h.nnodes = self.nnodes
        h.nedges = self.nedges
        h.row_start = self.row_start.ctypes.data_as(C.POINTER(C.c_uint32))
        h.edge_dst = self.edge_dst.ctypes.data_as(C.POINTER(C.c_uint32))
        h.edge_data = self.edge_data.ctypes.data_as(C.POINTER(C.c_int32))
        return h

    def degrees(self) -> np.ndarray:
        return np.diff(self.row_start.astype(np.int64))

    def write_gr(self, path, with_weights=True):
        h = self._as_host()
        check(_lib().gsrb_gr_write(os.fsencode(str(path)), C.byref(h), 1 if with_weights else 0), "gr_write")

    @staticmethod
    def read_gr(path) -> "Graph":
        h = HostCSR()
        check(_lib().gsrb_gr_read(os.fsencode(str(path)), C.byref(h)), "gr_read")
        return Graph._from_host(h)


def rmat(scale: int, edgefactor: int = 16, a=0.57, b=0.19, c=0.19, seed=0x5EED2022, wlo=1, whi=255) -> Graph:
    h = HostCSR()
    check(_lib().gsrb_gen_rmat(scale, edgefactor, a, b, c, seed, wlo, whi, C.byref(h)), "gen_rmat")
    return Graph._from_host(h)


def grid2d(width: int, height: int, seed=0x5EED2022, wlo=1, whi=1000) -> Graph:
    h = HostCSR()
    check(_lib().gsrb_gen_grid2d(width, height, seed, wlo, whi, C.byref(h)), "gen_grid2d")
    return Graph._from_host(h)


def csr_from_edges(n: int, src, dst, symmetrize=True, weight_seed=1, wlo=1, whi=255) -> Graph:
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    h = HostCSR()
    check(_lib().gsrb_csr_from_edges(n, len(src), _ptr(src), _ptr(dst), 1 if symmetrize else 0, weight_seed,
                                     wlo, whi, C.byref(h)), "csr_from_edges")
    return Graph._from_host(h)


def edge_weight(u: int, v: int, seed: int, lo: int, hi: int) -> int:
    return int(_lib().gsrb_edge_weight(u, v, seed, lo, hi))
