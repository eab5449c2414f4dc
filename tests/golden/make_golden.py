"""Generates the golden fixtures in this directory.

scan_u32_golden.npz -- inputs and outputs of the reference's own CPU scan,
    cpu_sum_scan (scan/main.cu:11-21), compiled from the reference sources by
    oracle/ref_build.sh into oracle/_ref/libref_scan.so.  Needs that library
    (built in a container that has the reference tree).
tiny.gr -- a 6-vertex weighted graph written byte by byte in the `.gr` v1
    layout that CSRGraph::readFromGR parses (LONESTAR/rt/src/csr_graph.cu:183-226):
    u64 version=1, u64 sizeEdgeTy=4, u64 n, u64 m, u64 outIdx[n] (row END
    offsets), u32 dst[m], u32 pad when m is odd, i32 weights[m].

Run: python tests/golden/make_golden.py
"""
import ctypes as C
import pathlib
import struct

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]


def scan_golden():
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libref_scan.so"))
    fn = getattr(lib, "_Z12cpu_sum_scanPjPKjm")  # cpu_sum_scan(unsigned*, const unsigned*, size_t)
    fn.restype = None
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
    rng = np.random.default_rng(2022)
    cases = {
        "ones_1000": np.ones(1000, dtype=np.uint32),                       # scan/main.cu:37-41
        "u15_4099": rng.integers(0, 16, 4099, dtype=np.uint32),            # the int32 scan run draws values in [0, 15]
        "wrap_777": rng.integers(2**31, 2**32, 777, dtype=np.uint64).astype(np.uint32),  # uint32 wraparound
        "single": np.array([7], dtype=np.uint32),
    }
    out = {}
    for k, a in cases.items():
        o = np.zeros_like(a)
        fn(o.ctypes.data, a.ctypes.data, a.size)
        out[k + "_in"] = a
        out[k + "_out"] = o
    np.savez_compressed(HERE / "scan_u32_golden.npz", **out)


# tiny graph: edges (undirected) with weights
TINY_N = 6
TINY_EDGES = [(0, 1, 7), (0, 2, 9), (0, 5, 14), (1, 2, 10), (1, 3, 15), (2, 3, 11), (2, 5, 2), (3, 4, 6),
              (4, 5, 9)]


def tiny_csr():
    adj = {v: [] for v in range(TINY_N)}
    for u, v, w in TINY_EDGES:
        adj[u].append((v, w))
        adj[v].append((u, w))
    row, dst, wt = [0], [], []
    for v in range(TINY_N):
        for d, w in sorted(adj[v]):
            dst.append(d)
            wt.append(w)
        row.append(len(dst))
    return row, dst, wt


def tiny_gr():
    row, dst, wt = tiny_csr()
    m = len(dst)
    b = struct.pack("<4Q", 1, 4, TINY_N, m)
    b += struct.pack(f"<{TINY_N}Q", *row[1:])
    b += struct.pack(f"<{m}I", *dst)
    if m % 2:
        b += struct.pack("<I", 0)
    b += struct.pack(f"<{m}i", *wt)
    (HERE / "tiny.gr").write_bytes(b)


if __name__ == "__main__":
    scan_golden()
    tiny_gr()
    print("golden fixtures written")
