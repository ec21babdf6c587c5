"""ctypes binding of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and the CPU-baseline / reference legs of
bench.py use this module, as the checker. The product library never imports
it. Each function follows the reference function named in oracle.cpp.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PATH = os.path.join(_HERE, "liboracle.so")


def build():
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


if not os.path.exists(_PATH):
    build()
_lib = C.CDLL(_PATH)
_vp, _sz = C.c_void_p, C.c_size_t

for name, res, args in [
    ("orc_dot", C.c_float, [_vp, _vp, _sz]),
    ("orc_l2", C.c_float, [_vp, _vp, _sz]),
    ("orc_dot_portable", C.c_float, [_vp, _vp, _sz]),
    ("orc_l2_portable", C.c_float, [_vp, _vp, _sz]),
    ("orc_dot_scalar", C.c_float, [_vp, _vp, _sz]),
    ("orc_l2_scalar", C.c_float, [_vp, _vp, _sz]),
    ("orc_distance", C.c_float, [C.c_int, _vp, _vp, _sz]),
    ("orc_i8_dot", C.c_int64, [_vp, _vp, _sz]),
    ("orc_i8_l2", C.c_int64, [_vp, _vp, _sz]),
    ("orc_sq_encode", None, [_vp, _vp, C.c_float, _sz, _vp]),
    ("orc_sq_distance", C.c_float, [C.c_int, C.c_float, _vp, _vp, _sz]),
    ("orc_prepare_query", C.c_int32, [C.c_int, _vp, _sz, _vp]),
    ("orc_crc32", C.c_uint32, [_vp, _sz]),
    ("orc_have_avx2", C.c_int, []),
    ("orc_splitmix", None, [C.c_uint64, _vp, _sz]),
    ("orc_gaussian", None, [_sz, _sz, _sz, C.c_uint64, _vp, _vp]),
    ("orc_clustered", None, [_sz, _sz, _sz, _sz, C.c_double, C.c_uint64, _vp, _vp]),
    ("orc_index_load", _vp, [_vp, _sz]),
    ("orc_index_free", None, [_vp]),
    ("orc_index_nodes", C.c_uint32, [_vp]),
    ("orc_index_dim", C.c_uint32, [_vp]),
    ("orc_index_metric", C.c_int, [_vp]),
    ("orc_search_batch", None, [_vp, _vp, _sz, _sz, _vp, _sz, _vp, C.c_int, _vp, C.c_uint64, _sz, _vp,
                                _vp, _vp, _vp, _vp, _vp, C.c_int, _sz, C.c_int]),
    ("orc_brute_batch", None, [C.c_int, _vp, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _vp, _vp, _vp, C.c_int]),
    ("orc_brute_filtered", None, [C.c_int, _vp, _vp, _sz, _sz, _vp, _sz, _sz, _vp, C.c_uint64, _sz, C.c_int, _vp,
                                  _vp, _vp, _vp, C.c_int]),
    ("orc_brute_f64", None, [C.c_int, _vp, _sz, _sz, _vp, _sz, _sz, _vp, _vp, C.c_int]),
    ("orc_recall_at_k", C.c_double, [_vp, _vp, _sz, _vp, _vp, _sz, _sz, _sz]),
    ("orc_build", _sz, [_sz, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_int, C.c_int, C.c_int,
                        C.c_uint64, _vp, _vp, _sz, _vp, _sz, C.c_int, C.POINTER(C.POINTER(C.c_uint8))]),
    ("orc_free_bytes", None, [C.POINTER(C.c_uint8)]),
    ("orc_mixture_split", None, [_sz, _sz, _sz, _sz, C.c_double, C.c_uint64, C.c_uint64, _vp, _vp]),
]:
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def dot(a, b):
    a, b = _f32(a), _f32(b)
    return float(np.float32(_lib.orc_dot(_p(a), _p(b), a.size)))


def l2(a, b):
    a, b = _f32(a), _f32(b)
    return float(np.float32(_lib.orc_l2(_p(a), _p(b), a.size)))


def dot_portable(a, b):
    a, b = _f32(a), _f32(b)
    return float(np.float32(_lib.orc_dot_portable(_p(a), _p(b), a.size)))


def l2_portable(a, b):
    a, b = _f32(a), _f32(b)
    return float(np.float32(_lib.orc_l2_portable(_p(a), _p(b), a.size)))


def dot_scalar(a, b):
    a, b = _f32(a), _f32(b)
    return float(np.float32(_lib.orc_dot_scalar(_p(a), _p(b), a.size)))


def l2_scalar(a, b):
    a, b = _f32(a), _f32(b)
    return float(np.float32(_lib.orc_l2_scalar(_p(a), _p(b), a.size)))


def distance(metric: int, a, b) -> np.float32:
    a, b = _f32(a), _f32(b)
    return np.float32(_lib.orc_distance(int(metric), _p(a), _p(b), a.size))


def i8_dot(a, b):
    a, b = np.ascontiguousarray(a, np.int8), np.ascontiguousarray(b, np.int8)
    return int(_lib.orc_i8_dot(_p(a), _p(b), a.size))


def i8_l2(a, b):
    a, b = np.ascontiguousarray(a, np.int8), np.ascontiguousarray(b, np.int8)
    return int(_lib.orc_i8_l2(_p(a), _p(b), a.size))


def sq_encode(x, offset, scale: float):
    x, offset = _f32(x), _f32(offset)
    out = np.zeros(x.size, np.int8)
    _lib.orc_sq_encode(_p(x), _p(offset), C.c_float(scale), x.size, _p(out))
    return out


def prepare_query(metric: int, q):
    q = _f32(q)
    out = np.zeros_like(q)
    st = _lib.orc_prepare_query(int(metric), _p(q), q.size, _p(out))
    return st, out


def crc32(data: bytes) -> int:
    buf = np.frombuffer(data, np.uint8) if data else np.zeros(1, np.uint8)
    return int(_lib.orc_crc32(_p(buf), len(data)))


def splitmix(seed: int, n: int):
    out = np.zeros(n, np.uint64)
    _lib.orc_splitmix(seed, _p(out), n)
    return out


def gaussian(nb, nq, dim, seed):
    base = np.zeros((nb, dim), np.float32)
    q = np.zeros((nq, dim), np.float32)
    _lib.orc_gaussian(nb, nq, dim, seed, _p(base), _p(q))
    return base, q


def clustered(nb, nq, dim, clusters, spread, seed):
    base = np.zeros((nb, dim), np.float32)
    q = np.zeros((nq, dim), np.float32)
    _lib.orc_clustered(nb, nq, dim, clusters, spread, seed, _p(base), _p(q))
    return base, q


def mixture_split(nb, nq, dim, clusters, spread, base_seed, query_seed):
    """Clustered data with the base (and centers) from base_seed and the
    queries on their own stream from query_seed (src/synthetic.rs:102-124 order)."""
    base = np.zeros((nb, dim), np.float32)
    q = np.zeros((nq, dim), np.float32)
    _lib.orc_mixture_split(nb, nq, dim, clusters, spread, base_seed, query_seed, _p(base), _p(q))
    return base, q


def build(base, keys=None, metric=0, m=16, m0=None, ef_construction=200, level_multiplier=None,
          selection=1, extend_candidates=False, keep_pruned=False, seed=0, threads=0, deleted_keys=()):
    """HnswIndex::insert_batch into an empty index, then to_bytes (format v1).
    threads=1 links in id order (the graph of repeated `insert`); otherwise
    the nodes are linked concurrently (0: all cores)."""
    import math

    base = _f32(base)
    n, dim = base.shape
    keys = np.arange(n, dtype=np.uint64) if keys is None else np.ascontiguousarray(keys, np.uint64)
    dk = np.ascontiguousarray(np.asarray(deleted_keys, np.uint64))
    m0 = 2 * m if m0 is None else m0
    ml = 1.0 / math.log(m) if level_multiplier is None else level_multiplier
    out = C.POINTER(C.c_uint8)()
    size = _lib.orc_build(dim, int(metric), m, m0, ef_construction, ml, int(selection), int(extend_candidates),
                          int(keep_pruned), seed, _p(keys), _p(base), n, _p(dk) if dk.size else None, dk.size,
                          int(threads), C.byref(out))
    if size == 0:
        raise ValueError("a row failed validation")
    data = C.string_at(out, size)
    _lib.orc_free_bytes(out)
    return data


class Index:
    """An index file loaded by the oracle (format v1)."""

    def __init__(self, data: bytes):
        self._buf = np.frombuffer(data, np.uint8)
        h = _lib.orc_index_load(_p(self._buf), self._buf.size)
        if not h:
            raise ValueError("oracle could not parse the index file")
        self._h = C.c_void_p(h)
        self.dim = int(_lib.orc_index_dim(self._h))
        self.nodes = int(_lib.orc_index_nodes(self._h))
        self.metric = int(_lib.orc_index_metric(self._h))

    def __del__(self):
        if getattr(self, "_h", None):
            _lib.orc_index_free(self._h)
            self._h = None

    def search(self, queries, k: int, ef: int, *, quantized=False, filter_bits=None, filter_nbits=0,
               filter_stride=0, filter_used=None, ks=None, efs=None, threads=0, stats=False, filter_by_node=False):
        """HnswIndex::search_batch / search_with (src/hnsw/mod.rs:412-536): arrays out."""
        q = _f32(queries).reshape(-1, self.dim)
        nq = q.shape[0]
        ks_a = None if ks is None else np.ascontiguousarray(ks, np.uint64)
        efs_a = None if efs is None else np.ascontiguousarray(efs, np.uint64)
        stride = max(int(ks_a.max()) if ks_a is not None and ks_a.size else k, 1)
        keys = np.zeros((nq, stride), np.uint64)
        dist = np.zeros((nq, stride), np.float32)
        counts = np.zeros(nq, np.uint32)
        status = np.zeros(nq, np.int32)
        st = np.zeros((nq, 4), np.uint64) if stats else None
        fb = None if filter_bits is None else np.ascontiguousarray(filter_bits, np.uint64)
        fu = None if filter_used is None else np.ascontiguousarray(filter_used, np.uint8)
        _lib.orc_search_batch(self._h, _p(q), nq, k, _p(ks_a), ef, _p(efs_a), int(quantized), _p(fb),
                              filter_nbits, filter_stride, _p(fu), _p(keys), _p(dist), _p(counts),
                              _p(status), _p(st), threads, stride, int(filter_by_node))
        if stats:
            return keys, dist, counts, status, st
        return keys, dist, counts, status


def brute(metric: int, base, queries, k: int, keys=None, threads=0):
    """BruteForceIndex::search_batch (src/brute.rs:122-180) over prepared rows."""
    base = _f32(base)
    q = _f32(queries)
    nb, dim = base.shape
    nq = q.shape[0]
    kk = max(k, 1)
    ok = np.zeros((nq, kk), np.uint64)
    od = np.zeros((nq, kk), np.float32)
    oc = np.zeros(nq, np.uint32)
    os_ = np.zeros(nq, np.int32)
    ka = None if keys is None else np.ascontiguousarray(keys, np.uint64)
    _lib.orc_brute_batch(int(metric), _p(base), _p(ka), nb, dim, _p(q), nq, k, _p(ok), _p(od), _p(oc), _p(os_),
                         threads)
    return ok, od, oc, os_


def brute_filtered(metric: int, base, queries, k: int, filter_bits, filter_nbits: int, filter_stride: int = 0,
                   by_row: bool = False, keys=None, threads=0):
    """BruteForceIndex::search_filtered (src/brute.rs:131-160) with a bitmap for the closure."""
    base = _f32(base)
    q = _f32(queries)
    nb, dim = base.shape
    nq = q.shape[0]
    kk = max(k, 1)
    ok = np.zeros((nq, kk), np.uint64)
    od = np.zeros((nq, kk), np.float32)
    oc = np.zeros(nq, np.uint32)
    os_ = np.zeros(nq, np.int32)
    ka = None if keys is None else np.ascontiguousarray(keys, np.uint64)
    fb = np.ascontiguousarray(filter_bits, np.uint64)
    _lib.orc_brute_filtered(int(metric), _p(base), _p(ka), nb, dim, _p(q), nq, k, _p(fb), filter_nbits, filter_stride,
                            int(by_row), _p(ok), _p(od), _p(oc), _p(os_), threads)
    return ok, od, oc, os_


def brute_f64(metric: int, base, queries, k: int, threads=0):
    base = _f32(base)
    q = _f32(queries)
    nb, dim = base.shape
    nq = q.shape[0]
    ok = np.zeros((nq, k), np.uint64)
    od = np.zeros((nq, k), np.float64)
    _lib.orc_brute_f64(int(metric), _p(base), nb, dim, _p(q), nq, k, _p(ok), _p(od), threads)
    return ok, od


def normalize_rows(x):
    """vector::normalized (src/vector.rs:42-45) applied to rows: f64 norm, f32 result."""
    x = _f32(x)
    out = np.empty_like(x)
    for i in range(x.shape[0]):
        st, out[i] = prepare_query(2, x[i])
        if st != 0:
            raise ValueError("row cannot be normalised")
    return out


def recall_at_k(truth_keys, truth_counts, found_keys, found_counts, k: int) -> float:
    tk = np.ascontiguousarray(truth_keys, np.uint64)
    tc = np.ascontiguousarray(truth_counts, np.uint32)
    fk = np.ascontiguousarray(found_keys, np.uint64)
    fc = np.ascontiguousarray(found_counts, np.uint32)
    return float(_lib.orc_recall_at_k(_p(tk), _p(tc), tk.shape[1], _p(fk), _p(fc), fk.shape[1], tc.size, k))
