"""Python mirror of the hnsw-index crate's query API over the C ABI.

The classes below keep the reference's names, argument meanings and error
behaviour (src/lib.rs:56-61): ``HnswIndex.search`` / ``search_filtered`` /
``search_with`` / ``search_batch`` (src/hnsw/mod.rs:412-536),
``SearchOptions`` (mod.rs:56-98), ``BruteForceIndex`` (src/brute.rs),
``Neighbor`` (src/neighbor.rs), ``Metric``, ``HnswParams`` and the
``Error`` / ``FormatError`` kinds (src/error.rs). Every search runs in
``libhnsw_gpu.so`` on the GPU; there is no CPU search path in this module, and
importing it fails loudly if the library is missing.

``IndexBuilder`` wraps the host-side construction (``HnswIndex::new`` /
``insert`` / ``insert_batch`` / ``remove`` / ``enable_quantization`` /
``to_bytes``), which produces the format-v1 files the device path opens.
"""

from __future__ import annotations

import ctypes as C
import enum
import os
from dataclasses import dataclass
from typing import Callable, NamedTuple, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# HNSW_GPU_LIB=checked loads the checked build (bounds checks in the
# traversal kernels, libhnsw_gpu_checked.so from `make -C <package> checked`).
_LIB_NAME = "libhnsw_gpu_checked.so" if os.environ.get("HNSW_GPU_LIB") == "checked" else "libhnsw_gpu.so"
_LIB_PATH = os.path.join(_HERE, _LIB_NAME)
if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"{_LIB_PATH} is missing: build it with `make -C {_HERE}` "
        "(the device path has no fallback)"
    )
_lib = C.CDLL(_LIB_PATH)

MAX_DIM = 1 << 16
MAX_NODES = (1 << 32) - 2


# ---------------------------------------------------------------------------
# Errors (src/error.rs:9-74)
# ---------------------------------------------------------------------------
class Status(enum.IntEnum):
    OK = 0
    DIMENSION_MISMATCH = 1
    INVALID_DIMENSION = 2
    NON_FINITE_VECTOR = 3
    ZERO_VECTOR = 4
    DUPLICATE_KEY = 5
    CAPACITY_EXCEEDED = 6
    QUANTIZATION_DISABLED = 7
    INVALID_PARAMETER = 8
    FORMAT_BAD_MAGIC = 10
    FORMAT_UNSUPPORTED_VERSION = 11
    FORMAT_TRUNCATED = 12
    FORMAT_CHECKSUM = 13
    FORMAT_TRAILING_BYTES = 14
    FORMAT_INVALID = 15
    MEMORY_LIMIT_EXCEEDED = 16
    CUDA = 20
    OUT_OF_DEVICE_MEMORY = 21
    TIMEOUT = 22
    ADMISSION_REJECTED = 23
    INVALID_ARGUMENT = 24
    SCRATCH_OVERFLOW = 25
    CANCELLED = 26


class Error(Exception):
    """Error of the crate (src/error.rs:9-51). ``status`` is the ABI code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = Status(status)
        self.message = message


class FormatError(Error):
    """Error::Format(FormatError) (src/error.rs:56-74)."""

    @property
    def invalid_field(self) -> Optional[str]:
        prefix = "invalid index file: invalid field: "
        if self.status == Status.FORMAT_INVALID and self.message.startswith(prefix):
            return self.message[len(prefix):]
        return None


def _raise(status: int):
    msg = _lib.hnsw_last_error().decode()
    if 10 <= status <= 15:
        raise FormatError(status, msg)
    raise Error(status, msg)


def _check(status: int):
    if status != 0:
        _raise(status)


class Metric(enum.IntEnum):
    """Metric (src/metric.rs:11-30); values are the file-format tags."""

    L2 = 0
    InnerProduct = 1
    Cosine = 2


def checked_build() -> bool:
    """True when the loaded library is the checked build."""
    return bool(_lib.hnsw_gpu_checked_build())


class Traversal(enum.IntEnum):
    """hnsw_search_opts.traversal: distances while the graph is walked. F32
    is the reference's search bit for bit; BF16 / BF16X3 use the tensor cores
    and re-rank the ef results with exact f32 distances."""

    F32 = 0
    BF16 = 1
    BF16X3 = 2


class Neighbor(NamedTuple):
    """Neighbor (src/neighbor.rs:7-12)."""

    key: int
    distance: float


# ---------------------------------------------------------------------------
# ctypes signatures
# ---------------------------------------------------------------------------
class _Info(C.Structure):
    _fields_ = [
        ("dim", C.c_uint32), ("metric", C.c_uint32), ("m", C.c_uint32), ("m0", C.c_uint32),
        ("ef_construction", C.c_uint32), ("quantized", C.c_uint32), ("nodes", C.c_uint32),
        ("live", C.c_uint32), ("top_level", C.c_uint32), ("entry", C.c_uint32),
        ("seed", C.c_uint64), ("level_multiplier", C.c_double), ("required_memory", C.c_uint64),
        ("device_bytes", C.c_uint64),
    ]


class _Opts(C.Structure):
    _fields_ = [
        ("k", C.c_uint32), ("ef", C.c_uint32), ("ks", C.c_void_p), ("efs", C.c_void_p),
        ("quantized", C.c_int32), ("filter_bits", C.c_void_p), ("filter_nbits", C.c_uint64),
        ("filter_stride", C.c_uint64), ("filter_used", C.c_void_p), ("out_stride", C.c_uint32),
        ("mode", C.c_int32), ("filter_ids", C.c_void_p), ("filter_by_node", C.c_int32),
        ("exact_below", C.c_float), ("traversal", C.c_int32),
    ]


class _Params(C.Structure):
    _fields_ = [
        ("m", C.c_uint32), ("m0", C.c_uint32), ("ef_construction", C.c_uint32),
        ("level_multiplier", C.c_double), ("selection", C.c_uint32),
        ("extend_candidates", C.c_uint32), ("keep_pruned", C.c_uint32), ("seed", C.c_uint64),
    ]


_vp = C.c_void_p
_sz = C.c_size_t
_lib.hnsw_last_error.restype = C.c_char_p
_lib.hnsw_validate_bytes.argtypes = [_vp, _sz, C.c_uint64, C.POINTER(_Info)]
_lib.hnsw_gpu_index_open.argtypes = [_vp, _sz, C.c_uint64, C.c_int, C.POINTER(_vp)]
_lib.hnsw_gpu_index_close.argtypes = [_vp]
_lib.hnsw_gpu_index_close.restype = None
_lib.hnsw_gpu_index_info.argtypes = [_vp, C.POINTER(_Info)]
_lib.hnsw_gpu_set_tombstones.argtypes = [_vp, _vp, _sz]
_lib.hnsw_gpu_search_batch.argtypes = [_vp, _vp, _sz, _sz, C.POINTER(_Opts), _vp, _vp, _vp, _vp]
_lib.hnsw_gpu_search_batch_device.argtypes = [_vp, _vp, _sz, _sz, C.POINTER(_Opts), _vp, _vp, _vp, _vp, _vp]
_lib.hnsw_gpu_set_counters.argtypes = [_vp, C.c_int]


class _Schedule(C.Structure):
    _fields_ = [("ef_cap", C.c_uint32), ("cand_cap", C.c_uint32), ("hash_cap", C.c_uint32),
                ("warps_per_block", C.c_uint32), ("cold_chunks", C.c_uint32), ("stage_rows", C.c_uint32),
                ("cold", C.c_uint32)]


_lib.hnsw_gpu_set_schedule.argtypes = [_vp, C.POINTER(_Schedule)]


class _TuneEntry(C.Structure):
    _fields_ = [("schedule", _Schedule), ("mode", C.c_int32), ("heuristic", C.c_int32), ("ms", C.c_float)]


_lib.hnsw_gpu_autotune.argtypes = [_vp, _vp, _sz, _sz, C.POINTER(_Opts), C.c_uint32, C.POINTER(_TuneEntry), _sz,
                                   C.POINTER(_sz), C.POINTER(_TuneEntry)]
_lib.hnsw_gpu_clear_tuning.argtypes = [_vp]

MODE_PLAIN, MODE_PERSISTENT, MODE_AUTO = 0, 1, 2
_lib.hnsw_gpu_graph_create.argtypes = [_vp, _vp, _sz, _sz, C.POINTER(_Opts), _vp, _vp, _vp, _vp, C.POINTER(_vp)]
_lib.hnsw_gpu_graph_launch.argtypes = [_vp, _vp]
_lib.hnsw_gpu_graph_destroy.argtypes = [_vp]
_lib.hnsw_gpu_graph_destroy.restype = None
_lib.hnsw_gpu_read_counters.argtypes = [_vp, _vp, _sz]
_lib.hnsw_gpu_brute_open.argtypes = [_vp, _vp, _sz, _sz, C.c_int, C.c_int, C.POINTER(_vp)]
_lib.hnsw_gpu_brute_close.argtypes = [_vp]
_lib.hnsw_gpu_brute_close.restype = None
_lib.hnsw_gpu_brute_search_batch.argtypes = [_vp, _vp, _sz, _sz, C.c_uint32, C.c_int, _vp, _vp, _vp, _vp]
class _BruteStats(C.Structure):
    _fields_ = [("candidates", C.c_uint64), ("queries", C.c_uint64), ("prep_ms", C.c_float),
                ("sample_ms", C.c_float), ("score_ms", C.c_float), ("rerank_ms", C.c_float)]


_lib.hnsw_gpu_brute_stats.argtypes = [_vp, C.POINTER(_BruteStats)]
_lib.hnsw_gpu_brute_set_wait_limits.argtypes = [_vp, C.c_uint64, C.c_int]
_lib.hnsw_gpu_brute_set_pairs.argtypes = [_vp, C.c_int]
_lib.hnsw_gpu_debug_fail_allocations.argtypes = [C.c_int]
_lib.hnsw_gpu_debug_fail_allocations.restype = None
_lib.hnsw_gpu_debug_visit_tags.argtypes = [C.c_int]
_lib.hnsw_gpu_debug_visit_tags.restype = None
_lib.hnsw_gpu_check_word.argtypes = [_vp, C.c_void_p, C.c_int]
_lib.hnsw_gpu_checked_build.argtypes = []


class _BruteFilter(C.Structure):
    _fields_ = [("bits", C.c_void_p), ("nbits", C.c_uint64), ("stride", C.c_uint64), ("used", C.c_void_p),
                ("ids", C.c_void_p), ("by_row", C.c_int32)]


_lib.hnsw_gpu_brute_search_filtered.argtypes = [_vp, _vp, _sz, _sz, C.c_uint32, C.POINTER(_BruteFilter), _vp, _vp,
                                                _vp, _vp]
_lib.hnsw_params_default.argtypes = [C.c_uint32, C.POINTER(_Params)]
_lib.hnsw_params_default.restype = None
_lib.hnsw_builder_new.argtypes = [_sz, C.c_int, C.POINTER(_Params), C.POINTER(_vp)]
_lib.hnsw_builder_free.argtypes = [_vp]
_lib.hnsw_builder_free.restype = None
_lib.hnsw_builder_insert.argtypes = [_vp, C.c_uint64, _vp, _sz]
_lib.hnsw_builder_insert_batch.argtypes = [_vp, _vp, _vp, _sz, _sz, C.c_int]
_lib.hnsw_builder_remove.argtypes = [_vp, C.c_uint64, C.POINTER(C.c_int)]
_lib.hnsw_builder_enable_quantization.argtypes = [_vp]
_lib.hnsw_builder_compact.argtypes = [_vp, C.c_int]


class _BuildOpts(C.Structure):
    _fields_ = [("wave_fraction", C.c_double), ("max_wave", C.c_uint32), ("hash_cap", C.c_uint32),
                ("timing", C.c_uint32)]


class _BuildStats(C.Structure):
    _fields_ = [("waves", C.c_uint32), ("nodes", C.c_uint32), ("spills", C.c_uint64), ("inexact", C.c_uint64),
                ("shrinks", C.c_uint64), ("records", C.c_uint64), ("device_ms", C.c_double),
                ("search_ms", C.c_double), ("connect_ms", C.c_double), ("dist_search", C.c_uint64),
                ("dist_select", C.c_uint64), ("dist_connect", C.c_uint64), ("lists0", C.c_uint64),
                ("listsU", C.c_uint64), ("search_warps_per_block", C.c_uint32), ("search_blocks_per_sm", C.c_uint32),
                ("connect_warps_per_block", C.c_uint32), ("connect_blocks_per_sm", C.c_uint32),
                ("hash_cap", C.c_uint32)]


_lib.hnsw_gpu_build_opts_default.argtypes = [C.POINTER(_BuildOpts)]
_lib.hnsw_gpu_build_opts_default.restype = None
_lib.hnsw_builder_insert_batch_gpu.argtypes = [_vp, _vp, _vp, _sz, _sz, C.c_int, C.POINTER(_BuildOpts)]
_lib.hnsw_builder_compact_gpu.argtypes = [_vp, C.c_int, C.POINTER(_BuildOpts)]
_lib.hnsw_builder_gpu_stats.argtypes = [_vp, C.POINTER(_BuildStats)]
_lib.hnsw_builder_to_bytes.argtypes = [_vp, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(_sz)]
_lib.hnsw_bytes_free.argtypes = [C.POINTER(C.c_uint8)]
_lib.hnsw_bytes_free.restype = None
_lib.hnsw_synthetic_gaussian.argtypes = [_sz, _sz, _sz, C.c_uint64, _vp, _vp]
_lib.hnsw_synthetic_gaussian.restype = None
_lib.hnsw_synthetic_mixture.argtypes = [_sz, _sz, _sz, _sz, C.c_double, C.c_uint64, _vp, _vp]
_lib.hnsw_synthetic_mixture.restype = None
_lib.hnsw_synthetic_mixture_split.argtypes = [_sz, _sz, _sz, _sz, C.c_double, C.c_uint64, C.c_uint64, _vp, _vp]
_lib.hnsw_synthetic_mixture_split.restype = None
_lib.hnsw_crc32.argtypes = [_vp, _sz]
_lib.hnsw_crc32.restype = C.c_uint32

EXPORTED_SYMBOLS = (
    "hnsw_last_error", "hnsw_validate_bytes", "hnsw_gpu_index_open", "hnsw_gpu_index_close",
    "hnsw_gpu_index_info", "hnsw_gpu_set_tombstones", "hnsw_gpu_search_batch",
    "hnsw_gpu_search_batch_device", "hnsw_gpu_set_counters", "hnsw_gpu_read_counters",
    "hnsw_gpu_brute_open", "hnsw_gpu_brute_close", "hnsw_gpu_brute_search_batch",
    "hnsw_params_default", "hnsw_builder_new", "hnsw_builder_free", "hnsw_builder_insert",
    "hnsw_builder_insert_batch", "hnsw_builder_remove", "hnsw_builder_enable_quantization",
    "hnsw_builder_to_bytes", "hnsw_bytes_free", "hnsw_synthetic_gaussian",
    "hnsw_synthetic_mixture", "hnsw_synthetic_mixture_split", "hnsw_crc32", "hnsw_gpu_autotune",
    "hnsw_gpu_clear_tuning", "hnsw_gpu_set_schedule", "hnsw_gpu_brute_search_filtered",
    "hnsw_builder_compact", "hnsw_gpu_build_opts_default", "hnsw_builder_insert_batch_gpu",
    "hnsw_builder_compact_gpu", "hnsw_builder_gpu_stats",
)

LIBRARY_PATH = _LIB_PATH


def _ptr(a: Optional[np.ndarray]) -> Optional[int]:
    return None if a is None else a.ctypes.data


# ---------------------------------------------------------------------------
# Parameters and options
# ---------------------------------------------------------------------------
@dataclass
class NeighborSelection:
    """NeighborSelection (src/params.rs:19-41): simple or heuristic."""

    heuristic: bool = True
    extend_candidates: bool = False
    keep_pruned: bool = False

    @staticmethod
    def simple() -> "NeighborSelection":
        return NeighborSelection(False, False, False)


@dataclass
class HnswParams:
    """HnswParams (src/params.rs:59-182); HnswParams(m) gives the paper's defaults."""

    m: int = 16
    m0: Optional[int] = None
    ef_construction: int = 200
    level_multiplier: Optional[float] = None
    selection: NeighborSelection = None
    seed: int = 0

    def _c(self) -> _Params:
        p = _Params()
        _lib.hnsw_params_default(C.c_uint32(min(self.m, 0xFFFFFFFF)), C.byref(p))
        if self.m0 is not None:
            p.m0 = self.m0
        p.ef_construction = self.ef_construction
        if self.level_multiplier is not None:
            p.level_multiplier = self.level_multiplier
        sel = self.selection or NeighborSelection()
        p.selection = 1 if sel.heuristic else 0
        p.extend_candidates = int(sel.extend_candidates)
        p.keep_pruned = int(sel.keep_pruned)
        p.seed = self.seed
        return p


class SearchOptions:
    """SearchOptions (src/hnsw/mod.rs:56-98).

    ``filter`` is either a callable over keys (evaluated on the host over the
    index's keys into a key bitmap, as the reference calls its closure per
    visited node) or a key bitmap: a uint64 array where key x passes iff bit x
    is set.
    """

    def __init__(self, ef: int):
        self._ef = ef
        self._filter = None
        self._quantized = False
        self._traversal = Traversal.F32

    def filter(self, f) -> "SearchOptions":
        self._filter = f
        return self

    def quantized(self, q: bool) -> "SearchOptions":
        self._quantized = bool(q)
        return self

    def traversal(self, t: "Traversal") -> "SearchOptions":
        """Distances while walking the graph (hnsw_search_opts.traversal); no
        counterpart in the reference, whose search is Traversal.F32."""
        self._traversal = Traversal(t)
        return self

    def ef(self) -> int:
        return self._ef


def key_bitmap(keys: np.ndarray, nbits: Optional[int] = None) -> np.ndarray:
    """A key bitmap (uint64 words) with the bits of `keys` set."""
    keys = np.asarray(keys, dtype=np.uint64)
    if nbits is None:
        nbits = int(keys.max()) + 1 if keys.size else 1
    words = np.zeros((nbits + 63) // 64, dtype=np.uint64)
    if keys.size:
        np.bitwise_or.at(words, (keys >> np.uint64(6)).astype(np.int64), np.uint64(1) << (keys & np.uint64(63)))
    return words


# ---------------------------------------------------------------------------
# Device HNSW index
# ---------------------------------------------------------------------------
class HnswIndex:
    """A format-v1 HNSW index resident on one GPU.

    Open with ``HnswIndex.from_bytes`` (src/hnsw/mod.rs:666-700). Searches
    take ``&self`` semantics: the handle may be used from many threads.
    """

    def __init__(self, handle: int, file_keys: np.ndarray, deleted: np.ndarray):
        self._h = C.c_void_p(handle)
        self._keys = file_keys
        self._deleted = deleted
        info = _Info()
        _check(_lib.hnsw_gpu_index_info(self._h, C.byref(info)))
        self._info = info

    @staticmethod
    def from_bytes(data: bytes, device: int = 0, max_memory: Optional[int] = None) -> "HnswIndex":
        buf = np.frombuffer(data, dtype=np.uint8)
        h = C.c_void_p()
        _check(_lib.hnsw_gpu_index_open(_ptr(buf), buf.size, max_memory or 0, device, C.byref(h)))
        n = int.from_bytes(data[48:52], "little")
        keys = np.frombuffer(data, dtype="<u8", count=n, offset=56).copy()
        deleted = np.frombuffer(data, dtype=np.uint8, count=n, offset=56 + 9 * n).copy()
        return HnswIndex(h.value, keys, deleted)

    @staticmethod
    def from_bytes_with_limit(data: bytes, max_memory: int, device: int = 0) -> "HnswIndex":
        if max_memory == 0:
            # A zero limit is a real limit here, not "default".
            max_memory = 1
            info = _Info()
            st = _lib.hnsw_validate_bytes(_ptr(np.frombuffer(data, np.uint8)), len(data), 1, C.byref(info))
            if st == Status.MEMORY_LIMIT_EXCEEDED:
                msg = _lib.hnsw_last_error().decode().replace("limit of 1", "limit of 0")
                raise Error(st, msg)
        return HnswIndex.from_bytes(data, device=device, max_memory=max_memory)

    def close(self):
        if self._h:
            _lib.hnsw_gpu_index_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- introspection --
    def dim(self) -> int:
        return self._info.dim

    def metric(self) -> Metric:
        return Metric(self._info.metric)

    def __len__(self) -> int:
        return self._info.live

    def len(self) -> int:
        return self._info.live

    def is_empty(self) -> bool:
        return self._info.live == 0

    def node_count(self) -> int:
        return self._info.nodes

    def is_quantized(self) -> bool:
        return bool(self._info.quantized)

    def info(self) -> _Info:
        return self._info

    def keys(self) -> np.ndarray:
        return self._keys

    # -- search --
    def _filter_bits(self, f):
        if f is None:
            return None, 0, False
        if callable(f):
            # The closure runs once per live node on the calling thread; the
            # bitmap is indexed by node id, so any u64 key set works.
            live = np.nonzero(self._deleted == 0)[0]
            keys = self._keys[live].tolist()
            accepted = np.fromiter((i for i, k in zip(live.tolist(), keys) if f(k)), dtype=np.uint64)
            nbits = max(int(self._keys.size), 1)
            return key_bitmap(accepted, nbits), nbits, True
        bits = np.ascontiguousarray(f, dtype=np.uint64)
        return bits, bits.size * 64, False

    @staticmethod
    def _opts(nq, k, ef, quantized=False, filter_bits=None, filter_nbits=0, filter_stride=0, filter_used=None,
              ks=None, efs=None, mode=0, filter_ids=None, filter_by_node=False, exact_below=0.0, traversal=0):
        """hnsw_search_opts for a batch, and the arrays it points into (keep them alive)."""
        ks_a = None if ks is None else np.ascontiguousarray(ks, dtype=np.uint32)
        efs_a = None if efs is None else np.ascontiguousarray(efs, dtype=np.uint32)
        kmax = int(ks_a.max()) if ks_a is not None and ks_a.size else k
        o = _Opts()
        o.k, o.ef = k, ef
        o.ks, o.efs = _ptr(ks_a), _ptr(efs_a)
        o.quantized = int(quantized)
        fb = None if filter_bits is None else np.ascontiguousarray(filter_bits, dtype=np.uint64)
        fu = None if filter_used is None else np.ascontiguousarray(filter_used, dtype=np.uint8)
        o.filter_bits = _ptr(fb)
        o.filter_nbits = filter_nbits if fb is not None else 0
        o.filter_stride = filter_stride
        o.filter_used = _ptr(fu)
        fi = None if filter_ids is None else np.ascontiguousarray(filter_ids, dtype=np.uint32)
        o.filter_ids = _ptr(fi)
        o.filter_by_node = int(filter_by_node)
        o.exact_below = float(exact_below)
        o.traversal = int(traversal)
        o.out_stride = max(kmax, 1)
        o.mode = mode
        return o, (ks_a, efs_a, fb, fu, fi)

    def search_arrays(self, queries: np.ndarray, k: int, ef: int, *, quantized: bool = False,
                      filter_bits: Optional[np.ndarray] = None, filter_nbits: int = 0,
                      filter_stride: int = 0, filter_used: Optional[np.ndarray] = None,
                      ks: Optional[np.ndarray] = None, efs: Optional[np.ndarray] = None,
                      mode: int = 0, raise_on_error: bool = True, filter_ids: Optional[np.ndarray] = None,
                      filter_by_node: bool = False, exact_below: float = 0.0, traversal: int = 0):
        """Batched search returning arrays (keys, dist, count, status).
        exact_below > 0 turns on the selectivity planner; traversal
        (Traversal.BF16 / BF16X3) walks the graph with tensor-core distances
        and re-ranks with exact f32 ones (hnsw_search_opts)."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        if q.ndim == 1:
            if q.size % max(self.dim(), 1):
                raise Error(Status.DIMENSION_MISMATCH,
                            f"dimension mismatch: expected {self.dim()}, got {q.size}")
            q = q.reshape(-1, self.dim())
        nq, dim = q.shape
        o, keep = self._opts(nq, k, ef, quantized=quantized, filter_bits=filter_bits, filter_nbits=filter_nbits,
                             filter_stride=filter_stride, filter_used=filter_used, ks=ks, efs=efs, mode=mode,
                             filter_ids=filter_ids, filter_by_node=filter_by_node, exact_below=exact_below,
                             traversal=traversal)
        stride = o.out_stride
        keys = np.zeros((nq, stride), dtype=np.uint64)
        dist = np.zeros((nq, stride), dtype=np.float32)
        count = np.zeros(nq, dtype=np.uint32)
        status = np.zeros(nq, dtype=np.int32)
        st = _lib.hnsw_gpu_search_batch(self._h, _ptr(q), nq, dim, C.byref(o), _ptr(keys), _ptr(dist),
                                        _ptr(count), _ptr(status))
        if st != 0 and raise_on_error:
            _raise(st)
        return keys, dist, count, status

    def _to_lists(self, keys, dist, count):
        return [[Neighbor(int(keys[i, j]), float(dist[i, j])) for j in range(int(count[i]))]
                for i in range(len(count))]

    def search(self, query: Sequence[float], k: int, ef: int):
        """HnswIndex::search (src/hnsw/mod.rs:412-414)."""
        return self.search_with(query, k, SearchOptions(ef))

    def search_filtered(self, query, k: int, ef: int, filter):
        """HnswIndex::search_filtered (src/hnsw/mod.rs:432-440)."""
        return self.search_with(query, k, SearchOptions(ef).filter(filter))

    def search_with(self, query, k: int, options: SearchOptions):
        """HnswIndex::search_with (src/hnsw/mod.rs:448-455)."""
        q = np.ascontiguousarray(query, dtype=np.float32).reshape(-1)
        if q.size != self.dim():
            raise Error(Status.DIMENSION_MISMATCH,
                        f"dimension mismatch: expected {self.dim()}, got {q.size}")
        bits, nbits, by_node = self._filter_bits(options._filter)
        keys, dist, count, _ = self.search_arrays(q.reshape(1, -1), k, options.ef(),
                                                  quantized=options._quantized,
                                                  filter_bits=bits, filter_nbits=nbits, filter_by_node=by_node,
                                                  traversal=int(options._traversal))
        return self._to_lists(keys, dist, count)[0]

    def search_batch(self, queries, k: int, ef: int):
        """HnswIndex::search_batch (src/hnsw/mod.rs:520-536)."""
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1)
        if q.size % self.dim():
            raise Error(Status.DIMENSION_MISMATCH,
                        f"dimension mismatch: expected {self.dim()}, got {q.size}")
        keys, dist, count, _ = self.search_arrays(q.reshape(-1, self.dim()), k, ef)
        return self._to_lists(keys, dist, count)

    def set_tombstones(self, deleted: np.ndarray):
        d = np.ascontiguousarray(deleted, dtype=np.uint8)
        _check(_lib.hnsw_gpu_set_tombstones(self._h, _ptr(d), d.size))
        self._deleted = d.copy()
        info = _Info()
        _check(_lib.hnsw_gpu_index_info(self._h, C.byref(info)))
        self._info = info

    def set_schedule(self, ef_cap=None, cand_cap=None, hash_cap=None, warps_per_block=None, cold_chunks=0,
                     stage_rows=0, cold=0):
        """Fixes the traversal scratch geometry; no arguments restores the automatic choice."""
        if ef_cap is None:
            _check(_lib.hnsw_gpu_set_schedule(self._h, None))
            return
        sc = _Schedule(ef_cap, cand_cap or 2 * ef_cap + 32, hash_cap, warps_per_block, cold_chunks, stage_rows,
                       int(cold))
        _check(_lib.hnsw_gpu_set_schedule(self._h, C.byref(sc)))

    def autotune(self, queries, k: int, ef: int, reps: int = 3, **search_kw):
        """Times the sample batch under every schedule of the tuner's grid and
        installs the fastest per mode for this ef bucket (hnsw_gpu_autotune).
        Returns (best, trials), each trial a dict of schedule, mode, ms."""
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, self.dim())
        o, keep = self._opts(q.shape[0], k, ef, **search_kw)
        entries = (_TuneEntry * 128)()
        n = C.c_size_t()
        best = _TuneEntry()
        _check(_lib.hnsw_gpu_autotune(self._h, _ptr(q), q.shape[0], q.shape[1], C.byref(o), reps, entries, 128,
                                      C.byref(n), C.byref(best)))
        del keep

        def d(e):
            s = e.schedule
            return {"ef_cap": s.ef_cap, "cand_cap": s.cand_cap, "hash_cap": s.hash_cap,
                    "warps_per_block": s.warps_per_block, "stage_rows": s.stage_rows, "cold": s.cold,
                    "mode": e.mode,
                    "heuristic": bool(e.heuristic),
                    "ms": e.ms}

        return d(best), [d(entries[i]) for i in range(n.value)]

    def clear_tuning(self):
        _check(_lib.hnsw_gpu_clear_tuning(self._h))

    def check_word(self, clear: bool = True):
        """(site, value) of the first bounds-check violation of the checked
        build (hnsw_gpu_check_word); (0, 0) when none or in the normal build."""
        out = (C.c_uint32 * 2)()
        _check(_lib.hnsw_gpu_check_word(self._h, out, int(clear)))
        return int(out[0]), int(out[1])

    def set_counters(self, enabled: bool):
        _check(_lib.hnsw_gpu_set_counters(self._h, int(enabled)))

    def read_counters(self, nq: int) -> np.ndarray:
        out = np.zeros((nq, 4), dtype=np.uint32)
        _check(_lib.hnsw_gpu_read_counters(self._h, _ptr(out), nq))
        return out

    def graph(self, d_queries: int, nq: int, k: int, ef: int, d_keys: int, d_dist: int, d_count: int,
              d_status: int, mode: int = 1, quantized: bool = False):
        """Captures the launch sequence of one device-pointer search (CUDA graph)."""
        o = _Opts()
        o.k, o.ef = k, ef
        o.quantized = int(quantized)
        o.out_stride = k
        o.mode = mode
        g = C.c_void_p()
        _check(_lib.hnsw_gpu_graph_create(self._h, d_queries, nq, self.dim(), C.byref(o), d_keys, d_dist, d_count,
                                          d_status, C.byref(g)))
        return SearchGraph(g)

    def search_device(self, d_queries: int, nq: int, k: int, ef: int, d_keys: int, d_dist: int,
                      d_count: int, d_status: int, stream: Optional[int] = None, quantized: bool = False,
                      mode: int = 0, out_stride: int = 0, traversal: int = 0):
        """hnsw_gpu_search_batch_device with raw device pointers."""
        o = _Opts()
        o.k, o.ef = k, ef
        o.quantized = int(quantized)
        o.traversal = int(traversal)
        o.out_stride = out_stride or k
        o.mode = mode
        # stream None = the library's own stream; 0 = the legacy default stream.
        handle = None if stream is None else (stream if stream != 0 else 1)
        _check(_lib.hnsw_gpu_search_batch_device(self._h, d_queries, nq, self.dim(), C.byref(o), d_keys,
                                                 d_dist, d_count, d_status, handle))


class _ServerConfig(C.Structure):
    _fields_ = [("max_batch", C.c_uint32), ("max_inflight", C.c_uint32), ("max_pending", C.c_uint32),
                ("max_k", C.c_uint32), ("max_ef", C.c_uint32), ("linger_us", C.c_uint32),
                ("filter_nbits", C.c_uint64), ("quantized", C.c_int32), ("filter_bank", C.c_void_p),
                ("filter_count", C.c_uint32), ("filter_by_node", C.c_int32), ("mode", C.c_int32)]


_lib.hnsw_server_config_default.argtypes = [C.POINTER(_ServerConfig)]
_lib.hnsw_server_config_default.restype = None
_lib.hnsw_gpu_server_start.argtypes = [_vp, C.POINTER(_ServerConfig), C.POINTER(_vp)]
_lib.hnsw_gpu_server_stop.argtypes = [_vp]
_lib.hnsw_gpu_server_stop.restype = None
_lib.hnsw_gpu_submit.argtypes = [_vp, _vp, C.c_uint32, C.c_uint32, C.c_int32, C.POINTER(C.c_uint64)]
_lib.hnsw_gpu_poll.argtypes = [_vp, C.c_uint64, C.POINTER(C.c_int)]
_lib.hnsw_gpu_cancel.argtypes = [_vp, C.c_uint64, C.POINTER(C.c_int)]
_lib.hnsw_gpu_wait.argtypes = [_vp, C.c_uint64, C.c_uint32, _vp, _vp, C.POINTER(C.c_uint32),
                               C.POINTER(C.c_int32), C.POINTER(C.c_double)]
_lib.hnsw_gpu_server_replay.argtypes = [_vp, _vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
_lib.hnsw_gpu_server_stats.argtypes = [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]


class Server:
    """Request loop over a resident HnswIndex: continuous batching."""

    def __init__(self, index: HnswIndex, *, max_batch=2048, max_inflight=4, max_pending=1 << 16, max_k=100,
                 max_ef=512, linger_us=100, filter_nbits=0, filter_bank: Optional[np.ndarray] = None,
                 quantized=False, filter_by_node=False, mode=1):
        cfg = _ServerConfig()
        _lib.hnsw_server_config_default(C.byref(cfg))
        cfg.max_batch, cfg.max_inflight, cfg.max_pending = max_batch, max_inflight, max_pending
        cfg.max_k, cfg.max_ef, cfg.linger_us = max_k, max_ef, linger_us
        cfg.filter_nbits, cfg.quantized = filter_nbits, int(quantized)
        cfg.filter_by_node = int(filter_by_node)
        cfg.mode = int(mode)
        bank = None if filter_bank is None else np.ascontiguousarray(filter_bank, np.uint64)
        if bank is not None:
            cfg.filter_bank = _ptr(bank)
            cfg.filter_count = bank.shape[0]
        h = C.c_void_p()
        _check(_lib.hnsw_gpu_server_start(index._h, C.byref(cfg), C.byref(h)))
        self._h = h
        self._index = index
        self.max_k = max_k
        self.words = (filter_nbits + 63) // 64

    def submit(self, query, k: int, ef: int, filter_id: int = -1) -> int:
        q = np.ascontiguousarray(query, np.float32)
        t = C.c_uint64()
        _check(_lib.hnsw_gpu_submit(self._h, _ptr(q), k, ef, filter_id, C.byref(t)))
        return t.value

    def cancel(self, ticket: int) -> bool:
        """hnsw_gpu_cancel: True if the request will report CANCELLED, False
        if it had already completed (its results stand)."""
        c = C.c_int()
        _check(_lib.hnsw_gpu_cancel(self._h, ticket, C.byref(c)))
        return bool(c.value)

    def wait(self, ticket: int, timeout_ms: int = 60000):
        keys = np.zeros(self.max_k, np.uint64)
        dist = np.zeros(self.max_k, np.float32)
        cnt, st, lat = C.c_uint32(), C.c_int32(), C.c_double()
        _check(_lib.hnsw_gpu_wait(self._h, ticket, timeout_ms, _ptr(keys), _ptr(dist), C.byref(cnt), C.byref(st),
                                  C.byref(lat)))
        c = cnt.value
        return keys[:c], dist[:c], st.value, lat.value

    def replay(self, queries, arrival_us, ks, efs, filter_ids=None):
        q = np.ascontiguousarray(queries, np.float32)
        n = q.shape[0]
        arr = np.ascontiguousarray(arrival_us, np.float64)
        ks_a = np.ascontiguousarray(ks, np.uint32)
        efs_a = np.ascontiguousarray(efs, np.uint32)
        fi = None if filter_ids is None else np.ascontiguousarray(filter_ids, np.int32)
        keys = np.zeros((n, self.max_k), np.uint64)
        dist = np.zeros((n, self.max_k), np.float32)
        cnt = np.zeros(n, np.uint32)
        st = np.zeros(n, np.int32)
        lat = np.zeros(n, np.float64)
        _check(_lib.hnsw_gpu_server_replay(self._h, _ptr(q), n, _ptr(arr), _ptr(ks_a), _ptr(efs_a), _ptr(fi),
                                           _ptr(keys), _ptr(dist), _ptr(cnt), _ptr(st), _ptr(lat)))
        return keys, dist, cnt, st, lat

    def stats(self):
        b, q = C.c_uint64(), C.c_uint64()
        _check(_lib.hnsw_gpu_server_stats(self._h, C.byref(b), C.byref(q)))
        return b.value, q.value

    def stop(self):
        if self._h:
            _lib.hnsw_gpu_server_stop(self._h)
            self._h = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


class SearchGraph:
    """A captured search launch sequence (hnsw_gpu_graph_*)."""

    def __init__(self, handle):
        self._h = handle

    def launch(self, stream: Optional[int] = None):
        handle = None if stream is None else (stream if stream != 0 else 1)
        _check(_lib.hnsw_gpu_graph_launch(self._h, handle))

    def close(self):
        if self._h:
            _lib.hnsw_gpu_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def debug_fail_allocations(count: int):
    """Test hook: the next `count` device allocations fail as out of memory."""
    _lib.hnsw_gpu_debug_fail_allocations(int(count))


def debug_visit_tags(mode: int):
    """Visited-hash storage of the traversal kernels: 0 automatic (16-bit
    tags where they fit), -1 always 32-bit ids, k > 0 ids treated as at least
    k bits wide (shorter recordable probes). Results are the same in every
    mode."""
    _lib.hnsw_gpu_debug_visit_tags(int(mode))


def validate_bytes(data: bytes, max_memory: Optional[int] = None) -> _Info:
    """Host-only validation with every check of HnswIndex::from_bytes."""
    buf = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
    info = _Info()
    _check(_lib.hnsw_validate_bytes(_ptr(buf), len(data), max_memory or 0, C.byref(info)))
    return info


# ---------------------------------------------------------------------------
# Device brute force
# ---------------------------------------------------------------------------
class Precision(enum.IntEnum):
    FP32 = 0
    BF16 = 1
    BF16X3 = 2


class BruteForceIndex:
    """BruteForceIndex (src/brute.rs:29-181) on the GPU."""

    def __init__(self, dim: int, metric: Metric, device: int = 0):
        if dim == 0 or dim > MAX_DIM:
            raise Error(Status.INVALID_DIMENSION, f"invalid dimension {dim}: must be between 1 and {MAX_DIM}")
        self._dim = dim
        self._metric = Metric(metric)
        self._device = device
        self._keys = np.zeros(0, np.uint64)
        self._vecs = np.zeros((0, dim), np.float32)
        self._h = None

    @staticmethod
    def new(dim: int, metric: Metric, device: int = 0) -> "BruteForceIndex":
        return BruteForceIndex(dim, metric, device)

    def insert_batch(self, keys, vectors):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        v = np.ascontiguousarray(vectors, dtype=np.float32).reshape(-1)
        if v.size != keys.size * self._dim:
            raise Error(Status.DIMENSION_MISMATCH,
                        f"dimension mismatch: expected {keys.size * self._dim}, got {v.size}")
        new_keys = np.concatenate([self._keys, keys])
        new_vecs = np.concatenate([self._vecs, v.reshape(-1, self._dim)])
        h = C.c_void_p()
        _check(_lib.hnsw_gpu_brute_open(_ptr(new_vecs), _ptr(new_keys), new_keys.size, self._dim,
                                        int(self._metric), self._device, C.byref(h)))
        self.close()
        self._h = h
        self._keys, self._vecs = new_keys, new_vecs

    def insert(self, key: int, vector):
        self.insert_batch(np.array([key], np.uint64), np.asarray(vector, np.float32).reshape(1, -1))

    def __len__(self):
        return int(self._keys.size)

    def len(self):
        return int(self._keys.size)

    def search_arrays(self, queries, k: int, precision: Precision = Precision.FP32, raise_on_error=True, *,
                      filter_bits=None, filter_nbits: int = 0, filter_stride: int = 0, filter_used=None,
                      filter_ids=None, filter_by_row: bool = False):
        """Batched exact search returning arrays (keys, dist, count, status).
        With filter_bits, hnsw_gpu_brute_search_filtered (FP32, any precision
        argument notwithstanding)."""
        q = np.ascontiguousarray(queries, dtype=np.float32)
        if q.ndim == 1:
            q = q.reshape(-1, self._dim)
        nq = q.shape[0]
        kk = max(int(k), 1)
        keys = np.zeros((nq, kk), np.uint64)
        dist = np.zeros((nq, kk), np.float32)
        count = np.zeros(nq, np.uint32)
        status = np.zeros(nq, np.int32)
        if self._h is None:
            self.insert_batch(np.zeros(0, np.uint64), np.zeros((0, self._dim), np.float32))
        if filter_bits is not None:
            fb = np.ascontiguousarray(filter_bits, np.uint64)
            fu = None if filter_used is None else np.ascontiguousarray(filter_used, np.uint8)
            fi = None if filter_ids is None else np.ascontiguousarray(filter_ids, np.uint32)
            f = _BruteFilter(_ptr(fb), filter_nbits, filter_stride, _ptr(fu), _ptr(fi), int(filter_by_row))
            st = _lib.hnsw_gpu_brute_search_filtered(self._h, _ptr(q), nq, q.shape[1], int(k), C.byref(f), _ptr(keys),
                                                     _ptr(dist), _ptr(count), _ptr(status))
        else:
            st = _lib.hnsw_gpu_brute_search_batch(self._h, _ptr(q), nq, q.shape[1], int(k), int(precision),
                                                  _ptr(keys), _ptr(dist), _ptr(count), _ptr(status))
        if st != 0 and raise_on_error:
            _raise(st)
        return keys, dist, count, status

    def search_filtered(self, query, k: int, filter):
        """BruteForceIndex::search_filtered (src/brute.rs:131-160). `filter` is a
        closure over keys (run once per row on the calling thread) or a key
        bitmap (uint64 words)."""
        if callable(filter):
            accepted = np.fromiter((i for i, key in enumerate(self._keys.tolist()) if filter(key)), dtype=np.uint64)
            nbits = max(int(self._keys.size), 1)
            bits, by_row = key_bitmap(accepted, nbits), True
        else:
            bits = np.ascontiguousarray(filter, np.uint64)
            nbits, by_row = bits.size * 64, False
        keys, dist, count, _ = self.search_arrays(np.asarray(query, np.float32).reshape(1, -1), k,
                                                  filter_bits=bits, filter_nbits=nbits, filter_by_row=by_row)
        return [Neighbor(int(keys[0, j]), float(dist[0, j])) for j in range(int(count[0]))]

    def set_wait_limits(self, budget_cycles: int = 0, inject_stall: bool = False):
        """Clock budget of the tensor-core pipeline's waits (0: the default);
        inject_stall makes the next tensor-core searches run out of it
        (hnsw_gpu_brute_set_wait_limits)."""
        _check(_lib.hnsw_gpu_brute_set_wait_limits(self._h, budget_cycles, int(inject_stall)))

    def set_pairs(self, enabled: bool = True):
        """Tensor-core kernel shape: paired CTAs per 256 x 256 tile (hnsw_gpu_brute_set_pairs)."""
        _check(_lib.hnsw_gpu_brute_set_pairs(self._h, int(enabled)))

    def last_stats(self) -> dict:
        """Candidates and device stage times of the last tensor-core search."""
        st = _BruteStats()
        _check(_lib.hnsw_gpu_brute_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def last_candidates_per_query(self) -> float:
        """Mean candidates kept by the threshold in the last tensor-core search."""
        st = _BruteStats()
        _check(_lib.hnsw_gpu_brute_stats(self._h, C.byref(st)))
        return st.candidates / max(st.queries, 1)

    def search(self, query, k: int, precision: Precision = Precision.FP32):
        keys, dist, count, _ = self.search_arrays(np.asarray(query, np.float32).reshape(1, -1), k, precision)
        return [Neighbor(int(keys[0, j]), float(dist[0, j])) for j in range(int(count[0]))]

    def search_batch(self, queries, k: int, precision: Precision = Precision.FP32):
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1)
        if q.size % self._dim:
            raise Error(Status.DIMENSION_MISMATCH, f"dimension mismatch: expected {self._dim}, got {q.size}")
        keys, dist, count, _ = self.search_arrays(q.reshape(-1, self._dim), k, precision)
        return [[Neighbor(int(keys[i, j]), float(dist[i, j])) for j in range(int(count[i]))]
                for i in range(len(count))]

    def close(self):
        if self._h:
            _lib.hnsw_gpu_brute_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Host-side construction
# ---------------------------------------------------------------------------
class IndexBuilder:
    """HnswIndex construction (src/hnsw/mod.rs:181-400), producing format-v1 bytes."""

    def __init__(self, dim: int, metric: Metric, params: Optional[HnswParams] = None):
        params = params or HnswParams()
        h = C.c_void_p()
        _check(_lib.hnsw_builder_new(dim, int(metric), C.byref(params._c()), C.byref(h)))
        self._h = h
        self._dim = dim

    def insert(self, key: int, vector):
        v = np.ascontiguousarray(vector, dtype=np.float32).reshape(-1)
        _check(_lib.hnsw_builder_insert(self._h, key, _ptr(v), v.size))

    def insert_batch(self, keys, vectors, threads: int = 0):
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        v = np.ascontiguousarray(vectors, dtype=np.float32).reshape(-1)
        if v.size != keys.size * self._dim:
            raise Error(Status.DIMENSION_MISMATCH,
                        f"dimension mismatch: expected {keys.size * self._dim}, got {v.size}")
        _check(_lib.hnsw_builder_insert_batch(self._h, _ptr(keys), _ptr(v), keys.size, self._dim, threads))

    def insert_batch_gpu(self, keys, vectors, device: int = 0, wave_fraction: Optional[float] = None,
                         max_wave: Optional[int] = None, hash_cap: Optional[int] = None, timing: bool = False):
        """insert_batch with the link step on a GPU (waves of nodes; see hnsw_gpu.h)."""
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        v = np.ascontiguousarray(vectors, dtype=np.float32).reshape(-1)
        if v.size != keys.size * self._dim:
            raise Error(Status.DIMENSION_MISMATCH,
                        f"dimension mismatch: expected {keys.size * self._dim}, got {v.size}")
        o = self._build_opts(wave_fraction, max_wave, hash_cap, timing)
        _check(_lib.hnsw_builder_insert_batch_gpu(self._h, _ptr(keys), _ptr(v), keys.size, self._dim, device,
                                                  C.byref(o)))

    def compact(self, threads: int = 0):
        """HnswIndex::compact: rebuild from the live nodes (no-op without tombstones)."""
        _check(_lib.hnsw_builder_compact(self._h, threads))

    def compact_gpu(self, device: int = 0, wave_fraction: Optional[float] = None, max_wave: Optional[int] = None,
                    hash_cap: Optional[int] = None, timing: bool = False):
        """compact with the link step on a GPU."""
        o = self._build_opts(wave_fraction, max_wave, hash_cap, timing)
        _check(_lib.hnsw_builder_compact_gpu(self._h, device, C.byref(o)))

    def gpu_stats(self) -> dict:
        """Figures of the last device link."""
        st = _BuildStats()
        _check(_lib.hnsw_builder_gpu_stats(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in _BuildStats._fields_}

    @staticmethod
    def _build_opts(wave_fraction, max_wave, hash_cap, timing=False) -> "_BuildOpts":
        o = _BuildOpts()
        _lib.hnsw_gpu_build_opts_default(C.byref(o))
        o.timing = int(bool(timing))
        if wave_fraction is not None:
            o.wave_fraction = wave_fraction
        if max_wave is not None:
            o.max_wave = max_wave
        if hash_cap is not None:
            o.hash_cap = hash_cap
        return o

    def remove(self, key: int) -> bool:
        r = C.c_int()
        _check(_lib.hnsw_builder_remove(self._h, key, C.byref(r)))
        return bool(r.value)

    def enable_quantization(self):
        _check(_lib.hnsw_builder_enable_quantization(self._h))

    def to_bytes(self) -> bytes:
        p = C.POINTER(C.c_uint8)()
        n = _sz()
        _check(_lib.hnsw_builder_to_bytes(self._h, C.byref(p), C.byref(n)))
        try:
            # ctypes.string_at takes a C int length: files above 2 GiB need a
            # 64-bit copy.
            if n.value == 0:
                return b""
            return np.ctypeslib.as_array(p, shape=(n.value,)).tobytes()
        finally:
            _lib.hnsw_bytes_free(p)

    def __del__(self):
        try:
            if self._h:
                _lib.hnsw_builder_free(self._h)
                self._h = None
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Synthetic data (src/synthetic.rs)
# ---------------------------------------------------------------------------
def gaussian(n_base: int, n_query: int, dim: int, seed: int):
    """Dataset::gaussian: (base, queries) float32 arrays."""
    base = np.empty((n_base, dim), np.float32)
    queries = np.empty((n_query, dim), np.float32)
    _lib.hnsw_synthetic_gaussian(n_base, n_query, dim, seed, _ptr(base), _ptr(queries))
    return base, queries


def mixture(n_base: int, n_query: int, dim: int, clusters: int, sigma: float, seed: int):
    """Dataset::clustered with spread `sigma`: (base, queries) float32 arrays."""
    base = np.empty((n_base, dim), np.float32)
    queries = np.empty((n_query, dim), np.float32)
    _lib.hnsw_synthetic_mixture(n_base, n_query, dim, clusters, sigma, seed, _ptr(base), _ptr(queries))
    return base, queries


def mixture_split(n_base: int, n_query: int, dim: int, clusters: int, sigma: float, base_seed: int,
                  query_seed: int):
    """Mixture with base (and centers) from base_seed and queries from query_seed."""
    base = np.empty((n_base, dim), np.float32)
    queries = np.empty((n_query, dim), np.float32)
    _lib.hnsw_synthetic_mixture_split(n_base, n_query, dim, clusters, sigma, base_seed, query_seed, _ptr(base),
                                      _ptr(queries))
    return base, queries


def crc32(data: bytes) -> int:
    buf = np.frombuffer(data, np.uint8) if data else np.zeros(1, np.uint8)
    return int(_lib.hnsw_crc32(_ptr(buf), len(data)))


def recall_at_k(truth_keys, truth_counts, found_keys, found_counts, k: int) -> float:
    """eval::recall_at_k (src/eval.rs:25-47) over array results."""
    hits = 0
    expected = 0
    for i in range(len(truth_counts)):
        t = truth_keys[i, : min(k, int(truth_counts[i]))]
        f = found_keys[i, : min(k, int(found_counts[i]))]
        expected += t.size
        hits += int(np.isin(f, t).sum())
    return 1.0 if expected == 0 else hits / expected
