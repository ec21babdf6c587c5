"""Host-side construction and the C ABI surface (no GPU needed).

Construction produces the index files the device path opens; its invariants
follow src/hnsw/tests.rs:28-79 and its determinism src/hnsw/tests.rs:129-135.
The ABI checks load libhnsw_gpu.so and confirm that every function
include/hnsw_gpu.h declares is exported, without calling into the device.
"""

import ctypes
import os
import re
import struct
from collections import deque

import numpy as np
import pytest

import hnsw_gpu as H
from conftest import ROOT, build_index, gpu_available


def parse(data: bytes):
    """Minimal parse of format v1 (src/hnsw/io.rs:3-28) for invariant checks."""
    dim, m, m0 = struct.unpack("<III", data[16:28])
    n, entry = struct.unpack("<II", data[48:56])
    off = 56 + 8 * n
    levels = list(data[off:off + n])
    off += 2 * n + 4 * n * dim
    lists = []
    for i in range(n):
        per = []
        for _layer in range(levels[i] + 1):
            c = struct.unpack("<I", data[off:off + 4])[0]
            per.append(list(struct.unpack(f"<{c}I", data[off + 4:off + 4 + 4 * c])))
            off += 4 + 4 * c
        lists.append(per)
    return dict(dim=dim, m=m, m0=m0, n=n, entry=entry, levels=levels, lists=lists)


def assert_invariants(p):
    n = p["n"]
    for i in range(n):
        for layer, nb in enumerate(p["lists"][i]):
            assert len(nb) <= (p["m0"] if layer == 0 else p["m"])
            assert len(set(nb)) == len(nb)
            for x in nb:
                assert x < n and x != i and p["levels"][x] >= layer
    if n:
        top = max(p["levels"])
        assert p["levels"][p["entry"]] == top


def reachable(p):
    n = p["n"]
    seen = [False] * n
    q = deque(i for i in range(n) if i == p["entry"] or p["levels"][i] > 0)
    for i in q:
        seen[i] = True
    count = len(q)
    while q:
        i = q.popleft()
        for x in p["lists"][i][0]:
            if not seen[x]:
                seen[x] = True
                count += 1
                q.append(x)
    return count


@pytest.mark.parametrize("selection", [H.NeighborSelection.simple(), H.NeighborSelection(),
                                       H.NeighborSelection(True, True, True)])
@pytest.mark.parametrize("parallel", [False, True])
def test_graphs_satisfy_invariants_and_stay_connected(selection, parallel):
    # src/hnsw/tests.rs:137-166.
    base, _ = H.mixture(3000, 1, 16, 20, 0.35, 5)
    b = H.IndexBuilder(16, H.Metric.L2, H.HnswParams(m=8, selection=selection))
    if parallel:
        b.insert_batch(np.arange(3000, dtype=np.uint64), base)
    else:
        for i in range(3000):
            b.insert(i, base[i])
    p = parse(b.to_bytes())
    assert_invariants(p)
    if selection.heuristic:
        assert reachable(p) >= 2970
    mean_degree = sum(len(p["lists"][i][0]) for i in range(3000)) / 3000
    assert 4.0 < mean_degree <= 16.0


def test_compaction_drops_tombstones_and_keeps_live_keys():
    # src/hnsw/tests.rs:266-291 (host link step; recall through the oracle's search).
    import oracle as O

    base, queries = H.gaussian(1000, 20, 16, 6)
    b = H.IndexBuilder(16, H.Metric.L2, H.HnswParams())
    for i in range(1000):
        b.insert(i, base[i])
    b.enable_quantization()
    for key in range(0, 1000, 3):
        assert b.remove(key)
    b.compact(threads=2)
    data = b.to_bytes()
    info = H.validate_bytes(data)
    live = 1000 - len(range(0, 1000, 3))
    assert (info.nodes, info.live, info.quantized) == (live, live, 1)
    p = parse(data)
    assert_invariants(p)
    assert reachable(p) * 100 >= live * 99
    keep = np.array([k for k in range(1000) if k % 3 != 0], np.uint64)
    tk, _, tc, _ = O.brute(0, base[keep.astype(np.int64)], queries, 10, keys=keep)
    fk, _, fc, _ = O.Index(data).search(queries, 10, 100)
    assert O.recall_at_k(tk, tc, fk, fc, 10) > 0.95
    b.compact()
    assert b.to_bytes() == data


def test_sequential_build_is_deterministic():
    base, _ = H.gaussian(500, 10, 8, 1)
    assert build_index(base, parallel=False, seed=0) == build_index(base, parallel=False, seed=0)


def test_levels_follow_geometric_distribution():
    # src/hnsw/build.rs:229-251 through the level column of a built file.
    base, _ = H.gaussian(20000, 0, 2, 3)
    p = parse(build_index(base, m=16, seed=42, ef_construction=16))
    levels = np.array(p["levels"])
    for l in (1, 2):
        expected = 20000 * 16.0 ** (-l)
        observed = (levels >= l).sum()
        assert abs(observed - expected) < 5 * np.sqrt(expected) + 2


def test_insert_rejects_invalid_input():
    # src/hnsw/tests.rs:168-206.
    b = H.IndexBuilder(2, H.Metric.Cosine)
    b.insert(1, [1.0, 0.0])
    with pytest.raises(H.Error) as e:
        b.insert(1, [0.0, 1.0])
    assert e.value.status == H.Status.DUPLICATE_KEY
    with pytest.raises(H.Error) as e:
        b.insert(2, [1.0])
    assert e.value.status == H.Status.DIMENSION_MISMATCH
    with pytest.raises(H.Error) as e:
        b.insert(2, [np.nan, 1.0])
    assert e.value.status == H.Status.NON_FINITE_VECTOR
    with pytest.raises(H.Error) as e:
        b.insert(2, [0.0, 0.0])
    assert e.value.status == H.Status.ZERO_VECTOR
    with pytest.raises(H.Error):
        b.insert_batch(np.array([2, 3], np.uint64), np.array([[1, 1], [0, 0]], np.float32))
    with pytest.raises(H.Error) as e:
        b.insert_batch(np.array([2, 2], np.uint64), np.array([[1, 1], [1, 2]], np.float32))
    assert e.value.status == H.Status.DUPLICATE_KEY
    assert H.validate_bytes(b.to_bytes()).nodes == 1


def test_constructor_validates_dimension_and_params():
    # src/hnsw/tests.rs:97-111 and src/params.rs:214-223.
    with pytest.raises(H.Error) as e:
        H.IndexBuilder(0, H.Metric.L2)
    assert e.value.status == H.Status.INVALID_DIMENSION
    with pytest.raises(H.Error):
        H.IndexBuilder(H.MAX_DIM + 1, H.Metric.L2)
    for p in [H.HnswParams(m=1), H.HnswParams(m=513), H.HnswParams(m=16, m0=15),
              H.HnswParams(m=16, m0=4096), H.HnswParams(m=16, ef_construction=0),
              H.HnswParams(m=16, level_multiplier=0.0), H.HnswParams(m=16, level_multiplier=float("nan")),
              H.HnswParams(m=16, level_multiplier=11.0)]:
        with pytest.raises(H.Error) as e:
            H.IndexBuilder(4, H.Metric.L2, p)
        assert e.value.status == H.Status.INVALID_PARAMETER


def header_functions():
    text = open(os.path.join(ROOT, "include", "hnsw_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hnsw_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(H.LIBRARY_PATH)
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/hnsw_gpu.h but not exported"
    assert set(H.EXPORTED_SYMBOLS) <= set(names)


@pytest.mark.skipif(gpu_available(), reason="checks the behaviour on a host without a CUDA device")
def test_device_paths_fail_loudly_without_a_gpu():
    # There is no CPU search path behind the device API: without a CUDA
    # device, opening an index and loading brute-force rows are CUDA errors.
    base, _ = H.gaussian(200, 0, 8, 1)
    data = build_index(base)
    with pytest.raises(H.Error) as e:
        H.HnswIndex.from_bytes(data)
    assert e.value.status == H.Status.CUDA
    bf = H.BruteForceIndex(8, H.Metric.L2)
    with pytest.raises(H.Error) as e:
        bf.insert_batch(np.arange(200, dtype=np.uint64), base)
    assert e.value.status == H.Status.CUDA


def test_null_handles_are_rejected_without_touching_the_device():
    # Every entry point checks its handle before any CUDA call: a null
    # handle is INVALID_ARGUMENT with a message, and the close/free calls
    # accept null (no compute is launched, so this runs on any host).
    lib = ctypes.CDLL(H.LIBRARY_PATH)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    lib.hnsw_last_error.restype = ctypes.c_char_p
    calls = {
        "hnsw_gpu_index_info": ([vp, vp], (None, None)),
        "hnsw_gpu_set_tombstones": ([vp, vp, sz], (None, None, 0)),
        "hnsw_gpu_search_batch": ([vp, vp, sz, sz, vp, vp, vp, vp, vp], (None, None, 1, 8, None, None, None, None,
                                                                         None)),
        "hnsw_gpu_search_batch_device": ([vp, vp, sz, sz, vp, vp, vp, vp, vp, vp],
                                         (None, None, 1, 8, None, None, None, None, None, None)),
        "hnsw_gpu_graph_launch": ([vp, vp], (None, None)),
        "hnsw_gpu_clear_tuning": ([vp], (None,)),
        "hnsw_gpu_set_counters": ([vp, ctypes.c_int], (None, 1)),
        "hnsw_gpu_read_counters": ([vp, vp, sz], (None, None, 1)),
        "hnsw_gpu_server_start": ([vp, vp, vp], (None, None, None)),
        "hnsw_gpu_server_stats": ([vp, vp, vp], (None, None, None)),
        "hnsw_builder_insert": ([vp, ctypes.c_uint64, vp, sz], (None, 1, None, 8)),
        "hnsw_builder_enable_quantization": ([vp], (None,)),
    }
    for name, (argtypes, args) in calls.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = ctypes.c_int
        assert fn(*args) == H.Status.INVALID_ARGUMENT, name
        assert lib.hnsw_last_error(), name
    for name in ("hnsw_gpu_index_close", "hnsw_gpu_graph_destroy", "hnsw_gpu_server_stop", "hnsw_gpu_brute_close",
                 "hnsw_builder_free"):
        fn = getattr(lib, name)
        fn.argtypes = [vp]
        fn.restype = None
        fn(None)
