"""Shared test setup: import paths for the product module and the oracle,
the `gpu` marker, and small index fixtures built with the host builder."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hnsw-index_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def build_index(base, metric=0, m=16, seed=7, ef_construction=200, parallel=True, keys=None,
                deleted_keys=(), quantize=False, selection=None, threads=0):
    """Builds a format-v1 file with the host builder (HnswIndex::insert_batch / insert)."""
    import hnsw_gpu as H

    base = np.ascontiguousarray(base, np.float32)
    n, dim = base.shape
    keys = np.arange(n, dtype=np.uint64) if keys is None else np.asarray(keys, np.uint64)
    params = H.HnswParams(m=m, ef_construction=ef_construction, seed=seed, selection=selection)
    b = H.IndexBuilder(dim, H.Metric(metric), params)
    if parallel:
        b.insert_batch(keys, base, threads=threads)
    else:
        for i in range(n):
            b.insert(int(keys[i]), base[i])
    for k in deleted_keys:
        b.remove(int(k))
    if quantize:
        b.enable_quantization()
    return b.to_bytes()
