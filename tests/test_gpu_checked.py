"""The checked build (libhnsw_gpu_checked.so, HNSW_DEVICE_CHECKS) on small
cases: every node id, array capacity, cold-list chunk and output row the
traversal kernels use is checked before the access; a violation is recorded
(site, value) and skipped instead of faulting. Each case must give the
oracle's results bit for bit and leave the check word at zero.

The checked library is loaded in a child process (HNSW_GPU_LIB=checked), so
this process keeps the normal one.
"""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r"""
import json, sys
import numpy as np
import hnsw_gpu as H
import oracle as O
from conftest import build_index

assert H.checked_build(), "the checked library did not load"
out = []

def same(got, ref):
    gk, gd, gc, gs = got
    rk, rd, rc, rs = ref
    if not (np.array_equal(gs, rs) and np.array_equal(gc, rc)):
        return False
    for i in range(len(gc)):
        c = int(gc[i])
        if not (np.array_equal(gk[i, :c], rk[i, :c]) and np.array_equal(gd[i, :c].view(np.uint32), rd[i, :c].view(np.uint32))):
            return False
    return True

def case(name, gi, got, ref):
    out.append({"case": name, "same": bool(same(got, ref)) if ref is not None else True, "check": gi.check_word()})

# Complete graph: 16 nodes with M = 16, so the search equals brute force.
base, queries = H.gaussian(16, 20, 8, 3)
data = build_index(base, metric=0, m=16, seed=1)
gi, oi = H.HnswIndex.from_bytes(data), O.Index(data)
for k, ef in [(1, 1), (5, 16), (16, 32)]:
    case(f"complete k={k} ef={ef}", gi, gi.search_arrays(queries, k, ef), oi.search(queries, k, ef))

# 2000 nodes, both modes, an ef sweep; then a small schedule that sends
# queries through the spill areas and retry passes.
base, queries = H.gaussian(2000, 100, 32, 5)
data = build_index(base, metric=0, m=8, seed=2)
gi, oi = H.HnswIndex.from_bytes(data), O.Index(data)
for mode in (0, 1):
    for ef in (1, 16, 64, 200):
        case(f"gaussian mode={mode} ef={ef}", gi, gi.search_arrays(queries, 10, ef, mode=mode),
             oi.search(queries, 10, ef))
keys = np.arange(2000, dtype=np.uint64)
bits = H.key_bitmap(keys[keys % 40 == 7], 2000)
for mode in (0, 1):
    for cold in (0, 1):
        gi.set_schedule(ef_cap=64, cand_cap=64, hash_cap=1024, warps_per_block=4, cold=cold)
        case(f"selective filter mode={mode} cold={cold}", gi,
             gi.search_arrays(queries, 10, 48, filter_bits=bits, filter_nbits=2000, mode=mode),
             oi.search(queries, 10, 48, filter_bits=bits, filter_nbits=2000))
gi.set_schedule()

# Tombstones, int8 traversal, inner product.
base, queries = H.mixture(2000, 100, 24, 10, 0.4, 9)
dead = list(range(0, 2000, 11))
data = build_index(base, metric=1, m=8, seed=3, deleted_keys=dead, quantize=True)
gi, oi = H.HnswIndex.from_bytes(data), O.Index(data)
for mode in (0, 1):
    case(f"int8 tombstones mode={mode}", gi, gi.search_arrays(queries, 10, 64, quantized=True, mode=mode),
         oi.search(queries, 10, 64, quantized=True))

# Tensor-core traversal (results checked against the f32 search elsewhere;
# here only the checks).
base, queries = H.gaussian(2000, 100, 64, 7)
data = build_index(base, metric=0, m=8, seed=4)
gi = H.HnswIndex.from_bytes(data)
for trav in (H.Traversal.BF16, H.Traversal.BF16X3):
    case(f"tensor-core traversal {int(trav)}", gi, gi.search_arrays(queries, 10, 64, traversal=trav), None)
print(json.dumps(out))
"""


def test_checked_build_small_cases_exact_and_clean():
    lib = os.path.join(ROOT, "hnsw-index_b200", "libhnsw_gpu_checked.so")
    if not os.path.exists(lib):
        pytest.fail(f"{lib} is missing: build it with `make -C hnsw-index_b200 checked`")
    env = dict(os.environ, HNSW_GPU_LIB="checked")
    env["PYTHONPATH"] = os.pathsep.join([os.path.join(ROOT, "hnsw-index_b200"), os.path.join(ROOT, "oracle"), HERE,
                                         env.get("PYTHONPATH", "")])
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=600,
                       cwd=HERE)
    assert r.returncode == 0, r.stderr[-3000:]
    results = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(results) == 19
    for res in results:
        assert res["same"], res
        assert res["check"] == [0, 0], res
