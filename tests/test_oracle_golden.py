"""The CPU oracle pinned against the reference's own known answers.

Each value comes from a test of the hnsw-index crate (file:line given); the
oracle must reproduce it before it is trusted as the checker of the GPU
path.
"""

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O


def test_splitmix64_reference_outputs():
    # src/synthetic.rs:182-187 (Vigna's splitmix64.c seeded with 1234567).
    assert list(O.splitmix(1_234_567, 2)) == [6_457_827_717_110_365_317, 3_203_168_211_198_807_973]


def test_dataset_matches_python_generator_golden():
    # tests/recall.rs:130-138: first components of Dataset::gaussian(10_000, 200, 128, 42).
    base, _ = O.gaussian(10, 0, 128, 42)
    want = [0.8822489, -0.45084986, 0.18835263]
    assert np.all(np.abs(base[0, :3] - np.array(want, np.float32)) < 1e-6)
    pb, _ = H.gaussian(10, 0, 128, 42)
    assert np.array_equal(base, pb)


def test_mixture_generator_matches_between_oracle_and_library():
    a = O.clustered(500, 20, 16, 7, 0.3, 1)
    b = H.mixture(500, 20, 16, 7, 0.3, 1)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_split_mixture_streams_match_sequential_generators():
    # Base (and centers) come from one SplitMix64 stream exactly as
    # Dataset::clustered draws them (src/synthetic.rs:102-124); queries from
    # their own stream. The library fills both in parallel chunks.
    base, queries = H.mixture_split(5000, 3, 16, 7, 0.3, 1, 2)
    ob, _ = O.clustered(5000, 0, 16, 7, 0.3, 1)
    assert np.array_equal(base, ob)
    centers, _ = O.gaussian(7, 0, 16, 1)  # the first 7*16 Gaussians of stream 1

    mask = (1 << 64) - 1

    def mix(z):
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        return z ^ (z >> 31)

    state = 2
    import math

    def nxt():
        nonlocal state
        state = (state + 0x9E3779B97F4A7C15) & mask
        return mix(state)

    for i in range(3):
        c = (nxt() * 7) >> 64
        for j in range(16):
            u1 = 1.0 - (nxt() >> 11) * (1.0 / (1 << 53))
            u2 = (nxt() >> 11) * (1.0 / (1 << 53))
            g = math.sqrt(-2.0 * math.log(u1)) * math.cos(math.tau * u2)
            # centers are float64 in the generator; the f32 copy from O.gaussian is only used
            # to locate the cluster (tolerance covers the f32 rounding of the center).
            assert abs(queries[i, j] - (float(centers[c, j]) + 0.3 * g)) < 1e-5


@pytest.mark.parametrize("data,want", [(b"123456789", 0xCBF43926), (b"", 0),
                                       (b"The quick brown fox jumps over the lazy dog", 0x414FA339)])
def test_crc32_check_values(data, want):
    # src/crc32.rs:103-111.
    assert O.crc32(data) == want
    assert H.crc32(data) == want


def test_crc32_matches_bitwise_reference_for_many_lengths():
    # src/crc32.rs:113-127 and tests/properties.rs:232-247 (bitwise CRC).
    data = bytes(((i * 31) ^ (i >> 3)) & 0xFF for i in range(1000))

    def bitwise(b):
        c = 0xFFFFFFFF
        for x in b:
            c ^= x
            for _ in range(8):
                c = (c >> 1) ^ 0xEDB88320 if c & 1 else c >> 1
        return c ^ 0xFFFFFFFF

    for n in [0, 1, 7, 8, 9, 63, 64, 65, 1000]:
        assert H.crc32(data[:n]) == bitwise(data[:n]) == O.crc32(data[:n])


def test_scalar_kernel_known_values():
    # src/kernels/scalar.rs:28-33.
    assert O.dot_scalar([1.0, -2.0, 0.5], [3.0, 4.0, 2.0]) == -4.0
    assert O.l2_scalar([1.0, -2.0, 0.5], [3.0, 4.0, 2.0]) == 42.25
    assert O.dot_scalar([], []) == 0.0


def test_kernels_exact_on_small_integers():
    # tests/kernels.rs:83-96: every summation order gives the exact result.
    a = np.array([(i % 7) - 3.0 for i in range(133)], np.float32)
    b = np.array([(i % 5) - 2.0 for i in range(133)], np.float32)
    want_dot = float(np.dot(a.astype(np.float64), b.astype(np.float64)))
    want_l2 = float(np.sum((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    for f_dot, f_l2 in [(O.dot, O.l2), (O.dot_portable, O.l2_portable)]:
        assert f_dot(a, b) == want_dot
        assert f_l2(a, b) == want_l2


def test_avx2_order_kernels_agree_with_scalar_within_tolerance():
    # tests/kernels.rs:11-71: |x - scalar| <= (len + 4) * eps * sum|terms|.
    rng = np.random.default_rng(0)
    for n in range(0, 81):
        a = rng.uniform(-100, 100, n).astype(np.float32)
        b = rng.uniform(-100, 100, n).astype(np.float32)
        eps = np.finfo(np.float32).eps
        tol_d = (n + 4) * eps * float(np.abs(a * b).sum()) + np.finfo(np.float32).tiny
        tol_l = (n + 4) * eps * float(((a - b) ** 2).sum()) + np.finfo(np.float32).tiny
        assert abs(O.dot(a, b) - O.dot_scalar(a, b)) <= tol_d
        assert abs(O.l2(a, b) - O.l2_scalar(a, b)) <= tol_l
        # The intrinsics and the portable restatement of the AVX2 order agree bit for bit.
        assert np.float32(O.dot(a, b)) == np.float32(O.dot_portable(a, b))
        assert np.float32(O.l2(a, b)) == np.float32(O.l2_portable(a, b))


def test_empty_slices_have_zero_distance():
    # src/kernels/mod.rs:268-274.
    assert O.dot([], []) == 0.0 and O.l2([], []) == 0.0


def test_metric_known_answers_including_negative_zero():
    # src/metric.rs:78-87.
    a, b = [1.0, 0.0], [0.0, 1.0]
    assert O.distance(0, a, b) == 2.0
    ip = O.distance(1, a, b)
    assert ip == 0.0 and np.signbit(ip)
    assert O.distance(2, a, b) == 1.0
    assert O.distance(2, a, a) == 0.0


def test_int8_kernels_match_naive_and_extremes():
    # src/kernels/int8.rs:68-85.
    for n in range(80):
        a = np.array([((i * 37) % 255) for i in range(n)], np.int64).astype(np.uint8).view(np.int8)
        b = np.array([((i * 91 + 13) % 255) for i in range(n)], np.int64).astype(np.uint8).view(np.int8)
        assert O.i8_dot(a, b) == int(np.dot(a.astype(np.int64), b.astype(np.int64)))
        assert O.i8_l2(a, b) == int(((a.astype(np.int64) - b.astype(np.int64)) ** 2).sum())
    dim = 1 << 16
    a = np.full(dim, 127, np.int8)
    b = np.full(dim, -127, np.int8)
    assert O.i8_dot(a, b) == -(127 * 127) * dim
    assert O.i8_l2(a, b) == 254 * 254 * dim


def test_quantizer_known_answer():
    # src/quantization.rs:126-136: offsets [1, 20], scale 10/127, clamping to +-127.
    b = H.IndexBuilder(2, H.Metric.L2)
    b.insert_batch(np.array([0, 1], np.uint64), np.array([[0.0, 10.0], [2.0, 30.0]], np.float32))
    b.enable_quantization()
    data = b.to_bytes()
    body = data[:-4]
    offsets = np.frombuffer(body[-12:-4], np.float32)
    scale = np.frombuffer(body[-4:], np.float32)[0]
    assert list(offsets) == [1.0, 20.0]
    assert abs(scale - 10.0 / 127.0) < 1e-6
    assert list(O.sq_encode([1000.0, -1000.0], offsets, scale)) == [127, -127]
    ip = H.IndexBuilder(2, H.Metric.InnerProduct)
    ip.insert_batch(np.array([0, 1], np.uint64), np.array([[0.0, 10.0], [2.0, 30.0]], np.float32))
    ip.enable_quantization()
    body = ip.to_bytes()[:-4]
    assert list(np.frombuffer(body[-12:-4], np.float32)) == [0.0, 0.0]


def test_degenerate_quantizer_scale_is_one():
    # src/quantization.rs:139-145.
    b = H.IndexBuilder(3, H.Metric.L2)
    b.insert_batch(np.array([0, 1], np.uint64), np.ones((2, 3), np.float32))
    b.enable_quantization()
    body = b.to_bytes()[:-4]
    assert np.frombuffer(body[-4:], np.float32)[0] == 1.0


def test_prepare_query_validation():
    # src/vector.rs:110-159.
    st, out = O.prepare_query(2, [3.0, 4.0])
    assert st == 0 and abs(out[0] - 0.6) < 1e-7 and abs(out[1] - 0.8) < 1e-7
    st, out = O.prepare_query(2, [0.0, 2.0])
    assert st == 0 and list(out) == [0.0, 1.0]
    assert O.prepare_query(0, [np.nan, 1.0])[0] == 3
    assert O.prepare_query(1, [np.inf, 1.0])[0] == 3
    assert O.prepare_query(0, [np.finfo(np.float32).max] * 2)[0] == 3
    assert O.prepare_query(2, [0.0, 0.0])[0] == 4
    assert O.prepare_query(0, [1.3e19])[0] == 3
    # Squared norm just above f32::MAX / 8 (and below 2^125) is rejected.
    assert O.prepare_query(0, [6.521909e18])[0] == 3
    assert O.prepare_query(0, [6.5219e18])[0] == 0
    assert O.prepare_query(0, [0.0, 0.0])[0] == 0


def test_brute_force_ties_break_by_key():
    # src/brute.rs:218-252.
    base = np.array([[5.0], [3.0], [9.0], [1.0]], np.float32)
    keys = np.array([5, 3, 9, 1], np.uint64)
    k, d, c, s = O.brute(0, base, np.array([[4.0]], np.float32), 3, keys=keys)
    assert list(k[0, :3]) == [3, 5, 1] and d[0, 0] == 1.0
    k, d, c, s = O.brute(0, base, np.array([[4.0]], np.float32), 100, keys=keys)
    assert c[0] == 4
    k, d, c, s = O.brute(0, np.array([[1.0], [-1.0], [1.0]], np.float32), np.array([[0.0]], np.float32), 3,
                         keys=np.array([7, 2, 4], np.uint64))
    assert list(k[0]) == [2, 4, 7]


def test_recall_at_k_known_answers():
    # src/eval.rs:59-73.
    t = np.array([[1, 2, 3], [4, 5, 6]], np.uint64)
    f = np.array([[3, 2, 1], [4, 9, 8]], np.uint64)
    c = np.array([3, 3], np.uint32)
    assert abs(O.recall_at_k(t, c, f, c, 3) - 4 / 6) < 1e-12
    assert O.recall_at_k(t, c, f, c, 1) == 0.5
    one = np.array([[1]], np.uint64)
    assert O.recall_at_k(one, np.array([1], np.uint32), one, np.array([1], np.uint32), 10) == 1.0
    assert O.recall_at_k(np.array([[1, 2]], np.uint64), np.array([2], np.uint32),
                         np.zeros((1, 2), np.uint64), np.array([0], np.uint32), 2) == 0.0


def _seq_build(base, m):
    # The oracle's own restatement of construction, one node at a time in id
    # order (the graph of repeated HnswIndex::insert).
    return O.build(base, metric=0, m=m, threads=1)


@pytest.fixture(scope="module")
def gaussian_10k_truth():
    base, queries = O.gaussian(10_000, 200, 128, 42)
    tk, td, tc, ts = O.brute(0, base, queries, 10)
    return base, queries, tk, tc


def test_recall_pin_m32(gaussian_10k_truth):
    # tests/recall.rs:43-51: >= 0.95 (0.9620 printed by the reference).
    base, queries, tk, tc = gaussian_10k_truth
    ix = O.Index(_seq_build(base, 32))
    k, d, c, s = ix.search(queries, 10, 100)
    r = O.recall_at_k(tk, tc, k, c, 10)
    assert r >= 0.95
    assert abs(r - 0.9620) <= 0.005


def test_recall_pin_m16_within_002_of_hnswlib(gaussian_10k_truth):
    # tests/recall.rs:53-72: within 0.02 of hnswlib's 0.889 (0.8900 printed).
    base, queries, tk, tc = gaussian_10k_truth
    ix = O.Index(_seq_build(base, 16))
    k, d, c, s = ix.search(queries, 10, 100)
    r = O.recall_at_k(tk, tc, k, c, 10)
    assert abs(r - 0.889) <= 0.02


def test_quantized_recall_pin(gaussian_10k_truth):
    # tests/recall.rs:115-128: int8 traversal + re-rank keeps recall >= 0.93.
    base, queries, tk, tc = gaussian_10k_truth
    b = H.IndexBuilder(128, H.Metric.L2, H.HnswParams(m=32))
    for i in range(base.shape[0]):
        b.insert(i, base[i])
    b.enable_quantization()
    ix = O.Index(b.to_bytes())
    k, d, c, s = ix.search(queries, 10, 100, quantized=True)
    assert O.recall_at_k(tk, tc, k, c, 10) >= 0.93


def test_clustered_recall_pin():
    # tests/recall.rs:74-82: clustered 10k (50 clusters, spread 0.35) >= 0.95 with M=16.
    base, queries = O.clustered(10_000, 200, 128, 50, 0.35, 42)
    tk, td, tc, ts = O.brute(0, base, queries, 10)
    ix = O.Index(_seq_build(base, 16))
    k, d, c, s = ix.search(queries, 10, 100)
    assert O.recall_at_k(tk, tc, k, c, 10) >= 0.95
