"""Device ingest (hnsw_gpu_index_open) against the host loader
(hnsw_validate_bytes): every corruption the reference's loader tests make
(src/hnsw/tests.rs:452-656, tests/properties.rs:197-230) must give the same
status and message through both, including the checksum message, whose
computed CRC comes from the device; valid files must open and search."""

import struct

import numpy as np
import pytest

import hnsw_gpu as H
from conftest import build_index

pytestmark = pytest.mark.gpu


def outcome(fn, b):
    try:
        fn(b)
        return None
    except H.Error as e:
        return (int(e.status), e.message)


def same_outcome(b):
    host = outcome(lambda x: H.validate_bytes(x), b)
    dev = outcome(lambda x: H.HnswIndex.from_bytes(x).close(), b)
    assert host == dev, (host, dev)
    return host


def with_valid_crc(b: bytes) -> bytes:
    body = b[:-4]
    return body + struct.pack("<I", H.crc32(body))


def test_envelope_and_checksum():
    base, _ = H.gaussian(20, 0, 4, 1)
    data = build_index(base, parallel=False)
    for b in [b"", b"HNSW", b"not an index file", data[:12], data[:40], data[:-1]]:
        assert same_outcome(b) is not None
    v2 = bytearray(data)
    v2[8] = 2
    assert same_outcome(bytes(v2))[0] == H.Status.FORMAT_UNSUPPORTED_VERSION
    for pos in (0, 13, 100, len(data) // 2, len(data) - 5, len(data) - 1):
        flipped = bytearray(data)
        flipped[pos] ^= 0x10
        same_outcome(bytes(flipped))


def test_structural_violations_at_exact_offsets():
    base, _ = H.gaussian(30, 0, 4, 1)
    data = build_index(base, parallel=False)

    def invalid(offset, value):
        b = bytearray(data)
        b[offset:offset + len(value)] = value
        return same_outcome(with_valid_crc(bytes(b)))

    levels = 56 + 30 * 8
    vectors = levels + 60
    links = vectors + 30 * 4 * 4
    count = struct.unpack("<I", data[links:links + 4])[0]
    first = data[links + 4:links + 8]
    cases = [(12, b"\x09"), (13, b"\x00\x01"), (15, b"\x02"), (16, struct.pack("<I", 0)), (20, struct.pack("<I", 1)),
             (32, struct.pack("<d", float("nan"))), (48, struct.pack("<I", 0xFFFFFFFF)),
             (48, struct.pack("<I", 1_000_000)), (52, struct.pack("<I", 30)), (56 + 8, struct.pack("<Q", 0)),
             (levels, b"\xc8"), (levels + 30, b"\x07"), (vectors, struct.pack("<f", float("inf"))),
             (vectors, struct.pack("<f", 3e38)), (links, struct.pack("<I", 1000)),
             (links + 4, struct.pack("<I", 999)), (links + 8, first)]
    assert count >= 2
    for off, val in cases:
        assert invalid(off, val) is not None
    longer = data[:-4] + b"\x00" * 5 + data[-4:]
    assert same_outcome(with_valid_crc(longer))[0] == H.Status.FORMAT_TRAILING_BYTES
    # The earliest failing list wins, as for a sequential reader.
    b = bytearray(data)
    b[links + 4:links + 8] = struct.pack("<I", 999)
    same_outcome(with_valid_crc(bytes(b)))


def test_cosine_and_quantized_files():
    b = H.IndexBuilder(2, H.Metric.Cosine)
    b.insert_batch(np.array([1, 2], np.uint64), np.array([[1, 0], [0, 1]], np.float32))
    data = bytearray(b.to_bytes())
    vectors = 56 + 2 * 10
    data[vectors:vectors + 4] = struct.pack("<f", 0.5)
    assert same_outcome(with_valid_crc(bytes(data)))[1].endswith("cosine vector is not unit length")
    base, _ = H.gaussian(300, 0, 12, 5)
    q = build_index(base, m=6, parallel=False, quantize=True, deleted_keys=[3, 7])
    assert same_outcome(q) is None
    qb = bytearray(q)
    qb[-8:-4] = struct.pack("<f", -1.0)  # quantizer scale
    same_outcome(with_valid_crc(bytes(qb)))


def test_mutated_and_truncated_files():
    base, _ = H.gaussian(60, 0, 3, 8)
    data = build_index(base, m=4, parallel=False, quantize=True)
    rng = np.random.default_rng(2)
    body = len(data) - 4
    links = 56 + 60 * (8 + 1 + 1 + 4 * 3)
    for trial in range(300):
        b = bytearray(data)
        start, span = (links, body - links) if trial % 2 else (0, body)
        for _ in range(int(rng.integers(1, 8))):
            b[start + int(rng.integers(span))] = int(rng.integers(256))
        same_outcome(with_valid_crc(bytes(b)))
    for n in range(0, len(data), max(1, len(data) // 61)):
        same_outcome(data[:n])


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 20000])
def test_device_crc_over_sizes_and_valid_opens(n):
    base, queries = H.gaussian(n, 5, 7, 40 + n)
    data = build_index(base, m=5, parallel=n > 100) if n else build_index(np.zeros((0, 7), np.float32))
    assert same_outcome(data) is None
    gi = H.HnswIndex.from_bytes(data)
    info = H.validate_bytes(data)
    assert gi.info().nodes == info.nodes and gi.info().live == info.live and gi.info().entry == info.entry
    if n:
        keys, _, count, _ = gi.search_arrays(queries, 3, 16)
        assert (count == min(3, n)).all()
    bad = bytearray(data)
    bad[len(bad) // 3] ^= 0x01
    same_outcome(bytes(bad))
