"""The validating loader (host side of hnsw_gpu_index_open), restating
io::read (src/hnsw/io.rs:236-540), against the reference's loader tests
(src/hnsw/tests.rs:452-656, tests/properties.rs:197-230). No GPU needed:
hnsw_validate_bytes runs every check that open runs before touching a device.
"""

import struct

import numpy as np
import pytest

import hnsw_gpu as H
import oracle as O
from conftest import build_index


def err(b, max_memory=None):
    with pytest.raises(H.Error) as e:
        H.validate_bytes(b, max_memory)
    return e.value


def with_valid_crc(b: bytes) -> bytes:
    body = b[:-4]
    return body + struct.pack("<I", H.crc32(body))


def test_envelope_errors():
    # src/hnsw/tests.rs:452-478.
    base, _ = H.gaussian(20, 0, 4, 1)
    data = build_index(base, parallel=False)
    assert err(b"").status == H.Status.FORMAT_TRUNCATED
    assert err(b"HNSW").status == H.Status.FORMAT_TRUNCATED
    assert err(b"not an index file").status == H.Status.FORMAT_BAD_MAGIC
    v2 = bytearray(data)
    v2[8] = 2
    e = err(bytes(v2))
    assert e.status == H.Status.FORMAT_UNSUPPORTED_VERSION and "version 2" in e.message
    flipped = bytearray(data)
    flipped[100] ^= 0x10
    e = err(bytes(flipped))
    assert e.status == H.Status.FORMAT_CHECKSUM and "checksum mismatch" in e.message
    for n in [12, 40, len(data) // 2, len(data) - 1]:
        err(data[:n])


def test_structural_violations_at_exact_offsets():
    # src/hnsw/tests.rs:488-573.
    base, _ = H.gaussian(30, 0, 4, 1)
    data = build_index(base, parallel=False)

    def invalid(offset, value):
        b = bytearray(data)
        b[offset:offset + len(value)] = value
        return err(with_valid_crc(bytes(b)))

    def field(e):
        assert e.status == H.Status.FORMAT_INVALID, e.message
        return e.invalid_field

    assert field(invalid(12, b"\x09")) == "metric"
    assert field(invalid(13, b"\x00\x01")) == "neighbor selection"
    assert field(invalid(15, b"\x02")) == "quantized flag"
    assert field(invalid(16, struct.pack("<I", 0))) == "dimension"
    assert field(invalid(20, struct.pack("<I", 1))) == "parameters"
    assert field(invalid(32, struct.pack("<d", float("nan")))) == "parameters"
    assert field(invalid(48, struct.pack("<I", 0xFFFFFFFF))) == "node count"
    assert invalid(48, struct.pack("<I", 1_000_000)).status == H.Status.FORMAT_TRUNCATED
    assert field(invalid(52, struct.pack("<I", 30))) == "entry point"
    assert field(invalid(56 + 8, struct.pack("<Q", 0))) == "duplicate live key"
    levels = 56 + 30 * 8
    assert field(invalid(levels, b"\xc8")) == "node level"
    assert field(invalid(levels + 30, b"\x07")) == "tombstone flag"
    vectors = levels + 60
    assert field(invalid(vectors, struct.pack("<f", float("inf")))) == "vector out of range"
    assert field(invalid(vectors, struct.pack("<f", 3e38))) == "vector out of range"
    links = vectors + 30 * 4 * 4
    assert field(invalid(links, struct.pack("<I", 1000))) == "neighbor count exceeds capacity"
    assert field(invalid(links + 4, struct.pack("<I", 999))) == "neighbor id"
    count = struct.unpack("<I", data[links:links + 4])[0]
    assert count >= 2
    first = data[links + 4:links + 8]
    assert field(invalid(links + 8, first)) == "duplicate neighbor id"
    longer = data[:-4] + b"\x00" * 5 + data[-4:]
    assert err(with_valid_crc(longer)).status == H.Status.FORMAT_TRAILING_BYTES


def test_implausible_levels_rejected_before_allocating():
    # src/hnsw/tests.rs:575-593.
    base, _ = H.gaussian(2000, 0, 1, 1)
    data = bytearray(build_index(base, m=64, parallel=False))
    levels = 56 + 2000 * 8
    data[levels:levels + 2000] = bytes([31]) * 2000
    assert err(with_valid_crc(bytes(data))).invalid_field == "implausible level distribution"


def test_cosine_vectors_must_be_unit_length():
    # src/hnsw/tests.rs:595-608.
    b = H.IndexBuilder(2, H.Metric.Cosine)
    b.insert_batch(np.array([1, 2], np.uint64), np.array([[1, 0], [0, 1]], np.float32))
    data = bytearray(b.to_bytes())
    vectors = 56 + 2 * 8 + 2 + 2
    data[vectors:vectors + 4] = struct.pack("<f", 2.0)
    assert err(with_valid_crc(bytes(data))).invalid_field == "cosine vector is not unit length"


@pytest.mark.parametrize("metric,quantize", [(0, False), (2, True)])
def test_memory_limit(metric, quantize):
    # src/hnsw/tests.rs:610-636: the limit is the loaded memory usage.
    base, _ = H.gaussian(3000, 0, 24, 4)
    data = build_index(base, metric=metric, m=12, quantize=quantize)
    e = err(data, max_memory=1)
    assert e.status == H.Status.MEMORY_LIMIT_EXCEEDED
    info = H.validate_bytes(data, max_memory=1 << 40)
    required = info.required_memory
    assert err(data, max_memory=required - 1).status == H.Status.MEMORY_LIMIT_EXCEEDED
    assert H.validate_bytes(data, max_memory=required).nodes == 3000


def test_default_limit_admits_low_dimensional_m0_256():
    # src/hnsw/tests.rs:638-656.
    base, _ = H.gaussian(20_000, 0, 1, 5)
    data = build_index(base, m=128)
    info = H.validate_bytes(data, max_memory=1 << 40)
    assert info.required_memory / len(data) < 48.0
    assert H.validate_bytes(data).nodes == 20_000


def test_round_trip_is_byte_identical_and_searchable():
    # src/hnsw/tests.rs:414-450 and docs/adr/0003 (saving a loaded index
    # reproduces it byte for byte): the oracle's own parser reads what the
    # library wrote, and a sequential build is deterministic.
    base, queries = H.mixture(500, 10, 8, 5, 0.35, 2)
    sel = H.NeighborSelection(True, True, False)
    b = H.IndexBuilder(8, H.Metric.Cosine, H.HnswParams(m=6, selection=sel))
    b.insert_batch(np.arange(500, dtype=np.uint64), base)
    for k in [3, 50, 499]:
        assert b.remove(k)
    b.enable_quantization()
    data = b.to_bytes()
    info = H.validate_bytes(data)
    assert (info.live, info.nodes - info.live, info.quantized) == (497, 3, 1)
    O.Index(data)  # the oracle parses it
    a1 = build_index(base, metric=0, parallel=False)
    a2 = build_index(base, metric=0, parallel=False)
    assert a1 == a2
    empty = H.IndexBuilder(3, H.Metric.L2).to_bytes()
    assert H.validate_bytes(empty).nodes == 0


def test_mutated_files_never_crash_the_loader():
    # tests/properties.rs:197-230: random mutations with a recomputed CRC are
    # either rejected or load; the loader never crashes.
    base, _ = H.gaussian(60, 0, 3, 8)
    data = build_index(base, m=4, parallel=False, quantize=True)
    rng = np.random.default_rng(1)
    body = len(data) - 4
    links = 56 + 60 * (8 + 1 + 1 + 4 * 3)
    for trial in range(1024):
        b = bytearray(data)
        start, span = (links, body - links) if trial % 2 else (0, body)
        for _ in range(int(rng.integers(1, 8))):
            b[start + int(rng.integers(span))] = int(rng.integers(256))
        try:
            H.validate_bytes(with_valid_crc(bytes(b)))
        except H.Error as e:
            assert e.status in {10, 11, 12, 13, 14, 15, 16}


def test_truncated_files_are_errors():
    base, _ = H.gaussian(40, 0, 5, 3)
    data = build_index(base, m=5, parallel=False)
    for n in range(0, len(data), max(1, len(data) // 97)):
        err(data[:n])
