"""CPU model of the traversal's 16-bit visited tags (visit / spill_visited in
hnsw-index_b200/csrc/traverse.cuh, set_hash_tags in csrc/device.hpp).

A hash of 2^b slots over ids below 2^B maps id to x = id * 0x9E3779B1 mod
2^B, probes linearly from home slot x >> (B - b) and stores the tag
(x mod 2^(B-b)) << dbits | d, d being the probe distance (dbits = 16 - (B -
b), d < 2^dbits - 1). The visited set decides which neighbors get distances
(src/hnsw/search.rs:120-136), so it must be exact: this model checks that
test-and-set answers equal a plain set's, that a probe longer than a tag
records is reported instead of mis-answered, and that the ids rebuilt from
slots and tags (the spill to the bitmap) are exactly the inserted ones.
"""

import numpy as np
import pytest

MUL = 0x9E3779B1
EMPTY = 0xFFFF


def inverse(k):
    x = k
    for _ in range(5):
        x = (x * (2 - k * x)) & 0xFFFFFFFF
    return x


def tag_params(n, cap, min_bits=0):
    """set_hash_tags: (sh, mask) or None when 32-bit ids are stored."""
    if min_bits < 0 or cap < 64 or cap & (cap - 1):
        return None
    b = cap.bit_length() - 1
    B = max((n - 1).bit_length() if n > 1 else 1, min_bits, b)
    B = min(B, 32)
    if B - b > (15 if min_bits > 0 else 10):
        return None
    return B - b, (1 << B) - 1


class TagHash:
    def __init__(self, cap, sh, mask):
        self.cap, self.sh, self.mask = cap, sh, mask
        self.dbits = 16 - sh
        self.slots = [EMPTY] * cap

    def visit(self, i):
        """'fresh', 'seen' or 'full', as visit() returns."""
        x = (i * MUL) & self.mask
        base = (x & ((1 << self.sh) - 1)) << self.dbits
        h = x >> self.sh
        for d in range(min((1 << self.dbits) - 1, self.cap)):
            tag = base | d
            if self.slots[h] == EMPTY:
                self.slots[h] = tag
                return "fresh"
            if self.slots[h] == tag:
                return "seen"
            h = (h + 1) & (self.cap - 1)
        return "full"

    def ids(self):
        inv = inverse(MUL)
        out = set()
        dmask = (1 << self.dbits) - 1
        for s, t in enumerate(self.slots):
            if t == EMPTY:
                continue
            home = (s - (t & dmask)) & (self.cap - 1)
            out.add((((home << self.sh) | (t >> self.dbits)) * inv) & self.mask)
        return out


def test_inverse_constant():
    assert (MUL * inverse(MUL)) & 0xFFFFFFFF == 1


@pytest.mark.parametrize("n,cap,min_bits", [(1_000_000, 4096, 0), (1_000_000, 2048, 0), (20_000, 4096, 0),
                                            (16, 64, 0), (10_000_000, 16384, 0), (5_000, 4096, 24),
                                            (5_000, 4096, 27)])
def test_tags_are_an_exact_set(n, cap, min_bits):
    sh, mask = tag_params(n, cap, min_bits)
    rng = np.random.default_rng(cap + n)
    h = TagHash(cap, sh, mask)
    truth = set()
    limit = cap * 3 // 4
    full = 0
    # Draws with repeats, up to the load limit the kernels keep.
    for i in rng.integers(0, n, size=4 * limit).tolist():
        if len(truth) >= limit:
            break
        got = h.visit(i)
        if got == "full":
            # Reported, never answered wrongly: the id is not in the set.
            assert i not in truth
            full += 1
            continue
        assert got == ("seen" if i in truth else "fresh")
        truth.add(i)
    assert h.ids() == truth
    if min_bits == 27:
        assert full > 0  # one distance bit: most collisions overflow


def test_tag_rule():
    assert tag_params(1_000_000, 4096) == (8, (1 << 20) - 1)
    assert tag_params(10_000_000, 4096) is None          # 12 bits beyond the hash
    assert tag_params(10_000_000, 16384) == (10, (1 << 24) - 1)
    assert tag_params(1_000_000, 2560) is None           # not a power of two
    assert tag_params(1_000_000, 4096, -1) is None       # turned off
    assert tag_params(5_000, 4096, 27) == (15, (1 << 27) - 1)
