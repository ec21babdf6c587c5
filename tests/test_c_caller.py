"""The C ABI from a plain C caller (what cgo or a Rust extern block binds):
include/hnsw_gpu.h compiles as strict C99, and a C program linked against
libhnsw_gpu.so runs the host-side entry points (CRC-32, synthetic data,
building, serialising and validating an index, error reporting). No GPU
entry point is called."""

import os
import shutil
import subprocess

import pytest

import hnsw_gpu as H
from conftest import ROOT

C_PROGRAM = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "hnsw_gpu.h"

#define CHECK(cond) do { if (!(cond)) { printf("FAILED %s:%d %s\n", __FILE__, __LINE__, #cond); return 1; } } while (0)

int main(void) {
    /* src/crc32.rs:103-111 check value. */
    CHECK(hnsw_crc32((const uint8_t*)"123456789", 9) == 0xCBF43926u);

    enum { N = 300, D = 16 };
    float* base = malloc(sizeof(float) * N * D);
    float* queries = malloc(sizeof(float) * 4 * D);
    hnsw_synthetic_gaussian(N, 4, D, 42, base, queries);

    hnsw_params p;
    hnsw_params_default(12, &p);
    CHECK(p.m == 12 && p.m0 == 24 && p.ef_construction == 200);
    hnsw_builder* b = NULL;
    CHECK(hnsw_builder_new(D, HNSW_METRIC_L2, &p, &b) == HNSW_OK && b != NULL);
    for (uint64_t i = 0; i < N; ++i) CHECK(hnsw_builder_insert(b, 1000 + i, base + i * D, D) == HNSW_OK);

    /* Errors: a duplicate key and a wrong dimension, with messages. */
    CHECK(hnsw_builder_insert(b, 1000, base, D) == HNSW_ERR_DUPLICATE_KEY);
    CHECK(strlen(hnsw_last_error()) > 0);
    CHECK(hnsw_builder_insert(b, 5, base, D - 1) == HNSW_ERR_DIMENSION_MISMATCH);

    int removed = 0;
    CHECK(hnsw_builder_remove(b, 1003, &removed) == HNSW_OK && removed == 1);

    uint8_t* bytes = NULL;
    size_t len = 0;
    CHECK(hnsw_builder_to_bytes(b, &bytes, &len) == HNSW_OK && len > 0);
    hnsw_index_info info;
    CHECK(hnsw_validate_bytes(bytes, len, 0, &info) == HNSW_OK);
    CHECK(info.dim == D && info.nodes == N && info.live == N - 1 && info.m == 12 && info.m0 == 24);

    /* A flipped body byte fails the checksum (FormatError::ChecksumMismatch). */
    bytes[len / 2] ^= 0x40;
    CHECK(hnsw_validate_bytes(bytes, len, 0, NULL) == HNSW_ERR_FORMAT_CHECKSUM);
    /* A short file is truncated (FormatError::Truncated). */
    CHECK(hnsw_validate_bytes(bytes, 20, 0, NULL) == HNSW_ERR_FORMAT_TRUNCATED);

    hnsw_bytes_free(bytes);
    hnsw_builder_free(b);
    free(base);
    free(queries);
    printf("ok\n");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_c_program_uses_the_host_entry_points(tmp_path):
    src = tmp_path / "caller.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(H.LIBRARY_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", libdir, "-lhnsw_gpu", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ok")
