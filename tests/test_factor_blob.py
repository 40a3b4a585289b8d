"""Factor blobs (Factor.save / load) on the host: the header, size and
checksum validation of mpchol_factor_blob_check, against blobs built here
from the documented layout (no device needed).  The device round trip is in
tests/test_gpu_solver.py."""
import struct

import numpy as np
import pytest

import cholesky_gpu_b200 as mp
from cholesky_gpu_b200 import MpcholError

STEP_BYTES = 32      # StepState: eight 32-bit fields
STATUS_BYTES = 16    # DevStatus: four 32-bit fields


def l_bytes(n, b):
    return sum((n - c) * min(b, n - c) * 4 for c in range(0, n, b))


def fnv64_words(payload: bytes) -> int:
    """64-bit FNV-1a over little-endian 8-byte words, the tail zero-padded."""
    h = 0xCBF29CE484222325
    pad = payload + b"\0" * (-len(payload) % 8)
    for (w,) in struct.iter_unpack("<Q", pad):
        h = ((h ^ w) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def make_blob(n, b, seed=0):
    ns = -(-n // b)
    lb = l_bytes(n, b)
    payload = np.random.default_rng(seed).bytes(lb + (ns + 1) * STEP_BYTES + 8 * n + STATUS_BYTES)
    total = 64 + len(payload)
    head = struct.pack("<8sIIiiiIQQQQ", b"MPCHOLF1", 1, 64, n, b, ns, STEP_BYTES, lb, total,
                       fnv64_words(payload), 0)
    assert len(head) == 64
    return head + payload


@pytest.mark.parametrize("n,b", [(70, 32), (256, 256), (1000, 128), (33, 64)])
def test_valid_blob_is_accepted(n, b):
    assert mp.factor_blob_info(make_blob(n, b)) == (n, b)


def corrupt(blob, offset, fmt, value):
    out = bytearray(blob)
    struct.pack_into(fmt, out, offset, value)
    return bytes(out)


@pytest.mark.parametrize("what", ["magic", "version", "n", "block", "nsteps", "l_bytes", "total",
                                  "checksum", "payload", "truncated", "short"])
def test_invalid_blob_is_rejected(what):
    blob = make_blob(300, 64, seed=3)
    bad = {
        "magic": lambda: b"MPCHOLF2" + blob[8:],
        "version": lambda: corrupt(blob, 8, "<I", 2),
        "n": lambda: corrupt(blob, 16, "<i", 301),
        "block": lambda: corrupt(blob, 20, "<i", 48),
        "nsteps": lambda: corrupt(blob, 24, "<i", 4),
        "l_bytes": lambda: corrupt(blob, 32, "<Q", l_bytes(300, 64) + 4),
        "total": lambda: corrupt(blob, 40, "<Q", len(blob) + 8),
        "checksum": lambda: corrupt(blob, 48, "<Q", 12345),
        "payload": lambda: blob[:100] + bytes([blob[100] ^ 1]) + blob[101:],
        "truncated": lambda: blob[:-1],
        "short": lambda: blob[:40],
    }[what]()
    with pytest.raises(MpcholError):
        mp.factor_blob_info(bad)


@pytest.mark.parametrize("n", [(1 << 24) + 1, 2**31 - 1, 2**31 - 200])
def test_hostile_order_is_rejected_before_size_arithmetic(n):
    """An order near INT_MAX (whose step count and size loop would overflow
    or run for a very long time) is rejected by the bound on n alone."""
    blob = make_blob(300, 64, seed=4)
    bad = corrupt(corrupt(blob, 16, "<i", n), 24, "<i", -(-n // 64))
    with pytest.raises(MpcholError):
        mp.factor_blob_info(bad)
