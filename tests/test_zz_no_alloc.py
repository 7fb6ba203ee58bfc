"""The scan entry point that allocates nothing (gpgmp_exclusive_scan_u32_noalloc).

It serves callers that may not allocate device memory themselves, such as code whose
device memory is owned by another allocator or that cannot afford cudaMalloc inside a
time loop; its scratch is a fixed array built into the library.  Called through the
C ABI on two calls in a row, its output must equal both the caller-scratch scan
(gpgmp_exclusive_scan_u32) and the oracle's prefix sums bit for bit -- the second
call also shows that the shared array is cleared between calls -- including at the
largest size the array serves (2^26 values, where it is an exact fit) and at the
edges of the scan's 16384-value tiles; its status query must report no look-back
timeout.  This file is collected last on purpose, and passes both alone in a fresh
process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

MAX_N = 1 << 26
TILE = 16384


def _lib():
    from inchman_b200 import _lib as L
    lib = L.lib()
    f = lib.gpgmp_exclusive_scan_u32_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    s = lib.gpgmp_exclusive_scan_u32_noalloc_status
    s.restype = C.c_int
    s.argtypes = [C.c_void_p, C.POINTER(C.c_int32)]
    g = lib.gpgmp_exclusive_scan_u32
    g.restype = C.c_int
    g.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_size_t, C.c_void_p]
    q = lib.gpgmp_scan_scratch_bytes
    q.restype = C.c_int
    q.argtypes = [C.c_int64, C.POINTER(C.c_size_t)]
    return lib


def _scratch_scan(lib, x, torch):
    n = x.numel()
    out = torch.empty_like(x)
    nb = C.c_size_t(0)
    assert lib.gpgmp_scan_scratch_bytes(n, C.byref(nb)) == 0
    scratch = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    rc = lib.gpgmp_exclusive_scan_u32(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), n,
                                      C.c_void_p(scratch.data_ptr()), nb.value, None)
    assert rc == 0
    return out


@pytest.mark.parametrize("n", [1, TILE - 1, TILE, TILE + 1, 2 * TILE + 1, 3_000_001, MAX_N])
def test_noalloc_scan_matches_oracle_and_scan_on_two_calls(n):
    import torch
    lib = _lib()
    rng = np.random.default_rng(n)
    for call in range(2):
        xh = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
        xh[: min(n, 5)] = 0xFFFFFFFF          # the sums wrap mod 2^32
        want = np.zeros(n, np.uint32)
        oracle.orc().orc_exclusive_scan_u32(oracle.ptr(xh), oracle.ptr(want), n)
        x = torch.from_numpy(xh.view(np.int32)).cuda()
        other = _scratch_scan(lib, x, torch)
        got = torch.full_like(x, -1)
        rc = lib.gpgmp_exclusive_scan_u32_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(got.data_ptr()), n, None)
        assert rc == 0, lib.gpgmp_last_error()
        st = C.c_int32(-1)
        assert lib.gpgmp_exclusive_scan_u32_noalloc_status(None, C.byref(st)) == 0
        assert st.value == 0, f"call {call}: look-back timeout reported"
        g = got.cpu().numpy().view(np.uint32)
        assert np.array_equal(g, want), f"call {call}: differs from the oracle"
        assert torch.equal(got, other), f"call {call}: differs from the caller-scratch scan"


def test_noalloc_scan_rejects_sizes_beyond_its_scratch():
    lib = _lib()
    rc = lib.gpgmp_exclusive_scan_u32_noalloc(C.c_void_p(16), C.c_void_p(16), MAX_N + 1, None)
    assert rc == 1
    assert b"exceeds" in lib.gpgmp_last_error()
