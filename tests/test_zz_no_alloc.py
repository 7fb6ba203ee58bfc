"""The scan entry point that allocates nothing (gpgmp_exclusive_scan_u32_noalloc).

It serves callers that may not allocate device memory themselves, such as code whose
device memory is owned by another allocator or that cannot afford cudaMalloc inside a
time loop; its scratch is a fixed array built into the library.  Called through the
C ABI, its output must equal the caller-scratch scan (gpgmp_exclusive_scan_u32) bit
for bit on two calls in a row, which also shows that the shared array is cleared
between calls.  This file is collected last on purpose, and passes both alone in a
fresh process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 1 << 26


def _lib():
    from inchman_b200 import _lib as L
    lib = L.lib()
    f = lib.gpgmp_exclusive_scan_u32_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    g = lib.gpgmp_exclusive_scan_u32
    g.restype = C.c_int
    g.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_size_t, C.c_void_p]
    q = lib.gpgmp_scan_scratch_bytes
    q.restype = C.c_int
    q.argtypes = [C.c_int64, C.POINTER(C.c_size_t)]
    return lib


def _reference_scan(lib, x, torch):
    n = x.numel()
    out = torch.empty_like(x)
    nb = C.c_size_t(0)
    assert lib.gpgmp_scan_scratch_bytes(n, C.byref(nb)) == 0
    scratch = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    rc = lib.gpgmp_exclusive_scan_u32(C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), n,
                                      C.c_void_p(scratch.data_ptr()), nb.value, None)
    assert rc == 0
    return out


@pytest.mark.parametrize("n", [1, 4097, 3_000_001])
def test_noalloc_scan_matches_scan_on_two_calls(n):
    import torch
    lib = _lib()
    rng = np.random.default_rng(n)
    for call in range(2):
        x = torch.from_numpy(rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32).view(np.int32)).cuda()
        want = _reference_scan(lib, x, torch)
        got = torch.full_like(x, -1)
        rc = lib.gpgmp_exclusive_scan_u32_noalloc(C.c_void_p(x.data_ptr()), C.c_void_p(got.data_ptr()), n, None)
        assert rc == 0, lib.gpgmp_last_error()
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}"


def test_noalloc_scan_rejects_sizes_beyond_its_scratch():
    lib = _lib()
    rc = lib.gpgmp_exclusive_scan_u32_noalloc(C.c_void_p(16), C.c_void_p(16), MAX_N + 1, None)
    assert rc == 1
    assert b"exceeds" in lib.gpgmp_last_error()
