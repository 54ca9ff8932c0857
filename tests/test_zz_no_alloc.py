"""decon_reduce_noalloc, the reduction for callers that cannot allocate
device memory (plug-ins inside a host that owns all device allocations,
pipelines that reserve memory up front), called through the C ABI and
checked against decon_reduce, which takes a caller-allocated workspace.

Both are FP64 sums of the same float32 data in different block orders, so
they agree to 1e-12 relative (MAX exactly).  The results are also checked
against torch's own float64 reductions of the same data (a check that shares
no code with the library).  Two calls in a row with
different data show that the shared scratch array keeps nothing stale
between calls.  This file sorts last so that a run stopping at the first
failure has already run every other test; it must also pass on its own.
"""

import ctypes as C
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                   "deconlib_b200", "libdecon_b200.so")
SUM, SUMSQ, DIFFSQ, MAX, DOT = range(5)
MAX_N = 67108864


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = C.CDLL(LIB)
    p, i64 = C.c_void_p, C.c_int64
    lib.decon_reduce_noalloc.argtypes = [p, p, i64, C.c_int, p, p]
    lib.decon_reduce_noalloc.restype = C.c_int
    lib.decon_reduce.argtypes = [p, p, i64, C.c_int, p, p, p]
    lib.decon_reduce.restype = C.c_int
    lib.decon_reduce_workspace_bytes.restype = i64
    lib.decon_last_error.restype = C.c_char_p
    return lib


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _reduce(lib, fn, a, b, op):
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    if fn == "noalloc":
        st = lib.decon_reduce_noalloc(_ptr(a), _ptr(b), a.numel(), op, _ptr(out), _stream())
    else:
        ws = torch.empty(lib.decon_reduce_workspace_bytes() // 8, dtype=torch.float64, device="cuda")
        st = lib.decon_reduce(_ptr(a), _ptr(b), a.numel(), op, _ptr(out), _ptr(ws), _stream())
    assert st == 0, lib.decon_last_error().decode()
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("n", [1, 4095, 4096, 4097, 1_000_003, 8_388_608])
def test_noalloc_matches_workspace_reduction_twice(lib, n):
    gen = torch.Generator(device="cuda").manual_seed(n)
    for call in range(2):  # two calls in a row, different data
        a = torch.randn(n, device="cuda", generator=gen) * (call + 1)
        b = torch.randn(n, device="cuda", generator=gen)
        for op in (SUM, SUMSQ, DIFFSQ, MAX, DOT):
            bb = b if op in (DIFFSQ, DOT) else None
            got = _reduce(lib, "noalloc", a, bb, op)
            ref = _reduce(lib, "workspace", a, bb, op)
            ad, bd = a.double(), b.double()
            ind = {SUM: ad.sum(), SUMSQ: (ad * ad).sum(), DIFFSQ: ((ad - bd) ** 2).sum(),
                   DOT: (ad * bd).sum(), MAX: a.max().double()}[op].item()
            if op == MAX:
                assert got == ref == ind
            else:
                scale = max(1.0, abs(ref))
                assert abs(got - ref) <= 1e-12 * scale, (op, got, ref)
                assert abs(got - ind) <= 1e-12 * max(1.0, abs(ind)), (op, got, ind)


def test_noalloc_rejects_sizes_beyond_its_scratch(lib):
    a = torch.zeros(16, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # rejected on the host before any launch: nothing reads past the 16 floats
    st = lib.decon_reduce_noalloc(_ptr(a), None, MAX_N + 1, SUM, _ptr(out), _stream())
    assert st == 1
    assert b"exceeds the fixed scratch capacity" in lib.decon_last_error()
