"""kf_prefix_sum_u32_noalloc: the allocation-free prefix sum.

Some callers may not allocate device memory at all (a frame loop under a fixed memory
budget, or a host framework that owns every device allocation), so the library offers a
variant of the prefix sum whose scratch lives in an array compiled into the library.  These
tests call it through the C ABI, several calls in a row (the array keeps the previous
call's contents), and check each result exactly (integer scan) against kf_prefix_sum_u32
and a numpy exclusive scan: one- and two-level sizes, a three-level size (more than
4096^2 elements), the exact 2^28-element limit, n = 0 and a NULL total; and that a call
lowers neither the device's free memory nor changes torch's reserved pool.  The file name makes
pytest collect it last.
"""
import ctypes as C
import gc

import numpy as np
import pytest

from oglfusionkinectv2_b200 import _lib as L

pytestmark = pytest.mark.gpu

LIMIT = 1 << 28  # the largest input the static scratch array serves


def _scan(fn, d_in, d_out, n, want_total=True):
    tot = C.c_uint32(0xDEADBEEF)
    st = fn(C.c_void_p(d_in.data_ptr() if d_in is not None else 0),
            C.c_void_p(d_out.data_ptr() if d_out is not None else 0), n,
            C.byref(tot) if want_total else None, None)
    return st, tot.value


def _numpy_exclusive(a: np.ndarray) -> np.ndarray:
    out = np.zeros_like(a, dtype=np.uint32)
    if len(a) > 1:
        np.cumsum(a[:-1], dtype=np.uint32, out=out[1:])
    return out


def _check(lib, torch, d_in, n):
    """Both entry points on the same device input; exact agreement with numpy; two
    allocation-free calls in a row, the second of which lowers neither the device's free
    memory nor changes torch's pool (the first follows the allocating call, whose freed scratch the
    driver's pool may return to the device while it runs)."""
    a = d_in.cpu().numpy().view(np.uint32)
    out_ref = torch.empty_like(d_in)
    out_new = torch.full_like(d_in, -1)
    out_new2 = torch.full_like(d_in, -1)
    st, tot_ref = _scan(lib.kf_prefix_sum_u32, d_in, out_ref, n)
    assert st == L.KF_OK
    torch.cuda.synchronize()
    st, tot_new = _scan(lib.kf_prefix_sum_u32_noalloc, d_in, out_new, n)
    assert st == L.KF_OK
    # objects of earlier tests that the garbage collector frees release device memory: collect
    # them first, so that only an allocation by the call could change the figures below
    gc.collect()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    st, tot_new2 = _scan(lib.kf_prefix_sum_u32_noalloc, d_in, out_new2, n)
    assert st == L.KF_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 >= free0, (free0, free1)  # nothing allocated (memory freed elsewhere may return)
    assert torch.cuda.memory_reserved() == reserved0
    assert torch.equal(out_new, out_ref) and torch.equal(out_new2, out_ref)
    assert tot_new2 == tot_new
    expect = _numpy_exclusive(a)
    np.testing.assert_array_equal(out_new.cpu().numpy().view(np.uint32), expect)
    assert tot_new == tot_ref == int(a.astype(np.uint64).sum()) % 2 ** 32


def test_noalloc_prefix_sum_matches_allocating_entry_point():
    import torch
    lib = L.load()
    rng = np.random.default_rng(11)
    # calls in a row with different sizes and contents: one tile, two levels, and three
    # levels (4096^2 + 1 elements make 4097 tile totals, scanned in two more levels)
    for n, hi in [(5_000_000, 9), (123_457, 2 ** 20), (3_000, 7), (4096 * 4096 + 1, 3)]:
        a = rng.integers(0, hi, n, dtype=np.uint32)
        d_in = torch.from_numpy(a.view(np.int32)).cuda()
        _check(lib, torch, d_in, n)


def test_noalloc_prefix_sum_at_the_size_limit():
    """Exactly 2^28 elements, the most the static array serves (and a 32-bit wrap of the
    running sum along the way)."""
    import torch
    lib = L.load()
    g = torch.Generator(device="cuda").manual_seed(5)
    d_in = torch.randint(0, 64, (LIMIT,), dtype=torch.int32, device="cuda", generator=g)
    _check(lib, torch, d_in, LIMIT)
    del d_in
    torch.cuda.empty_cache()


def test_noalloc_prefix_sum_empty_and_null_total():
    import torch
    lib = L.load()
    # n = 0: no pointer is read, the total is 0
    st, tot = _scan(lib.kf_prefix_sum_u32_noalloc, None, None, 0)
    assert st == L.KF_OK and tot == 0
    # total == NULL: the scan still runs (asynchronously on the stream)
    a = np.arange(10_000, dtype=np.uint32) % 5
    d_in = torch.from_numpy(a.view(np.int32)).cuda()
    out = torch.full_like(d_in, -1)
    st, _ = _scan(lib.kf_prefix_sum_u32_noalloc, d_in, out, len(a), want_total=False)
    assert st == L.KF_OK
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), _numpy_exclusive(a))


def test_noalloc_prefix_sum_rejects_oversized_input():
    lib = L.load()
    tot = C.c_uint32()
    # the size check comes before any pointer is touched
    st = lib.kf_prefix_sum_u32_noalloc(C.c_void_p(16), C.c_void_p(16), LIMIT + 1, C.byref(tot), None)
    assert st == L.KF_ERR_CAPACITY
