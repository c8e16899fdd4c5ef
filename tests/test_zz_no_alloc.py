"""kf_prefix_sum_u32_noalloc: the allocation-free prefix sum.

Some callers may not allocate device memory at all (a frame loop under a fixed memory
budget, or a host framework that owns every device allocation), so the library offers a
variant of the prefix sum whose scratch lives in an array compiled into the library.  This
test calls it through the C ABI twice in a row (the array keeps the previous call's
contents) and checks each result against kf_prefix_sum_u32, exactly (integer scan).  The
file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

from oglfusionkinectv2_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _scan(fn, d_in, d_out, n):
    tot = C.c_uint32()
    st = fn(C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), n, C.byref(tot), None)
    return st, tot.value


def test_noalloc_prefix_sum_matches_allocating_entry_point():
    import torch
    lib = L.load()
    rng = np.random.default_rng(11)
    # two calls in a row with different sizes and contents
    for n, hi in [(5_000_000, 9), (123_457, 2 ** 20)]:
        a = rng.integers(0, hi, n, dtype=np.uint32)
        d_in = torch.from_numpy(a.view(np.int32)).cuda()
        out_ref = torch.empty_like(d_in)
        out_new = torch.full_like(d_in, -1)
        st, tot_ref = _scan(lib.kf_prefix_sum_u32, d_in, out_ref, n)
        assert st == L.KF_OK
        st, tot_new = _scan(lib.kf_prefix_sum_u32_noalloc, d_in, out_new, n)
        assert st == L.KF_OK
        torch.cuda.synchronize()
        assert torch.equal(out_new, out_ref)
        assert tot_new == tot_ref == int(a.astype(np.uint64).sum()) % 2 ** 32


def test_noalloc_prefix_sum_rejects_oversized_input():
    lib = L.load()
    tot = C.c_uint32()
    # the size check comes before any pointer is touched
    st = lib.kf_prefix_sum_u32_noalloc(C.c_void_p(16), C.c_void_p(16), (1 << 28) + 1, C.byref(tot), None)
    assert st == L.KF_ERR_CAPACITY
