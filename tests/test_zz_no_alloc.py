"""The no-allocation entry point (bgpu_mul_u64_device_noalloc), called
through the C-ABI and checked bit-exact against the allocating device entry
point (bgpu_mul_u64_device) on two calls in a row.

It is for callers that cannot allocate device memory when they multiply (a
fixed memory budget or pool that must not grow; threads that may not call
cudaMalloc because it can synchronize the device).  The file sorts last so a
run that stops at the first failure has already run every other test."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import SEED, rand_limbs

pytestmark = pytest.mark.gpu
MAX_LIMBS = 65536


def _entry(lib):
    f = lib.bgpu_mul_u64_device_noalloc
    f.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _dev(torch, x):
    return torch.from_numpy(x.view(np.int64)).cuda()


def test_noalloc_matches_allocating_entry_point(bb):
    torch = pytest.importorskip("torch")
    noalloc = _entry(bb.lib)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    rng = np.random.default_rng(SEED + 77)
    cases = [(40000, MAX_LIMBS - 40000), (3000, 2000), (7, 5)]
    for na, nb in cases:
        outs = []
        for call in range(2):  # two calls in a row, fresh operands each time
            a, b = rand_limbs(rng, na), rand_limbs(rng, nb)
            da, db = _dev(torch, a), _dev(torch, b)
            want = torch.empty(na + nb, dtype=torch.int64, device="cuda")
            got = torch.full((na + nb,), -1, dtype=torch.int64, device="cuda")
            with torch.cuda.stream(stream):
                bb.mul_device(da.data_ptr(), na, db.data_ptr(), nb, want.data_ptr(), stream=sp,
                              method=bb.BGPU_METHOD_NTT)
                bb.device_status(sp)
                rc = noalloc(da.data_ptr(), na, db.data_ptr(), nb, got.data_ptr(), sp)
            assert rc == 0, rc
            assert torch.equal(got, want), (na, nb, call)
            outs.append(got.cpu())
        assert not torch.equal(outs[0], outs[1])  # the second call really recomputed


def test_noalloc_square_and_repeat_without_new_device_memory(bb):
    torch = pytest.importorskip("torch")
    noalloc = _entry(bb.lib)
    rng = np.random.default_rng(SEED + 78)
    a = rand_limbs(rng, MAX_LIMBS // 2)
    da = _dev(torch, a)
    want = torch.empty(a.size * 2, dtype=torch.int64, device="cuda")
    bb.mul_device(da.data_ptr(), a.size, da.data_ptr(), a.size, want.data_ptr(),
                  method=bb.BGPU_METHOD_NTT)
    bb.device_status(0)
    got = torch.empty_like(want)
    assert noalloc(da.data_ptr(), a.size, da.data_ptr(), a.size, got.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    torch0 = torch.cuda.memory_allocated()
    for _ in range(2):
        got.fill_(-1)
        assert noalloc(da.data_ptr(), a.size, da.data_ptr(), a.size, got.data_ptr(), None) == 0
        assert torch.equal(got, want)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # nothing new on the device: neither through torch's allocator nor directly
    assert torch.cuda.memory_allocated() == torch0
    assert free1 == free0


def test_noalloc_rejects_sizes_beyond_its_static_scratch(bb):
    torch = pytest.importorskip("torch")
    noalloc = _entry(bb.lib)
    buf = torch.zeros(MAX_LIMBS + 1, dtype=torch.int64, device="cuda")
    p = buf.data_ptr()
    assert noalloc(p, MAX_LIMBS, p + 8, 1, p, None) == -4  # BGPU_ERR_CAPACITY
    assert noalloc(p, 0, p, 1, p, None) == -1              # BGPU_ERR_INVALID_ARG
