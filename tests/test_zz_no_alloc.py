"""pmb_unknown_index_static: the unknown-pixel index without any allocation.

Some callers cannot call cudaMalloc — a host program that gives the library
only buffers from its own fixed, pre-sized device pool, or a language binding
with no device allocator of its own — so they cannot provide the scan scratch
that pmb_unknown_index takes. The static variant keeps that scratch in a
fixed array inside the library. These tests call both entry points through
the C ABI and require identical results (integer output: exact), on two
calls in a row so that leftovers of the first call in the shared array
cannot hide an error. The file is named to be collected last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 33553407   # PMB_UNKNOWN_INDEX_STATIC_MAX_N in include/pymatting_b200.h


def _lib():
    from pymatting_b200 import _ffi
    return _ffi.lib()


def _with_scratch(known_t):
    import torch
    lib = _lib()
    n = known_t.numel()
    cidx = torch.full((n + 1,), -7, dtype=torch.int64, device=known_t.device)
    scratch = torch.empty(int(lib.pmb_scan_scratch_elems(n)), dtype=torch.int64,
                          device=known_t.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.pmb_unknown_index(ctypes.c_void_p(known_t.data_ptr()), n,
                               ctypes.c_void_p(cidx.data_ptr()),
                               ctypes.c_void_p(scratch.data_ptr()), stream)
    assert rc == 0, lib.pmb_last_error()
    return cidx


def _static(known_t, cidx):
    import torch
    lib = _lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.pmb_unknown_index_static(ctypes.c_void_p(known_t.data_ptr()), known_t.numel(),
                                        ctypes.c_void_p(cidx.data_ptr()), stream)


@pytest.mark.parametrize("n,frac", [(1, 0.5), (1023, 0.3), (1024, 0.1), (307201, 0.12),
                                    (4096 * 4096, 0.15)])
def test_static_matches_scratch_variant_twice(gpu, n, frac):
    import torch
    rng = np.random.default_rng(n)
    known = (rng.random(n) >= frac).astype(np.uint8)
    known_t = torch.as_tensor(known, device=gpu)
    ref = _with_scratch(known_t)
    for _ in range(2):
        out = torch.full((n + 1,), -7, dtype=torch.int64, device=gpu)
        assert _static(known_t, out) == 0, _lib().pmb_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
    expect = np.concatenate([[0], np.cumsum(1 - known)])
    assert np.array_equal(ref.cpu().numpy(), expect)


def test_static_two_sizes_in_a_row(gpu):
    """A large call then a small one: the small one must not read the large
    call's chunk totals."""
    import torch
    rng = np.random.default_rng(5)
    for n in (3_000_000, 2049):
        known_t = torch.as_tensor((rng.random(n) >= 0.2).astype(np.uint8), device=gpu)
        out = torch.empty(n + 1, dtype=torch.int64, device=gpu)
        assert _static(known_t, out) == 0, _lib().pmb_last_error()
        assert torch.equal(out, _with_scratch(known_t))


def test_static_rejects_sizes_beyond_the_limit(gpu):
    """The size check runs on the host before any launch."""
    import torch
    lib = _lib()
    known_t = torch.zeros(16, dtype=torch.uint8, device=gpu)
    cidx = torch.zeros(17, dtype=torch.int64, device=gpu)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.pmb_unknown_index_static(ctypes.c_void_p(known_t.data_ptr()), MAX_N + 1,
                                      ctypes.c_void_p(cidx.data_ptr()), stream)
    assert rc == -1
    assert b"limit" in lib.pmb_last_error()
