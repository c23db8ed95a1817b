"""Every device wait of the library ends: a wait that runs out reports an
error status and the context stays usable.

The waits are run on a barrier or word that nothing completes (no copy is
issued, no producer runs), so giving up is the only way out and nothing is
in flight when the kernel returns. After each, a normal solve and a normal
foreground estimate on the same context must succeed."""

import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(gpu):
    from pymatting_b200 import _ffi
    return _ffi.lib()


def _selftest(lib, which, limit):
    import torch
    scratch = torch.empty(64, dtype=torch.uint8, device="cuda")
    out = ctypes.c_int(-1)
    rc = lib.pmb_selftest_wait(which, limit, ctypes.c_void_p(scratch.data_ptr()),
                               ctypes.byref(out), ctypes.c_void_p(
                                   torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.pmb_last_error()
    return out.value


def _normal_calls_still_work():
    import pymatting_b200 as pm
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _a, _f = make_matting_problem(40, 56, 7, sigma=2.0, band=3, unknown_fraction=0.25)
    A, b = pm.make_linear_system(pm.cf_laplacian(img), tri)
    x = pm.cg(A, b, M=pm.vcycle(A, tri.shape), rtol=1e-7)
    x_ref, _it = oracle.solve_soft(img, tri, preconditioner="vcycle", rtol=1e-7)
    assert np.abs(x - x_ref).max() < 1e-6
    a32 = np.clip(x, 0, 1).reshape(tri.shape).astype(np.float32)
    i32 = img.astype(np.float32)
    F = pm.estimate_foreground_ml(i32, a32, seed_colors=oracle.fg_mean_colors(i32, a32))
    assert np.array_equal(F, oracle.estimate_foreground_ml(i32, a32))


@pytest.mark.parametrize("polls", [1, 1000])
def test_mbarrier_wait_gives_up(lib, polls):
    """The TMA kernels' mbarrier wait (limit in polls; the kernels use 2^24)."""
    assert _selftest(lib, 0, polls) == 1
    _normal_calls_still_work()


def test_foreground_epoch_poll_gives_up(lib):
    """The foreground sweep's epoch poll (deadline in ns; the sweep uses 2 s):
    a 1 ms deadline expires and sets the timeout status."""
    assert _selftest(lib, 1, 1_000_000) == 1
    _normal_calls_still_work()


@pytest.mark.parametrize("polls", [1, 1000])
def test_ichol_stream_wait_gives_up(lib, polls):
    """The streamed ichol solve's chunk wait (limit in polls; the solve uses
    2^24): a chunk whose copy is never issued makes it give up, the result is
    NaN, and an ichol factor and solve on the same context still match the
    oracle."""
    import scipy.sparse
    import pymatting_b200 as pm
    assert _selftest(lib, 2, polls) == 1
    _normal_calls_still_work()
    g = np.random.default_rng(5)
    n = 300
    B = scipy.sparse.random(n, n, density=0.02, random_state=5) + scipy.sparse.eye(n) * 4.0
    A = scipy.sparse.csc_matrix(B @ B.T)
    rhs = g.standard_normal(n)
    np.testing.assert_allclose(pm.ichol(A)(rhs), oracle.ichol(A)(rhs), rtol=1e-9, atol=1e-12)


def test_selftest_rejects_bad_arguments(lib):
    import torch
    scratch = torch.empty(64, dtype=torch.uint8, device="cuda")
    out = ctypes.c_int()
    assert lib.pmb_selftest_wait(3, 10, ctypes.c_void_p(scratch.data_ptr()), ctypes.byref(out),
                                 None) == -1
    assert lib.pmb_selftest_wait(0, 0, ctypes.c_void_p(scratch.data_ptr()), ctypes.byref(out),
                                 None) == -1
