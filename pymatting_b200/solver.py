"""Preconditioned conjugate gradient on the GPU.

Drop-in for ``pymatting.solver.cg`` (pymatting/solver/cg.py:4-117) and its
callbacks (pymatting/solver/callback.py:1-23). The iteration, exit tests
(strict ``<`` on ``atol`` and ``rtol * |b|``), ``x0`` copy, optional
reorthogonalisation and the ``ValueError`` after ``maxiter`` follow the
reference. Where the work happens:

* ``A`` assembled by this package (``cf_laplacian`` / ``make_linear_system``)
  with ``M`` = None / ``jacobi(A)`` / ``vcycle(A, shape)``: the whole solve
  runs in the stencil engine (fused kernels replayed from CUDA graphs);
* any other matrix ``A`` (scipy sparse, dense array): device CSR engine, with
  ``M`` = None, ``jacobi``, ``ichol``, a matrix, or any callable;
* ``A`` given as a function: the vector algebra stays on the device and the
  function is called on host copies of ``p``.

A callback receives host copies ``(A, x, b, norm_b, r, norm_r)`` after every
iteration, before the exit test, as in the reference. ``CounterCallback``
does not need the vectors and is updated from the device iteration count.
"""

import numpy as np
import scipy.sparse
import torch

from . import _device as dev
from .laplacian import DeviceCSRMatrix, device_source
from .preconditioner import (CholeskyDecomposition, GridPlanes, JacobiPreconditioner,
                             VCyclePreconditioner)
from .sparse import to_device_csr
from .systems import (FP64, M_EXTERNAL, M_ICHOL, M_JACOBI, M_MATRIX, M_NONE, PREC_JACOBI,
                      PREC_NONE, CsrSystem, StencilSystem, cg_error)

__all__ = ["cg", "CounterCallback", "ProgressCallback"]


class CounterCallback:
    """Counts iterations (``.n``)."""

    def __init__(self):
        self.n = 0

    def __call__(self, A, x, b, norm_b, r, norm_r):
        self.n += 1


class ProgressCallback:
    """Counts iterations and prints the residual norm of each."""

    def __init__(self):
        self.n = 0

    def __call__(self, A, x, b, norm_b, r, norm_r):
        self.n += 1
        print("iteration %7d - %e (%.20f)" % (self.n, norm_r, norm_r))


def _stencil_system(A, src, M):
    """The stencil engine to use for (A, M), or None if (A, M) does not fit."""
    if (src is None and isinstance(M, VCyclePreconditioner) and M.A is A and
            M._direct is None and isinstance(M.source, GridPlanes)):
        # A matrix from elsewhere that vcycle already turned into planes.
        return M.system
    if src is None or src.radius != 1:
        return None
    if M is None:
        sys_ = A.__dict__.get("_pmb_sys_none")
        if sys_ is None:
            sys_ = StencilSystem([src], FP64, PREC_NONE)
            A.__dict__["_pmb_sys_none"] = sys_
        return sys_
    if isinstance(M, JacobiPreconditioner) and M.source is src:
        sys_ = A.__dict__.get("_pmb_sys_jacobi")
        if sys_ is None:
            sys_ = StencilSystem([src], FP64, PREC_JACOBI)
            A.__dict__["_pmb_sys_jacobi"] = sys_
        return sys_
    if isinstance(M, VCyclePreconditioner) and M.source is src and M._direct is None:
        return M.system
    return None


def _finish(stats, maxiter, callback):
    if callback is not None and type(callback).__name__ == "CounterCallback":
        callback.n += stats.iters
    if stats.status == 1:
        return
    raise cg_error(maxiter)


def _to_out(host, x, like):
    if host:
        return dev.to_host(x).reshape(np.shape(like)).astype(np.result_type(like, np.float64),
                                                             copy=False)
    return x.reshape(like.shape)


def cg(A, b, x0=None, atol=0.0, rtol=1e-7, maxiter=10000, callback=None, M=None,
       reorthogonalize=False):
    """Solve ``A x = b`` by preconditioned conjugate gradients on the GPU.

    ``A``: matrix (scipy sparse, numpy array, this package's device matrix)
    or a function ``x -> A x``. ``M``: None, a preconditioner of this
    package, a function, or a matrix. ``b`` / ``x0``: numpy vectors (the
    result is numpy) or CUDA tensors (the result stays on the device).

    >>> A = np.array([[3.0, 1.0], [1.0, 2.0]])
    >>> cg(A, np.array([4.0, 3.0]), M=jacobi(A))     # array([1., 1.])
    """
    host = not dev.is_device_tensor(b)
    b_t = dev.to_device(np.asarray(b, dtype=np.float64) if host else b, torch.float64).reshape(-1)
    x0_t = None
    if x0 is not None:
        x0_t = dev.to_device(np.asarray(x0, dtype=np.float64) if not dev.is_device_tensor(x0)
                             else x0, torch.float64).reshape(-1).clone()
    n = b_t.numel()

    counter_only = callback is None or type(callback).__name__ == "CounterCallback"
    src = device_source(A)
    system = _stencil_system(A, src, M) if counter_only else None
    if system is not None:
        x = system.solve(b_t, x0_t, atol, rtol, maxiter, reorthogonalize)
        _finish(system.stats(0), maxiter, callback)
        return _to_out(host, x, b)

    # General path: CSR engine (or A applied by the caller).
    a_is_function = callable(A) and not scipy.sparse.issparse(A) and not isinstance(A, np.ndarray)
    csr = None
    if not a_is_function:
        indptr, indices, data, nr, nc = to_device_csr(A)
        csr = (indptr, indices, data)
    mkind, inv_diag, m_csr, ich, m_fn = M_NONE, None, None, None, None
    if M is None:
        pass
    elif isinstance(M, JacobiPreconditioner):
        mkind, inv_diag = M_JACOBI, M.inv_diag
    elif isinstance(M, CholeskyDecomposition) and M.factor.n == n:
        mkind, ich = M_ICHOL, M.factor
    elif callable(M):
        mkind, m_fn = M_EXTERNAL, M
    else:
        mi, mx, md, _r, _c = to_device_csr(M)
        mkind, m_csr = M_MATRIX, (mi, mx, md)
    system = CsrSystem(n, mkind, csr=csr, inv_diag=inv_diag, m_csr=m_csr, ichol=ich)

    if csr is not None and mkind != M_EXTERNAL and counter_only:
        x = system.solve(b_t, x0_t, atol, rtol, maxiter, reorthogonalize)
        _finish(system.stats(), maxiter, callback)
        return _to_out(host, x, b)

    return _cg_steps(system, A, a_is_function, m_fn, b, b_t, x0_t, host, atol, rtol, maxiter,
                     callback, reorthogonalize)


def _apply_function(fn, v_t, host_io):
    """Call a user function on a vector; host functions get numpy."""
    if isinstance(fn, (VCyclePreconditioner, JacobiPreconditioner, CholeskyDecomposition)):
        return fn.apply_device(v_t)
    if host_io:
        out = fn(dev.to_host(v_t).copy())
        return dev.to_device(np.asarray(out, dtype=np.float64), torch.float64).reshape(-1)
    out = fn(v_t)
    return dev.to_device(out, torch.float64).reshape(-1)


def _cg_steps(system, A, a_is_function, m_fn, b, b_t, x0_t, host, atol, rtol, maxiter, callback,
              reorthogonalize):
    """Iteration-by-iteration driver for callbacks and caller-applied A / M."""
    rhs = b_t
    if a_is_function and x0_t is not None:
        # The caller's A gives r0 = b - A x0; the exit test still uses |b|
        # (cg.py:66-73), folded into one absolute tolerance.
        rhs = b_t - _apply_function(A, x0_t, host)
        nb = float(np.linalg.norm(dev.to_host(b_t)))
        atol, rtol = max(atol, rtol * nb), 0.0
    system.begin(rhs, x0_t, atol, rtol, maxiter, reorthogonalize)
    if m_fn is not None:
        st = system.stats()
        if st.status == 0:
            system.row(system.Z).copy_(_apply_function(m_fn, system.row(system.R), host))
            system.finish_precondition()
    st = system.stats()
    norm_b = float(np.linalg.norm(dev.to_host(b_t))) if a_is_function and x0_t is not None else st.norm_b
    if st.status == 1:
        return _to_out(host, system.row(system.X).clone(), b)
    if st.status != 0:
        raise cg_error(maxiter)
    while True:
        if a_is_function:
            system.step(1)
            p = system.p_row()
            system.row(system.AP).copy_(_apply_function(A, p, host))
            system.step(2)
        else:
            system.step(0)
        st = system.stats()
        if callback is not None:
            x_h = dev.to_host(system.row(system.X)).copy()
            r_h = dev.to_host(system.row(system.R)).copy()
            b_h = b if host else dev.to_host(b_t)
            callback(A, x_h, b_h, norm_b, r_h, st.norm_r)
        if st.status == 1:
            return _to_out(host, system.row(system.X).clone(), b)
        if st.status != 0:
            raise cg_error(maxiter)
        if m_fn is not None:
            system.row(system.Z).copy_(_apply_function(m_fn, system.row(system.R), host))
            system.finish_precondition()
