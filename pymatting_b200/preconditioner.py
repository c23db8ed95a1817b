"""Preconditioner factories: ``jacobi``, ``vcycle`` and ``ichol``.

Same signatures and calling convention as pymatting.preconditioner
(jacobi.py:1-31, vcycle.py:103-153, ichol.py:184-301): each factory returns
a callable ``M`` with ``M(r) -> z``. Here every ``M`` computes on the GPU.
``M(r)`` accepts a numpy vector (and returns one) or a CUDA tensor (and
returns one); ``cg`` of this package drives them without host copies.
"""

import numpy as np
import scipy.sparse
import torch

from . import _device as dev
from . import _ffi
from .laplacian import DeviceCSRMatrix, device_csr_arrays, device_source
from .sparse import to_device_csr
from .systems import (FP64, PREC_JACOBI, PREC_VCYCLE, CsrSystem, IcholFactor, StencilSystem,
                      csc_profile)

__all__ = ["jacobi", "vcycle", "ichol", "CholeskyDecomposition", "JacobiPreconditioner",
           "VCyclePreconditioner", "GridPlanes"]


def _vec_in(r):
    host = not dev.is_device_tensor(r)
    t = dev.to_device(np.asarray(r, dtype=np.float64) if host else r, torch.float64)
    return host, t.reshape(-1)


def _vec_out(host, t, like=None):
    if host:
        out = dev.to_host(t)
        return out.reshape(np.shape(like)) if like is not None else out
    return t


class JacobiPreconditioner:
    """``M(x) = x * (1 / diag(A))`` (pymatting/preconditioner/jacobi.py:24-31)."""

    def __init__(self, A):
        self.A = A
        self.source = device_source(A)
        if self.source is not None and self.source.radius == 1:
            n = self.source.n
            self.inv_diag = dev.empty(n, torch.float64)
            _ffi.check(_ffi.lib().pmb_planes_inv_diag(
                dev.ptr(self.source.planes()), self.source.h, self.source.w,
                dev.ptr(self.inv_diag), dev.stream()), "jacobi")
        else:
            indptr, indices, data, n, _m = to_device_csr(A)
            self.inv_diag = dev.empty(n, torch.float64)
            _ffi.check(_ffi.lib().pmb_csr_inv_diag(n, dev.ptr(indptr), dev.ptr(indices),
                                                   dev.ptr(data), dev.ptr(self.inv_diag),
                                                   dev.stream()), "jacobi")

    @classmethod
    def from_inverse_diagonal(cls, inv_diag):
        """Jacobi preconditioner of an operator given only as a function
        (e.g. lkm_laplacian): ``inv_diag`` is 1 / diag(A) on the device."""
        obj = cls.__new__(cls)
        obj.A = None
        obj.source = None
        obj.inv_diag = inv_diag
        return obj

    def apply_device(self, r):
        z = dev.empty(r.numel(), torch.float64)
        _ffi.check(_ffi.lib().pmb_vec_mul(r.numel(), dev.ptr(r), dev.ptr(self.inv_diag),
                                          dev.ptr(z), dev.stream()), "jacobi")
        return z

    def __call__(self, x):
        host, t = _vec_in(x)
        return _vec_out(host, self.apply_device(t))


def jacobi(A):
    """Jacobi preconditioner of ``A``: a callable applying ``1 / diag(A)``.

    >>> A = np.array([[2, 3], [3, 5]])
    >>> jacobi(A)(np.array([1, 2]))      # array([0.5, 0.4])
    """
    return JacobiPreconditioner(A)


class _DenseDirect:
    """Exact solve of a small matrix on the device (the n <= direct_solve_size
    branch, vcycle.py:59-60, where the reference calls spsolve)."""

    def __init__(self, A):
        indptr, indices, data, n, m = to_device_csr(A)
        if n != m:
            raise ValueError("matrix must be square")
        self.n = n
        self.csr = (indptr, indices, data)

    def apply_device(self, r):
        x = r.reshape(-1).clone()
        scratch = dev.empty(self.n * self.n, torch.float64)
        singular = dev.zeros(1, torch.int32)
        _ffi.check(_ffi.lib().pmb_dense_solve(self.n, dev.ptr(self.csr[0]), dev.ptr(self.csr[1]),
                                              dev.ptr(self.csr[2]), dev.ptr(scratch), dev.ptr(x),
                                              dev.ptr(singular), dev.stream()), "dense solve")
        return x


class GridPlanes:
    """Half-stencil planes of a grid matrix this package did not assemble.

    ``A`` is any ``(h w, h w)`` matrix (scipy sparse, dense, or device CSR)
    whose entries couple each pixel only with pixels at most two rows and two
    columns away — the pattern of the radius-1 matting Laplacian and of
    ``make_linear_system``'s matrix, whatever computed them. The conversion
    runs on the device; matrices outside that pattern, or not symmetric
    (the stencil engine stores one triangle), raise ``NotImplementedError``.
    Stands in for a CFSource in the stencil solver.
    """

    radius = 1

    def __init__(self, A, h, w, rel_tol=1e-10):
        indptr, indices, data, n, m = to_device_csr(A)
        if n != m or n != h * w:
            raise ValueError("A must be square with h * w rows")
        self.h, self.w = int(h), int(w)
        lib = _ffi.lib()
        self.pitch = int(lib.pmb_grid_pitch(self.w))
        ps = self.h * self.pitch
        self._planes = dev.empty(13 * ps, torch.float64)
        back = dev.empty(12 * ps, torch.float64)
        bad = dev.zeros(2, torch.int64)
        _ffi.check(lib.pmb_csr_to_planes(dev.ptr(indptr), dev.ptr(indices), dev.ptr(data),
                                         self.h, self.w, dev.ptr(self._planes), dev.ptr(back),
                                         float(rel_tol), dev.ptr(bad), dev.stream()),
                   "pmb_csr_to_planes")
        outside, asym = (int(v) for v in bad.cpu())
        if outside:
            raise NotImplementedError(
                "vcycle on the device needs a matrix whose entries couple pixels at most two "
                "rows and columns apart (%d entries are farther)" % outside)
        if asym:
            raise NotImplementedError(
                "vcycle on the device needs a symmetric matrix (%d entry pairs differ)" % asym)

    @property
    def n(self):
        return self.h * self.w

    @property
    def plane_elems(self):
        return 13 * self.h * self.pitch

    def planes(self):
        return self._planes

    def assemble_planes(self, out):
        out.copy_(self._planes)
        return out


class VCyclePreconditioner:
    """Geometric multigrid V-cycle (pymatting/preconditioner/vcycle.py).

    For a device-resident radius-1 matting system the whole hierarchy
    (Galerkin coarse operators, dense coarsest inverse) is built and applied
    on the GPU. ``cache``, when given, keeps that hierarchy keyed by shape so
    several factories can share it, as the reference shares its coarse
    matrices.
    """

    def __init__(self, A, shape, num_pre_iter=1, num_post_iter=1, omega=0.8,
                 direct_solve_size=64, cache=None):
        self.A = A
        self.shape = tuple(int(s) for s in shape)
        self.params = (int(num_pre_iter), int(num_post_iter), float(omega),
                       int(direct_solve_size))
        self.cache = cache
        self.source = device_source(A)
        self._system = None
        self._direct = None
        h, w = self.shape
        if h * w <= direct_solve_size:
            self._direct = _DenseDirect(A)
        elif (self.source is None or self.source.radius != 1 or
              (self.source.h, self.source.w) != self.shape):
            # Any other matrix of the grid (a host scipy matrix, another
            # Laplacian): converted to the stencil planes on the device.
            self.source = GridPlanes(A, h, w)

    @property
    def system(self):
        if self._system is None:
            key = ("pymatting_b200", self.shape, self.params, id(self.source))
            if self.cache is not None and key in self.cache:
                self._system = self.cache[key]
            else:
                pre, post, omega, direct = self.params
                self._system = StencilSystem([self.source], FP64, PREC_VCYCLE, pre, post, omega,
                                             direct)
                if self.cache is not None:
                    self.cache[key] = self._system
        return self._system

    def apply_device(self, r):
        if self._direct is not None:
            return self._direct.apply_device(r)
        return self.system.precondition(r)

    def __call__(self, r):
        host, t = _vec_in(r)
        return _vec_out(host, self.apply_device(t))


def vcycle(A, shape, num_pre_iter=1, num_post_iter=1, omega=0.8, direct_solve_size=64,
           cache=None):
    """V-cycle preconditioner for the matting system ``A`` of an image of
    ``shape == (h, w)``; same parameters as pymatting's ``vcycle``."""
    return VCyclePreconditioner(A, shape, num_pre_iter, num_post_iter, omega, direct_solve_size,
                                cache)


class CholeskyDecomposition:
    """Incomplete Cholesky factor ``L`` (CSC) held on the device.

    Calling it applies ``x = L^-T L^-1 b`` with level-scheduled triangular
    solves (pymatting/preconditioner/ichol.py:148-181).
    """

    def __init__(self, factor):
        self.factor = factor

    @property
    def Ltuple(self):
        lv, lr, lp = self.factor.arrays()
        return dev.to_host(lv).copy(), dev.to_host(lr).copy(), dev.to_host(lp).copy()

    @property
    def L(self):
        lv, lr, lp = self.Ltuple
        n = len(lp) - 1
        return scipy.sparse.csc_matrix((lv, lr, lp), (n, n))

    def apply_device(self, b):
        return self.factor.apply(b)

    def __call__(self, b):
        host, t = _vec_in(b)
        return _vec_out(host, self.apply_device(t))


ICHOL_SHIFTS = [0.0, 1e-4, 1e-3, 1e-2, 0.1, 0.5, 1.0, 10.0, 100, 1e3, 1e4, 1e5]


def _csc_arrays(A):
    """Device CSC arrays of ``A`` as ichol reads it (ichol.py:240-249)."""
    if isinstance(A, DeviceCSRMatrix) and A.pmb_on_device:
        # The CSC view of A.T has A's CSR arrays; the reference transposes a
        # CSR input before factorising, so these are the arrays it uses.
        indptr, indices, data = device_csr_arrays(A)
        return (indptr, indices, data), A.shape[0]
    if isinstance(A, scipy.sparse.csr_matrix):
        A = A.T
    if not isinstance(A, scipy.sparse.csc_matrix):
        raise ValueError("Matrix A must be a scipy.sparse.csc_matrix")
    if not A.has_canonical_format:
        A.sum_duplicates()
    m, n = A.shape
    assert m == n
    t = (dev.to_device(np.asarray(A.indptr, dtype=np.int64), torch.int64),
         dev.to_device(np.asarray(A.indices, dtype=np.int64), torch.int64),
         dev.to_device(np.asarray(A.data, dtype=np.float64), torch.float64))
    return t, n


def ichol(A, discard_threshold=1e-4, shifts=ICHOL_SHIFTS, max_nnz=int(4e9 / 16),
          relative_discard_threshold=0.0, diag_keep_discarded=True):
    """Thresholded incomplete Cholesky decomposition, factorised on the GPU.

    Same parameters, shift retries, warnings and errors as pymatting's
    ``ichol`` (ichol.py:184-301).
    """
    csc, n = _csc_arrays(A)
    band, envelope = csc_profile(csc, n)
    capacity = max(min(int(max_nnz), int(envelope)), n, 1)
    factor = IcholFactor(n, band, capacity)
    nnz = -1
    for shift in shifts:
        nnz = factor.factor(csc, discard_threshold, shift, max_nnz, relative_discard_threshold,
                            diag_keep_discarded)
        if nnz >= 0:
            break
        if nnz == -1:
            print("PERFORMANCE WARNING:")
            print("Thresholded incomplete Cholesky decomposition failed due to insufficient "
                  "positive-definiteness of matrix A with parameters:")
            print("    discard_threshold = %e" % discard_threshold)
            print("    shift = %e" % shift)
            print("Try decreasing discard_threshold or start with a larger shift")
            print("")
        if nnz == -2:
            raise ValueError(
                "Thresholded incomplete Cholesky decomposition failed because more than "
                "max_nnz non-zero elements were created. Try increasing max_nnz or "
                "discard_threshold.")
    if nnz < 0:
        raise ValueError(
            "Thresholded incomplete Cholesky decomposition failed due to insufficient "
            "positive-definiteness of matrix A and diagonal shifts did not help.")
    return CholeskyDecomposition(factor)
