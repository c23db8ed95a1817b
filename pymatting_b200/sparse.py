"""Moving general matrices to the device.

The solvers accept whatever the reference accepts for ``A`` and ``M``: scipy
sparse matrices, dense numpy arrays, or this package's device-resident
matrices. This module turns the first two into device CSR arrays (int64
indices, float64 values) so the CUDA kernels can use them.
"""

import numpy as np
import scipy.sparse
import torch

from . import _device as dev
from . import _ffi
from .laplacian import DeviceCSRMatrix, device_csr_arrays

__all__ = ["to_device_csr", "add_diagonal"]


def to_device_csr(A):
    """``(indptr, indices, data, n_rows, n_cols)`` of ``A`` on the device."""
    if isinstance(A, DeviceCSRMatrix) and A.pmb_on_device:
        indptr, indices, data = device_csr_arrays(A)
        return indptr, indices, data, A.shape[0], A.shape[1]
    if scipy.sparse.issparse(A):
        M = A.tocsr()
    else:
        M = scipy.sparse.csr_matrix(np.asarray(A, dtype=np.float64))
    indptr = dev.to_device(np.asarray(M.indptr, dtype=np.int64), torch.int64)
    indices = dev.to_device(np.asarray(M.indices, dtype=np.int64), torch.int64)
    data = dev.to_device(np.asarray(M.data, dtype=np.float64), torch.float64)
    return indptr, indices, data, M.shape[0], M.shape[1]


def add_diagonal(L, c):
    """``L + diag(c)`` in canonical CSR form, computed on the device.

    Mirrors ``(L + scipy.sparse.diags(c)).tocsr()`` followed by
    ``sum_duplicates()`` (pymatting/laplacian/laplacian.py:50-55): columns
    sorted, duplicates summed, explicit zeros dropped.
    """
    indptr, indices, data, n, m = to_device_csr(L)
    c_t = dev.to_device(np.asarray(c, dtype=np.float64), torch.float64)
    lib = _ffi.lib()
    rowptr = dev.empty(n + 1, torch.int64)
    overflow = dev.zeros(1, torch.int32)
    scratch = dev.empty(int(lib.pmb_scan_scratch_elems(n + 1)), torch.int64)
    _ffi.check(lib.pmb_csr_add_diag_rowptr(n, dev.ptr(indptr), dev.ptr(indices), dev.ptr(data),
                                           dev.ptr(c_t), dev.ptr(rowptr), dev.ptr(overflow),
                                           dev.ptr(scratch), dev.stream()), "add_diagonal")
    nnz = int(rowptr[n].item())
    cols = dev.empty(max(nnz, 1), torch.int64)
    vals = dev.empty(max(nnz, 1), torch.float64)
    _ffi.check(lib.pmb_csr_add_diag_fill(n, dev.ptr(indptr), dev.ptr(indices), dev.ptr(data),
                                         dev.ptr(c_t), dev.ptr(rowptr), dev.ptr(cols),
                                         dev.ptr(vals), dev.stream()), "add_diagonal")
    return DeviceCSRMatrix(shape=(n, m), pmb_arrays=(rowptr, cols[:nnz], vals[:nnz]))
