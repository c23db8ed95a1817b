"""Closed-form alpha matting (pymatting/alpha/estimate_alpha_cf.py:8-78).

The hard-constraint system ``L_U x_U = -R is_fg_K`` is built on the GPU:
the reference Laplacian rows (with windows inside the known region
skipped), the compaction of the unknown pixels, ``L_U`` in CSR form and the
right-hand side ``-R m``. The preconditioner factory is called with
``L_U`` as a scipy CSR matrix — a DeviceCSRMatrix whose host arrays are only
produced if the factory reads them — and ``cg`` solves on the device. The
known pixels keep their trimap values, then everything is clipped to [0, 1].
"""

import numpy as np
import torch

from . import _device as dev
from . import _ffi
from .laplacian import DeviceCSRMatrix, _image_to_device, _mask_to_device
from .preconditioner import ichol
from .solver import cg
from .util import sanity_check_image, trimap_split

__all__ = ["estimate_alpha_cf", "estimate_alpha", "estimate_alpha_knn", "estimate_alpha_lbdm",
           "estimate_alpha_rw"]


def hard_system(image, trimap, epsilon=1e-7, radius=1, is_fg=None, is_known=None):
    """Device ``(L_U, b_U, context)`` of the hard-constraint system."""
    if int(radius) != radius or radius < 1:
        raise ValueError("radius must be a positive integer")
    radius = int(radius)
    lib = _ffi.lib()
    h, w = trimap.shape[:2]
    n = h * w
    image_t = _image_to_device(image)
    known_t = _mask_to_device(is_known, h, w).reshape(-1)
    fg_t = _mask_to_device(is_fg, h, w).reshape(-1)
    S = (4 * radius + 1) ** 2
    values = dev.empty(n * S, torch.float64)
    indices = dev.empty(n * S, torch.int64)
    indptr = dev.empty(n + 1, torch.int64)
    _ffi.check(lib.pmb_cf_laplacian_ell(dev.ptr(image_t), dev.ptr(known_t), h, w, radius,
                                        float(epsilon), None, 0.0, dev.ptr(values),
                                        dev.ptr(indices), dev.ptr(indptr), dev.stream()),
               "cf_laplacian")
    del indices, indptr
    cidx = dev.empty(n + 1, torch.int64)
    scratch = dev.empty(int(lib.pmb_scan_scratch_elems(n + 1)), torch.int64)
    _ffi.check(lib.pmb_unknown_index(dev.ptr(known_t), n, dev.ptr(cidx), dev.ptr(scratch),
                                     dev.stream()), "unknown index")
    nu = int(cidx[n].item())
    rowptr = dev.empty(nu + 1, torch.int64)
    scratch_u = dev.empty(int(lib.pmb_scan_scratch_elems(nu + 1)), torch.int64)
    _ffi.check(lib.pmb_hard_lu_rowptr(dev.ptr(known_t), h, w, radius, dev.ptr(cidx), nu,
                                      dev.ptr(rowptr), dev.ptr(scratch_u), dev.stream()),
               "L_U rowptr")
    nnz = int(rowptr[nu].item())
    cols = dev.empty(max(nnz, 1), torch.int64)
    data = dev.empty(max(nnz, 1), torch.float64)
    rhs = dev.empty(max(nu, 1), torch.float64)
    _ffi.check(lib.pmb_hard_lu_fill(dev.ptr(values), dev.ptr(known_t), dev.ptr(fg_t), h, w,
                                    radius, dev.ptr(cidx), dev.ptr(rowptr), dev.ptr(cols),
                                    dev.ptr(data), dev.ptr(rhs), dev.stream()), "L_U fill")
    L_U = DeviceCSRMatrix(shape=(nu, nu), pmb_arrays=(rowptr, cols[:nnz], data[:nnz]))
    return L_U, rhs[:nu], (known_t, cidx, n)


def estimate_alpha_cf(image, trimap, preconditioner=None, laplacian_kwargs={}, cg_kwargs={}):
    """Estimate alpha with closed-form matting (Levin et al.), on the GPU.

    Same contract as pymatting's ``estimate_alpha_cf``: ``image`` is
    ``(h, w, 3)``, ``trimap`` ``(h, w)``; ``preconditioner`` is a factory
    called with ``L_U`` (default: ``ichol``); ``laplacian_kwargs`` go to the
    Laplacian (``epsilon``, ``radius``) and ``cg_kwargs`` to ``cg``. Returns
    the ``(h, w)`` alpha matte as a numpy array (a CUDA tensor if the trimap
    was one).
    """
    if preconditioner is None:
        preconditioner = ichol
    host_trimap = not dev.is_device_tensor(trimap)
    trimap_np = trimap if host_trimap else dev.to_host(trimap)
    image_np = image if not dev.is_device_tensor(image) else None
    if image_np is not None:
        sanity_check_image(image_np)
    is_fg, is_bg, is_known, is_unknown = trimap_split(trimap_np)
    kw = dict(laplacian_kwargs)
    epsilon = kw.pop("epsilon", 1e-7)
    radius = kw.pop("radius", 1)
    if kw:
        raise TypeError("unexpected laplacian_kwargs: %s" % sorted(kw))
    L_U, b_U, (known_t, cidx, n) = hard_system(image, trimap_np, epsilon, radius, is_fg, is_known)
    x_U = cg(L_U, b_U, M=preconditioner(L_U), **cg_kwargs)
    x_U = dev.to_device(x_U, torch.float64).reshape(-1)
    trimap_t = dev.to_device(np.asarray(trimap_np, dtype=np.float64), torch.float64).reshape(-1)
    alpha = dev.empty(n, torch.float64)
    _ffi.check(_ffi.lib().pmb_alpha_compose(dev.ptr(trimap_t), dev.ptr(known_t), dev.ptr(cidx),
                                            dev.ptr(x_U), n, dev.ptr(alpha), dev.stream()),
               "alpha compose")
    alpha = alpha.reshape(trimap_np.shape)
    if host_trimap:
        return dev.to_host(alpha).astype(np.result_type(trimap_np.dtype, np.float64), copy=False)
    return alpha


estimate_alpha = estimate_alpha_cf


def _estimate_alpha_with(laplacian, default_preconditioner, image, trimap, preconditioner,
                         laplacian_kwargs, cg_kwargs):
    """make_linear_system(laplacian(image), trimap), preconditioned cg, clip:
    the common body of estimate_alpha_knn / _lbdm / _rw."""
    from .laplacian import make_linear_system
    if preconditioner is None:
        preconditioner = default_preconditioner
    sanity_check_image(image)
    A, b = make_linear_system(laplacian(image, **laplacian_kwargs), trimap)
    x = cg(A, b, M=preconditioner(A), **cg_kwargs)
    return np.clip(x, 0, 1).reshape(trimap.shape)


def estimate_alpha_knn(image, trimap, preconditioner=None, laplacian_kwargs={}, cg_kwargs={}):
    """pymatting/alpha/estimate_alpha_knn.py: knn_laplacian, Jacobi-
    preconditioned cg (by default), clipped."""
    from .laplacian import knn_laplacian
    from .preconditioner import jacobi
    return _estimate_alpha_with(knn_laplacian, jacobi, image, trimap, preconditioner,
                                laplacian_kwargs, cg_kwargs)


def estimate_alpha_lbdm(image, trimap, preconditioner=None, laplacian_kwargs={}, cg_kwargs={}):
    """pymatting/alpha/estimate_alpha_lbdm.py: lbdm_laplacian, ichol-
    preconditioned cg (by default), clipped."""
    from .laplacian import lbdm_laplacian
    return _estimate_alpha_with(lbdm_laplacian, ichol, image, trimap, preconditioner,
                                laplacian_kwargs, cg_kwargs)


def estimate_alpha_rw(image, trimap, preconditioner=None, laplacian_kwargs={}, cg_kwargs={}):
    """pymatting/alpha/estimate_alpha_rw.py: rw_laplacian, Jacobi-
    preconditioned cg (by default), clipped."""
    from .laplacian import rw_laplacian
    from .preconditioner import jacobi
    return _estimate_alpha_with(rw_laplacian, jacobi, image, trimap, preconditioner,
                                laplacian_kwargs, cg_kwargs)
