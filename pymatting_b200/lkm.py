"""Large-kernel matting Laplacian and its alpha estimator on the device.

Drop-ins for ``lkm_laplacian(image, epsilon=1e-7, radius=10,
return_diagonal=True)`` (pymatting/laplacian/lkm_laplacian.py:6-76) and
``estimate_alpha_lkm(image, trimap, laplacian_kwargs={}, cg_kwargs={})``
(pymatting/alpha/estimate_alpha_lkm.py:8-64). The operator is matrix-free:
``pmb_lkm_setup`` computes the per-window coefficients once, ``pmb_lkm_apply``
evaluates L p with separable box filters, ``pmb_lkm_diagonal`` the diagonal.
Like the reference, ``L_matvec`` takes and returns flat vectors; numpy in
gives numpy out, CUDA tensors stay on the device.
"""

import numpy as np
import torch

from . import _device as dev
from . import _ffi
from .preconditioner import JacobiPreconditioner
from .solver import cg
from .util import sanity_check_image, trimap_split

__all__ = ["lkm_laplacian", "estimate_alpha_lkm", "LKMOperator"]


class LKMOperator:
    """``L_matvec`` of lkm_laplacian, with the window coefficients on the device."""

    def __init__(self, image, epsilon=1e-7, radius=10):
        img = image if dev.is_device_tensor(image) else np.asarray(image)
        self.image = dev.to_device(img, torch.float64)
        h, w, depth = self.image.shape
        if depth != 3:
            raise ValueError("lkm_laplacian expects an (h, w, 3) image")
        self.h, self.w, self.radius = int(h), int(w), int(radius)
        self.n = self.h * self.w
        lib = _ffi.lib()
        elems = int(lib.pmb_lkm_scratch_elems(self.h, self.w, self.radius))
        if elems < 0:
            raise ValueError("image of %dx%d is too small for radius %d" % (h, w, radius))
        self.scratch = dev.empty(elems, torch.float64)
        nw = (self.h - 2 * self.radius) * (self.w - 2 * self.radius)
        self.windows = dev.empty(nw * 10, torch.float64)
        _ffi.check(lib.pmb_lkm_setup(dev.ptr(self.image), self.h, self.w, self.radius,
                                     float(epsilon), dev.ptr(self.windows), dev.ptr(self.scratch),
                                     dev.stream()), "pmb_lkm_setup")

    def apply_device(self, p, diag_add=None):
        """L p (+ diag_add * p) for a flat device vector p."""
        out = dev.empty(self.n, torch.float64)
        _ffi.check(_ffi.lib().pmb_lkm_apply(dev.ptr(self.image), self.h, self.w, self.radius,
                                            dev.ptr(self.windows), dev.ptr(diag_add),
                                            dev.ptr(p.reshape(-1)), dev.ptr(out),
                                            dev.ptr(self.scratch), dev.stream()),
                   "pmb_lkm_apply")
        return out

    def diagonal(self, diag_add=None, inverse=False):
        """diag(L) (+ diag_add); with ``inverse`` also its reciprocal."""
        d = dev.empty(self.n, torch.float64)
        inv = dev.empty(self.n, torch.float64) if inverse else None
        _ffi.check(_ffi.lib().pmb_lkm_diagonal(dev.ptr(self.image), self.h, self.w, self.radius,
                                               dev.ptr(self.windows), dev.ptr(diag_add),
                                               dev.ptr(d), dev.ptr(inv), dev.ptr(self.scratch),
                                               dev.stream()), "pmb_lkm_diagonal")
        return (d, inv) if inverse else d

    def __call__(self, p):
        if dev.is_device_tensor(p):
            return self.apply_device(dev.to_device(p, torch.float64))
        t = dev.to_device(np.asarray(p, dtype=np.float64).reshape(-1), torch.float64)
        return dev.to_host(self.apply_device(t))


def lkm_laplacian(image, epsilon=1e-7, radius=10, return_diagonal=True):
    """Large-kernel matting Laplacian as a function (see module docstring);
    with ``return_diagonal`` also ``diag_L`` (numpy for numpy images)."""
    op = LKMOperator(image, epsilon, radius)
    if not return_diagonal:
        return op
    d = op.diagonal()
    return op, (d if dev.is_device_tensor(image) else dev.to_host(d))


def estimate_alpha_lkm(image, trimap, laplacian_kwargs={}, cg_kwargs={}):
    """Alpha from the large-kernel Laplacian: cg on L + lambda C with the
    Jacobi preconditioner 1 / (diag_L + lambda C), lambda = 100
    (estimate_alpha_lkm.py:44-64); the solve stays on the device."""
    host = not dev.is_device_tensor(image)
    sanity_check_image(dev.to_host(image) if not host else image)
    op = LKMOperator(image, **laplacian_kwargs)
    tri = dev.to_host(trimap) if dev.is_device_tensor(trimap) else np.asarray(trimap)
    is_fg, is_bg, is_known, is_unknown = trimap_split(tri)
    lambda_value = 100.0
    lib = _ffi.lib()
    n = op.n
    c = dev.empty(n, torch.float64)
    b = dev.empty(n, torch.float64)
    known_t = dev.to_device(is_known.astype(np.uint8), torch.uint8)
    fg_t = dev.to_device(is_fg.astype(np.uint8), torch.uint8)
    _ffi.check(lib.pmb_mask_scale(dev.ptr(known_t), n, lambda_value, dev.ptr(c), dev.stream()), "c")
    _ffi.check(lib.pmb_mask_scale(dev.ptr(fg_t), n, lambda_value, dev.ptr(b), dev.stream()), "b")
    _d, inv_diag = op.diagonal(diag_add=c, inverse=True)
    M = JacobiPreconditioner.from_inverse_diagonal(inv_diag)
    x = cg(lambda v: op.apply_device(v, diag_add=c), b, M=M, **cg_kwargs)
    alpha = dev.empty(n, torch.float64)
    _ffi.check(lib.pmb_clip01(dev.ptr(x), n, dev.ptr(alpha), dev.stream()), "clip")
    alpha = alpha.reshape(tri.shape)
    return dev.to_host(alpha) if host else alpha
