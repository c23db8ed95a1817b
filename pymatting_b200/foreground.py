"""Foreground and background estimation on the device.

Drop-in for ``estimate_foreground_ml(image, alpha, regularization=1e-5,
n_small_iterations=10, n_big_iterations=2, small_size=32,
return_background=False, gradient_weight=1.0)``
(pymatting/foreground/estimate_foreground_ml.py:186-253). The library runs
the reference's multi-level Gauss-Seidel sweeps in their exact raster order
(``pmb_fg_ml``), so with the same starting colours F and B are bit-identical
to the reference.

The starting colours are the mean foreground (alpha > 0.9) and background
(alpha < 0.1) colours of the input. The library sums them in float64, while
the reference keeps a running float32 sum. The seeds can therefore differ in
their last bits, which moves a few output values by float32 rounding (about
4e-7 on a 440x680 photograph). ``seed_colors`` (2 * depth values, F then B)
replaces the computed seeds.

numpy inputs give float32 numpy outputs, like the reference; CUDA tensors
stay on the device.
"""

import numpy as np
import torch

from . import _device as dev
from . import _ffi

__all__ = ["estimate_foreground_ml", "estimate_foreground_ml_cupy", "estimate_foreground_cf",
           "foreground_levels"]


def foreground_levels(h, w, n_small_iterations=10, n_big_iterations=2, small_size=32):
    """(h, w) of every level, coarsest first (estimate_foreground_ml.py:101-105)."""
    lib = _ffi.lib()
    hw = np.zeros(128, dtype=np.int32)
    n = lib.pmb_fg_levels(int(h), int(w), int(n_small_iterations), int(n_big_iterations),
                          int(small_size), hw.ctypes.data, 64)
    if n == -4:
        raise ZeroDivisionError("division by zero")
    _ffi.check(0 if n > 0 else n, "pmb_fg_levels")
    return [(int(hw[2 * i]), int(hw[2 * i + 1])) for i in range(n)]


def _to_f32(a):
    return dev.to_device(a if dev.is_device_tensor(a) else np.asarray(a), torch.float32)


def estimate_foreground_ml(image, alpha, regularization=1e-5, n_small_iterations=10,
                           n_big_iterations=2, small_size=32, return_background=False,
                           gradient_weight=1.0, seed_colors=None):
    """Estimate the foreground (and background) colours of a matte.

    image: (h, w, depth) and alpha: (h, w), cast to float32 as the reference
    does. Returns F, or (F, B) with ``return_background``, each (h, w, depth)
    float32. Raises ZeroDivisionError for a 1x1 image, like the reference.
    """
    on_device = dev.is_device_tensor(image)
    img = _to_f32(image)
    al = _to_f32(alpha)
    if img.dim() != 3 or al.dim() != 2 or tuple(img.shape[:2]) != tuple(al.shape):
        raise ValueError("image must be (h, w, depth) and alpha (h, w) of the same size")
    h, w, depth = (int(v) for v in img.shape)
    if not 1 <= depth <= 8:
        raise ValueError("images with 1 to 8 channels are supported, got %d" % depth)
    seed = None
    if seed_colors is not None:
        seed = _to_f32(seed_colors).reshape(-1)
        if seed.numel() != 2 * depth:
            raise ValueError("seed_colors needs %d values" % (2 * depth))
    lib = _ffi.lib()
    nbytes = int(lib.pmb_fg_workspace_bytes(h, w, depth))
    if nbytes <= 0:
        raise ValueError("bad image shape %r" % ((h, w, depth),))
    ws = dev.workspace(nbytes)
    F = dev.empty((h, w, depth), torch.float32)
    B = dev.empty((h, w, depth), torch.float32) if return_background else None
    rc = lib.pmb_fg_ml(dev.ptr(img), dev.ptr(al), h, w, depth, float(regularization),
                       int(n_small_iterations), int(n_big_iterations), int(small_size),
                       float(gradient_weight), dev.ptr(seed), dev.ptr(F), dev.ptr(B),
                       dev.ptr(ws), nbytes, dev.stream())
    if rc == -4:
        raise ZeroDivisionError("division by zero")
    _ffi.check(rc, "pmb_fg_ml")
    _ffi.check(lib.pmb_fg_status(dev.ptr(ws), dev.stream()), "pmb_fg_ml")
    if not on_device:
        F = dev.to_host(F)
        B = dev.to_host(B) if B is not None else None
    if return_background:
        return F, B
    return F


def estimate_foreground_ml_cupy(input_image, input_alpha, regularization=1e-5,
                                n_small_iterations=10, n_big_iterations=2, small_size=32,
                                block_size=(32, 32), return_background=False, to_numpy=True):
    """Drop-in for the reference's GPU backend ``estimate_foreground_ml_cupy``
    (pymatting/foreground/estimate_foreground_ml_cupy.py:110-230): Jacobi
    iterations in float32, seeded with the colour of pixel (0, 0), with the
    reference's buffer handling. Much faster than ``estimate_foreground_ml``
    (every pixel of an iteration is independent) and a different algorithm.
    Its results agree with the reference to float32 rounding, not bitwise:
    the reference's kernel is compiled with fused multiply-adds allowed.

    ``block_size`` is accepted for compatibility and ignored (launch shapes
    are chosen here). ``to_numpy=False`` returns CUDA tensors.
    """
    img = _to_f32(input_image)
    al = _to_f32(input_alpha)
    h0, w0, depth = (int(v) for v in img.shape)
    assert depth == 3
    if tuple(al.shape) != (h0, w0):
        raise ValueError("alpha must be (h, w) like the image")
    lib = _ffi.lib()
    nbytes = int(lib.pmb_fg_jacobi_workspace_bytes(h0, w0))
    ws = dev.workspace(nbytes)
    F = dev.empty((h0, w0, depth), torch.float32)
    B = dev.empty((h0, w0, depth), torch.float32) if return_background else None
    rc = lib.pmb_fg_ml_jacobi(dev.ptr(img), dev.ptr(al), h0, w0, float(regularization),
                              int(n_small_iterations), int(n_big_iterations), int(small_size),
                              dev.ptr(F), dev.ptr(B), dev.ptr(ws), nbytes, dev.stream())
    if rc == -4:
        raise ZeroDivisionError("division by zero")
    _ffi.check(rc, "pmb_fg_ml_jacobi")
    if to_numpy:
        F = dev.to_host(F)
        B = dev.to_host(B) if B is not None else None
    if return_background:
        return F, B
    return F


def _fg_cf_matrix(alpha_t, h, w, regularization):
    """Device CSR of A = U^T U + diag(S, S) (pmb_fg_cf_system)."""
    from .laplacian import DeviceCSRMatrix
    lib = _ffi.lib()
    n2 = 2 * h * w
    rowptr = dev.empty(n2 + 1, torch.int64)
    scratch = dev.empty((n2 + 1023) // 1024 + 2, torch.int64)
    _ffi.check(lib.pmb_fg_cf_system(dev.ptr(alpha_t), h, w, float(regularization),
                                    dev.ptr(rowptr), None, None, dev.ptr(scratch), dev.stream()),
               "pmb_fg_cf_system")
    nnz = int(rowptr[n2].item())
    cols = dev.empty(nnz, torch.int64)
    vals = dev.empty(nnz, torch.float64)
    _ffi.check(lib.pmb_fg_cf_system(dev.ptr(alpha_t), h, w, float(regularization),
                                    dev.ptr(rowptr), dev.ptr(cols), dev.ptr(vals),
                                    dev.ptr(scratch), dev.stream()), "pmb_fg_cf_system")
    return DeviceCSRMatrix(shape=(n2, n2), pmb_arrays=(rowptr, cols, vals))


def estimate_foreground_cf(image, alpha, regularization=1e-5, rtol=1e-5,
                           neighbors=[(-1, 0), (1, 0), (0, -1), (0, 1)],
                           return_background=False, foreground_guess=None,
                           background_guess=None, ichol_kwargs={}, cg_kwargs={}):
    """Closed-form foreground / background estimation:
    pymatting/foreground/estimate_foreground_cf.py. The 2 h w system
    A = U^T U + diag(S, S) is assembled on the device (default neighbours),
    preconditioned with the device ``ichol`` and solved per colour channel
    with the device ``cg`` from the image (or the guesses). Results are
    clipped to [0, 1]; numpy arrays like the reference."""
    from .preconditioner import ichol
    from .solver import cg
    if sorted(tuple(d) for d in neighbors) != [(-1, 0), (0, -1), (0, 1), (1, 0)]:
        raise NotImplementedError("estimate_foreground_cf on the device supports the default "
                                  "4-neighbourhood")
    image = np.asarray(image)
    h, w, d = image.shape
    alpha = np.asarray(alpha)
    assert alpha.shape == (h, w)
    n = h * w
    a = alpha.astype(np.float64).ravel()
    A = _fg_cf_matrix(dev.to_device(a, torch.float64), h, w, regularization)
    precondition = ichol(A, **ichol_kwargs)
    foreground = (image if foreground_guess is None else foreground_guess).copy()
    background = (image if background_guess is None else background_guess).copy()
    for channel in range(d):
        image_channel = image[:, :, channel].ravel()
        b = np.concatenate([a * image_channel, (1 - a) * image_channel])
        fb = np.concatenate([foreground[:, :, channel].ravel(), background[:, :, channel].ravel()])
        fb = cg(A, b, x0=fb, M=precondition, rtol=rtol, **cg_kwargs)
        foreground[:, :, channel] = fb[:n].reshape(h, w)
        background[:, :, channel] = fb[n:].reshape(h, w)
    foreground = np.clip(foreground, 0, 1)
    background = np.clip(background, 0, 1)
    if return_background:
        return foreground, background
    return foreground
