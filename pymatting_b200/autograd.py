"""Differentiable closed-form alpha (no reference counterpart).

``cf_alpha(images, trimaps)`` returns the soft-constraint alpha
``x = (L(image) + lambda C)^-1 lambda f`` — the system of
``make_linear_system(cf_laplacian(image), trimap)``
(pymatting/laplacian/laplacian.py:5-60, pymatting/laplacian/cf_laplacian.py)
— as a torch tensor that back-propagates to the image.

Backward pass, for a cotangent g = d loss / d x:
  * adjoint solve  A mu = g  with the same V-cycle PCG engine (A is
    symmetric, so the forward operator serves);
  * d loss / d image = -d(mu' L(image) x) / d image, computed by the
    ``pmb_cf_laplacian_vjp`` kernel, which recomputes every window's colour
    mean and inverse covariance from the image instead of storing them.
The trimap enters only through C and f, which are piecewise constant in it,
so it receives no gradient. Solves run in FP64.
"""

import torch

from . import _device as dev
from . import _ffi
from .batch import AlphaBatch
from .systems import cg_error

__all__ = ["cf_alpha", "CFAlphaFunction"]

_TINY = 1e-300


class CFAlphaFunction(torch.autograd.Function):
    """images (B, h, w, 3), trimaps (B, h, w) on the device -> alphas (B, h, w)."""

    @staticmethod
    def forward(ctx, images, trimaps, lambda_value, epsilon, rtol, maxiter):
        B, h, w, _ = images.shape
        img64 = images.detach().to(torch.float64).contiguous()
        tri64 = trimaps.detach().to(torch.float64).contiguous()
        batch = AlphaBatch([img64[k] for k in range(B)], [tri64[k] for k in range(B)],
                           lambda_value, epsilon, "vcycle", "fp64")
        x = batch.solve(rtol=rtol, maxiter=maxiter)
        ctx.batch = batch
        ctx.shape = (B, h, w)
        ctx.epsilon = epsilon
        ctx.rtol = rtol
        ctx.maxiter = maxiter
        ctx.image_dtype = images.dtype
        ctx.save_for_backward(img64, x)
        return x.reshape(B, h, w).to(images.dtype)

    @staticmethod
    def backward(ctx, g):
        img64, x = ctx.saved_tensors
        B, h, w = ctx.shape
        n = h * w
        g64 = g.detach().to(torch.float64).contiguous().reshape(-1)
        system = ctx.batch.system
        # A zero cotangent (gradcheck sends some) has |b| = 0, where a purely
        # relative test never passes; the tiny absolute tolerance ends those
        # solves at mu = 0 and leaves every other solve unchanged.
        mu = system.solve(g64, atol=_TINY, rtol=ctx.rtol, maxiter=ctx.maxiter)
        for k in range(B):
            if system.stats(k).status != 1:
                raise cg_error(ctx.maxiter)
        grad = dev.empty((B, h, w, 3), torch.float64)
        lib = _ffi.lib()
        for k in range(B):
            _ffi.check(lib.pmb_cf_laplacian_vjp(dev.ptr(img64[k]), None, h, w,
                                                float(ctx.epsilon), dev.ptr(x[k * n:(k + 1) * n]),
                                                dev.ptr(mu[k * n:(k + 1) * n]),
                                                dev.ptr(grad[k]), dev.stream()),
                       "pmb_cf_laplacian_vjp")
        return (-grad).to(ctx.image_dtype), None, None, None, None, None


def cf_alpha(images, trimaps, lambda_value=100.0, epsilon=1e-7, rtol=1e-10, maxiter=10000):
    """Soft-constraint alpha that is differentiable with respect to the image.

    ``images``: ``(h, w, 3)`` or ``(B, h, w, 3)`` CUDA tensor (float32 or
    float64); ``trimaps``: ``(h, w)`` or ``(B, h, w)``. Returns ``(h, w)`` or
    ``(B, h, w)`` in the image dtype, not clipped (clipping has no useful
    gradient). ``rtol`` is the relative residual of the forward and the
    adjoint solve.
    """
    single = images.dim() == 3
    if single:
        images = images.unsqueeze(0)
        trimaps = trimaps.unsqueeze(0)
    if not (dev.is_device_tensor(images) and dev.is_device_tensor(trimaps)):
        raise TypeError("cf_alpha takes CUDA tensors")
    out = CFAlphaFunction.apply(images, trimaps, float(lambda_value), float(epsilon), float(rtol),
                                int(maxiter))
    return out[0] if single else out
