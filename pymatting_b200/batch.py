"""Batched soft-constraint alpha solves (no reference counterpart).

``solve_alpha`` solves ``(L_k + lambda C_k) x_k = lambda f_k`` for many
images of different sizes at once — the system ``make_linear_system``
builds (pymatting/laplacian/laplacian.py:5-60) — in one stencil engine:
every kernel launch covers the tiles of all images, each image keeps its own
CG scalars and stops when it converges, and the iteration is replayed from
a CUDA graph. ``precision="mixed"`` runs the Laplacian apply and the inner
V-cycle PCG in FP32 inside FP64 iterative refinement; ``"fp64"`` is the
plain FP64 solve. Both stop at the same FP64 relative residual.
"""

import numpy as np
import torch

from . import _device as dev
from . import _ffi
from .laplacian import CFSource, _image_to_device
from .systems import FP64, MIXED, PREC_JACOBI, PREC_NONE, PREC_VCYCLE, StencilSystem, cg_error

__all__ = ["AlphaBatch", "solve_alpha"]

_PREC = {"none": PREC_NONE, None: PREC_NONE, "jacobi": PREC_JACOBI, "vcycle": PREC_VCYCLE}
_PRECISION = {"fp64": FP64, "mixed": MIXED}


def _device_masks(trimap_t):
    """Foreground / known masks of a device trimap (thresholds 0.9 / 0.1)."""
    n = trimap_t.numel()
    fg = dev.empty(n, torch.uint8)
    known = dev.empty(n, torch.uint8)
    counts = dev.empty(2, torch.int64)     # zeroed by pmb_trimap_masks
    _ffi.check(_ffi.lib().pmb_trimap_masks(dev.ptr(trimap_t), n, 0.9, 0.1, dev.ptr(fg),
                                           dev.ptr(known), dev.ptr(counts), dev.stream()),
               "trimap masks")
    return fg, known, counts


class AlphaBatch:
    """A prepared batch: device inputs, assembled systems, solver."""

    def __init__(self, images, trimaps, lambda_value=100.0, epsilon=1e-7,
                 preconditioner="vcycle", precision="mixed", check_trimaps=True, tune=None):
        if len(images) != len(trimaps) or not images:
            raise ValueError("images and trimaps must be non-empty lists of equal length")
        self.shapes = []
        sources, fgs, counts = [], [], []
        for img, tri in zip(images, trimaps):
            h, w = tri.shape[:2]
            self.shapes.append((h, w))
            tri_t = dev.to_device(tri if isinstance(tri, torch.Tensor)
                                  else np.asarray(tri, dtype=np.float64), torch.float64).reshape(-1)
            fg, known, cnt = _device_masks(tri_t)
            counts.append(cnt)
            src = CFSource(_image_to_device(img), None, h, w, epsilon, 1,
                           known.reshape(h, w), lambda_value)
            sources.append(src)
            fgs.append(fg)
        if check_trimaps:
            # one device-to-host read for every image's counts
            for nf, nb in torch.stack(counts).cpu().tolist():
                if nb == 0:
                    raise ValueError("Trimap did not contain background values (values <= %f)" % 0.1)
                if nf == 0:
                    raise ValueError("Trimap did not contain foreground values (values >= %f)" % 0.9)
        self.n = sum(h * w for h, w in self.shapes)
        self.b = dev.empty(self.n, torch.float64)
        off = 0
        for fg, (h, w) in zip(fgs, self.shapes):
            _ffi.check(_ffi.lib().pmb_mask_scale(dev.ptr(fg), h * w, float(lambda_value),
                                                 dev.ptr(self.b[off:off + h * w]), dev.stream()),
                       "rhs")
            off += h * w
        self.system = StencilSystem(sources, _PRECISION[precision], _PREC[preconditioner])
        self.system.setup()
        # Launch shapes: None keeps the defaults, "cached" applies a tuning
        # found earlier for this shape (if any), "auto" tunes now if needed.
        self.tuning = None
        if tune is not None:
            from . import autotune
            if tune == "auto":
                self.tuning = autotune.autotune(self)
            elif tune == "cached":
                hit = autotune.cached(self)
                if hit is not None:
                    autotune.apply_tuning(self.system, hit["knobs"])
                    self.tuning = hit
            else:
                raise ValueError("tune must be None, 'cached' or 'auto'")

    def solve(self, rtol=1e-7, atol=0.0, maxiter=10000, inner_rtol=1e-4, max_outer=50,
              check=True):
        x = self.system.solve(self.b, None, atol, rtol, maxiter, False, inner_rtol, max_outer)
        if check:
            for k in range(len(self.shapes)):
                if self.system.stats(k).status != 1:
                    raise cg_error(maxiter)
        return x

    def alphas(self, x):
        out = dev.empty(self.n, torch.float64)
        _ffi.check(_ffi.lib().pmb_clip01(dev.ptr(x), self.n, dev.ptr(out), dev.stream()), "clip")
        res, off = [], 0
        for h, w in self.shapes:
            res.append(out[off:off + h * w].reshape(h, w))
            off += h * w
        return res

    def stats(self):
        return [self.system.stats(k) for k in range(len(self.shapes))]


def solve_alpha(images, trimaps, lambda_value=100.0, epsilon=1e-7, preconditioner="vcycle",
                precision="mixed", rtol=1e-7, atol=0.0, maxiter=10000, inner_rtol=1e-4,
                return_stats=False, tune=None):
    """Alpha mattes of a batch of images from the soft-constraint system.

    ``images``: list of ``(h, w, 3)`` arrays or tensors; ``trimaps``: list of
    ``(h, w)``. Returns a list of ``(h, w)`` alphas (numpy for numpy inputs,
    CPU tensors for CPU tensors, device tensors for device tensors), clipped to
    [0, 1]; with ``return_stats`` also per-image solve statistics. ``tune``:
    None (default launch shapes), ``"cached"`` (a tuning found earlier for
    this shape) or ``"auto"`` (run the autotuner if nothing is cached).
    """
    host_tensor = isinstance(trimaps[0], torch.Tensor) and not trimaps[0].is_cuda
    host = not dev.is_device_tensor(trimaps[0])
    batch = AlphaBatch(images, trimaps, lambda_value, epsilon, preconditioner, precision,
                       tune=tune)
    x = batch.solve(rtol, atol, maxiter, inner_rtol)
    alphas = batch.alphas(x)
    if host_tensor:
        # CPU tensors in, CPU tensors out (pinned inputs copy at full speed).
        alphas = [a.cpu() for a in alphas]
    elif host:
        alphas = [dev.to_host(a) for a in alphas]
    if return_stats:
        return alphas, batch.stats()
    return alphas
