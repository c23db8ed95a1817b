"""pymatting_b200 — PyMatting's matting paths on NVIDIA B200.

Drop-in replacements, computed by hand-written sm_100a kernels behind a C ABI
(``include/pymatting_b200.h``):

* the closed-form alpha path: ``cf_laplacian``, ``make_linear_system``, ``cg``
  (with ``CounterCallback`` / ``ProgressCallback``), the ``jacobi`` /
  ``vcycle`` / ``ichol`` preconditioner factories and ``estimate_alpha_cf``;
* the other Laplacians and their estimators: ``lkm_laplacian``,
  ``uniform_laplacian``, ``rw_laplacian``, ``lbdm_laplacian``,
  ``knn_laplacian`` (``LAPLACIANS``), ``estimate_alpha_lkm`` / ``_knn`` /
  ``_lbdm`` / ``_rw``;
* foreground estimation: ``estimate_foreground_ml`` (the reference's sweep
  order), ``estimate_foreground_ml_cupy`` (its GPU backend's Jacobi variant)
  and ``estimate_foreground_cf``;
* ``cutout`` with ``load_image`` / ``save_image`` / ``stack_images`` /
  ``blend``.

Extensions without a reference counterpart: ``solve_alpha`` / ``AlphaBatch``
(batched, mixed-precision soft-constraint solves), ``solve_alpha_sharded``
(a batch split over GPUs, results gathered to rank 0) and ``cf_alpha``
(alpha differentiable with respect to the image).
"""

from .util import trimap_split, sanity_check_image
from .laplacian import (cf_laplacian, make_linear_system, DeviceCSRMatrix, rw_laplacian,
                        uniform_laplacian, lbdm_laplacian, knn_laplacian)
from .preconditioner import jacobi, vcycle, ichol, CholeskyDecomposition
from .solver import cg, CounterCallback, ProgressCallback
from .alpha import (estimate_alpha_cf, estimate_alpha, estimate_alpha_knn, estimate_alpha_lbdm,
                    estimate_alpha_rw)
from .autograd import cf_alpha
from .batch import AlphaBatch, solve_alpha
from .shard import solve_alpha_sharded
from .lkm import lkm_laplacian, estimate_alpha_lkm
from .foreground import (estimate_foreground_ml, estimate_foreground_ml_cupy,
                         estimate_foreground_cf)
from .cutout import cutout, load_image, save_image, stack_images, blend

__version__ = "0.1.0"

__all__ = [
    "trimap_split", "sanity_check_image", "cf_laplacian", "make_linear_system",
    "DeviceCSRMatrix", "jacobi", "vcycle", "ichol", "CholeskyDecomposition", "cg",
    "CounterCallback", "ProgressCallback", "estimate_alpha_cf", "estimate_alpha", "cf_alpha",
    "lkm_laplacian", "estimate_alpha_lkm", "estimate_foreground_ml",
    "estimate_foreground_ml_cupy", "cutout", "load_image", "save_image", "stack_images", "blend",
    "rw_laplacian", "uniform_laplacian", "lbdm_laplacian", "knn_laplacian", "LAPLACIANS",
    "estimate_alpha_knn", "estimate_alpha_lbdm", "estimate_alpha_rw", "estimate_foreground_cf",
    "AlphaBatch", "solve_alpha", "solve_alpha_sharded",
]

# the reference's list (pymatting/laplacian/__init__.py)
LAPLACIANS = [cf_laplacian, knn_laplacian, lbdm_laplacian, rw_laplacian, uniform_laplacian]
