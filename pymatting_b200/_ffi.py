"""ctypes binding of ``libpmb200.so`` (the C ABI in include/pymatting_b200.h).

The pattern follows the reference's own native bindings (ctypes ``CDLL``,
declared ``argtypes``, integer status turned into a Python exception). The
library is the only compute path: there is no CPU fallback, so a missing
library or a missing CUDA device raises at first use.
"""

import ctypes
import os

_lib = None

c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_flt = ctypes.c_float
c_vp = ctypes.c_void_p

# name: (restype, argtypes)
_SIGNATURES = {
    "pmb_last_error": (ctypes.c_char_p, []),
    "pmb_version": (c_int, []),
    "pmb_grid_pitch": (c_int, [c_int]),
    "pmb_cf_laplacian_ell": (c_int, [c_vp, c_vp, c_int, c_int, c_int, c_dbl, c_vp, c_dbl,
                                     c_vp, c_vp, c_vp, c_vp]),
    "pmb_cf_laplacian_planes": (c_int, [c_vp, c_vp, c_int, c_int, c_dbl, c_vp, c_dbl, c_vp,
                                        c_vp]),
    "pmb_lkm_scratch_elems": (c_i64, [c_int, c_int, c_int]),
    "pmb_lkm_setup": (c_int, [c_vp, c_int, c_int, c_int, c_dbl, c_vp, c_vp, c_vp]),
    "pmb_lkm_apply": (c_int, [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_lkm_diagonal": (c_int, [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_cf_laplacian_vjp": (c_int, [c_vp, c_vp, c_int, c_int, c_dbl, c_vp, c_vp, c_vp, c_vp]),
    "pmb_fg_workspace_bytes": (c_i64, [c_int, c_int, c_int]),
    "pmb_fg_ml": (c_int, [c_vp, c_vp, c_int, c_int, c_int, c_flt, c_int, c_int, c_int, c_flt,
                          c_vp, c_vp, c_vp, c_vp, c_i64, c_vp]),
    "pmb_fg_status": (c_int, [c_vp, c_vp]),
    "pmb_fg_levels": (c_int, [c_int, c_int, c_int, c_int, c_int, c_vp, c_int]),
    "pmb_fg_jacobi_workspace_bytes": (c_i64, [c_int, c_int]),
    "pmb_fg_ml_jacobi": (c_int, [c_vp, c_vp, c_int, c_int, c_flt, c_int, c_int, c_int, c_vp, c_vp,
                                 c_vp, c_i64, c_vp]),
    "pmb_window_laplacian": (c_int, [c_int, c_vp, c_int, c_int, c_int, c_dbl, c_vp, c_vp, c_vp,
                                     c_vp, c_vp, c_vp]),
    "pmb_lbdm_scratch_elems": (c_i64, [c_int, c_int, c_int]),
    "pmb_lbdm_laplacian": (c_int, [c_vp, c_int, c_int, c_int, c_dbl, c_vp, c_vp, c_vp, c_vp, c_vp,
                                   c_vp, c_vp]),
    "pmb_knn_scratch_elems": (c_i64, [c_i64, c_int, c_int]),
    "pmb_knn_laplacian": (c_int, [c_vp, c_int, c_int, c_vp, c_vp, c_int, c_int, c_vp, c_vp, c_vp,
                                  c_vp, c_vp, c_vp]),
    "pmb_fg_cf_system": (c_int, [c_vp, c_int, c_int, c_dbl, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_cf_hard_system": (c_int, [c_vp, c_vp, c_vp, c_int, c_int, c_dbl, c_vp, c_vp, c_vp]),
    "pmb_scan_scratch_elems": (c_i64, [c_i64]),
    "pmb_ell_csr_rowptr": (c_int, [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp]),
    "pmb_ell_csr_fill": (c_int, [c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp]),
    "pmb_trimap_masks": (c_int, [c_vp, c_i64, c_dbl, c_dbl, c_vp, c_vp, c_vp, c_vp]),
    "pmb_unknown_index": (c_int, [c_vp, c_i64, c_vp, c_vp, c_vp]),
    "pmb_unknown_index_static": (c_int, [c_vp, c_i64, c_vp, c_vp]),
    "pmb_hard_lu_rowptr": (c_int, [c_vp, c_int, c_int, c_int, c_vp, c_i64, c_vp, c_vp, c_vp]),
    "pmb_hard_lu_fill": (c_int, [c_vp, c_vp, c_vp, c_int, c_int, c_int, c_vp, c_vp, c_vp, c_vp,
                                 c_vp, c_vp]),
    "pmb_alpha_compose": (c_int, [c_vp, c_vp, c_vp, c_vp, c_i64, c_vp, c_vp]),
    "pmb_stencil_create": (c_int, [c_int, c_vp, c_vp, c_int, c_int, c_int, c_int, c_dbl, c_int,
                                   ctypes.POINTER(c_vp)]),
    "pmb_stencil_workspace_bytes": (c_i64, [c_vp]),
    "pmb_stencil_plane_offset": (c_i64, [c_vp, c_int]),
    "pmb_stencil_plane_elems": (c_i64, [c_vp]),
    "pmb_stencil_levels": (c_int, [c_vp, c_int]),
    "pmb_stencil_bind": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "pmb_stencil_setup": (c_int, [c_vp, c_vp]),
    "pmb_stencil_solve": (c_int, [c_vp, c_vp, c_vp, c_vp, c_dbl, c_dbl, c_int, c_int, c_dbl,
                                  c_int, c_vp]),
    "pmb_stencil_precondition": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "pmb_stencil_apply": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "pmb_stencil_stats": (c_int, [c_vp, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                  ctypes.POINTER(c_dbl), ctypes.POINTER(c_dbl),
                                  ctypes.POINTER(c_int)]),
    "pmb_stencil_launch_count": (c_i64, [c_vp]),
    "pmb_stencil_time_apply": (c_int, [c_vp, c_int, ctypes.POINTER(c_dbl), c_vp]),
    "pmb_stencil_profile": (c_int, [c_vp, c_vp, c_int, c_vp, c_vp]),
    "pmb_stencil_destroy": (c_int, [c_vp]),
    "pmb_stencil_tune": (c_int, [c_vp, c_int, c_int]),
    "pmb_stencil_tuning": (c_int, [c_vp, c_int]),
    "pmb_csr_create": (c_int, [c_i64, c_i64, c_int, ctypes.POINTER(c_vp)]),
    "pmb_csr_workspace_bytes": (c_i64, [c_vp]),
    "pmb_csr_bind": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_csr_set_matrix_preconditioner": (c_int, [c_vp, c_i64, c_vp, c_vp, c_vp, c_vp]),
    "pmb_csr_set_ichol": (c_int, [c_vp, c_vp, c_vp]),
    "pmb_csr_solve": (c_int, [c_vp, c_vp, c_vp, c_vp, c_dbl, c_dbl, c_int, c_int, c_vp]),
    "pmb_csr_begin": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_dbl, c_int, c_int, c_vp]),
    "pmb_csr_step": (c_int, [c_vp, c_int, c_vp]),
    "pmb_csr_finish_precondition": (c_int, [c_vp, c_vp]),
    "pmb_csr_p_index": (c_int, [c_vp]),
    "pmb_csr_stats": (c_int, [c_vp, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                              ctypes.POINTER(c_dbl), ctypes.POINTER(c_dbl)]),
    "pmb_csr_spmv": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_csr_inv_diag": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_vec_mul": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp]),
    "pmb_csr_destroy": (c_int, [c_vp]),
    "pmb_csc_profile": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_ichol_create": (c_int, [c_i64, c_i64, c_i64, ctypes.POINTER(c_vp)]),
    "pmb_ichol_workspace_bytes": (c_i64, [c_vp]),
    "pmb_ichol_bind": (c_int, [c_vp, c_vp]),
    "pmb_ichol_factor": (c_int, [c_vp, c_vp, c_vp, c_vp, c_dbl, c_dbl, c_i64, c_dbl, c_int,
                                 ctypes.POINTER(c_i64), c_vp]),
    "pmb_ichol_levels": (c_int, [c_vp]),
    "pmb_ichol_cluster": (c_int, [c_vp]),
    "pmb_ichol_factor_ms": (ctypes.c_float, [c_vp]),
    "pmb_ichol_factor_arrays": (c_int, [c_vp, ctypes.POINTER(c_vp), ctypes.POINTER(c_vp),
                                        ctypes.POINTER(c_vp)]),
    "pmb_ichol_apply": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "pmb_ichol_destroy": (c_int, [c_vp]),
    "pmb_planes_inv_diag": (c_int, [c_vp, c_int, c_int, c_vp, c_vp]),
    "pmb_csr_add_diag_rowptr": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_selftest_wait": (c_int, [c_int, c_i64, c_vp, ctypes.POINTER(c_int), c_vp]),
    "pmb_csr_to_planes": (c_int, [c_vp, c_vp, c_vp, c_int, c_int, c_vp, c_vp, c_dbl, c_vp,
                                  c_vp]),
    "pmb_csr_add_diag_fill": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_dense_solve": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_mask_scale": (c_int, [c_vp, c_i64, c_dbl, c_vp, c_vp]),
    "pmb_clip01": (c_int, [c_vp, c_i64, c_vp, c_vp]),
}


class LibraryError(RuntimeError):
    """A call into the CUDA library failed."""


def _path():
    here = os.path.dirname(os.path.abspath(__file__))
    return os.path.join(here, "_lib", "libpmb200.so")


def lib():
    """Load (building first if needed) and return the CUDA library."""
    global _lib
    if _lib is None:
        path = _path()
        if not os.path.exists(path):
            from . import build
            build.build()
        handle = ctypes.CDLL(path)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def exported_symbols():
    """Names of the C-ABI functions this binding expects."""
    return sorted(_SIGNATURES)


def last_error():
    msg = lib().pmb_last_error()
    return msg.decode() if msg else ""


def check(rc, what=""):
    """Raise on a negative status from the library."""
    if rc != 0:
        raise LibraryError("%s failed (status %d): %s" % (what or "pymatting_b200", rc, last_error()))
    return rc
