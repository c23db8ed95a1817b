"""Python owners of the native solver objects.

``StencilSystem`` wraps ``pmb_stencil`` (a batch of pixel-grid systems with
a none / Jacobi / V-cycle preconditioner, FP64 or FP32-inner refinement),
``CsrSystem`` wraps ``pmb_csr`` (one general sparse system) and
``IcholFactor`` wraps ``pmb_ichol``. Each owns the torch tensors that back
its workspace and releases the native handle when garbage-collected.
"""

import ctypes

import numpy as np
import torch

from . import _device as dev
from . import _ffi

PREC_NONE, PREC_JACOBI, PREC_VCYCLE = 0, 1, 2
FP64, MIXED = 0, 1
STATUS = {1: "converged", 2: "maxiter", 3: "nonfinite"}


class SolveStats:
    __slots__ = ("iters", "status", "norm_r", "norm_b", "outer_iters")

    def __init__(self, iters, status, norm_r, norm_b, outer_iters=0):
        self.iters, self.status = iters, status
        self.norm_r, self.norm_b, self.outer_iters = norm_r, norm_b, outer_iters

    def __repr__(self):
        return ("SolveStats(iters=%d, status=%s, norm_r=%.3e, norm_b=%.3e, outer=%d)"
                % (self.iters, STATUS.get(self.status, self.status), self.norm_r, self.norm_b,
                   self.outer_iters))


def cg_error(maxiter):
    return ValueError(
        "Conjugate gradient descent did not converge within %d iterations" % maxiter)


class StencilSystem:
    """A batch of half-stencil systems solved together on the device.

    ``sources`` are CFSource objects (one per image). Level-0 planes are
    assembled into one buffer in the native layout.
    """

    def __init__(self, sources, precision=FP64, preconditioner=PREC_VCYCLE, num_pre_iter=1,
                 num_post_iter=1, omega=0.8, direct_solve_size=64):
        lib = _ffi.lib()
        self.sources = list(sources)
        self.precision = precision
        self.preconditioner = preconditioner
        k = len(self.sources)
        hs = (ctypes.c_int * k)(*[s.h for s in self.sources])
        ws = (ctypes.c_int * k)(*[s.w for s in self.sources])
        handle = ctypes.c_void_p()
        _ffi.check(lib.pmb_stencil_create(k, hs, ws, precision, preconditioner, num_pre_iter,
                                          num_post_iter, float(omega), int(direct_solve_size),
                                          ctypes.byref(handle)), "pmb_stencil_create")
        self._h = handle
        self.sizes = [(s.h, s.w) for s in self.sources]
        self.n_user = sum(h * w for h, w in self.sizes)
        if k == 1:
            self.planes = self.sources[0].planes()
        else:
            total = int(lib.pmb_stencil_plane_elems(handle))
            self.planes = dev.empty(total, torch.float64)
            for i, s in enumerate(self.sources):
                off = int(lib.pmb_stencil_plane_offset(handle, i))
                s.assemble_planes(self.planes[off:off + s.plane_elems])
        self.workspace = dev.workspace(lib.pmb_stencil_workspace_bytes(handle))
        _ffi.check(lib.pmb_stencil_bind(handle, dev.ptr(self.workspace), dev.ptr(self.planes),
                                        dev.stream()), "pmb_stencil_bind")

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        try:
            if h is not None and _ffi._lib is not None:
                _ffi.lib().pmb_stencil_destroy(h)
        except (AttributeError, TypeError):
            pass    # interpreter shutdown: module globals already cleared

    def setup(self):
        _ffi.check(_ffi.lib().pmb_stencil_setup(self._h, dev.stream()), "pmb_stencil_setup")

    def levels(self, image=0):
        return int(_ffi.lib().pmb_stencil_levels(self._h, image))

    def solve(self, b, x0=None, atol=0.0, rtol=1e-7, maxiter=10000, reorthogonalize=False,
              inner_rtol=1e-4, max_outer=50, out=None):
        """Solve every image; ``b`` / ``x0`` / result are concatenated device vectors."""
        b = b.reshape(-1)
        x = out if out is not None else dev.empty(self.n_user, torch.float64)
        _ffi.check(_ffi.lib().pmb_stencil_solve(
            self._h, dev.ptr(b), dev.ptr(None if x0 is None else x0.reshape(-1)), dev.ptr(x),
            float(atol), float(rtol), int(maxiter), int(bool(reorthogonalize)),
            float(inner_rtol), int(max_outer), dev.stream()), "pmb_stencil_solve")
        return x

    def stats(self, image=0):
        it, st, onr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nr, nb = ctypes.c_double(), ctypes.c_double()
        _ffi.check(_ffi.lib().pmb_stencil_stats(self._h, image, ctypes.byref(it),
                                                ctypes.byref(st), ctypes.byref(nr),
                                                ctypes.byref(nb), ctypes.byref(onr)),
                   "pmb_stencil_stats")
        return SolveStats(it.value, st.value, nr.value, nb.value, onr.value)

    def precondition(self, r):
        z = dev.empty(self.n_user, torch.float64)
        _ffi.check(_ffi.lib().pmb_stencil_precondition(self._h, dev.ptr(r.reshape(-1)),
                                                       dev.ptr(z), dev.stream()),
                   "pmb_stencil_precondition")
        return z

    def apply(self, x):
        y = dev.empty(self.n_user, torch.float64)
        _ffi.check(_ffi.lib().pmb_stencil_apply(self._h, dev.ptr(x.reshape(-1)), dev.ptr(y),
                                                dev.stream()), "pmb_stencil_apply")
        return y

    def launch_count(self):
        """Kernel launches issued by this system so far (graph replays included)."""
        return int(_ffi.lib().pmb_stencil_launch_count(self._h))

    PROFILE_KINDS = ("cg_apply", "cg_update", "refine", "vc_down_l0", "vc_down", "vc_tail",
                     "vc_direct", "vc_up", "vc_up_l0", "other")

    def profile_kernels(self, b=None, iters=8):
        """Milliseconds per iteration in each kind of launch (``PROFILE_KINDS``)
        over ``iters`` live iterations of a solve with right-hand side ``b``
        (default: all ones), CUDA events after every launch."""
        if b is None:
            b = torch.ones(self.n_user, dtype=torch.float64, device=dev.device())
        out = np.zeros(len(self.PROFILE_KINDS), dtype=np.float64)
        _ffi.check(_ffi.lib().pmb_stencil_profile(self._h, dev.ptr(b.reshape(-1)), int(iters),
                                                  out.ctypes.data, dev.stream()),
                   "pmb_stencil_profile")
        return {k: float(v) for k, v in zip(self.PROFILE_KINDS, out) if v > 0}

    def time_apply(self, iters=20):
        """Average milliseconds of one level-0 operator apply (CUDA events on
        the solver's stream)."""
        ms = ctypes.c_double()
        _ffi.check(_ffi.lib().pmb_stencil_time_apply(self._h, int(iters), ctypes.byref(ms),
                                                     dev.stream()), "pmb_stencil_time_apply")
        return ms.value


M_NONE, M_JACOBI, M_MATRIX, M_ICHOL, M_EXTERNAL = 0, 1, 2, 3, 4


class CsrSystem:
    """One general sparse system on the device (A as CSR, or applied by the
    caller), with the preconditioner kind fixed at construction."""

    # rows of the vector block
    X, R, Z, P0, P1, AP, DR, INVD = range(8)

    def __init__(self, n, mkind, csr=None, inv_diag=None, m_csr=None, ichol=None):
        lib = _ffi.lib()
        self.n = int(n)
        self.mkind = mkind
        handle = ctypes.c_void_p()
        _ffi.check(lib.pmb_csr_create(self.n, 0, mkind, ctypes.byref(handle)), "pmb_csr_create")
        self._h = handle
        self.workspace = dev.workspace(lib.pmb_csr_workspace_bytes(handle))
        self.vectors = dev.zeros((8, self.n), torch.float64)
        self.csr = csr
        if inv_diag is not None:
            self.vectors[self.INVD].copy_(inv_diag.reshape(-1))
        ip, ix, dt = (csr[0], csr[1], csr[2]) if csr is not None else (None, None, None)
        _ffi.check(lib.pmb_csr_bind(handle, dev.ptr(self.workspace), dev.ptr(self.vectors),
                                    dev.ptr(ip), dev.ptr(ix), dev.ptr(dt)), "pmb_csr_bind")
        self.m_csr = m_csr
        if m_csr is not None:
            _ffi.check(lib.pmb_csr_set_matrix_preconditioner(
                handle, 0, dev.ptr(m_csr[0]), dev.ptr(m_csr[1]), dev.ptr(m_csr[2]),
                dev.stream()), "set matrix preconditioner")
        self.ichol = ichol
        if ichol is not None:
            _ffi.check(lib.pmb_csr_set_ichol(handle, ichol._h, dev.stream()), "set ichol")

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        try:
            if h is not None and _ffi._lib is not None:
                _ffi.lib().pmb_csr_destroy(h)
        except (AttributeError, TypeError):
            pass    # interpreter shutdown: module globals already cleared

    def row(self, k):
        return self.vectors[k]

    def solve(self, b, x0=None, atol=0.0, rtol=1e-7, maxiter=10000, reorthogonalize=False):
        x = dev.empty(self.n, torch.float64)
        _ffi.check(_ffi.lib().pmb_csr_solve(self._h, dev.ptr(b), dev.ptr(x0), dev.ptr(x),
                                            float(atol), float(rtol), int(maxiter),
                                            int(bool(reorthogonalize)), dev.stream()),
                   "pmb_csr_solve")
        return x

    def begin(self, b, x0=None, atol=0.0, rtol=1e-7, maxiter=10000, reorthogonalize=False):
        _ffi.check(_ffi.lib().pmb_csr_begin(self._h, dev.ptr(b), dev.ptr(x0), float(atol),
                                            float(rtol), int(maxiter),
                                            int(bool(reorthogonalize)), dev.stream()),
                   "pmb_csr_begin")

    def step(self, mode=0):
        _ffi.check(_ffi.lib().pmb_csr_step(self._h, int(mode), dev.stream()), "pmb_csr_step")

    def finish_precondition(self):
        _ffi.check(_ffi.lib().pmb_csr_finish_precondition(self._h, dev.stream()),
                   "pmb_csr_finish_precondition")

    def p_row(self):
        idx = int(_ffi.lib().pmb_csr_p_index(self._h))
        if idx < 0:
            raise _ffi.LibraryError(_ffi.last_error())
        return self.vectors[self.P0 + idx]

    def stats(self):
        it, st = ctypes.c_int(), ctypes.c_int()
        nr, nb = ctypes.c_double(), ctypes.c_double()
        _ffi.check(_ffi.lib().pmb_csr_stats(self._h, ctypes.byref(it), ctypes.byref(st),
                                            ctypes.byref(nr), ctypes.byref(nb)), "pmb_csr_stats")
        return SolveStats(it.value, st.value, nr.value, nb.value)


class IcholFactor:
    """Device thresholded incomplete Cholesky factor (pmb_ichol)."""

    def __init__(self, n, bandwidth, capacity):
        lib = _ffi.lib()
        handle = ctypes.c_void_p()
        _ffi.check(lib.pmb_ichol_create(int(n), int(bandwidth), int(capacity),
                                        ctypes.byref(handle)), "pmb_ichol_create")
        self._h = handle
        self.n = int(n)
        self.workspace = dev.workspace(lib.pmb_ichol_workspace_bytes(handle))
        _ffi.check(lib.pmb_ichol_bind(handle, dev.ptr(self.workspace)), "pmb_ichol_bind")
        self.nnz = -1

    def __del__(self):
        h = getattr(self, "_h", None)
        self._h = None
        try:
            if h is not None and _ffi._lib is not None:
                _ffi.lib().pmb_ichol_destroy(h)
        except (AttributeError, TypeError):
            pass    # interpreter shutdown: module globals already cleared

    def factor(self, csc, discard_threshold, shift, max_nnz, relative_discard_threshold,
               diag_keep_discarded):
        res = ctypes.c_int64()
        _ffi.check(_ffi.lib().pmb_ichol_factor(
            self._h, dev.ptr(csc[0]), dev.ptr(csc[1]), dev.ptr(csc[2]), float(discard_threshold),
            float(shift), int(max_nnz), float(relative_discard_threshold),
            int(bool(diag_keep_discarded)), ctypes.byref(res), dev.stream()), "pmb_ichol_factor")
        self.nnz = int(res.value)
        return self.nnz

    def levels(self):
        return int(_ffi.lib().pmb_ichol_levels(self._h))

    def factor_ms(self):
        """Device time of the last factorisation kernel (ms)."""
        return float(_ffi.lib().pmb_ichol_factor_ms(self._h))

    def cluster(self):
        """CTAs that held the band front on chip in the last factorisation
        (0: the front was in global memory)."""
        return int(_ffi.lib().pmb_ichol_cluster(self._h))

    def apply(self, b):
        x = dev.empty(self.n, torch.float64)
        _ffi.check(_ffi.lib().pmb_ichol_apply(self._h, dev.ptr(b), dev.ptr(x), dev.stream()),
                   "pmb_ichol_apply")
        return x

    def arrays(self):
        """Device views (Lv, Lr, Lp) of the CSC factor."""
        lv, lr, lp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _ffi.check(_ffi.lib().pmb_ichol_factor_arrays(self._h, ctypes.byref(lv),
                                                      ctypes.byref(lr), ctypes.byref(lp)),
                   "pmb_ichol_factor_arrays")
        # Copy out through a device-to-device view of the workspace.
        base = self.workspace.data_ptr()
        nnz, n = self.nnz, self.n
        ws = self.workspace

        def view(ptr, count, dtype, esize):
            off = ptr - base
            return ws[off:off + count * esize].view(dtype)

        return (view(lv.value, nnz, torch.float64, 8), view(lr.value, nnz, torch.int64, 8),
                view(lp.value, n + 1, torch.int64, 8))


def csc_profile(csc, n):
    """(bandwidth, envelope) of a device CSC matrix's lower part."""
    lib = _ffi.lib()
    scratch = dev.empty(n + 2, torch.int64)
    out = dev.zeros(2, torch.int64)
    _ffi.check(lib.pmb_csc_profile(int(n), dev.ptr(csc[0]), dev.ptr(csc[1]), dev.ptr(csc[2]),
                                   dev.ptr(scratch), dev.ptr(out), dev.stream()),
               "pmb_csc_profile")
    band, env = (int(v) for v in out.cpu().numpy().astype(np.uint64))
    return band, env
