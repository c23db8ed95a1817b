"""ORACLE — test infrastructure, not product code.

A CPU restatement of PyMatting's closed-form alpha path. Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` import it, and only as the checker or the timed CPU baseline;
the product package ``pymatting_b200`` never imports it.

Pieces and the reference code each restates (paths inside PyMatting 1.1.15):

* ``cf_laplacian``       pymatting/laplacian/cf_laplacian.py:5-177 (C, bit-exact)
* ``make_linear_system`` pymatting/laplacian/laplacian.py:5-60
* ``trimap_split``       pymatting/util/util.py:439-525
* ``cg``                 pymatting/solver/cg.py:4-117
* ``jacobi``             pymatting/preconditioner/jacobi.py:1-31
* ``make_P`` / ``vcycle`` pymatting/preconditioner/vcycle.py:6-153
* ``ichol``              pymatting/preconditioner/ichol.py:6-301 (C)
* ``estimate_alpha_cf``  pymatting/alpha/estimate_alpha_cf.py:8-78
* ``lkm_laplacian``      pymatting/laplacian/lkm_laplacian.py:6-76
* ``estimate_foreground_ml`` pymatting/foreground/estimate_foreground_ml.py:5-253 (C)
* ``estimate_foreground_ml_cupy`` pymatting/foreground/estimate_foreground_ml_cupy.py:5-230
* ``window_laplacian``, ``lbdm_laplacian``, ``knn_laplacian`` pymatting/laplacian/*.py

Parity of this restatement with the reference itself is pinned by
``tests/test_oracle.py`` against the fixtures in ``tests/golden/`` that
``tests/golden/make_golden.py`` produced by running the reference.
"""

import ctypes
import os

import numpy as np
import scipy.sparse
import scipy.sparse.linalg

from . import build as _build

_lib = None


def _load():
    global _lib
    if _lib is None:
        path = _build.build()
        lib = ctypes.CDLL(path)
        i64 = ctypes.c_int64
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int64)
        up = ctypes.POINTER(ctypes.c_uint8)
        lib.oracle_cf_laplacian.argtypes = [dp, i64, i64, ctypes.c_double, i64,
                                            up, dp, ip, ip]
        lib.oracle_cf_laplacian.restype = ctypes.c_int
        lib.oracle_ichol.argtypes = [i64, dp, ip, ip, dp, ip, ip, ctypes.c_double,
                                     ctypes.c_double, i64, ctypes.c_double,
                                     ctypes.c_int]
        lib.oracle_ichol.restype = i64
        lib.oracle_backsub_L.argtypes = [dp, ip, ip, dp, i64]
        lib.oracle_backsub_LT.argtypes = [dp, ip, ip, dp, i64]
        _lib = lib
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


# --------------------------------------------------------------------------
# Laplacian and linear system
# --------------------------------------------------------------------------

def cf_laplacian_arrays(image, epsilon=1e-7, radius=1, is_known=None):
    """Return ``(values, indices, indptr)`` exactly as the reference fills them."""
    lib = _load()
    image = np.ascontiguousarray(image, dtype=np.float64)
    h, w, d = image.shape
    assert d == 3
    n = h * w
    if is_known is None:
        is_known = np.zeros((h, w), dtype=np.bool_)
    known = np.ascontiguousarray(np.asarray(is_known).reshape(h, w), dtype=np.uint8)
    slots = (4 * radius + 1) ** 2
    values = np.zeros(n * slots, dtype=np.float64)
    indices = np.zeros(n * slots, dtype=np.int64)
    indptr = np.zeros(n + 1, dtype=np.int64)
    rc = lib.oracle_cf_laplacian(_p(image, ctypes.c_double), h, w, float(epsilon),
                                 int(radius), _p(known, ctypes.c_uint8),
                                 _p(values, ctypes.c_double),
                                 _p(indices, ctypes.c_int64),
                                 _p(indptr, ctypes.c_int64))
    if rc != 0:
        raise MemoryError("oracle_cf_laplacian failed")
    return values, indices, indptr


def cf_laplacian(image, epsilon=1e-7, radius=1, is_known=None):
    h, w, _ = image.shape
    n = h * w
    values, indices, indptr = cf_laplacian_arrays(image, epsilon, radius, is_known)
    return scipy.sparse.csr_matrix((values, indices, indptr), (n, n))


def trimap_split(trimap, flatten=True, bg_threshold=0.1, fg_threshold=0.9):
    if flatten:
        trimap = trimap.flatten()
    is_fg = trimap >= fg_threshold
    is_bg = trimap <= bg_threshold
    if is_bg.sum() == 0:
        raise ValueError(
            "Trimap did not contain background values (values <= %f)" % bg_threshold)
    if is_fg.sum() == 0:
        raise ValueError(
            "Trimap did not contain foreground values (values >= %f)" % fg_threshold)
    is_known = is_fg | is_bg
    return is_fg, is_bg, is_known, ~is_known


def make_linear_system(L, trimap, lambda_value=100.0, return_c=False):
    is_fg, _bg, is_known, _unk = trimap_split(trimap)
    c = lambda_value * is_known
    b = lambda_value * is_fg
    A = (L + scipy.sparse.diags(c)).tocsr()
    A.sum_duplicates()
    if return_c:
        return A, b, c
    return A, b


# --------------------------------------------------------------------------
# Solver and preconditioners
# --------------------------------------------------------------------------

def cg(A, b, x0=None, atol=0.0, rtol=1e-7, maxiter=10000, callback=None, M=None,
       reorthogonalize=False):
    """Preconditioned CG with the reference's update order and exit tests."""
    if M is None:
        def precondition(v):
            return v
    elif callable(M):
        precondition = M
    else:
        def precondition(v):
            return M.dot(v)
    apply = A if callable(A) else A.dot

    x = np.zeros_like(b) if x0 is None else x0.copy()
    norm_b = np.linalg.norm(b)
    r = b - apply(x)
    norm_r = np.linalg.norm(r)
    if norm_r < atol or norm_r < rtol * norm_b:
        return x
    z = precondition(r)
    p = z.copy()
    rz = np.inner(r, z)
    for _ in range(maxiter):
        r_old = r.copy()
        Ap = apply(p)
        alpha = rz / np.inner(p, Ap)
        x += alpha * p
        r -= alpha * Ap
        norm_r = np.linalg.norm(r)
        if callback is not None:
            callback(A, x, b, norm_b, r, norm_r)
        if norm_r < atol or norm_r < rtol * norm_b:
            return x
        z = precondition(r)
        if reorthogonalize:
            beta = np.inner(r - r_old, z) / rz
            rz = np.inner(r, z)
        else:
            beta = 1.0 / rz
            rz = np.inner(r, z)
            beta *= rz
        p *= beta
        p += z
    raise ValueError(
        "Conjugate gradient descent did not converge within %d iterations" % maxiter)


class CounterCallback:
    def __init__(self):
        self.n = 0

    def __call__(self, A, x, b, norm_b, r, norm_r):
        self.n += 1


def jacobi(A):
    inverse_diagonal = 1.0 / A.diagonal()
    return lambda v: v * inverse_diagonal


def make_P(shape):
    """Full-weighting prolongation/restriction pair (upsample, downsample)."""
    h, w = shape
    h2, w2 = h // 2, w // 2
    n, n2 = h * w, h2 * w2
    wts = np.float64([1, 2, 1, 2, 4, 2, 1, 2, 1]) / 16
    cy, cx = np.divmod(np.arange(n2), w2)
    oy = np.array([-1, -1, -1, 0, 0, 0, 1, 1, 1])
    ox = np.array([-1, 0, 1, -1, 0, 1, -1, 0, 1])
    fx = (2 * cx)[:, None] + ox[None, :]
    fy = (2 * cy)[:, None] + oy[None, :]
    keep = (fx >= 0) & (fx < w) & (fy >= 0) & (fy <= h)
    rows = np.broadcast_to(np.arange(n2)[:, None], keep.shape)[keep]
    cols = (fx + fy * w)[keep]
    vals = np.broadcast_to(wts[None, :], keep.shape)[keep]
    down = scipy.sparse.csr_matrix((vals, (rows, cols)), (n2, n))
    return down.T, down


def _jacobi_sweeps(A, diag, b, x, count, omega):
    if x is None:
        if count > 0:
            x = omega * b / diag
            count -= 1
        else:
            x = np.zeros_like(b)
    for _ in range(count):
        x = x + omega * (b - A.dot(x)) / diag
    return x


def _vcycle(A, b, shape, cache, pre, post, omega, direct):
    h, w = shape
    if h * w <= direct:
        return scipy.sparse.linalg.spsolve(A, b)
    if shape not in cache:
        up, down = make_P(shape)
        cache[shape] = (up, down, down.dot(A).dot(up), A.diagonal())
    up, down, coarse_A, diag = cache[shape]
    x = _jacobi_sweeps(A, diag, b, None, pre, omega)
    coarse_b = down.dot(b - A.dot(x))
    x += up.dot(_vcycle(coarse_A, coarse_b, (h // 2, w // 2), cache, pre, post,
                        omega, direct))
    return _jacobi_sweeps(A, diag, b, x, post, omega)


def vcycle(A, shape, num_pre_iter=1, num_post_iter=1, omega=0.8,
           direct_solve_size=64, cache=None):
    if cache is None:
        cache = {}
    return lambda r: _vcycle(A, r, shape, cache, num_pre_iter, num_post_iter,
                             omega, direct_solve_size)


class CholeskyDecomposition:
    def __init__(self, Ltuple):
        self.Ltuple = Ltuple

    @property
    def L(self):
        Lv, Lr, Lp = self.Ltuple
        n = len(Lp) - 1
        return scipy.sparse.csc_matrix(self.Ltuple, (n, n))

    def __call__(self, b):
        lib = _load()
        Lv, Lr, Lp = self.Ltuple
        x = np.array(b, dtype=np.float64, copy=True)
        n = len(x)
        lib.oracle_backsub_L(_p(Lv, ctypes.c_double), _p(Lr, ctypes.c_int64),
                             _p(Lp, ctypes.c_int64), _p(x, ctypes.c_double), n)
        lib.oracle_backsub_LT(_p(Lv, ctypes.c_double), _p(Lr, ctypes.c_int64),
                              _p(Lp, ctypes.c_int64), _p(x, ctypes.c_double), n)
        return x


ICHOL_SHIFTS = [0.0, 1e-4, 1e-3, 1e-2, 0.1, 0.5, 1.0, 10.0, 100, 1e3, 1e4, 1e5]


def ichol(A, discard_threshold=1e-4, shifts=ICHOL_SHIFTS, max_nnz=int(4e9 / 16),
          relative_discard_threshold=0.0, diag_keep_discarded=True):
    lib = _load()
    if isinstance(A, scipy.sparse.csr_matrix):
        A = A.T
    if not isinstance(A, scipy.sparse.csc_matrix):
        raise ValueError("Matrix A must be a scipy.sparse.csc_matrix")
    if not A.has_canonical_format:
        A.sum_duplicates()
    m, n = A.shape
    assert m == n
    Av = np.ascontiguousarray(A.data, dtype=np.float64)
    Ar = np.ascontiguousarray(A.indices, dtype=np.int64)
    Ap = np.ascontiguousarray(A.indptr, dtype=np.int64)
    # Fill stays inside the row envelope of A (row i spans columns
    # first_col[i]..i), so that envelope bounds the factor; sizing by it
    # instead of max_nnz keeps memory small. The max_nnz test stays exact.
    first_col = np.arange(n, dtype=np.int64)
    if A.nnz:
        cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(Ap))
        np.minimum.at(first_col, Ar, cols)
    envelope = int(np.sum(np.arange(n, dtype=np.int64) - np.minimum(first_col, np.arange(n)) + 1))
    cap = int(max(min(max_nnz, envelope), 1))
    Lv = np.empty(cap, dtype=np.float64)
    Lr = np.empty(cap, dtype=np.int64)
    Lp = np.zeros(n + 1, dtype=np.int64)
    nnz = -1
    for shift in shifts:
        nnz = lib.oracle_ichol(n, _p(Av, ctypes.c_double), _p(Ar, ctypes.c_int64),
                               _p(Ap, ctypes.c_int64), _p(Lv, ctypes.c_double),
                               _p(Lr, ctypes.c_int64), _p(Lp, ctypes.c_int64),
                               float(discard_threshold), float(shift), int(max_nnz),
                               float(relative_discard_threshold),
                               int(bool(diag_keep_discarded)))
        if nnz >= 0:
            break
        if nnz == -2 or (nnz == -3):
            raise ValueError(
                "Thresholded incomplete Cholesky decomposition failed because more "
                "than max_nnz non-zero elements were created. Try increasing max_nnz "
                "or discard_threshold.")
    if nnz < 0:
        raise ValueError(
            "Thresholded incomplete Cholesky decomposition failed due to insufficient "
            "positive-definiteness of matrix A and diagonal shifts did not help.")
    return CholeskyDecomposition((Lv[:nnz].copy(), Lr[:nnz].copy(), Lp))


# --------------------------------------------------------------------------
# Alpha estimation
# --------------------------------------------------------------------------

def estimate_alpha_cf(image, trimap, preconditioner=None, laplacian_kwargs={},
                      cg_kwargs={}):
    if preconditioner is None:
        preconditioner = ichol
    is_fg, _bg, is_known, is_unknown = trimap_split(trimap)
    L = cf_laplacian(image, **laplacian_kwargs, is_known=is_known)
    L_U = L[is_unknown, :][:, is_unknown]
    R = L[is_unknown, :][:, is_known]
    m = is_fg[is_known]
    x = trimap.copy().ravel()
    x[is_unknown] = cg(L_U, -R.dot(m), M=preconditioner(L_U), **cg_kwargs)
    return np.clip(x, 0, 1).reshape(trimap.shape)


def solve_soft(image, trimap, preconditioner="vcycle", rtol=1e-7, atol=0.0,
               lambda_value=100.0, maxiter=10000, epsilon=1e-7):
    """Soft-constraint full-grid solve: returns ``(x, iterations)``."""
    h, w = trimap.shape
    A, b = make_linear_system(cf_laplacian(image, epsilon=epsilon), trimap,
                              lambda_value)
    if preconditioner == "vcycle":
        M = vcycle(A, (h, w))
    elif preconditioner == "jacobi":
        M = jacobi(A)
    elif preconditioner == "ichol":
        M = ichol(A)
    else:
        M = None
    cb = CounterCallback()
    x = cg(A, b, M=M, rtol=rtol, atol=atol, maxiter=maxiter, callback=cb)
    return x, cb.n


# --------------------------------------------------------------------------
# Gradients of the soft-constraint alpha (no reference counterpart: PyMatting
# has no autodiff). FP64 restatement used to check the adjoint kernels.
# --------------------------------------------------------------------------

def soft_alpha_exact(image, trimap, lambda_value=100.0, epsilon=1e-7):
    """alpha = A^-1 b for make_linear_system(cf_laplacian(image), trimap), solved
    directly (sparse LU), as a smooth function of the image."""
    L = cf_laplacian(image, epsilon)
    A, b = make_linear_system(L, trimap, lambda_value)
    return scipy.sparse.linalg.spsolve(A.tocsc(), b)


def cf_laplacian_vjp(image, x, mu, epsilon=1e-7):
    """d(mu' L(image) x) / d image, shape (h, w, 3), for the radius-1 matting
    Laplacian with every window active (cf_laplacian.py:31-129 differentiated):
    per window, mu' L_w x = sum mu_i x_i - 9 mu_bar x_bar - u' D v / 9 with
    u = sum mu_i c_i, v = sum x_i c_i, D = ((eps I + sum c_i c_i') / 9)^-1."""
    image = np.asarray(image, dtype=np.float64)
    h, w, _ = image.shape
    x = np.asarray(x, dtype=np.float64).reshape(h, w)
    mu = np.asarray(mu, dtype=np.float64).reshape(h, w)
    ys, xs = np.mgrid[1:h - 1, 1:w - 1]
    ys, xs = ys.ravel(), xs.ravel()
    offs = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    py = np.stack([ys + dy for dy, dx in offs], axis=1)          # (nw, 9)
    px = np.stack([xs + dx for dy, dx in offs], axis=1)
    I = image[py, px]                                            # (nw, 9, 3)
    c = I - I.mean(axis=1, keepdims=True)
    a = (epsilon * np.eye(3) + np.einsum("wki,wkj->wij", c, c)) / 9.0
    D = np.linalg.inv(a)
    m = mu[py, px]
    xv = x[py, px]
    u = np.einsum("wk,wki->wi", m, c)
    v = np.einsum("wk,wki->wi", xv, c)
    p = np.einsum("wij,wj->wi", D, u)
    q = np.einsum("wij,wj->wi", D, v)
    dm = m - m.mean(axis=1, keepdims=True)
    dx = xv - xv.mean(axis=1, keepdims=True)
    cq = np.einsum("wki,wi->wk", c, q)
    cp = np.einsum("wki,wi->wk", c, p)
    term = (dm[:, :, None] * q[:, None, :] + dx[:, :, None] * p[:, None, :]
            - (p[:, None, :] * cq[:, :, None] + q[:, None, :] * cp[:, :, None]) / 9.0) / 9.0
    grad = np.zeros((h, w, 3))
    np.add.at(grad, (py.ravel(), px.ravel()), -term.reshape(-1, 3))
    return grad


def soft_alpha_grad(image, trimap, g, lambda_value=100.0, epsilon=1e-7):
    """d(g . alpha) / d image with alpha = soft_alpha_exact(image, trimap):
    adjoint solve A mu = g, then -d(mu' L x) / d image."""
    L = cf_laplacian(image, epsilon)
    A, b = make_linear_system(L, trimap, lambda_value)
    lu = scipy.sparse.linalg.splu(A.tocsc())
    x = lu.solve(b)
    mu = lu.solve(np.asarray(g, dtype=np.float64).ravel())
    return -cf_laplacian_vjp(image, x, mu, epsilon)


# --------------------------------------------------------------------------
# Large-kernel matting Laplacian (pymatting/laplacian/lkm_laplacian.py:6-76)
# --------------------------------------------------------------------------

def _box(a, r, mode):
    """Box sums over (2r+1)^2 windows along the first two axes: 'valid'
    (h-2r, w-2r) or 'full' (h+2r, w+2r, zeros outside), by cumulative sums
    (pymatting/util/boxfilter.py:6-82 restated)."""
    if mode == "full":
        pad = [(2 * r, 2 * r), (2 * r, 2 * r)] + [(0, 0)] * (a.ndim - 2)
        a = np.pad(a, pad)
    k = 2 * r + 1
    c = np.cumsum(a, axis=0)
    c = np.concatenate([np.zeros_like(c[:1]), c], axis=0)
    a = c[k:] - c[:-k]
    c = np.cumsum(a, axis=1)
    c = np.concatenate([np.zeros_like(c[:, :1]), c], axis=1)
    return c[:, k:] - c[:, :-k]


def lkm_laplacian(image, epsilon=1e-7, radius=10):
    """(L_matvec, diag_L) of the large-kernel Laplacian."""
    image = np.asarray(image, dtype=np.float64)
    r = radius
    area = (2 * r + 1) ** 2
    h, w, _ = image.shape
    means = _box(image, r, "valid") / area
    covs = _box(image[:, :, :, None] * image[:, :, None, :], r, "valid") / area
    covs -= means[:, :, :, None] * means[:, :, None, :]
    V = np.linalg.inv(covs + epsilon / area * np.eye(3)) / area
    Vm = np.einsum("...ij,...j->...i", V, means)
    mVm = 1.0 / area + np.einsum("...i,...i->...", means, Vm)
    c = _box(np.ones((h - 2 * r, w - 2 * r)), r, "full")

    def L_matvec(p):
        p = np.asarray(p, dtype=np.float64).reshape(h, w)
        ps = _box(p, r, "valid")
        pI = _box(p[:, :, None] * image, r, "valid")
        out = c * p
        t3 = ps[:, :, None] * Vm - np.einsum("...ij,...j->...i", V, pI)
        out += np.einsum("...i,...i->...", image, _box(t3, r, "full"))
        t1 = ps * mVm - np.einsum("...i,...i->...", pI, Vm)
        out -= _box(t1, r, "full")
        return out.ravel()

    diag = _box(1.0 - mVm, r, "full")
    t = 2 * _box(Vm, r, "full") - np.einsum("...ij,...j->...i", _box(V, r, "full"), image)
    diag += np.einsum("...i,...i->...", image, t)
    return L_matvec, diag.ravel()


# --------------------------------------------------------------------------
# Foreground / background estimation
# --------------------------------------------------------------------------

def _fg_inputs(image, alpha):
    image = np.ascontiguousarray(image, dtype=np.float32)
    alpha = np.ascontiguousarray(alpha, dtype=np.float32)
    h, w = alpha.shape
    assert image.ndim == 3 and image.shape[:2] == (h, w) and 1 <= image.shape[2] <= 8
    return image, alpha, h, w


def fg_mean_colors(image, alpha):
    """estimate_foreground_ml.py:79-95: the 2 depth seed colours (F then B)."""
    lib = _load()
    image, alpha, h, w = _fg_inputs(image, alpha)
    depth = image.shape[2]
    seed = np.zeros(2 * depth, dtype=np.float32)
    lib.oracle_fg_mean_colors(_p(image, ctypes.c_float), _p(alpha, ctypes.c_float),
                              ctypes.c_int64(h), ctypes.c_int64(w), ctypes.c_int(depth),
                              _p(seed, ctypes.c_float))
    return seed


def fg_levels(h, w):
    """estimate_foreground_ml.py:101-105: the (h, w) of every level."""
    lib = _load()
    hs = np.zeros(64, dtype=np.int64)
    ws = np.zeros(64, dtype=np.int64)
    lib.oracle_fg_levels.restype = ctypes.c_int
    n = lib.oracle_fg_levels(ctypes.c_int64(h), ctypes.c_int64(w), _p(hs, ctypes.c_int64),
                             _p(ws, ctypes.c_int64), 64)
    if n < 0:
        raise ZeroDivisionError("division by zero")
    return list(zip(hs[:n].tolist(), ws[:n].tolist()))


def estimate_foreground_ml(image, alpha, regularization=1e-5, n_small_iterations=10,
                           n_big_iterations=2, small_size=32, return_background=False,
                           gradient_weight=1.0, seed=None):
    """estimate_foreground_ml.py:186-253 over _estimate_fb_ml (:61-183).

    ``seed`` replaces the 2 depth mean colours the reference starts from."""
    lib = _load()
    image, alpha, h, w = _fg_inputs(image, alpha)
    depth = image.shape[2]
    F = np.zeros((h, w, depth), dtype=np.float32)
    B = np.zeros((h, w, depth), dtype=np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    sp = None
    if seed is not None:
        seed = np.ascontiguousarray(seed, dtype=np.float32).reshape(2 * depth)
        sp = _p(seed, ctypes.c_float)
    lib.oracle_fg_ml.restype = ctypes.c_int
    lib.oracle_fg_ml.argtypes = [fp, fp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                 ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_float, fp, fp, fp]
    rc = lib.oracle_fg_ml(_p(image, ctypes.c_float), _p(alpha, ctypes.c_float), h, w, depth,
                          float(regularization), int(n_small_iterations),
                          int(n_big_iterations), int(small_size), float(gradient_weight),
                          sp, _p(F, ctypes.c_float), _p(B, ctypes.c_float))
    if rc == -1:
        raise ZeroDivisionError("division by zero")
    if rc != 0:
        raise ValueError("oracle_fg_ml failed (%d)" % rc)
    if return_background:
        return F, B
    return F


def estimate_foreground_ml_cupy(input_image, input_alpha, regularization=1e-5,
                                n_small_iterations=10, n_big_iterations=2, small_size=32,
                                return_background=False):
    """pymatting/foreground/estimate_foreground_ml_cupy.py:110-230 and its
    kernels :5-107 (Jacobi iterations), in float32 numpy.

    Restates the reference's flat buffers exactly. F and B start as the
    colour of pixel (0, 0). Each level resizes the buffer named ``F`` (read
    with the previous level's shape) into ``F_prev`` and iterates with
    swaps. The result is ``F``, which is the second newest iterate when the
    last level runs iterations. The reference compiles its kernel with
    NVRTC (fused multiply-adds allowed), so results agree to float32
    rounding, not bitwise."""
    image = np.ascontiguousarray(input_image, dtype=np.float32)
    alpha0 = np.ascontiguousarray(input_alpha, dtype=np.float32)
    h0, w0, depth = image.shape
    assert depth == 3
    f32 = np.float32
    reg = f32(regularization)
    n = h0 * w0 * depth

    def resize(dst, src, ws, hs, wd, hd, d):
        ys = np.minimum(np.arange(hd) * hs // hd, hs - 1)
        xs = np.minimum(np.arange(wd) * ws // wd, ws - 1)
        s3 = src[:hs * ws * d].reshape(hs, ws, d)
        dst[:hd * wd * d] = s3[ys][:, xs].reshape(-1)

    F_prev = np.zeros(n, np.float32)
    B_prev = np.zeros(n, np.float32)
    F = np.zeros(n, np.float32)
    B = np.zeros(n, np.float32)
    image_level = np.zeros(n, np.float32)
    alpha_level = np.zeros(h0 * w0, np.float32)
    flat_image = image.reshape(-1)
    flat_alpha = alpha0.reshape(-1)
    n_levels = (max(w0, h0) - 1).bit_length()
    w_prev = h_prev = 1
    resize(F, flat_image, w0, h0, w_prev, h_prev, depth)
    resize(B, flat_image, w0, h0, w_prev, h_prev, depth)
    for i_level in range(n_levels + 1):
        w = round(w0 ** (i_level / n_levels))
        h = round(h0 ** (i_level / n_levels))
        resize(image_level, flat_image, w0, h0, w, h, depth)
        resize(alpha_level, flat_alpha, w0, h0, w, h, 1)
        resize(F_prev, F, w_prev, h_prev, w, h, depth)
        resize(B_prev, B, w_prev, h_prev, w, h, depth)
        n_iter = n_big_iterations
        if min(w, h) <= small_size:
            n_iter = n_small_iterations
        m = h * w
        img = image_level[:m * 3].reshape(h, w, 3)
        a0 = alpha_level[:m].reshape(h, w)
        a1 = f32(1.0) - a0
        xm = np.maximum(np.arange(w) - 1, 0)
        xp = np.minimum(np.arange(w) + 1, w - 1)
        ym = np.maximum(np.arange(h) - 1, 0)
        yp = np.minimum(np.arange(h) + 1, h - 1)
        for _ in range(n_iter):
            Fp = F_prev[:m * 3].reshape(h, w, 3)
            Bp = B_prev[:m * 3].reshape(h, w, 3)
            b0 = a0[:, :, None] * img
            b1 = a1[:, :, None] * img
            a_sum = np.zeros_like(a0)
            for an, Fn, Bn in ((a0[:, xm], Fp[:, xm], Bp[:, xm]),
                               (a0[:, xp], Fp[:, xp], Bp[:, xp]),
                               (a0[ym, :], Fp[ym, :], Bp[ym, :]),
                               (a0[yp, :], Fp[yp, :], Bp[yp, :])):
                da = reg + np.abs(a0 - an)
                a_sum = a_sum + da
                b0 = b0 + da[:, :, None] * Fn
                b1 = b1 + da[:, :, None] * Bn
            a00 = a0 * a0 + a_sum
            a11 = a1 * a1 + a_sum
            a01 = a0 * a1
            inv_det = (f32(1.0) / (a00 * a11 - a01 * a01))[:, :, None]
            # fmaxf(0, fminf(1, v)): NaN-ignoring, like the CUDA functions
            Fo = np.fmax(f32(0.0), np.fmin(f32(1.0), inv_det * (a11[:, :, None] * b0 -
                                                               a01[:, :, None] * b1)))
            Bo = np.fmax(f32(0.0), np.fmin(f32(1.0), inv_det * (a00[:, :, None] * b1 -
                                                               a01[:, :, None] * b0)))
            F[:m * 3] = Fo.reshape(-1)
            B[:m * 3] = Bo.reshape(-1)
            F_prev, F = F, F_prev
            B_prev, B = B, B_prev
        w_prev, h_prev = w, h
    F = F.reshape(h0, w0, depth).copy()
    B = B.reshape(h0, w0, depth).copy()
    if return_background:
        return F, B
    return F


# --------------------------------------------------------------------------
# uniform_laplacian / rw_laplacian (through weights_to_laplacian)
# --------------------------------------------------------------------------

def window_laplacian(image, radius=1, regularization=0.0, kind="uniform"):
    """pymatting/laplacian/uniform_laplacian.py and rw_laplacian.py with
    util/util.py weights_to_laplacian (:840-875), row by row in the
    reference's operation order: W's duplicate (clamped) entries summed,
    rowsum(W) over ascending columns, W' = W / rowsum, rowsum(W') over
    descending columns (the order scipy's sparse product leaves each row
    in), L = diag(regularization + rowsum(W')) - W'. Returns a CSR matrix
    with sorted columns."""
    image = np.asarray(image, dtype=np.float64)
    h, w = image.shape[:2]
    r = int(radius)
    flat = image.reshape(-1, image.shape[2]) if image.ndim == 3 else None
    indptr = [0]
    indices, data = [], []
    for y in range(h):
        for x in range(w):
            i = x + y * w
            cnt = {}
            for dy in range(-r, r + 1):
                for dx in range(-r, r + 1):
                    j = min(max(x + dx, 0), w - 1) + min(max(y + dy, 0), h - 1) * w
                    cnt[j] = cnt.get(j, 0) + 1
            cols = sorted(cnt)
            vals = []
            for j in cols:
                if kind == "uniform":
                    wv = 1.0
                else:
                    nrm = float(np.linalg.norm(flat[i] - flat[j]))
                    wv = float(np.exp(-900 * nrm ** 2))
                v = wv
                for _ in range(cnt[j] - 1):
                    v = v + wv
                vals.append(v)
            s1 = 0.0
            for v in vals:
                s1 = s1 + v
            f = 1.0 / s1
            wp = [f * v for v in vals]
            s2 = 0.0
            for v in reversed(wp):
                s2 = s2 + v
            d = regularization + s2
            for j, v in zip(cols, wp):
                indices.append(j)
                data.append(d - v if j == i else -v)
            indptr.append(len(indices))
    n = h * w
    return scipy.sparse.csr_matrix((np.array(data), np.array(indices), np.array(indptr)),
                                   shape=(n, n))


def lbdm_laplacian(image, epsilon=1e-7, radius=1):
    """pymatting/laplacian/lbdm_laplacian.py restated with numpy: per
    interior window X = [colours, 1], K = X X^T, F = solve(K + eps I, K),
    T = (I - F)(I - F)^T, summed over windows into a CSR matrix by scipy (the
    same COO -> CSR conversion as the reference)."""
    image = np.asarray(image, dtype=np.float64)
    h, w = image.shape[:2]
    r = int(radius)
    n = h * w
    s = 2 * r + 1
    area = s * s
    idx = np.arange(n).reshape(h, w)
    rows, cols, vals = [np.zeros(1, np.int64)], [np.zeros(1, np.int64)], [np.zeros(1)]
    for y in range(r, h - r):
        for x in range(r, w - r):
            win = image[y - r:y + r + 1, x - r:x + r + 1].reshape(area, 3)
            X = np.concatenate([win, np.ones((area, 1))], axis=1)
            K = X @ X.T
            F = np.linalg.solve(K + epsilon * np.eye(area), K)
            T2 = np.eye(area) - F
            T = T2 @ T2.T
            wi = idx[y - r:y + r + 1, x - r:x + r + 1].ravel()
            rows.append(np.repeat(wi, area))
            cols.append(np.tile(wi, area))
            vals.append(T.ravel())
    return scipy.sparse.csr_matrix((np.concatenate(vals), (np.concatenate(rows),
                                                           np.concatenate(cols))), shape=(n, n))



def knn(f, k):
    """Indices of the k nearest feature rows of every row (oracle/knn.c: the
    k-d tree's distance, the k smallest by (distance, index))."""
    lib = _load()
    f = np.ascontiguousarray(f, dtype=np.float32)
    n, dims = f.shape
    out = np.zeros((n, k), dtype=np.int64)
    lib.oracle_knn.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int64, ctypes.c_int,
                               ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    lib.oracle_knn(_p(f, ctypes.c_float), n, dims, k, _p(out, ctypes.c_int64))
    return out


def knn_laplacian(image, n_neighbors=[20, 10], distance_weights=[2.0, 0.1], kernel="binary"):
    """pymatting/laplacian/knn_laplacian.py restated with oracle.knn in place
    of the reference's k-d tree (same neighbours except among equal
    distances), then the reference's own scipy assembly: W = B + B^T,
    normalize_rows, L = I - W."""
    image = np.asarray(image, dtype=np.float64)
    h, w = image.shape[:2]
    r, g, b = image.reshape(-1, 3).T
    n = w * h
    x = np.tile(np.linspace(0, 1, w), h)
    y = np.repeat(np.linspace(0, 1, h), w)
    i, j, coo_data = [], [], []
    for k, dw in zip(n_neighbors, distance_weights):
        f = np.stack([r, g, b, dw * x, dw * y], axis=1, out=np.zeros((n, 5), dtype=np.float32))
        nbr = knn(f, k)
        i.append(np.repeat(np.arange(n), k))
        j.append(nbr.ravel())
        W_ij = np.ones(k * n)
        if kernel == "soft":
            W_ij -= np.abs(f[i[-1]] - f[j[-1]]).sum(axis=1) / f.shape[1]
        coo_data.append(W_ij)
    ij = np.concatenate(i + j)
    ji = np.concatenate(j + i)
    coo_data = np.concatenate(coo_data + coo_data)
    W = scipy.sparse.csr_matrix((coo_data, (ij, ji)), (n, n))
    rs = W.dot(np.ones(n))
    W = scipy.sparse.diags(1.0 / rs).dot(W)
    return scipy.sparse.identity(n) - W
