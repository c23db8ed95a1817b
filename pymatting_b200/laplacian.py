"""Closed-form matting Laplacian and the soft-constraint linear system.

Drop-in for ``pymatting.laplacian.cf_laplacian`` (cf_laplacian.py:132-177)
and ``pymatting.laplacian.make_linear_system`` (laplacian.py:5-60).

Both return ``scipy.sparse.csr_matrix`` objects, as the reference does, but
the matrix is assembled on the GPU and stays there: the returned object is a
``DeviceCSRMatrix`` (a ``csr_matrix`` subclass) whose ``data`` / ``indices``
/ ``indptr`` arrays are only copied to the host the first time host code
touches them. Solvers of this package recognise a matrix whose host arrays
were never exposed and use its device form directly (the 13-plane half
stencil for the solve, the exact CSR arrays for everything else). Once the
host arrays exist the matrix is treated like any other scipy matrix, so
in-place edits are always honoured.
"""

import numpy as np
import scipy.sparse
import torch

from . import _device as dev
from . import _ffi
from .util import trimap_split

__all__ = ["cf_laplacian", "uniform_laplacian", "rw_laplacian", "lbdm_laplacian", "knn_laplacian",
           "make_linear_system",
           "DeviceCSRMatrix", "CFSource", "device_source", "device_csr_arrays"]


class CFSource:
    """Device-side description of a closed-form Laplacian system.

    Holds the image and masks on the device and assembles, on demand, the
    forms the solvers need: the half-stencil planes (radius 1), the
    reference's CSR arrays (exactly as ``cf_laplacian`` builds them) and
    the canonical CSR of ``L + diag(diag_value * diag_mask)``.
    """

    def __init__(self, image_t, known_t, h, w, epsilon, radius, diag_mask_t=None,
                 diag_value=0.0):
        self.image = image_t
        self.known = known_t
        self.h, self.w = int(h), int(w)
        self.epsilon = float(epsilon)
        self.radius = int(radius)
        self.diag_mask = diag_mask_t
        self.diag_value = float(diag_value)
        self._planes = None
        self._csr = None

    @property
    def n(self):
        return self.h * self.w

    @property
    def pitch(self):
        return int(_ffi.lib().pmb_grid_pitch(self.w))

    @property
    def plane_elems(self):
        return 13 * self.h * self.pitch

    def with_diag(self, mask_t, value):
        return CFSource(self.image, self.known, self.h, self.w, self.epsilon, self.radius,
                        mask_t, value)

    def assemble_planes(self, out):
        """Write the 13 half-stencil planes into device tensor ``out``."""
        if self.radius != 1:
            raise NotImplementedError("the stencil solver supports radius=1 Laplacians")
        _ffi.check(_ffi.lib().pmb_cf_laplacian_planes(
            dev.ptr(self.image), dev.ptr(self.known), self.h, self.w, self.epsilon,
            dev.ptr(self.diag_mask), self.diag_value, dev.ptr(out), dev.stream()),
            "cf_laplacian planes")
        return out

    def planes(self):
        if self._planes is None:
            self._planes = self.assemble_planes(dev.empty(self.plane_elems, torch.float64))
        return self._planes

    def ell(self):
        """Reference CSR arrays of L (+ diagonal): (values, indices, indptr)."""
        S = (4 * self.radius + 1) ** 2
        values = dev.empty(self.n * S, torch.float64)
        indices = dev.empty(self.n * S, torch.int64)
        indptr = dev.empty(self.n + 1, torch.int64)
        _ffi.check(_ffi.lib().pmb_cf_laplacian_ell(
            dev.ptr(self.image), dev.ptr(self.known), self.h, self.w, self.radius,
            self.epsilon, dev.ptr(self.diag_mask), self.diag_value, dev.ptr(values),
            dev.ptr(indices), dev.ptr(indptr), dev.stream()), "cf_laplacian")
        return values, indices, indptr

    def csr(self):
        """Device CSR arrays identical to the host matrix this source stands for.

        Without a diagonal term this is ``cf_laplacian``'s non-canonical CSR
        ((4r+1)^2 slots per row). With one it is the canonical CSR of
        ``L + C`` that scipy forms in ``make_linear_system`` (explicit zeros
        and the out-of-image slots dropped)."""
        if self._csr is not None:
            return self._csr
        values, indices, indptr = self.ell()
        if self.diag_mask is None:
            self._csr = (indptr, indices, values)
            return self._csr
        lib = _ffi.lib()
        n = self.n
        rowptr = dev.empty(n + 1, torch.int64)
        scratch = dev.empty(int(lib.pmb_scan_scratch_elems(n + 1)), torch.int64)
        _ffi.check(lib.pmb_ell_csr_rowptr(dev.ptr(values), self.h, self.w, self.radius,
                                          dev.ptr(rowptr), dev.ptr(scratch), dev.stream()),
                   "make_linear_system rowptr")
        nnz = int(rowptr[n].item())
        cidx = dev.empty(max(nnz, 1), torch.int64)
        data = dev.empty(max(nnz, 1), torch.float64)
        _ffi.check(lib.pmb_ell_csr_fill(dev.ptr(values), self.h, self.w, self.radius,
                                        dev.ptr(rowptr), dev.ptr(cidx), dev.ptr(data),
                                        dev.stream()), "make_linear_system fill")
        self._csr = (rowptr, cidx[:nnz], data[:nnz])
        return self._csr


class DeviceCSRMatrix(scipy.sparse.csr_matrix):
    """``csr_matrix`` whose arrays live on the GPU until host code reads them.

    ``data``, ``indices`` and ``indptr`` are deliberately absent from the
    instance until first access; ``__getattr__`` then copies them from the
    device. Every scipy operation therefore works unchanged. Construction by
    scipy itself (results of arithmetic, ``copy()``...) falls through to the
    plain ``csr_matrix`` constructor.
    """

    def __init__(self, arg1=None, shape=None, dtype=None, copy=False, maxprint=None, *,
                 pmb_source=None, pmb_arrays=None):
        if pmb_source is None and pmb_arrays is None:
            super().__init__(arg1, shape=shape, dtype=dtype, copy=copy, maxprint=maxprint)
            return
        d = self.__dict__
        d["_pmb_source"] = pmb_source
        d["_pmb_arrays"] = pmb_arrays
        self._shape = tuple(int(s) for s in shape)
        self.maxprint = 50 if maxprint is None else maxprint

    def __getattr__(self, name):
        d = self.__dict__
        if name in ("data", "indices", "indptr") and (
                "_pmb_source" in d or "_pmb_arrays" in d):
            self._pmb_materialize()
            return d[name]
        raise AttributeError(name)

    def _pmb_materialize(self):
        d = self.__dict__
        if "data" in d:
            return
        indptr, indices, data = device_csr_arrays(self)
        d["indptr"] = dev.to_host(indptr)
        d["indices"] = dev.to_host(indices)
        d["data"] = dev.to_host(data)

    @property
    def dtype(self):
        if "data" not in self.__dict__:
            return np.dtype(np.float64)
        return self.data.dtype

    @dtype.setter
    def dtype(self, newtype):
        self.data = self.data.view(newtype)

    @property
    def pmb_on_device(self):
        """True while the host arrays were never exposed."""
        return "data" not in self.__dict__

    def __reduce__(self):
        self._pmb_materialize()
        return (scipy.sparse.csr_matrix, ((self.data, self.indices, self.indptr), self.shape))


def device_source(A):
    """The CFSource behind ``A`` if its host arrays were never exposed."""
    if isinstance(A, DeviceCSRMatrix) and A.pmb_on_device:
        return A.__dict__.get("_pmb_source")
    return None


def device_csr_arrays(A):
    """Device (indptr, indices, data) of a DeviceCSRMatrix."""
    d = A.__dict__
    arrays = d.get("_pmb_arrays")
    if arrays is None:
        arrays = d["_pmb_source"].csr()
        d["_pmb_arrays"] = arrays
    return arrays


def _image_to_device(image):
    if dev.is_device_tensor(image):
        t = image.to(torch.float64).contiguous()
    elif isinstance(image, torch.Tensor):
        t = dev.to_device(image, torch.float64)     # pinned host tensors copy directly
    else:
        t = dev.to_device(np.asarray(image), torch.float64)
    return t


def _mask_to_device(mask, h, w):
    if mask is None:
        return None
    if dev.is_device_tensor(mask):
        return mask.reshape(h, w).to(torch.uint8).contiguous()
    return dev.to_device(np.asarray(mask).reshape(h, w).astype(np.uint8), torch.uint8)


def cf_laplacian(image, epsilon=1e-7, radius=1, is_known=None):
    """Closed-form matting Laplacian of Levin et al., assembled on the GPU.

    Same signature and result as pymatting's ``cf_laplacian``
    (pymatting/laplacian/cf_laplacian.py:132): an ``(h*w, h*w)`` CSR matrix
    with ``(4r+1)^2`` stored entries per row, out-of-image slots holding
    column 0 and value 0, and values bitwise equal to the reference.
    ``image`` is ``(h, w, 3)`` (numpy or a CUDA tensor); windows whose pixels
    are all in ``is_known`` are skipped. ``radius`` 1 or 2.
    """
    h, w, d = image.shape
    assert d == 3
    if radius not in (1, 2):
        raise NotImplementedError("cf_laplacian on the device supports radius 1 and 2")
    src = CFSource(_image_to_device(image), _mask_to_device(is_known, h, w), h, w,
                   epsilon, radius)
    n = h * w
    return DeviceCSRMatrix(shape=(n, n), pmb_source=src)


def make_linear_system(L, trimap, lambda_value=100.0, return_c=False):
    """``A = L + lambda * diag(is_known)``, ``b = lambda * is_fg``.

    Same contract as pymatting/laplacian/laplacian.py:5-60. When ``L`` is a
    device-resident Laplacian of this package, ``A`` is assembled on the GPU
    (the diagonal folded into the centre plane) and returned as a
    DeviceCSRMatrix whose host arrays equal scipy's canonical ``L + C``.
    """
    h, w = trimap.shape[:2]
    is_fg, is_bg, is_known, is_unknown = trimap_split(trimap)
    c = lambda_value * is_known
    b = lambda_value * is_fg
    src = device_source(L)
    if src is not None and src.diag_mask is None and src.n == h * w:
        known_t = _mask_to_device(is_known, h, w)
        A = DeviceCSRMatrix(shape=L.shape, pmb_source=src.with_diag(known_t, lambda_value))
    else:
        from .sparse import add_diagonal
        A = add_diagonal(L, c)
    if return_c:
        return A, b, c
    return A, b


def _window_extents(n, r):
    """Prefix sums of the clamped window extent min(v + r, n - 1) - max(v - r, 0) + 1."""
    v = np.arange(n)
    ext = np.minimum(v + r, n - 1) - np.maximum(v - r, 0) + 1
    return np.concatenate([[0], np.cumsum(ext)]).astype(np.int64)


def _window_laplacian(mode, image, radius, regularization):
    h, w = image.shape[:2]
    r = int(radius)
    px = _window_extents(w, r)
    py = _window_extents(h, r)
    nnz = int(py[-1] * px[-1])
    n = h * w
    img = _image_to_device(image) if mode == 1 else None
    rowptr = dev.empty(n + 1, torch.int64)
    cols = dev.empty(max(nnz, 1), torch.int64)
    vals = dev.empty(max(nnz, 1), torch.float64)
    # held in names until the launch is queued: a freed temporary's block
    # could be handed to the next upload before the kernel reads it
    px_t = dev.to_device(px)
    py_t = dev.to_device(py)
    _ffi.check(_ffi.lib().pmb_window_laplacian(
        mode, dev.ptr(img), h, w, r, float(regularization), dev.ptr(px_t), dev.ptr(py_t),
        dev.ptr(rowptr), dev.ptr(cols), dev.ptr(vals), dev.stream()), "pmb_window_laplacian")
    return DeviceCSRMatrix(shape=(n, n), pmb_arrays=(rowptr, cols[:nnz], vals[:nnz]))


def uniform_laplacian(image, radius=1):
    """Uniform-weight Laplacian over (2 radius + 1)^2 windows, normalised:
    pymatting/laplacian/uniform_laplacian.py (weights_to_laplacian of a box
    convolution matrix). Canonical CSR on the device."""
    return _window_laplacian(0, image, radius, 0.0)


def rw_laplacian(image, sigma=0.033, radius=1, regularization=1e-8):
    """Random-walk Laplacian: pymatting/laplacian/rw_laplacian.py. Weights
    exp(-900 |z_i - z_j|^2) over (2 radius + 1)^2 windows with clamped
    neighbours, row-normalised, plus ``regularization`` on the diagonal. As
    in the reference, ``sigma`` does not enter the weights."""
    return _window_laplacian(1, image, radius, regularization)


def _lbdm_extents(n, r):
    """Prefix sums of the number of coordinates sharing a window with v:
    window centres [max(r, v - r), min(n - 1 - r, v + r)] widened by r."""
    v = np.arange(n)
    ext = np.minimum(n - 1 - r, v + r) - np.maximum(r, v - r) + 2 * r + 1
    return np.concatenate([[0], np.cumsum(ext)]).astype(np.int64)


def lbdm_laplacian(image, epsilon=1e-7, radius=1):
    """Learning-based digital matting Laplacian:
    pymatting/laplacian/lbdm_laplacian.py. Canonical CSR on the device;
    radius 1 or 2. An image with no interior window gives the reference's
    matrix of a single stored zero at (0, 0)."""
    h, w = image.shape[:2]
    r = int(radius)
    if r not in (1, 2):
        raise NotImplementedError("lbdm_laplacian on the device supports radius 1 and 2")
    n = h * w
    if h <= 2 * r or w <= 2 * r:
        rowptr = torch.ones(n + 1, dtype=torch.int64, device=dev.device())
        rowptr[0] = 0
        return DeviceCSRMatrix(shape=(n, n), pmb_arrays=(rowptr, dev.zeros(1, torch.int64),
                                                         dev.zeros(1, torch.float64)))
    lib = _ffi.lib()
    img = _image_to_device(image)
    scratch = dev.empty(int(lib.pmb_lbdm_scratch_elems(h, w, r)), torch.float64)
    px_t = dev.to_device(_lbdm_extents(w, r))
    py_t = dev.to_device(_lbdm_extents(h, r))
    nnz = int(_lbdm_extents(h, r)[-1] * _lbdm_extents(w, r)[-1])
    rowptr = dev.empty(n + 1, torch.int64)
    cols = dev.empty(nnz, torch.int64)
    vals = dev.empty(nnz, torch.float64)
    _ffi.check(lib.pmb_lbdm_laplacian(dev.ptr(img), h, w, r, float(epsilon), dev.ptr(scratch),
                                      dev.ptr(px_t), dev.ptr(py_t), dev.ptr(rowptr),
                                      dev.ptr(cols), dev.ptr(vals), dev.stream()),
               "pmb_lbdm_laplacian")
    return DeviceCSRMatrix(shape=(n, n), pmb_arrays=(rowptr, cols, vals))


def knn_laplacian(image, n_neighbors=[20, 10], distance_weights=[2.0, 0.1], kernel="binary"):
    """k-nearest-neighbour Laplacian: pymatting/laplacian/knn_laplacian.py.

    For each (k, weight) pass, the k nearest pixels in the float32 feature
    space (r, g, b, weight x, weight y) are found by an exact search on the
    device with the reference k-d tree's distance, keeping the k smallest by
    (distance, index); the reference resolves equal distances in its tree
    order. Candidate tiles are pruned by their bounding boxes. W = sum of
    B + B^T (binary or soft weights), L = I - D^-1 W as canonical CSR on the
    device.
    """
    if kernel not in ["binary", "soft"]:
        raise ValueError("kernel must be binary/soft, but not " + kernel + ".")
    h, w = image.shape[:2]
    n = h * w
    ks = np.ascontiguousarray(list(n_neighbors), dtype=np.int32)
    dws = np.ascontiguousarray(list(distance_weights), dtype=np.float64)
    passes = min(len(ks), len(dws))
    ks, dws = ks[:passes], dws[:passes]
    lib = _ffi.lib()
    img = _image_to_device(image)
    elems = int(lib.pmb_knn_scratch_elems(n, int(ks.sum()), passes))
    if elems <= 0:
        raise ValueError("knn_laplacian: unsupported neighbour counts %r" % (list(ks),))
    scratch = dev.empty(elems, torch.int64)
    rowptr = dev.empty(n + 1, torch.int64)
    nnz = np.zeros(1, dtype=np.int64)
    soft = 1 if kernel == "soft" else 0
    _ffi.check(lib.pmb_knn_laplacian(dev.ptr(img), h, w, ks.ctypes.data, dws.ctypes.data,
                                     passes, soft, dev.ptr(scratch), dev.ptr(rowptr), None, None,
                                     nnz.ctypes.data, dev.stream()), "pmb_knn_laplacian")
    m = int(nnz[0])
    cols = dev.empty(max(m, 1), torch.int64)
    vals = dev.empty(max(m, 1), torch.float64)
    _ffi.check(lib.pmb_knn_laplacian(dev.ptr(img), h, w, ks.ctypes.data, dws.ctypes.data,
                                     passes, soft, dev.ptr(scratch), dev.ptr(rowptr),
                                     dev.ptr(cols), dev.ptr(vals), nnz.ctypes.data, dev.stream()),
               "pmb_knn_laplacian")
    return DeviceCSRMatrix(shape=(n, n), pmb_arrays=(rowptr, cols[:m], vals[:m]))
