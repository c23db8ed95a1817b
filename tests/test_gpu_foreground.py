"""estimate_foreground_ml on the device against the oracle's C restatement
(itself bit-exact with PyMatting, tests/test_oracle.py) and against fixtures
produced by PyMatting (tests/golden/foreground_small.npz).

Tolerances: with the reference's seed colours (``seed_colors``) F and B
must be bit-identical. With the library's own seeds (a float64 mean, where
the reference keeps a running float32 sum) every value must be within
DEFAULT_TOL of the reference."""

import numpy as np
import pytest

import oracle
from tests.conftest import golden

pytestmark = pytest.mark.gpu

DEFAULT_TOL = 2e-6


def _kwargs(p):
    return dict(regularization=float(p[0]), n_small_iterations=int(p[1]),
                n_big_iterations=int(p[2]), small_size=int(p[3]), gradient_weight=float(p[4]))


def _case(rng, h, w, depth=3):
    img = rng.random((h, w, depth)).astype(np.float32)
    alpha = np.clip(rng.random((h, w)) * 1.4 - 0.2, 0.0, 1.0).astype(np.float32)
    return img, alpha


def _seeded(img, alpha, **kw):
    import pymatting_b200 as pm
    seed = oracle.fg_mean_colors(img, alpha)
    return pm.estimate_foreground_ml(img, alpha, return_background=True, seed_colors=seed, **kw)


def test_fixture_cases_bit_exact(gpu):
    g = golden("foreground_small.npz")
    for i in range(int(g["n_cases"][0])):
        img, alpha = g[f"c{i}_image"], g[f"c{i}_alpha"]
        F, B = _seeded(img, alpha, **_kwargs(g[f"c{i}_params"]))
        assert F.dtype == np.float32 and F.shape == img.shape
        assert np.array_equal(F, g[f"c{i}_F"]), i
        assert np.array_equal(B, g[f"c{i}_B"]), i


def test_reference_lemur_test(gpu):
    """tests/test_foreground.py of the reference (lemur, scale 0.1): mse
    threshold 0.022, and bit-exact with the reference's output."""
    import pymatting_b200 as pm
    g = golden("foreground_small.npz")
    image, alpha, trimap = g["lemur_image"], g["lemur_alpha"], g["lemur_trimap"]
    F, B = pm.estimate_foreground_ml(image, alpha, return_background=True)
    unknown = (trimap > 0.1) & (trimap < 0.9)
    mse = np.mean((alpha[:, :, None] * np.abs(F - g["lemur_expected"]))[unknown])
    assert mse <= 0.022
    assert np.abs(F - g["lemur_F"]).max() <= DEFAULT_TOL
    F, B = _seeded(image, alpha)
    assert np.array_equal(F, g["lemur_F"]) and np.array_equal(B, g["lemur_B"])


@pytest.mark.parametrize("h,w", [(1, 2), (2, 1), (5, 1), (1, 40), (31, 33), (32, 32), (33, 31),
                                 (64, 65), (97, 130), (257, 300)])
def test_sizes_bit_exact_with_seed(gpu, h, w):
    rng = np.random.default_rng(h * 1000 + w)
    img, alpha = _case(rng, h, w)
    F, B = _seeded(img, alpha)
    Fr, Br = oracle.estimate_foreground_ml(img, alpha, return_background=True)
    assert np.array_equal(F, Fr) and np.array_equal(B, Br)


@pytest.mark.parametrize("depth", [1, 2, 4, 8])
def test_depths_bit_exact_with_seed(gpu, depth):
    rng = np.random.default_rng(depth)
    img, alpha = _case(rng, 70, 45, depth)
    F, B = _seeded(img, alpha)
    Fr, Br = oracle.estimate_foreground_ml(img, alpha, return_background=True)
    assert np.array_equal(F, Fr) and np.array_equal(B, Br)


@pytest.mark.parametrize("kw", [dict(n_big_iterations=0), dict(n_small_iterations=0),
                                dict(n_big_iterations=7, small_size=8),
                                dict(regularization=0.1, gradient_weight=3.0),
                                dict(gradient_weight=0.0), dict(small_size=1000)])
def test_parameters_bit_exact_with_seed(gpu, kw):
    rng = np.random.default_rng(7)
    img, alpha = _case(rng, 83, 61)
    F, B = _seeded(img, alpha, **kw)
    Fr, Br = oracle.estimate_foreground_ml(img, alpha, return_background=True, **kw)
    assert np.array_equal(F, Fr) and np.array_equal(B, Br)


def test_full_hd_bit_exact_and_default_seed_close(gpu):
    """1080x1920: 34 strips, two sweeps in flight per level."""
    import pymatting_b200 as pm
    from pymatting_b200.synthetic import make_matting_problem
    img, _, alpha, _ = make_matting_problem(1080, 1920, 1, sigma=2.0, band=7,
                                            unknown_fraction=0.12, dtype=np.float32)
    Fr, Br = oracle.estimate_foreground_ml(img, alpha, return_background=True)
    F, B = _seeded(img, alpha)
    assert np.array_equal(F, Fr) and np.array_equal(B, Br)
    F, B = pm.estimate_foreground_ml(img, alpha, return_background=True)
    assert np.abs(F - Fr).max() <= DEFAULT_TOL and np.abs(B - Br).max() <= DEFAULT_TOL


def test_device_tensors_stay_on_device(gpu):
    import torch
    import pymatting_b200 as pm
    rng = np.random.default_rng(3)
    img, alpha = _case(rng, 48, 50)
    ti = torch.as_tensor(img, device=gpu)
    ta = torch.as_tensor(alpha, device=gpu)
    seed = torch.as_tensor(oracle.fg_mean_colors(img, alpha), device=gpu)
    F = pm.estimate_foreground_ml(ti, ta, seed_colors=seed)
    assert F.is_cuda and F.dtype == torch.float32
    assert np.array_equal(F.cpu().numpy(), oracle.estimate_foreground_ml(img, alpha))


def test_errors(gpu):
    import pymatting_b200 as pm
    with pytest.raises(ZeroDivisionError):
        pm.estimate_foreground_ml(np.zeros((1, 1, 3)), np.zeros((1, 1)))
    with pytest.raises(ValueError):
        pm.estimate_foreground_ml(np.zeros((4, 4, 3)), np.zeros((4, 5)))


# --- the reference's GPU backend (estimate_foreground_ml_cupy, Jacobi) ---
# Its kernel is built by NVRTC with fused multiply-adds allowed, as is ours;
# the oracle restates it in numpy without them. Where alpha is 0 or 1 the
# per-pixel 2x2 system is nearly singular (determinant ~ regularization), so
# a float32 rounding difference can grow to ~1e-4 over ten iterations.
# Tolerances: JACOBI_TOL elementwise, JACOBI_MEAN_TOL on the mean.

JACOBI_TOL = 1e-3
JACOBI_MEAN_TOL = 2e-6


@pytest.mark.parametrize("h,w", [(1, 2), (2, 1), (7, 9), (33, 31), (97, 130), (257, 300)])
def test_jacobi_matches_oracle(gpu, h, w):
    import pymatting_b200 as pm
    rng = np.random.default_rng(h * 7 + w)
    img, alpha = _case(rng, h, w)
    F, B = pm.estimate_foreground_ml_cupy(img, alpha, return_background=True)
    Fr, Br = oracle.estimate_foreground_ml_cupy(img, alpha, return_background=True)
    assert F.dtype == np.float32 and F.shape == (h, w, 3)
    assert np.abs(F - Fr).max() <= JACOBI_TOL and np.abs(B - Br).max() <= JACOBI_TOL
    if h * w >= 1000:   # in tiny images the mean is one near-singular pixel
        assert np.abs(F - Fr).mean() <= JACOBI_MEAN_TOL
        assert np.abs(B - Br).mean() <= JACOBI_MEAN_TOL


@pytest.mark.parametrize("kw", [dict(n_big_iterations=0), dict(n_small_iterations=0),
                                dict(n_big_iterations=1), dict(n_big_iterations=3, small_size=8),
                                dict(regularization=0.05), dict(small_size=1000)])
def test_jacobi_parameters(gpu, kw):
    import pymatting_b200 as pm
    rng = np.random.default_rng(11)
    img, alpha = _case(rng, 120, 95)
    F, B = pm.estimate_foreground_ml_cupy(img, alpha, return_background=True, **kw)
    Fr, Br = oracle.estimate_foreground_ml_cupy(img, alpha, return_background=True, **kw)
    assert np.abs(F - Fr).max() <= JACOBI_TOL and np.abs(B - Br).max() <= JACOBI_TOL


def test_jacobi_reference_lemur_test_and_full_hd(gpu):
    """tests/test_foreground.py of the reference runs the cupy backend
    through the same mse <= 0.022 check; and a 1080x1920 case."""
    import pymatting_b200 as pm
    from pymatting_b200.synthetic import make_matting_problem
    g = golden("foreground_small.npz")
    alpha = g["lemur_alpha"]
    F = pm.estimate_foreground_ml_cupy(g["lemur_image"], alpha)
    unknown = (g["lemur_trimap"] > 0.1) & (g["lemur_trimap"] < 0.9)
    assert np.mean((alpha[:, :, None] * np.abs(F - g["lemur_expected"]))[unknown]) <= 0.022
    img, _, alpha, _ = make_matting_problem(1080, 1920, 2, sigma=2.0, band=7,
                                            unknown_fraction=0.12, dtype=np.float32)
    F = pm.estimate_foreground_ml_cupy(img, alpha)
    Fr = oracle.estimate_foreground_ml_cupy(img, alpha)
    assert np.abs(F - Fr).max() <= JACOBI_TOL and np.abs(F - Fr).mean() <= JACOBI_MEAN_TOL


def test_jacobi_device_output_and_errors(gpu):
    import torch
    import pymatting_b200 as pm
    rng = np.random.default_rng(5)
    img, alpha = _case(rng, 40, 50)
    F = pm.estimate_foreground_ml_cupy(torch.as_tensor(img, device=gpu),
                                       torch.as_tensor(alpha, device=gpu), to_numpy=False)
    assert F.is_cuda and F.dtype == torch.float32
    assert np.abs(F.cpu().numpy() - oracle.estimate_foreground_ml_cupy(img, alpha)).max() <= JACOBI_TOL
    with pytest.raises(ZeroDivisionError):
        pm.estimate_foreground_ml_cupy(np.zeros((1, 1, 3)), np.zeros((1, 1)))
    with pytest.raises(AssertionError):
        pm.estimate_foreground_ml_cupy(np.zeros((4, 4, 4)), np.zeros((4, 4)))


# --- closed-form foreground (estimate_foreground_cf) ---

def test_foreground_cf_system_matches_reference(gpu):
    """A = U^T U + diag(S, S) assembled on the device against the matrix
    the reference builds with scipy (same entries; values within 1e-15,
    the reference sums the same terms in its sparse-product order)."""
    import scipy.sparse
    from pymatting_b200.foreground import _fg_cf_matrix
    import pymatting_b200._device as dev
    import torch
    g = golden("foreground_small.npz")
    a = g["cf_small_alpha"]
    h, w = a.shape
    A = _fg_cf_matrix(dev.to_device(a.ravel(), torch.float64), h, w, 1e-5)
    R = scipy.sparse.csr_matrix((g["cf_small_data"], g["cf_small_indices"], g["cf_small_indptr"]),
                                shape=A.shape)
    assert np.array_equal(A.indptr, R.indptr) and np.array_equal(A.indices, R.indices)
    assert np.abs(A.data - R.data).max() <= 1e-15


def test_foreground_cf_lemur(gpu):
    """The reference test's check (mse <= 0.022) and closeness to the
    reference's own result (CG to rtol 1e-5 from the image, ichol
    preconditioner)."""
    import pymatting_b200 as pm
    g = golden("foreground_small.npz")
    image, alpha, trimap = g["lemur_image"], g["lemur_alpha"], g["lemur_trimap"]
    F, B = pm.estimate_foreground_cf(image, alpha, return_background=True)
    unknown = (trimap > 0.1) & (trimap < 0.9)
    mse = np.mean((alpha[:, :, None] * np.abs(F - g["lemur_expected"]))[unknown])
    assert mse <= 0.022
    assert np.abs(F - g["lemur_F_cf"]).mean() <= 1e-3 and np.abs(B - g["lemur_B_cf"]).mean() <= 1e-3
