"""Large-kernel matting Laplacian (lkm_laplacian, estimate_alpha_lkm) against
fixtures produced by PyMatting itself and the reference test's comparison
with the closed-form system (tests/test_lkm.py)."""

import numpy as np
import pytest

from tests.conftest import golden

pytestmark = pytest.mark.gpu


def test_lkm_apply_and_diagonal(gpu):
    import pymatting_b200 as pm
    d = golden("lkm_small.npz")
    for name in "abc":
        r = int(d[f"{name}_radius"][0])
        L, diag = pm.lkm_laplacian(d[f"{name}_image"], epsilon=1e-7, radius=r)
        lp = L(d[f"{name}_p"])
        ref_lp, ref_diag = d[f"{name}_Lp"], d[f"{name}_diag"]
        assert isinstance(lp, np.ndarray) and lp.shape == ref_lp.shape
        assert np.abs(lp - ref_lp).max() <= 1e-9 * np.abs(ref_lp).max(), name
        assert np.abs(diag - ref_diag).max() <= 1e-9 * np.abs(ref_diag).max(), name


def test_lkm_against_cf_like_the_reference(gpu):
    """tests/test_lkm.py:12-49 on the same lemur image: the LKM and CF solves
    agree to 1e-5 and their CG iteration counts differ by at most 2."""
    import pymatting_b200 as pm
    d = golden("lkm_small.npz")
    lem = golden("lemur.npz")
    image, trimap = lem["s0125_image"], lem["s0125_trimap"]
    L_lkm, diag_lkm = pm.lkm_laplacian(image, epsilon=1e-7, radius=2)
    A_cf, b, c = pm.make_linear_system(pm.cf_laplacian(image, epsilon=1e-7, radius=2), trimap,
                                       return_c=True)
    inv = 1.0 / (diag_lkm + c)
    cb_l, cb_c = pm.CounterCallback(), pm.CounterCallback()
    x_lkm = pm.cg(lambda x: L_lkm(x) + c * x, b, M=lambda r: inv * r, callback=cb_l)
    x_cf = pm.cg(A_cf, b, M=pm.jacobi(A_cf), callback=cb_c)
    assert np.linalg.norm(x_lkm - x_cf) < 1e-5
    assert abs(cb_l.n - cb_c.n) <= 2
    # and against the reference's own runs of the same two solves
    assert abs(cb_l.n - int(d["lemur_it_lkm"][0])) <= 2
    assert np.abs(x_lkm - d["lemur_x_lkm"]).max() < 1e-5


def test_estimate_alpha_lkm(gpu):
    import pymatting_b200 as pm
    d = golden("lkm_small.npz")
    lem = golden("lemur.npz")
    alpha = pm.estimate_alpha_lkm(lem["s0125_image"], lem["s0125_trimap"])
    assert alpha.shape == lem["s0125_trimap"].shape
    assert np.abs(alpha - d["lemur_alpha_lkm"]).max() < 1e-4


def test_lkm_device_tensors_stay_on_device(gpu):
    import torch
    import pymatting_b200 as pm
    d = golden("lkm_small.npz")
    img = torch.as_tensor(d["a_image"], device=gpu)
    L, diag = pm.lkm_laplacian(img, radius=2)
    p = torch.as_tensor(d["a_p"], device=gpu)
    out = L(p)
    assert out.is_cuda and diag.is_cuda
    assert np.abs(out.cpu().numpy() - d["a_Lp"]).max() <= 1e-9 * np.abs(d["a_Lp"]).max()


def test_lkm_small_image_rejected(gpu):
    import pymatting_b200 as pm
    with pytest.raises(ValueError):
        pm.lkm_laplacian(np.zeros((8, 30, 3)), radius=4)
