"""cutout (pymatting/cutout/cutout.py) end to end on the reference test's
files: the reference test's thresholds (tests/test_simple_api.py: alpha
error < 3.1, foreground error < 4) and the cutout file the reference itself
wrote for the same inputs (uint8; channels may differ by one level where
alpha or F sit on a quantisation boundary)."""

import numpy as np
import pytest

from tests.conftest import golden

pytestmark = pytest.mark.gpu


def test_cutout_matches_reference(gpu, tmp_path):
    from PIL import Image
    import pymatting_b200 as pm
    g = golden("cutout_test.npz")
    img, tri, out = (str(tmp_path / n) for n in ("test.png", "test_trimap.png", "cutout.png"))
    Image.fromarray(g["test_u8"]).save(img)
    Image.fromarray(g["test_trimap_u8"]).save(tri)
    pm.cutout(img, tri, out)
    cut = pm.load_image(out)
    alpha, fg = cut[:, :, 3], cut[:, :, :3]
    assert np.linalg.norm(alpha - g["true_alpha"]) < 3.1
    assert np.linalg.norm(alpha[:, :, None] * np.abs(fg - g["true_foreground"])) < 4
    ours = np.array(Image.open(out)).astype(np.int16)
    ref = g["reference_cutout_u8"].astype(np.int16)
    assert ours.shape == ref.shape
    assert np.abs(ours - ref).max() <= 1
    assert np.mean(ours == ref) >= 0.99
