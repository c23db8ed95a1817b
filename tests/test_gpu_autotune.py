"""Launch-shape knobs and the autotuner (no reference counterpart): knobs
are clamped to what the kernels support, and any setting gives the same
solution as the defaults."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(gpu):
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _a, _f = make_matting_problem(180, 260, 31, sigma=2.0, band=4, unknown_fraction=0.15)
    return img, tri


def test_knobs_clamp_and_read_back(problem):
    from pymatting_b200.batch import AlphaBatch
    from pymatting_b200 import autotune
    img, tri = problem
    b64 = AlphaBatch([img], [tri], precision="fp64")
    assert autotune.apply_tuning(b64.system, {"vec_apply": 4})["vec_apply"] == 2   # FP64: 2 only
    bm = AlphaBatch([img], [tri], precision="mixed")
    assert autotune.apply_tuning(bm.system, {"vec_apply": 4})["vec_apply"] == 4
    got = autotune.apply_tuning(bm.system, {"ctas_fine": 99, "chunk": 0})
    assert 1 <= got["ctas_fine"] <= 4 and got["chunk"] == 1
    assert autotune.tuning(bm.system)["ctas_fine"] == got["ctas_fine"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_setting_gives_the_same_solution(problem, precision):
    import torch
    from pymatting_b200.batch import AlphaBatch
    from pymatting_b200 import autotune
    img, tri = problem
    batch = AlphaBatch([img], [tri], precision=precision)
    ref = batch.solve().clone()
    for knobs in [{"vec_apply": 4, "vec_up": 4}, {"ctas_fine": 1, "ctas_up": 1, "ctas_down": 1},
                  {"ctas_flat": 2, "chunk": 8}, {"chunk": 1, "ctas_fine": 3},
                  {"stages": 1}, {"stages": 1, "vec_up": 4, "ctas_up": 2}, {"stages": 2}]:
        autotune.apply_tuning(batch.system, knobs)
        x = batch.solve()
        assert batch.stats()[0].status == 1
        tol = 1e-9 if precision == "fp64" else 1e-5
        assert float((x - ref).abs().max()) <= tol


def test_autotune_caches_and_applies(problem):
    from pymatting_b200.batch import AlphaBatch
    from pymatting_b200 import autotune
    img, tri = problem
    tuned = AlphaBatch([img], [tri], precision="mixed", tune="auto").tuning
    assert set(tuned["knobs"]) == set(autotune.KNOBS) and tuned["ms"] > 0
    again = AlphaBatch([img], [tri], precision="mixed", tune="cached")
    assert again.tuning == tuned
    assert autotune.tuning(again.system) == tuned["knobs"]
    x = again.solve()
    assert again.stats()[0].status == 1 and np.isfinite(float(x.sum()))


def test_largest_launch_shapes_on_a_batch(gpu):
    """The largest CTA counts on a batch of uneven images: per-image partial
    sums stay within their buffer and the solution is unchanged."""
    from pymatting_b200.batch import AlphaBatch
    from pymatting_b200 import autotune
    from pymatting_b200.synthetic import make_matting_problem
    sizes = [(96, 128), (64, 64), (200, 150), (120, 90), (80, 200), (64, 96), (150, 150), (72, 72)]
    probs = [make_matting_problem(h, w, 60 + k, sigma=2.0, band=3, unknown_fraction=0.2)[:2]
             for k, (h, w) in enumerate(sizes)]
    batch = AlphaBatch([p[0] for p in probs], [p[1] for p in probs], precision="mixed")
    ref = batch.solve().clone()
    autotune.apply_tuning(batch.system, {"ctas_flat": 16, "ctas_fine": 4, "ctas_up": 4,
                                         "ctas_down": 4})
    x = batch.solve()
    assert all(s.status == 1 for s in batch.stats())
    assert float((x - ref).abs().max()) <= 1e-5
