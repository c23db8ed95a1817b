"""Batched solves: many images of different sizes in one stencil engine,
each with its own CG scalars and convergence status."""

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problems(gpu):
    from pymatting_b200.synthetic import make_matting_problem
    sizes = [(64, 96, 0.2), (37, 53, 0.25), (128, 80, 0.15), (8, 8, 0.3), (200, 300, 0.1)]
    out = []
    for k, (h, w, f) in enumerate(sizes):
        img, tri, _a, _f = make_matting_problem(h, w, 40 + k, sigma=2.0, band=3,
                                                unknown_fraction=f)
        out.append((img, tri))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_single_solves(problems, precision):
    from pymatting_b200.batch import solve_alpha
    imgs = [p[0] for p in problems]
    tris = [p[1] for p in problems]
    alphas, stats = solve_alpha(imgs, tris, precision=precision, return_stats=True)
    for (img, tri), a, st in zip(problems, alphas, stats):
        assert st.status == 1
        A, b = oracle.make_linear_system(oracle.cf_laplacian(img), tri)
        # Solve the same system alone and through the reference algorithm.
        single = solve_alpha([img], [tri], precision=precision)[0]
        np.testing.assert_allclose(a, single, rtol=0, atol=1e-12 if precision == "fp64" else 1e-5)
        x_ref, _it = oracle.solve_soft(img, tri, preconditioner="vcycle", rtol=1e-7)
        assert np.abs(a.ravel() - np.clip(x_ref, 0, 1)).max() < 1e-3


def test_batch_per_image_failure_is_isolated(problems):
    """A non-finite image stops with its own status; the others converge."""
    from pymatting_b200.batch import AlphaBatch
    imgs = [p[0].copy() for p in problems]
    tris = [p[1] for p in problems]
    imgs[1][5, 7, 0] = np.nan
    batch = AlphaBatch(imgs, tris, precision="fp64")
    batch.solve(check=False)
    stats = batch.stats()
    assert stats[1].status == 3
    assert all(s.status == 1 for k, s in enumerate(stats) if k != 1)


def test_batch_trimap_errors(problems):
    from pymatting_b200.batch import solve_alpha
    img, tri = problems[0]
    with pytest.raises(ValueError, match="foreground"):
        solve_alpha([img], [np.where(tri > 0.9, 0.5, tri)])


def test_batch_jacobi_and_none(problems):
    from pymatting_b200.batch import solve_alpha
    imgs = [p[0] for p in problems[:3]]
    tris = [p[1] for p in problems[:3]]
    for pre in ["jacobi", "none"]:
        for precision in ["fp64", "mixed"]:
            alphas, stats = solve_alpha(imgs, tris, preconditioner=pre, precision=precision,
                                        return_stats=True)
            assert all(s.status == 1 for s in stats)


def test_solve_alpha_host_tensor_io(problems):
    """Pinned CPU tensors in, CPU tensors out; same alphas as numpy inputs."""
    import torch
    from pymatting_b200.batch import solve_alpha
    imgs = [torch.from_numpy(p[0]).pin_memory() for p in problems[:2]]
    tris = [torch.from_numpy(p[1]).pin_memory() for p in problems[:2]]
    out = solve_alpha(imgs, tris, precision="fp64")
    ref = solve_alpha([p[0] for p in problems[:2]], [p[1] for p in problems[:2]], precision="fp64")
    for a, r in zip(out, ref):
        assert isinstance(a, torch.Tensor) and not a.is_cuda
        assert np.array_equal(a.numpy(), r)


def test_sharded_solve_on_one_rank(problems):
    """solve_alpha_sharded with one rank: the shard is the whole batch, the
    gather returns every image in batch order, equal to solve_alpha's."""
    import torch
    from pymatting_b200 import solve_alpha, solve_alpha_sharded
    from pymatting_b200.shard import STAT_FIELDS
    imgs = [p[0] for p in problems]
    tris = [p[1] for p in problems]
    alphas, stats = solve_alpha_sharded(imgs, tris, 0, 1, torch.device("cuda", 0),
                                        precision="fp64")
    ref = solve_alpha(imgs, tris, precision="fp64")
    assert len(alphas) == len(ref) and stats.shape == (len(ref), len(STAT_FIELDS))
    for a, r, t in zip(alphas, ref, tris):
        assert a.shape == t.shape
        np.testing.assert_allclose(a.cpu().numpy(), r, rtol=0, atol=1e-12)
    assert bool((stats[:, 1] == 1).all())
