"""The device ichol factor against the oracle's restatement of the reference
(pymatting/preconditioner/ichol.py:6-113) on matrices whose bandwidth selects
each factor kernel: the front held by one CTA, by clusters of 2 to 8 CTAs in
distributed shared memory, and in global memory for bands too wide for a
cluster. Structure (Lp, Lr) exact; values within 1e-12 relative."""

import numpy as np
import pytest
import scipy.sparse

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pm(gpu):
    import pymatting_b200
    return pymatting_b200


def cluster_size(W):
    """Host mirror of the factor's kernel choice (ichol.cu, ichol_cluster_size)."""
    if W < 1 or W - 1 > 32 * 14:
        return 0
    for C in range(1, 9):
        Wp = (W + 7) & ~7
        S = (W + C - 1) // C
        size = S * Wp * 8 + S * 8 + 2 * W * 8 + S * 4 + 4 * W * 4 + S * Wp
        if (size + 15) & ~15 <= 227 * 1024 - 256:
            return C
    return 0


def grid_laplacian(h, w, shift, seed):
    """5-point Laplacian of an h x w grid with random positive edge weights
    plus a diagonal shift: SPD, bandwidth w."""
    rng = np.random.default_rng(seed)
    n = h * w
    idx = np.arange(n).reshape(h, w)
    rows, cols, vals = [], [], []
    for a, b in [(idx[:, :-1], idx[:, 1:]), (idx[:-1, :], idx[1:, :])]:
        wt = rng.uniform(0.5, 1.5, a.size)
        rows += [a.ravel(), b.ravel()]
        cols += [b.ravel(), a.ravel()]
        vals += [-wt, -wt]
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    off = scipy.sparse.csc_matrix((v, (r, c)), (n, n))
    deg = -np.asarray(off.sum(axis=1)).ravel()
    A = off + scipy.sparse.diags(deg + shift)
    A = scipy.sparse.csc_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    return A


def check_factor(pm, A, cluster=None, **kw):
    d = pm.ichol(A, **kw)
    if cluster is not None:
        assert d.factor.cluster() == cluster
    ref = oracle.ichol(A, **kw)
    Lv, Lr, Lp = d.Ltuple
    Rv, Rr, Rp = ref.Ltuple
    np.testing.assert_array_equal(Lp, Rp)
    np.testing.assert_array_equal(Lr, Rr)
    np.testing.assert_allclose(Lv, Rv, rtol=1e-12, atol=1e-14)
    rhs = np.random.default_rng(0).standard_normal(A.shape[0])
    np.testing.assert_allclose(d(rhs), ref(rhs), rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize("w,expect", [(20, 1), (150, 1), (200, 2), (300, 4), (420, 8),
                                      (500, 0)])
def test_ichol_grid_bandwidths(pm, w, expect):
    A = grid_laplacian(10, w, 1e-2, w)
    assert cluster_size(w + 1) == expect
    check_factor(pm, A, cluster=expect)
    check_factor(pm, A, cluster=expect, discard_threshold=1e-2, diag_keep_discarded=False)


def test_ichol_320x240_unknown_block(pm):
    """The 320x240 workload's L_U (bandwidth 241: a cluster of 3)."""
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _a, _f = make_matting_problem(240, 320, 1, sigma=2.0, band=7, unknown_fraction=0.12)
    L = oracle.cf_laplacian(img)
    u = (tri > 0.1) & (tri < 0.9)
    A = scipy.sparse.csc_matrix(L[u.ravel()][:, u.ravel()])
    low = scipy.sparse.tril(A, -1).tocoo()
    W = int((low.row - low.col).max()) + 1
    assert cluster_size(W) == 3
    check_factor(pm, A, cluster=3)


def test_ichol_cluster_failure_codes(pm):
    """Not positive definite at every shift, and too many entries, in the
    cluster kernel (bandwidth 30)."""
    A = grid_laplacian(6, 30, 1e-2, 1)
    bad = scipy.sparse.csc_matrix(A - scipy.sparse.diags(np.full(A.shape[0], 50.0)))
    with pytest.raises(ValueError, match="positive-definiteness"):
        pm.ichol(bad, shifts=[0.0, 1e-4])
    with pytest.raises(ValueError, match="max_nnz"):
        pm.ichol(A, discard_threshold=0.0, max_nnz=A.shape[0] + 10)
