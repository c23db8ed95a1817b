"""Pin the oracle (CPU restatement) against the reference's own outputs.

The fixtures in tests/golden were produced by running PyMatting itself
(tests/golden/make_golden.py). Here the oracle must reproduce them: the
Laplacian bit for bit, the solver and preconditioners within rounding.
"""

import numpy as np
import pytest
import scipy.sparse

import oracle
from tests.conftest import golden


def test_cf_laplacian_bit_exact():
    g = golden("cf_laplacian_small.npz")
    for k in range(int(g["count"][0])):
        h, w, r = (int(v) for v in g[f"c{k}_meta"])
        values, indices, indptr = oracle.cf_laplacian_arrays(
            g[f"c{k}_image"], float(g[f"c{k}_eps"][0]), r, g[f"c{k}_known"])
        np.testing.assert_array_equal(indices, g[f"c{k}_indices"])
        np.testing.assert_array_equal(indptr, g[f"c{k}_indptr"])
        # Same IEEE operation order as the reference: identical bits.
        np.testing.assert_array_equal(values, g[f"c{k}_values"])


def test_cg_reference_cases():
    g = golden("cg_small.npz")
    for k in range(int(g["count"][0])):
        A, b = g[f"k{k}_A"], g[f"k{k}_b"]
        x0 = g[f"k{k}_x0"]
        x0 = None if x0.size == 0 else x0
        mk = int(g[f"k{k}_M"][0])
        Mj = np.diag(1.0 / np.diag(A))
        M = [None, Mj, lambda v: Mj.dot(v)][mk]
        cb = oracle.CounterCallback()
        x = oracle.cg(A, b, x0=x0, M=M, rtol=0, atol=1e-10, callback=cb)
        assert cb.n == int(g[f"k{k}_iters"][0])
        np.testing.assert_allclose(x, g[f"k{k}_x"], rtol=0, atol=1e-12)
        assert np.linalg.norm(A.dot(x) - b) < 1e-10


def test_docstring_examples():
    g = golden("cg_small.npz")
    A = np.array([[3.0, 1.0], [1.0, 2.0]])
    np.testing.assert_allclose(oracle.cg(A, np.array([4.0, 3.0]), M=oracle.jacobi(A)),
                               g["doc_cg"], atol=1e-12)
    np.testing.assert_allclose(
        oracle.jacobi(np.array([[2, 3], [3, 5]]))(np.array([1, 2])), g["doc_jacobi"])
    np.testing.assert_allclose(
        oracle.vcycle(np.array([[2, 3], [3, 5]]), (2, 2))(np.array([1, 2])),
        g["doc_vcycle"], atol=1e-12)
    d = oracle.ichol(scipy.sparse.csc_matrix(np.array([[2.0, 3.0], [3.0, 5.0]])))
    np.testing.assert_allclose(d(np.array([1.0, 2.0])), g["doc_ichol"], atol=1e-12)


def _csc(g, k):
    n = len(g[f"k{k}_A_indptr"]) - 1
    return scipy.sparse.csc_matrix(
        (g[f"k{k}_A_data"], g[f"k{k}_A_indices"], g[f"k{k}_A_indptr"]), (n, n))


def test_ichol_factors_match_reference():
    g = golden("ichol_small.npz")
    for k in range(int(g["count"][0])):
        A = _csc(g, k)
        thr, rel, keep = (float(v) for v in g[f"k{k}_params"])
        d = oracle.ichol(A, discard_threshold=thr, relative_discard_threshold=rel,
                         diag_keep_discarded=bool(keep),
                         max_nnz=100000 if thr == 0.0 else int(4e9 / 16))
        Lv, Lr, Lp = d.Ltuple
        np.testing.assert_array_equal(Lp, g[f"k{k}_Lp"])
        np.testing.assert_array_equal(Lr, g[f"k{k}_Lr"])
        np.testing.assert_array_equal(Lv, g[f"k{k}_Lv"])


def test_soft_system_and_vcycle():
    g = golden("soft_small.npz")
    for k in range(int(g["count"][0])):
        img, tri = g[f"k{k}_image"], g[f"k{k}_trimap"]
        h, w = tri.shape
        A, b = oracle.make_linear_system(oracle.cf_laplacian(img), tri)
        np.testing.assert_array_equal(A.indptr, g[f"k{k}_A_indptr"])
        np.testing.assert_array_equal(A.indices, g[f"k{k}_A_indices"])
        np.testing.assert_array_equal(A.data, g[f"k{k}_A_data"])
        np.testing.assert_array_equal(b, g[f"k{k}_b"])
        v = g[f"k{k}_v"]
        np.testing.assert_allclose(oracle.vcycle(A, (h, w))(v), g[f"k{k}_vcycle_v"],
                                   rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(
            oracle.vcycle(A, (h, w), num_pre_iter=2, num_post_iter=3, omega=0.7)(v),
            g[f"k{k}_vcycle_v_2_3"], rtol=1e-10, atol=1e-12)
        for name in ["none", "jacobi", "vcycle", "ichol"]:
            M = {"none": None, "jacobi": oracle.jacobi(A),
                 "vcycle": oracle.vcycle(A, (h, w)), "ichol": oracle.ichol(A)}[name]
            cb = oracle.CounterCallback()
            x = oracle.cg(A, b, M=M, rtol=1e-7, callback=cb)
            assert abs(cb.n - int(g[f"k{k}_it_{name}"][0])) <= 1
            np.testing.assert_allclose(x, g[f"k{k}_x_{name}"], rtol=0, atol=1e-6)


def test_lemur_pins():
    """The reference tests' iteration caps and the Laplacian error pin."""
    g = golden("lemur.npz")
    image, trimap = g["s0125_image"], g["s0125_trimap"]
    A, b = oracle.make_linear_system(oracle.cf_laplacian(image), trimap)
    caps = {"none": 378, "jacobi": 197, "icholt": 3, "vcycle": 48}
    for name, fac in [("none", lambda A: None), ("jacobi", oracle.jacobi),
                      ("icholt", lambda A: oracle.ichol(A, max_nnz=500000)),
                      ("vcycle", lambda A: oracle.vcycle(A, trimap.shape))]:
        cb = oracle.CounterCallback()
        x = oracle.cg(A, b, M=fac(A), atol=1e-6, rtol=0, callback=cb)
        assert np.linalg.norm(b - A.dot(x)) <= 1e-6
        assert cb.n <= caps[name]
        assert cb.n == int(g[f"s0125_it_{name}"][0])
    image, trimap, good = g["s01_image"], g["s01_trimap"], g["s01_good"]
    alpha = oracle.estimate_alpha_cf(image, trimap)
    np.testing.assert_allclose(alpha, g["s01_alpha_cf"], rtol=0, atol=1e-9)
    assert np.linalg.norm(alpha - good) < 1.68


def test_synthetic_320x240_estimate_alpha_cf():
    """The first workload: estimate_alpha_cf (ichol default) on 320x240."""
    from pymatting_b200.synthetic import make_matting_problem
    g = golden("synthetic_320x240.npz")
    img, tri, _, frac = make_matting_problem(240, 320, 1, sigma=2.0, band=7,
                                             unknown_fraction=0.12)
    np.testing.assert_allclose([img.sum(), tri.sum()], g["image_sum"], rtol=1e-12)
    alpha = oracle.estimate_alpha_cf(img, tri)
    unknown = (tri > 0.1) & (tri < 0.9)
    np.testing.assert_allclose(alpha[unknown], g["alpha_unknown"], rtol=0, atol=1e-9)


def test_estimate_alpha_cf_radius2_matches_reference():
    """estimate_alpha_cf with laplacian_kwargs={"radius": 2}: the oracle's
    composition (radius-2 Laplacian, L_U slicing, ichol, cg) against the
    reference's own result on the image the device test of that option uses."""
    from pymatting_b200.synthetic import make_matting_problem
    g = golden("alpha_cf_radius2.npz")
    img, tri, _, _ = make_matting_problem(48, 64, 9, sigma=2.0, band=4, unknown_fraction=0.2)
    np.testing.assert_allclose([img.sum(), tri.sum()], g["image_sum"], rtol=1e-12)
    alpha = oracle.estimate_alpha_cf(img, tri, laplacian_kwargs={"radius": 2})
    np.testing.assert_allclose(alpha, g["alpha"], rtol=0, atol=1e-9)
    r1 = oracle.estimate_alpha_cf(img, tri)
    assert np.abs(g["alpha"] - r1).max() > 1e-6     # radius 2 is a different system


def test_oracle_laplacian_vjp_matches_finite_differences():
    """The FP64 restatement of d(mu' L(I) x)/dI that the adjoint kernels are
    checked against, pinned by central differences of the oracle Laplacian."""
    rng = np.random.default_rng(3)
    h, w = 9, 11
    img = rng.random((h, w, 3))
    x = rng.standard_normal(h * w)
    mu = rng.standard_normal(h * w)
    eps = 1e-2   # keeps the window covariances well conditioned for differences

    def phi(im):
        return mu @ (oracle.cf_laplacian(im, eps) @ x)

    grad = oracle.cf_laplacian_vjp(img, x, mu, eps)
    step = 1e-6
    for (y, xx, c) in [(0, 0, 0), (4, 5, 1), (8, 10, 2), (3, 7, 0), (6, 2, 2)]:
        e = np.zeros_like(img)
        e[y, xx, c] = step
        fd = (phi(img + e) - phi(img - e)) / (2 * step)
        assert abs(fd - grad[y, xx, c]) <= 1e-6 * max(1.0, abs(fd)), (y, xx, c, fd, grad[y, xx, c])


def test_oracle_lkm_matches_reference():
    d = golden("lkm_small.npz")
    for name in "abc":
        L, diag = oracle.lkm_laplacian(d[f"{name}_image"], 1e-7, int(d[f"{name}_radius"][0]))
        ref_lp, ref_diag = d[f"{name}_Lp"], d[f"{name}_diag"]
        assert np.abs(L(d[f"{name}_p"]) - ref_lp).max() <= 1e-8 * np.abs(ref_lp).max()
        assert np.abs(diag - ref_diag).max() <= 1e-8 * np.abs(ref_diag).max()


def _fg_kwargs(p):
    return dict(regularization=float(p[0]), n_small_iterations=int(p[1]),
                n_big_iterations=int(p[2]), small_size=int(p[3]), gradient_weight=float(p[4]))


def test_oracle_foreground_matches_reference():
    """estimate_foreground_ml (numba, sequential Gauss-Seidel) against the C
    restatement: bit-exact F and B on every fixture case, including depths 1
    and 4, zero-iteration levels and the cases whose output keeps the seed
    colours (which pins the running float32 mean)."""
    g = golden("foreground_small.npz")
    for i in range(int(g["n_cases"][0])):
        kw = _fg_kwargs(g[f"c{i}_params"])
        F, B = oracle.estimate_foreground_ml(g[f"c{i}_image"], g[f"c{i}_alpha"],
                                             return_background=True, **kw)
        assert np.array_equal(F, g[f"c{i}_F"]), i
        assert np.array_equal(B, g[f"c{i}_B"]), i
    F, B = oracle.estimate_foreground_ml(g["lemur_image"], g["lemur_alpha"],
                                         return_background=True)
    assert np.array_equal(F, g["lemur_F"]) and np.array_equal(B, g["lemur_B"])


def test_oracle_foreground_reference_test_threshold():
    """tests/test_foreground.py of the reference: alpha-weighted mean error
    against the expected lemur foreground over unknown pixels <= 0.022."""
    g = golden("foreground_small.npz")
    alpha = g["lemur_alpha"]
    F = oracle.estimate_foreground_ml(g["lemur_image"], alpha)
    unknown = (g["lemur_trimap"] > 0.1) & (g["lemur_trimap"] < 0.9)
    diff = (alpha[:, :, None] * np.abs(F - g["lemur_expected"]))[unknown]
    assert np.mean(diff) <= 0.022


def test_oracle_foreground_levels_and_errors():
    assert oracle.fg_levels(1, 2) == [(1, 1), (1, 2)]
    lv = oracle.fg_levels(1080, 1920)
    assert len(lv) == 12 and lv[0] == (1, 1) and lv[-1] == (1080, 1920)
    with pytest.raises(ZeroDivisionError):
        oracle.estimate_foreground_ml(np.zeros((1, 1, 3)), np.zeros((1, 1)))


def test_oracle_foreground_cupy_variant_reference_threshold():
    """The reference's test runs its cupy backend through the same lemur
    check (mse <= 0.022); the oracle's restatement of that backend passes it.
    CuPy is not installed here, so this is the only pin of that restatement."""
    g = golden("foreground_small.npz")
    alpha = g["lemur_alpha"]
    F = oracle.estimate_foreground_ml_cupy(g["lemur_image"], alpha)
    unknown = (g["lemur_trimap"] > 0.1) & (g["lemur_trimap"] < 0.9)
    assert np.mean((alpha[:, :, None] * np.abs(F - g["lemur_expected"]))[unknown]) <= 0.022
    with pytest.raises(ZeroDivisionError):
        oracle.estimate_foreground_ml_cupy(np.zeros((1, 1, 3)), np.zeros((1, 1)))


def _ref_csr(g, k, name):
    n = g[f"c{k}_image"].shape[0] * g[f"c{k}_image"].shape[1]
    return scipy.sparse.csr_matrix((g[f"c{k}_{name}_data"], g[f"c{k}_{name}_indices"],
                                    g[f"c{k}_{name}_indptr"]), shape=(n, n))


def test_oracle_window_laplacians_match_reference():
    """uniform_laplacian: identical values. rw_laplacian: within 1e-15 (the
    reference's exp and norm run through numba/libm; a few weights near the
    underflow range round differently). Entries the reference's sparse
    arithmetic drops as exact zeros are kept here as zeros."""
    g = golden("laplacians_small.npz")
    for k in range(int(g["n_cases"][0])):
        img, r = g[f"c{k}_image"], int(g[f"c{k}_radius"][0])
        for name, reg, tol in (("uniform", 0.0, 0.0), ("rw", 1e-8, 1e-15)):
            L = oracle.window_laplacian(img, r, reg, name)
            D = abs(L - _ref_csr(g, k, name))
            assert (D.max() if D.nnz else 0.0) <= tol, (k, name)


def test_oracle_lbdm_matches_reference():
    """lbdm_laplacian: the per-window solve (K + eps I)^-1 K is
    ill-conditioned (K = X X^T has rank 4 of (2r+1)^2), so two LAPACK builds
    agree only to ~1e-9 of the matrix scale; tolerance 1e-8 of max |L|."""
    g = golden("laplacians_small.npz")
    for k in range(int(g["lbdm_n"][0])):
        img, r = g[f"lbdm{k}_image"], int(g[f"lbdm{k}_radius"][0])
        n = img.shape[0] * img.shape[1]
        R = scipy.sparse.csr_matrix((g[f"lbdm{k}_data"], g[f"lbdm{k}_indices"],
                                     g[f"lbdm{k}_indptr"]), shape=(n, n))
        D = abs(oracle.lbdm_laplacian(img, radius=r) - R)
        assert (D.max() if D.nnz else 0.0) <= 1e-8 * max(abs(R).max(), 1.0), k


def test_oracle_knn_laplacian_matches_reference():
    """The index-order search with the k-d tree's insertion rule gives the
    reference's knn_laplacian exactly on random images (binary and soft);
    on the lemur image only rows whose k-th neighbour is tied can differ."""
    g = golden("laplacians_small.npz")

    def ref(prefix, n):
        return scipy.sparse.csr_matrix((g[prefix + "_data"], g[prefix + "_indices"],
                                        g[prefix + "_indptr"]), shape=(n, n))

    for k in range(int(g["knn_n"][0])):
        img = g[f"knn{k}_image"]
        n = img.shape[0] * img.shape[1]
        L = oracle.knn_laplacian(img, kernel="soft" if g[f"knn{k}_soft"][0] else "binary")
        D = abs(scipy.sparse.csr_matrix(L) - ref(f"knn{k}", n))
        assert (D.max() if D.nnz else 0.0) == 0.0, k
    img = g["lemur_image"]
    n = img.shape[0] * img.shape[1]
    L = scipy.sparse.csr_matrix(oracle.knn_laplacian(img))
    D = (L - ref("lemur_knn", n)).tocsr()
    D.eliminate_zeros()
    # two rows have a tied k-th neighbour; the neighbours they swap change
    # their own reverse entries too (6 rows in all)
    assert np.count_nonzero(np.diff(D.indptr)) <= 10
