"""uniform_laplacian and rw_laplacian assembled on the device, against the
reference's matrices (tests/golden/laplacians_small.npz) and the reference
test's lemur errors (tests/test_laplacians.py: error of the clipped solve
against the good alpha on unknown pixels, 1 % regression allowed).

Tolerances: uniform values identical; rw within 1e-15 absolute (entries are
at most 1 in size; the reference's exp and norm come from numba/libm)."""

import numpy as np
import pytest
import scipy.sparse

import oracle
from tests.conftest import golden

pytestmark = pytest.mark.gpu


def _ref_csr(g, k, name):
    n = g[f"c{k}_image"].shape[0] * g[f"c{k}_image"].shape[1]
    return scipy.sparse.csr_matrix((g[f"c{k}_{name}_data"], g[f"c{k}_{name}_indices"],
                                    g[f"c{k}_{name}_indptr"]), shape=(n, n))


def _maxdiff(A, B):
    D = abs(scipy.sparse.csr_matrix(A) - B)
    return D.max() if D.nnz else 0.0


def test_window_laplacians_match_reference(gpu):
    import pymatting_b200 as pm
    g = golden("laplacians_small.npz")
    for k in range(int(g["n_cases"][0])):
        img, r = g[f"c{k}_image"], int(g[f"c{k}_radius"][0])
        U = pm.uniform_laplacian(img, radius=r)
        assert isinstance(U, scipy.sparse.csr_matrix) and U.shape == _ref_csr(g, k, "uniform").shape
        assert _maxdiff(U, _ref_csr(g, k, "uniform")) == 0.0, k
        assert _maxdiff(pm.rw_laplacian(img, radius=r), _ref_csr(g, k, "rw")) <= 1e-15, k


def test_window_laplacians_match_oracle_bitwise_structure(gpu):
    import pymatting_b200 as pm
    rng = np.random.default_rng(9)
    img = rng.random((37, 53, 3))
    for name, fn, reg in (("uniform", pm.uniform_laplacian, 0.0), ("rw", pm.rw_laplacian, 1e-8)):
        L = fn(img)
        Lr = oracle.window_laplacian(img, 1, reg, name)
        assert np.array_equal(L.indptr, Lr.indptr) and np.array_equal(L.indices, Lr.indices)
        tol = 0.0 if name == "uniform" else 1e-15
        assert np.abs(L.data - Lr.data).max() <= tol


def test_reference_laplacian_errors_on_lemur(gpu):
    """Both Laplacians are row-normalised, hence not symmetric: like the
    reference test, solve with scipy's spsolve (here on the matrix assembled
    on the device) rather than CG."""
    import scipy.sparse.linalg
    import pymatting_b200 as pm
    g = golden("laplacians_small.npz")
    image, trimap, good = g["lemur_image"], g["lemur_trimap"], g["lemur_good"]
    is_unknown = pm.trimap_split(trimap, flatten=False)[3]
    for name, fn in (("uniform", pm.uniform_laplacian), ("rw", pm.rw_laplacian)):
        A, b = pm.make_linear_system(fn(image), trimap)
        x = scipy.sparse.linalg.spsolve(scipy.sparse.csr_matrix(A), b)
        alpha = np.clip(x, 0, 1).reshape(trimap.shape)
        error = np.linalg.norm(np.abs(alpha - good)[is_unknown])
        expected = float(g[f"lemur_{name}_error"][0])
        assert (error - expected) / expected <= 0.01, (name, error, expected)
        assert abs(error - expected) <= 1e-6 * expected, (name, error, expected)


LBDM_TOL = 1e-8   # of max |L|: the per-window solve is ill-conditioned (rank-4 K)


def test_lbdm_matches_reference(gpu):
    import pymatting_b200 as pm
    g = golden("laplacians_small.npz")
    for k in range(int(g["lbdm_n"][0])):
        img, r = g[f"lbdm{k}_image"], int(g[f"lbdm{k}_radius"][0])
        n = img.shape[0] * img.shape[1]
        R = scipy.sparse.csr_matrix((g[f"lbdm{k}_data"], g[f"lbdm{k}_indices"],
                                     g[f"lbdm{k}_indptr"]), shape=(n, n))
        L = pm.lbdm_laplacian(img, radius=r)
        assert np.array_equal(L.indptr, R.indptr) and np.array_equal(L.indices, R.indices), k
        assert np.abs(L.data - R.data).max() <= LBDM_TOL * max(np.abs(R.data).max(), 1.0), k


def test_lbdm_larger_against_oracle_and_lemur_error(gpu):
    import scipy.sparse.linalg
    import pymatting_b200 as pm
    rng = np.random.default_rng(4)
    img = rng.random((48, 61, 3))
    L = pm.lbdm_laplacian(img)
    R = oracle.lbdm_laplacian(img)
    assert _maxdiff(L, R) <= LBDM_TOL * abs(R).max()
    g = golden("laplacians_small.npz")
    image, trimap, good = g["lemur_image"], g["lemur_trimap"], g["lemur_good"]
    is_unknown = pm.trimap_split(trimap, flatten=False)[3]
    A, b = pm.make_linear_system(pm.lbdm_laplacian(image), trimap)
    x = scipy.sparse.linalg.spsolve(scipy.sparse.csr_matrix(A), b)
    error = np.linalg.norm(np.abs(np.clip(x, 0, 1).reshape(trimap.shape) - good)[is_unknown])
    expected = float(g["lemur_lbdm_error"][0])
    assert (error - expected) / expected <= 0.01
    assert abs(error - expected) <= 1e-5 * expected, (error, expected)


def _knn_ref(g, prefix, n):
    return scipy.sparse.csr_matrix((g[prefix + "_data"], g[prefix + "_indices"],
                                    g[prefix + "_indptr"]), shape=(n, n))


def test_knn_matches_reference_and_oracle(gpu):
    """Same neighbour rule and candidate order as the oracle: identical
    matrices. Against the reference: identical on random images; on the
    lemur image rows whose k-th neighbour is tied may differ (the reference
    resolves ties in its k-d tree's order)."""
    import pymatting_b200 as pm
    g = golden("laplacians_small.npz")
    for k in range(int(g["knn_n"][0])):
        img = g[f"knn{k}_image"]
        n = img.shape[0] * img.shape[1]
        kern = "soft" if g[f"knn{k}_soft"][0] else "binary"
        L = pm.knn_laplacian(img, kernel=kern)
        assert _maxdiff(L, _knn_ref(g, f"knn{k}", n)) == 0.0, k
    img = g["lemur_image"]
    n = img.shape[0] * img.shape[1]
    L = pm.knn_laplacian(img)
    Lo = scipy.sparse.csr_matrix(oracle.knn_laplacian(img))
    Lo.sum_duplicates()
    Lo.sort_indices()
    assert np.array_equal(L.indptr, Lo.indptr) and np.array_equal(L.indices, Lo.indices)
    assert np.array_equal(L.data, Lo.data)
    D = (scipy.sparse.csr_matrix(L) - _knn_ref(g, "lemur_knn", n)).tocsr()
    D.eliminate_zeros()
    # two rows have a tied k-th neighbour; the neighbours they swap change
    # their own reverse entries too (6 rows in all)
    assert np.count_nonzero(np.diff(D.indptr)) <= 10


def test_knn_lemur_error_and_errors(gpu):
    import scipy.sparse.linalg
    import pymatting_b200 as pm
    g = golden("laplacians_small.npz")
    image, trimap, good = g["lemur_image"], g["lemur_trimap"], g["lemur_good"]
    is_unknown = pm.trimap_split(trimap, flatten=False)[3]
    A, b = pm.make_linear_system(pm.knn_laplacian(image), trimap)
    x = scipy.sparse.linalg.spsolve(scipy.sparse.csr_matrix(A), b)
    error = np.linalg.norm(np.abs(np.clip(x, 0, 1).reshape(trimap.shape) - good)[is_unknown])
    expected = float(g["lemur_knn_error"][0])
    assert (error - expected) / expected <= 0.01, (error, expected)
    with pytest.raises(ValueError):
        pm.knn_laplacian(image, kernel="gaussian")


@pytest.mark.parametrize("name,limit,tol", [("knn", 2.2, 1e-3), ("lbdm", 1.68, 1e-4),
                                            ("rw", 6.0, 1e-4)])
def test_other_alpha_estimators(gpu, name, limit, tol):
    """tests/test_estimate_alpha.py of the reference (error against the good
    alpha below its limit) and the reference's own alpha for the same lemur
    inputs: mean difference within `tol` (CG stops at rtol 1e-7; the knn
    matrix differs in the rows with tied neighbours)."""
    import pymatting_b200 as pm
    g = golden("laplacians_small.npz")
    image, trimap, good = g["lemur_image"], g["lemur_trimap"], g["lemur_good"]
    alpha = getattr(pm, "estimate_alpha_" + name)(image, trimap)
    assert alpha.shape == trimap.shape
    assert np.linalg.norm(alpha - good) < limit
    assert np.abs(alpha - g["lemur_alpha_" + name]).mean() <= tol


def test_laplacians_list(gpu):
    import pymatting_b200 as pm
    assert [f.__name__ for f in pm.LAPLACIANS] == [
        "cf_laplacian", "knn_laplacian", "lbdm_laplacian", "rw_laplacian", "uniform_laplacian"]


def test_knn_pruned_search_on_a_larger_image(gpu):
    """96x128 pixels, 48 candidate tiles, so tile pruning is exercised:
    identical to the oracle's brute force."""
    import pymatting_b200 as pm
    from pymatting_b200.synthetic import make_matting_problem
    img, _, _, _ = make_matting_problem(96, 128, 3, sigma=2.0, band=5, unknown_fraction=0.1)
    for kern in ("binary", "soft"):
        L = pm.knn_laplacian(img, kernel=kern)
        Lo = scipy.sparse.csr_matrix(oracle.knn_laplacian(img, kernel=kern))
        Lo.sum_duplicates()
        Lo.sort_indices()
        assert np.array_equal(L.indptr, Lo.indptr) and np.array_equal(L.indices, Lo.indices)
        assert np.array_equal(L.data, Lo.data)
