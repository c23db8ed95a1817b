"""Parity of the CUDA path with the reference (through the golden fixtures
and the oracle). Every call goes through the C ABI of libpmb200.so.

Tolerances: the assembled Laplacian and ichol structure are exact; solver
results are compared at 1e-6 absolute (the reference's own CG stops at
relative residual 1e-7); alpha within 1e-4 max-abs of the reference solve;
FP64 relative residuals <= 1e-7."""

import numpy as np
import pytest
import scipy.sparse

import oracle
from tests.conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pm(gpu):
    import pymatting_b200
    return pymatting_b200


def test_cf_laplacian_bit_exact(pm):
    g = golden("cf_laplacian_small.npz")
    for k in range(int(g["count"][0])):
        h, w, r = (int(v) for v in g[f"c{k}_meta"])
        L = pm.cf_laplacian(g[f"c{k}_image"], float(g[f"c{k}_eps"][0]), r, g[f"c{k}_known"])
        assert isinstance(L, scipy.sparse.csr_matrix)
        assert L.shape == (h * w, h * w)
        np.testing.assert_array_equal(L.indptr, g[f"c{k}_indptr"])
        np.testing.assert_array_equal(L.indices, g[f"c{k}_indices"])
        np.testing.assert_array_equal(L.data, g[f"c{k}_values"])


def test_make_linear_system_bit_exact(pm):
    g = golden("soft_small.npz")
    for k in range(int(g["count"][0])):
        A, b = pm.make_linear_system(pm.cf_laplacian(g[f"k{k}_image"]), g[f"k{k}_trimap"])
        np.testing.assert_array_equal(A.indptr, g[f"k{k}_A_indptr"])
        np.testing.assert_array_equal(A.indices, g[f"k{k}_A_indices"])
        np.testing.assert_array_equal(A.data, g[f"k{k}_A_data"])
        np.testing.assert_array_equal(b, g[f"k{k}_b"])


def test_make_linear_system_of_host_matrix(pm):
    """A host scipy Laplacian goes through the device canonicalisation."""
    g = golden("soft_small.npz")
    img, tri = g["k0_image"], g["k0_trimap"]
    L = oracle.cf_laplacian(img)
    A, b, c = pm.make_linear_system(L, tri, return_c=True)
    Ar, br, cr = oracle.make_linear_system(L, tri, return_c=True)
    np.testing.assert_array_equal(A.indptr, Ar.indptr)
    np.testing.assert_array_equal(A.indices, Ar.indices)
    np.testing.assert_array_equal(A.data, Ar.data)
    np.testing.assert_array_equal(c, cr)


@pytest.mark.parametrize("name", ["none", "jacobi", "vcycle"])
def test_soft_system_cg(pm, name):
    g = golden("soft_small.npz")
    for k in range(int(g["count"][0])):
        img, tri = g[f"k{k}_image"], g[f"k{k}_trimap"]
        h, w = tri.shape
        A, b = pm.make_linear_system(pm.cf_laplacian(img), tri)
        M = {"none": None, "jacobi": pm.jacobi(A), "vcycle": pm.vcycle(A, (h, w))}[name]
        cb = pm.CounterCallback()
        x = pm.cg(A, b, M=M, rtol=1e-7, callback=cb)
        assert abs(cb.n - int(g[f"k{k}_it_{name}"][0])) <= 1
        np.testing.assert_allclose(x, g[f"k{k}_x_{name}"], rtol=0, atol=1e-6)


def test_vcycle_apply_matches_reference(pm):
    g = golden("soft_small.npz")
    for k in range(int(g["count"][0])):
        img, tri = g[f"k{k}_image"], g[f"k{k}_trimap"]
        h, w = tri.shape
        A, b = pm.make_linear_system(pm.cf_laplacian(img), tri)
        v = g[f"k{k}_v"]
        np.testing.assert_allclose(pm.vcycle(A, (h, w))(v), g[f"k{k}_vcycle_v"],
                                   rtol=1e-11, atol=1e-12)
        A2, _ = pm.make_linear_system(pm.cf_laplacian(img), tri)
        z2 = pm.vcycle(A2, (h, w), num_pre_iter=2, num_post_iter=3, omega=0.7)(v)
        np.testing.assert_allclose(z2, g[f"k{k}_vcycle_v_2_3"], rtol=1e-11, atol=1e-12)


def test_cg_reference_cases(pm):
    g = golden("cg_small.npz")
    for k in range(int(g["count"][0])):
        A, b = g[f"k{k}_A"], g[f"k{k}_b"]
        x0 = g[f"k{k}_x0"]
        x0 = None if x0.size == 0 else x0
        mk = int(g[f"k{k}_M"][0])
        Mj = np.diag(1.0 / np.diag(A))
        M = [None, Mj, lambda v, Mj=Mj: Mj.dot(v)][mk]
        for cb in [pm.CounterCallback(), pm.ProgressCallback()]:
            x = pm.cg(A, b, x0=x0, M=M, rtol=0, atol=1e-10, callback=cb)
            assert np.linalg.norm(A.dot(x) - b) < 1e-10
            assert 0 < cb.n < 20
            assert abs(cb.n - int(g[f"k{k}_iters"][0])) <= 1


def test_cg_function_operator_and_reorthogonalize(pm):
    g = golden("cg_small.npz")
    A, b = g["k12_A"], g["k12_b"]
    x = pm.cg(lambda v: A.dot(v), b, x0=np.ones_like(b), rtol=0, atol=1e-10)
    assert np.linalg.norm(A.dot(x) - b) < 1e-10
    x = pm.cg(A, b, M=pm.jacobi(A), reorthogonalize=True, rtol=0, atol=1e-10)
    assert np.linalg.norm(A.dot(x) - b) < 1e-10


def test_cg_maxiter_raises(pm):
    g = golden("soft_small.npz")
    A, b = pm.make_linear_system(pm.cf_laplacian(g["k0_image"]), g["k0_trimap"])
    with pytest.raises(ValueError, match="did not converge within 3 iterations"):
        pm.cg(A, b, maxiter=3)


def test_docstring_examples(pm):
    g = golden("cg_small.npz")
    A = np.array([[3.0, 1.0], [1.0, 2.0]])
    np.testing.assert_allclose(pm.cg(A, np.array([4.0, 3.0]), M=pm.jacobi(A)), g["doc_cg"],
                               atol=1e-12)
    np.testing.assert_allclose(pm.jacobi(np.array([[2, 3], [3, 5]]))(np.array([1, 2])),
                               g["doc_jacobi"])
    np.testing.assert_allclose(pm.vcycle(np.array([[2, 3], [3, 5]]), (2, 2))(np.array([1, 2])),
                               g["doc_vcycle"], atol=1e-12)
    d = pm.ichol(scipy.sparse.csc_matrix(np.array([[2.0, 3.0], [3.0, 5.0]])))
    np.testing.assert_allclose(d(np.array([1.0, 2.0])), g["doc_ichol"], atol=1e-12)


def test_ichol_factors(pm):
    g = golden("ichol_small.npz")
    for k in range(int(g["count"][0])):
        n = len(g[f"k{k}_A_indptr"]) - 1
        A = scipy.sparse.csc_matrix(
            (g[f"k{k}_A_data"], g[f"k{k}_A_indices"], g[f"k{k}_A_indptr"]), (n, n))
        thr, rel, keep = (float(v) for v in g[f"k{k}_params"])
        d = pm.ichol(A, discard_threshold=thr, relative_discard_threshold=rel,
                     diag_keep_discarded=bool(keep),
                     max_nnz=100000 if thr == 0.0 else int(4e9 / 16))
        Lv, Lr, Lp = d.Ltuple
        np.testing.assert_array_equal(Lp, g[f"k{k}_Lp"])
        np.testing.assert_array_equal(Lr, g[f"k{k}_Lr"])
        np.testing.assert_allclose(Lv, g[f"k{k}_Lv"], rtol=1e-12, atol=1e-13)
        rhs = np.random.default_rng(k).standard_normal(n)
        ref = oracle.CholeskyDecomposition((g[f"k{k}_Lv"], g[f"k{k}_Lr"], g[f"k{k}_Lp"]))(rhs)
        np.testing.assert_allclose(d(rhs), ref, rtol=1e-10, atol=1e-12)


def test_ichol_errors(pm):
    A = scipy.sparse.csc_matrix(np.array([[1.0, 2.0], [2.0, 1.0]]))   # indefinite
    with pytest.raises(ValueError, match="positive-definiteness"):
        pm.ichol(A, shifts=[0.0])
    g = golden("ichol_small.npz")
    n = len(g["k0_A_indptr"]) - 1
    A = scipy.sparse.csc_matrix((g["k0_A_data"], g["k0_A_indices"], g["k0_A_indptr"]), (n, n))
    with pytest.raises(ValueError, match="max_nnz"):
        pm.ichol(A, discard_threshold=0.0, max_nnz=100)
    with pytest.raises(ValueError, match="csc_matrix"):
        pm.ichol(scipy.sparse.coo_matrix(A))


def test_lemur_reference_pins(pm):
    """The reference tests' own pins: iteration caps, residual, alpha error."""
    g = golden("lemur.npz")
    image, trimap = g["s0125_image"], g["s0125_trimap"]
    caps = {"none": 378, "jacobi": 197, "icholt": 3, "vcycle": 48}
    Ah, _ = oracle.make_linear_system(oracle.cf_laplacian(image), trimap)
    for name in ["none", "jacobi", "icholt", "vcycle"]:
        A, b = pm.make_linear_system(pm.cf_laplacian(image), trimap)
        M = {"none": lambda: None, "jacobi": lambda: pm.jacobi(A),
             "icholt": lambda: pm.ichol(A, max_nnz=500000),
             "vcycle": lambda: pm.vcycle(A, trimap.shape)}[name]()
        cb = pm.CounterCallback()
        x = pm.cg(A, b, M=M, atol=1e-6, rtol=0, maxiter=10000, callback=cb)
        assert np.linalg.norm(b - Ah.dot(x)) <= 1e-6
        assert cb.n <= caps[name]
        assert cb.n == int(g[f"s0125_it_{name}"][0])
    image, trimap, good = g["s01_image"], g["s01_trimap"], g["s01_good"]
    alpha = pm.estimate_alpha_cf(image, trimap)
    np.testing.assert_allclose(alpha, g["s01_alpha_cf"], rtol=0, atol=1e-6)
    assert np.linalg.norm(alpha - good) < 1.68
    assert pm.estimate_alpha is pm.estimate_alpha_cf


def test_estimate_alpha_cf_320x240(pm):
    """The 320x240 workload (default ichol): alpha within 1e-4 of the reference."""
    from pymatting_b200.synthetic import make_matting_problem
    g = golden("synthetic_320x240.npz")
    img, tri, _, _ = make_matting_problem(240, 320, 1, sigma=2.0, band=7, unknown_fraction=0.12)
    alpha = pm.estimate_alpha_cf(img, tri)
    unknown = (tri > 0.1) & (tri < 0.9)
    assert np.abs(alpha[unknown] - g["alpha_unknown"]).max() <= 1e-4
    known = ~unknown
    np.testing.assert_array_equal(alpha[known], np.clip(tri[known], 0, 1))
    a2 = pm.estimate_alpha_cf(img, tri, preconditioner=pm.jacobi, cg_kwargs={"maxiter": 5000})
    assert np.abs(a2[unknown] - g["alpha_unknown"]).max() <= 1e-3


def test_soft_1080p_fp64_and_mixed(pm):
    """1920x1080 soft system: FP64 path against the reference CPU solve, mixed
    path by FP64 relative residual."""
    from pymatting_b200.batch import solve_alpha
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _, _ = make_matting_problem(1080, 1920, 2, sigma=3.0, band=10, unknown_fraction=0.08)
    A, b = oracle.make_linear_system(oracle.cf_laplacian(img), tri)
    x_ref, it_ref = oracle.solve_soft(img, tri, preconditioner="vcycle", rtol=1e-7)
    (a64,), (s64,) = solve_alpha([img], [tri], precision="fp64", return_stats=True)
    assert abs(s64.iters - it_ref) <= 1
    assert np.abs(a64.ravel() - np.clip(x_ref, 0, 1)).max() <= 1e-4
    Lp = pm.cf_laplacian(img)
    A_dev, b_dev = pm.make_linear_system(Lp, tri)
    x64 = pm.cg(A_dev, b_dev, M=pm.vcycle(A_dev, tri.shape), rtol=1e-7)
    assert np.linalg.norm(b - A.dot(x64)) / np.linalg.norm(b) <= 1e-7
    from pymatting_b200.batch import AlphaBatch
    batch = AlphaBatch([img], [tri], precision="mixed")
    xm = batch.solve().cpu().numpy()
    assert np.linalg.norm(b - A.dot(xm)) / np.linalg.norm(b) <= 1e-7
    # The last FP32 phase stops at the FP64 tolerance, so FP32 arithmetic
    # costs no extra iterations here.
    sm = batch.stats()[0]
    assert sm.iters <= s64.iters + 1, (sm.iters, s64.iters)
