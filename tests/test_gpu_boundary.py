"""The drop-in boundary on inputs this package did not produce: host scipy
matrices in the reference's own arithmetic, rows longer than a radius-1
Laplacian's, and radius-2 Laplacians in estimate_alpha_cf. Every call goes
through the C ABI of libpmb200.so.

Tolerances: matrices exact; iteration counts within one of the reference's
and under the reference test's caps; alphas within 1e-6 of the reference
solve with the same stopping rule (rel-res 1e-7 with ichol, whose iterations
the device path repeats)."""

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


def test_reference_preconditioner_sequence_on_host_matrix(pm):
    """pymatting's tests/test_preconditioners.py sequence with A and b from
    the reference's own make_linear_system (a host scipy CSR matrix): every
    preconditioner factory of this package takes it, and vcycle converts it
    to the stencil planes on the device."""
    from pymatting_b200.preconditioner import GridPlanes
    g = golden("lemur.npz")
    image, trimap = g["s0125_image"], g["s0125_trimap"]
    A, b = oracle.make_linear_system(oracle.cf_laplacian(image), trimap)
    assert isinstance(A, scipy.sparse.csr_matrix)
    caps = {"none": 378, "jacobi": 197, "icholt": 3, "vcycle": 48}
    factories = {"none": lambda A: None, "jacobi": lambda A: pm.jacobi(A),
                 "icholt": lambda A: pm.ichol(A, max_nnz=500000),
                 "vcycle": lambda A: pm.vcycle(A, trimap.shape)}
    for name, make in factories.items():
        cb = pm.CounterCallback()
        M = make(A)
        if name == "vcycle":
            assert isinstance(M.source, GridPlanes)
        x = pm.cg(A, b, M=M, atol=1e-6, rtol=0, maxiter=10000, callback=cb)
        assert isinstance(x, np.ndarray)
        assert np.linalg.norm(b - A.dot(x)) <= 1e-6
        assert cb.n <= caps[name]
        assert abs(cb.n - int(g[f"s0125_it_{name}"][0])) <= 1


def test_vcycle_on_host_matrix_matches_device_matrix(pm):
    """The planes built from the host matrix give the same V-cycle as the
    planes this package assembles for the same image."""
    g = golden("soft_small.npz")
    img, tri = g["k0_image"], g["k0_trimap"]
    h, w = tri.shape
    Ah, _ = oracle.make_linear_system(oracle.cf_laplacian(img), tri)
    Ad, _ = pm.make_linear_system(pm.cf_laplacian(img), tri)
    v = np.random.default_rng(3).standard_normal(h * w)
    np.testing.assert_allclose(pm.vcycle(Ah, (h, w))(v), pm.vcycle(Ad, (h, w))(v),
                               rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(pm.vcycle(Ah, (h, w))(v), oracle.vcycle(Ah, (h, w))(v),
                               rtol=1e-11, atol=1e-12)


def test_vcycle_rejects_matrices_outside_the_stencil(pm):
    g = golden("soft_small.npz")
    img, tri = g["k0_image"], g["k0_trimap"]
    h, w = tri.shape
    A, _ = oracle.make_linear_system(oracle.cf_laplacian(img), tri)
    far = A.tolil()
    far[0, 3 * w] = 1e-3          # three rows away
    far[3 * w, 0] = 1e-3
    with pytest.raises(NotImplementedError, match="two"):
        pm.vcycle(far.tocsr(), (h, w))
    skew = A.tolil()
    skew[0, 1] = skew[0, 1] + 0.5   # A[0, 1] != A[1, 0]
    with pytest.raises(NotImplementedError, match="symmetric"):
        pm.vcycle(skew.tocsr(), (h, w))


def test_make_linear_system_radius2(pm):
    """Radius-2 Laplacians have 81 stored entries per row: the device
    canonicalisation handles rows of any length, bit-exact."""
    g = golden("soft_small.npz")
    img, tri = g["k0_image"], g["k0_trimap"]
    L2 = oracle.cf_laplacian(img, radius=2)
    assert np.diff(L2.indptr).max() == 81
    A, b, c = pm.make_linear_system(L2, tri, return_c=True)
    Ar, br, cr = oracle.make_linear_system(L2, tri, return_c=True)
    np.testing.assert_array_equal(A.indptr, Ar.indptr)
    np.testing.assert_array_equal(A.indices, Ar.indices)
    np.testing.assert_array_equal(A.data, Ar.data)
    np.testing.assert_array_equal(b, br)
    Ad, bd = pm.make_linear_system(pm.cf_laplacian(img, radius=2), tri)
    np.testing.assert_array_equal(Ad.indptr, Ar.indptr)
    np.testing.assert_array_equal(Ad.indices, Ar.indices)
    np.testing.assert_array_equal(Ad.data, Ar.data)


def test_estimate_alpha_cf_radius2(pm):
    """estimate_alpha_cf(..., laplacian_kwargs={"radius": 2}) (the reference
    passes laplacian_kwargs to cf_laplacian, estimate_alpha_cf.py:55)."""
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _a, _f = make_matting_problem(48, 64, 9, sigma=2.0, band=4, unknown_fraction=0.2)
    kw = {"radius": 2}
    alpha = pm.estimate_alpha_cf(img, tri, laplacian_kwargs=kw)
    ref = oracle.estimate_alpha_cf(img, tri, laplacian_kwargs=kw)
    np.testing.assert_allclose(alpha, ref, rtol=0, atol=1e-6)
    r1 = pm.estimate_alpha_cf(img, tri)
    assert np.abs(alpha - r1).max() > 1e-6      # the radius really changed the system
    with pytest.raises(ValueError):
        pm.estimate_alpha_cf(img, tri, laplacian_kwargs={"radius": 0})
