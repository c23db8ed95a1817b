"""Generate the golden fixtures in this folder by running PyMatting itself.

Run in a container where the reference source tree is available:

    python tests/golden/make_golden.py /path/to/pymatting-checkout

The reference is imported in place. Its package ``__init__`` asks
``importlib.metadata`` for its own version, which fails for a source tree
that is not pip-installed, so the lookup is answered with "1.1.15" for that
one name. Outputs are small ``.npz`` files; the tests read only those, never
the reference tree.
"""

import importlib.metadata
import os
import sys

import numpy as np
import scipy.sparse

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def import_reference(root):
    real_version = importlib.metadata.version

    def version(name):
        if name.lower() == "pymatting":
            return "1.1.15"
        return real_version(name)

    importlib.metadata.version = version
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
    sys.path.insert(0, root)
    import pymatting  # noqa: E402
    return pymatting


def small_image(rng, h, w):
    base = rng.uniform(0.1, 0.9, size=(1, 1, 3))
    img = base + 0.15 * rng.standard_normal((h, w, 3))
    # A few flat clipped patches exercise the near-singular covariance case.
    img[: max(h // 3, 1), : max(w // 3, 1), :] = 1.0
    return np.clip(img, 0.0, 1.0)


def gen_cf(pm, rng):
    cases = [(1, 1, 1, False), (2, 5, 1, False), (3, 3, 1, False), (5, 5, 1, True),
             (7, 9, 1, False), (16, 13, 1, True), (24, 20, 1, False),
             (11, 17, 2, False), (9, 8, 2, True)]
    out = {}
    for k, (h, w, r, with_known) in enumerate(cases):
        img = small_image(rng, h, w)
        if with_known:
            known = rng.uniform(size=(h, w)) < 0.6
        else:
            known = np.zeros((h, w), dtype=bool)
        eps = 1e-7 if k % 3 else 1e-5
        L = pm.cf_laplacian(img, epsilon=eps, radius=r, is_known=known)
        out[f"c{k}_image"] = img
        out[f"c{k}_known"] = known
        out[f"c{k}_meta"] = np.array([h, w, r], dtype=np.int64)
        out[f"c{k}_eps"] = np.array([eps])
        out[f"c{k}_values"] = L.data
        out[f"c{k}_indices"] = L.indices.astype(np.int64)
        out[f"c{k}_indptr"] = L.indptr.astype(np.int64)
    out["count"] = np.array([len(cases)])
    np.savez_compressed(os.path.join(HERE, "cf_laplacian_small.npz"), **out)


def gen_cg(pm):
    """The reference's own CG test matrices, with the reference's answers."""
    np.random.seed(0)
    out = {}
    k = 0
    for n in [1, 5, 10]:
        x_true = np.random.rand(n)
        A = np.random.rand(n, n)
        A += A.T + n * np.eye(n)
        b = A.dot(x_true)
        M_jacobi = np.diag(1.0 / np.diag(A))
        for x0 in [None, np.random.rand(n)]:
            for mk in ["none", "matrix", "callable"]:
                M = {"none": None, "matrix": M_jacobi,
                     "callable": (lambda v, M_=M_jacobi: M_.dot(v))}[mk]
                cb = pm.CounterCallback()
                x = pm.cg(A, b, x0=x0, M=M, rtol=0, atol=1e-10, callback=cb)
                out[f"k{k}_A"] = A
                out[f"k{k}_b"] = b
                out[f"k{k}_x0"] = np.zeros(0) if x0 is None else x0
                out[f"k{k}_M"] = np.array([["none", "matrix", "callable"].index(mk)])
                out[f"k{k}_x"] = x
                out[f"k{k}_iters"] = np.array([cb.n])
                k += 1
    out["count"] = np.array([k])
    # Docstring examples of cg / jacobi / vcycle / ichol.
    A = np.array([[3.0, 1.0], [1.0, 2.0]])
    out["doc_cg"] = pm.cg(A, np.array([4.0, 3.0]), M=pm.jacobi(A))
    out["doc_jacobi"] = pm.jacobi(np.array([[2, 3], [3, 5]]))(np.array([1, 2]))
    out["doc_vcycle"] = pm.vcycle(np.array([[2, 3], [3, 5]]), (2, 2))(np.array([1, 2]))
    out["doc_ichol"] = pm.ichol(scipy.sparse.csc_matrix(np.array([[2.0, 3.0], [3.0, 5.0]])))(
        np.array([1.0, 2.0]))
    np.savez_compressed(os.path.join(HERE, "cg_small.npz"), **out)


def _store_csc(out, k, A):
    A = scipy.sparse.csc_matrix(A)
    A.sum_duplicates()
    out[f"k{k}_A_data"] = A.data
    out[f"k{k}_A_indices"] = A.indices.astype(np.int64)
    out[f"k{k}_A_indptr"] = A.indptr.astype(np.int64)


def gen_ichol(pm, rng):
    """Reference factors: the test_ichol matrices plus thresholded CF systems."""
    out = {}
    np.random.seed(0)
    k = 0
    for _ in range(4):
        n = 50
        A = np.random.rand(n, n)
        A[np.random.rand(n, n) < 0.8] = 0
        A += A.T + n * np.eye(n)
        Ac = scipy.sparse.csc_matrix(A)
        dec = pm.ichol(Ac, discard_threshold=0.0, max_nnz=100000)
        Lv, Lr, Lp = dec.Ltuple
        _store_csc(out, k, Ac)
        out[f"k{k}_params"] = np.array([0.0, 0.0, 1.0])
        out[f"k{k}_Lv"], out[f"k{k}_Lr"], out[f"k{k}_Lp"] = Lv, Lr, Lp
        k += 1
    # Hard-constraint CF system L_U of a small synthetic problem, with the
    # default and stronger thresholds (both the absolute and relative paths).
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _, _ = make_matting_problem(30, 40, 11, sigma=2.0, band=3,
                                          unknown_fraction=0.3)
    is_fg, is_bg, is_known, is_unknown = pm.trimap_split(tri)
    L = pm.cf_laplacian(img, is_known=is_known)
    L_U = L[is_unknown, :][:, is_unknown]
    for params in [(1e-4, 0.0, 1.0), (1e-2, 0.0, 1.0), (1e-4, 0.05, 1.0),
                   (1e-3, 0.0, 0.0)]:
        thr, rel, keep = params
        dec = pm.ichol(L_U.copy(), discard_threshold=thr,
                       relative_discard_threshold=rel,
                       diag_keep_discarded=bool(keep))
        Lv, Lr, Lp = dec.Ltuple
        # ichol factors the CSC view of L_U's transpose (a CSR input is
        # transposed first), whose bits differ from L_U's own columns.
        _store_csc(out, k, L_U.T)
        out[f"k{k}_params"] = np.array(params)
        out[f"k{k}_Lv"], out[f"k{k}_Lr"], out[f"k{k}_Lp"] = Lv, Lr, Lp
        k += 1
    out["count"] = np.array([k])
    np.savez_compressed(os.path.join(HERE, "ichol_small.npz"), **out)


def gen_soft(pm):
    """Soft-constraint system of a small synthetic image: vcycle output and
    CG results for every preconditioner."""
    from pymatting_b200.synthetic import make_matting_problem
    out = {}
    for k, (h, w, seed) in enumerate([(30, 40, 3), (37, 29, 4)]):
        img, tri, _, _ = make_matting_problem(h, w, seed, sigma=2.0, band=3,
                                              unknown_fraction=0.25)
        A, b = pm.make_linear_system(pm.cf_laplacian(img), tri)
        rng = np.random.default_rng(seed)
        v = rng.standard_normal(h * w)
        out[f"k{k}_image"], out[f"k{k}_trimap"] = img, tri
        out[f"k{k}_b"] = b
        out[f"k{k}_A_data"] = A.data
        out[f"k{k}_A_indices"] = A.indices.astype(np.int64)
        out[f"k{k}_A_indptr"] = A.indptr.astype(np.int64)
        out[f"k{k}_v"] = v
        out[f"k{k}_vcycle_v"] = pm.vcycle(A, (h, w))(v)
        out[f"k{k}_vcycle_v_2_3"] = pm.vcycle(A, (h, w), num_pre_iter=2,
                                              num_post_iter=3, omega=0.7)(v)
        for name, fac in [("none", lambda A: None), ("jacobi", pm.jacobi),
                          ("vcycle", lambda A: pm.vcycle(A, (h, w))),
                          ("ichol", pm.ichol)]:
            cb = pm.CounterCallback()
            x = pm.cg(A, b, M=fac(A), rtol=1e-7, callback=cb)
            out[f"k{k}_x_{name}"] = x
            out[f"k{k}_it_{name}"] = np.array([cb.n])
    out["count"] = np.array([2])
    np.savez_compressed(os.path.join(HERE, "soft_small.npz"), **out)


def gen_lemur(pm, root):
    """The reference tests' lemur inputs and the values they pin."""
    cwd = os.getcwd()
    os.chdir(root)
    try:
        out = {}
        image = pm.load_image("data/lemur/lemur.png", "rgb", 0.125, "bilinear")
        trimap = pm.load_image("data/lemur/lemur_trimap.png", "gray", 0.125, "nearest")
        out["s0125_image"], out["s0125_trimap"] = image, trimap
        A, b = pm.make_linear_system(pm.cf_laplacian(image), trimap)
        for name, fac in [("none", lambda A: None), ("jacobi", pm.jacobi),
                          ("icholt", lambda A: pm.ichol(A, max_nnz=500000)),
                          ("vcycle", lambda A: pm.vcycle(A, trimap.shape))]:
            cb = pm.CounterCallback()
            x = pm.cg(A, b, M=fac(A), atol=1e-6, rtol=0, maxiter=10000, callback=cb)
            out[f"s0125_it_{name}"] = np.array([cb.n])
            out[f"s0125_x_{name}"] = x

        image = pm.load_image("data/lemur/lemur.png", "rgb", 0.1, "bilinear")
        trimap = pm.load_image("data/lemur/lemur_trimap.png", "gray", 0.1, "nearest")
        good = pm.load_image("data/lemur/lemur_alpha_fba.png", "gray", 0.1, "bilinear")
        out["s01_image"], out["s01_trimap"], out["s01_good"] = image, trimap, good
        out["s01_alpha_cf"] = pm.estimate_alpha_cf(image, trimap)
        A, b = pm.make_linear_system(pm.cf_laplacian(image), trimap)
        import scipy.sparse.linalg
        out["s01_x_soft_direct"] = scipy.sparse.linalg.spsolve(A, b)
        np.savez_compressed(os.path.join(HERE, "lemur.npz"), **out)
    finally:
        os.chdir(cwd)


def gen_lkm(pm, root, rng):
    """lkm_laplacian on small random images (L p and diag_L), and the
    reference test's lemur comparison of the LKM and CF solves
    (tests/test_lkm.py), plus estimate_alpha_lkm on that image."""
    out = {}
    for name, (h, w, r) in {"a": (29, 37, 2), "b": (41, 53, 4), "c": (47, 45, 10)}.items():
        img = rng.random((h, w, 3))
        p = rng.standard_normal(h * w)
        L, diag = pm.lkm_laplacian(img, epsilon=1e-7, radius=r)
        out[f"{name}_image"], out[f"{name}_p"] = img, p
        out[f"{name}_Lp"], out[f"{name}_diag"] = L(p), diag
        out[f"{name}_radius"] = np.array([r])
    cwd = os.getcwd()
    os.chdir(root)
    try:
        image = pm.load_image("data/lemur/lemur.png", "rgb", 0.125, "bilinear")
        trimap = pm.load_image("data/lemur/lemur_trimap.png", "gray", 0.125, "nearest")
    finally:
        os.chdir(cwd)
    L_lkm, diag_lkm = pm.lkm_laplacian(image, epsilon=1e-7, radius=2)
    A_cf, b, c = pm.make_linear_system(pm.cf_laplacian(image, epsilon=1e-7, radius=2), trimap,
                                       return_c=True)
    inv = 1.0 / (diag_lkm + c)
    cb_l, cb_c = pm.CounterCallback(), pm.CounterCallback()
    out["lemur_x_lkm"] = pm.cg(lambda x: L_lkm(x) + c * x, b, M=lambda r: inv * r, callback=cb_l)
    out["lemur_x_cf"] = pm.cg(A_cf, b, M=pm.jacobi(A_cf), callback=cb_c)
    out["lemur_it_lkm"], out["lemur_it_cf"] = np.array([cb_l.n]), np.array([cb_c.n])
    out["lemur_alpha_lkm"] = pm.estimate_alpha_lkm(image, trimap)
    np.savez_compressed(os.path.join(HERE, "lkm_small.npz"), **out)


def gen_c1(pm):
    """estimate_alpha_cf on the 320x240 synthetic workload (default ichol)."""
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _, frac = make_matting_problem(240, 320, 1, sigma=2.0, band=7,
                                             unknown_fraction=0.12)
    alpha = pm.estimate_alpha_cf(img, tri)
    unknown = (tri > 0.1) & (tri < 0.9)
    np.savez_compressed(os.path.join(HERE, "synthetic_320x240.npz"),
                        image_sum=np.array([img.sum(), tri.sum()]),
                        alpha_unknown=alpha[unknown], frac=np.array([frac]))


def gen_alpha_r2(pm):
    """estimate_alpha_cf with laplacian_kwargs={"radius": 2} (default ichol),
    on the 48x64 synthetic image of the device test of that option."""
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _, _ = make_matting_problem(48, 64, 9, sigma=2.0, band=4, unknown_fraction=0.2)
    alpha = pm.estimate_alpha_cf(img, tri, laplacian_kwargs={"radius": 2})
    np.savez_compressed(os.path.join(HERE, "alpha_cf_radius2.npz"),
                        image_sum=np.array([img.sum(), tri.sum()]), alpha=alpha)


def _fg_case(rng, h, w, depth=3, kind="random"):
    img = rng.random((h, w, depth)).astype(np.float32)
    if kind == "random":
        alpha = np.clip(rng.random((h, w)) * 1.4 - 0.2, 0.0, 1.0)
    elif kind == "mostly_bg":
        # alpha 0 almost everywhere: F there keeps the seed colour, which pins
        # the seed computation
        alpha = np.zeros((h, w))
        alpha[h // 3: h // 3 + 2, w // 2: w // 2 + 3] = 1.0
    else:  # "mostly_fg"
        alpha = np.ones((h, w))
        alpha[: 2, : 3] = 0.0
        alpha[h // 2, w // 2] = 0.5
    return img, alpha.astype(np.float32)


def gen_foreground(pm, root, rng):
    """estimate_foreground_ml on small float32 inputs with several parameter
    sets and depths, and the reference test's lemur case
    (tests/test_foreground.py: scale 0.1, box resize, mse <= 0.022)."""
    from pymatting.foreground.estimate_foreground_ml import estimate_foreground_ml
    cases = [
        ((1, 2), {}, 3, "random"), ((2, 1), {}, 3, "random"), ((1, 7), {}, 3, "random"),
        ((7, 9), {}, 3, "random"), ((33, 17), {}, 3, "random"), ((40, 65), {}, 3, "random"),
        ((64, 64), {}, 3, "random"), ((100, 37), {}, 3, "random"),
        ((45, 70), dict(regularization=1e-3, gradient_weight=0.5, n_small_iterations=3,
                        n_big_iterations=4, small_size=16), 3, "random"),
        ((29, 31), dict(n_big_iterations=0), 3, "random"),
        ((50, 20), dict(n_small_iterations=0, n_big_iterations=1), 3, "random"),
        ((24, 36), {}, 1, "random"), ((37, 23), {}, 4, "random"),
        ((16, 16), {}, 3, "mostly_bg"), ((21, 18), {}, 3, "mostly_fg"),
    ]
    out = {"n_cases": np.array([len(cases)])}
    for i, ((h, w), kw, depth, kind) in enumerate(cases):
        img, alpha = _fg_case(rng, h, w, depth, kind)
        F, B = estimate_foreground_ml(img, alpha, return_background=True, **kw)
        out[f"c{i}_image"], out[f"c{i}_alpha"] = img, alpha
        out[f"c{i}_F"], out[f"c{i}_B"] = F, B
        out[f"c{i}_params"] = np.array([kw.get("regularization", 1e-5),
                                        kw.get("n_small_iterations", 10),
                                        kw.get("n_big_iterations", 2),
                                        kw.get("small_size", 32),
                                        kw.get("gradient_weight", 1.0)])
    cwd = os.getcwd()
    os.chdir(root)
    try:
        image = pm.load_image("data/lemur/lemur.png", "RGB", 0.1, "box")
        trimap = pm.load_image("data/lemur/lemur_trimap.png", "GRAY", 0.1, "nearest")
        alpha = pm.load_image("data/lemur/lemur_alpha.png", "GRAY", 0.1, "box")
        expected = pm.load_image("data/lemur/lemur_foreground.png", "RGB", 0.1, "box")
    finally:
        os.chdir(cwd)
    F, B = estimate_foreground_ml(image, alpha, return_background=True)
    Fc, Bc = pm.estimate_foreground_cf(image, alpha, return_background=True)
    out["lemur_F_cf"], out["lemur_B_cf"] = Fc, Bc
    # the system matrix of estimate_foreground_cf on a small image
    import scipy.sparse
    rs = np.random.default_rng(12)
    a_small = np.clip(rs.random((5, 7)) * 1.4 - 0.2, 0.0, 1.0)
    n_s = a_small.size
    S = None
    for dx, dy in [(-1, 0), (1, 0), (0, -1), (0, 1)]:
        from pymatting.util.util import sparse_conv_matrix_with_offsets
        D = sparse_conv_matrix_with_offsets(7, 5, [1.0, -1.0], [0, dx], [0, dy])
        S2 = D.T.dot(scipy.sparse.diags(1e-5 + np.abs(D.dot(a_small.ravel())))).dot(D)
        S = S2 if S is None else S + S2
    V = scipy.sparse.bmat([[S, None], [None, S]])
    a_f = a_small.ravel()
    U = scipy.sparse.bmat([[scipy.sparse.diags(a_f), scipy.sparse.diags(1 - a_f)]])
    A = (U.T.dot(U) + V).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    out["cf_small_alpha"] = a_small
    out["cf_small_indptr"], out["cf_small_indices"] = A.indptr.astype(np.int64), A.indices.astype(np.int64)
    out["cf_small_data"] = A.data
    out["lemur_image"], out["lemur_alpha"], out["lemur_trimap"] = image, alpha, trimap
    out["lemur_expected"], out["lemur_F"], out["lemur_B"] = expected, F, B
    np.savez_compressed(os.path.join(HERE, "foreground_small.npz"), **out)


def gen_cutout(pm, root):
    """The reference's cutout test (tests/test_simple_api.py): its input
    files as uint8 arrays, the files it compares against, and the cutout the
    reference itself writes for them (read back with its load_image)."""
    import tempfile
    from PIL import Image
    out = {}
    d = os.path.join(root, "data", "test")
    for name in ["test", "test_trimap", "test_alpha", "test_foreground"]:
        out[name + "_u8"] = np.array(Image.open(os.path.join(d, name + ".png")))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "cutout.png")
        pm.cutout(os.path.join(d, "test.png"), os.path.join(d, "test_trimap.png"), path)
        out["reference_cutout"] = pm.load_image(path)
        out["reference_cutout_u8"] = np.array(Image.open(path))
    out["true_alpha"] = pm.load_image(os.path.join(d, "test_alpha.png"), "GRAY")
    out["true_foreground"] = pm.load_image(os.path.join(d, "test_foreground.png"), "RGB")
    np.savez_compressed(os.path.join(HERE, "cutout_test.npz"), **out)


def gen_laplacians(pm, root, rng):
    """uniform_laplacian, rw_laplacian and lbdm_laplacian on small random
    images (CSR arrays of the reference's matrices), and the reference
    test's lemur errors
    (tests/test_laplacians.py: spsolve of make_linear_system, error of the
    clipped alpha against the good alpha on unknown pixels)."""
    import scipy.sparse.linalg
    out = {}
    cases = [(1, 1, 1), (1, 5, 1), (4, 1, 1), (2, 2, 1), (7, 9, 1), (16, 13, 1), (12, 17, 2),
             (5, 6, 3)]
    out["n_cases"] = np.array([len(cases)])
    for k, (h, w, r) in enumerate(cases):
        img = rng.random((h, w, 3))
        out[f"c{k}_image"], out[f"c{k}_radius"] = img, np.array([r])
        for name, L in (("uniform", pm.uniform_laplacian(img, radius=r)),
                        ("rw", pm.rw_laplacian(img, radius=r))):
            L = scipy.sparse.csr_matrix(L)
            L.sum_duplicates()
            L.sort_indices()
            out[f"c{k}_{name}_indptr"] = L.indptr.astype(np.int64)
            out[f"c{k}_{name}_indices"] = L.indices.astype(np.int64)
            out[f"c{k}_{name}_data"] = L.data
    cwd = os.getcwd()
    os.chdir(root)
    try:
        image = pm.load_image("data/lemur/lemur.png", "rgb", 0.1, "bilinear")
        trimap = pm.load_image("data/lemur/lemur_trimap.png", "gray", 0.1, "nearest")
        good = pm.load_image("data/lemur/lemur_alpha_fba.png", "gray", 0.1, "bilinear")
    finally:
        os.chdir(cwd)
    is_unknown = pm.trimap_split(trimap, flatten=False)[3]
    for name, fn in (("uniform", pm.uniform_laplacian), ("rw", pm.rw_laplacian)):
        A, b = pm.make_linear_system(fn(image), trimap)
        x = scipy.sparse.linalg.spsolve(A, b)
        alpha = np.clip(x, 0, 1).reshape(trimap.shape)
        out[f"lemur_{name}_error"] = np.array([np.linalg.norm(np.abs(alpha - good)[is_unknown])])
    A, b = pm.make_linear_system(pm.lbdm_laplacian(image), trimap)
    x = scipy.sparse.linalg.spsolve(A, b)
    alpha = np.clip(x, 0, 1).reshape(trimap.shape)
    out["lemur_lbdm_error"] = np.array([np.linalg.norm(np.abs(alpha - good)[is_unknown])])
    lb = [(3, 3, 1), (2, 6, 1), (5, 7, 1), (12, 9, 1), (7, 8, 2), (9, 11, 2)]
    out["lbdm_n"] = np.array([len(lb)])
    for k, (h, w, r) in enumerate(lb):
        img = rng.random((h, w, 3))
        L = scipy.sparse.csr_matrix(pm.lbdm_laplacian(img, radius=r))
        L.sum_duplicates()
        L.sort_indices()
        out[f"lbdm{k}_image"], out[f"lbdm{k}_radius"] = img, np.array([r])
        out[f"lbdm{k}_indptr"] = L.indptr.astype(np.int64)
        out[f"lbdm{k}_indices"] = L.indices.astype(np.int64)
        out[f"lbdm{k}_data"] = L.data
    A, b = pm.make_linear_system(pm.knn_laplacian(image), trimap)
    x = scipy.sparse.linalg.spsolve(A, b)
    alpha = np.clip(x, 0, 1).reshape(trimap.shape)
    out["lemur_knn_error"] = np.array([np.linalg.norm(np.abs(alpha - good)[is_unknown])])
    kc = [((6, 7), "binary"), ((9, 8), "soft"), ((13, 17), "binary"), ((20, 15), "soft")]
    out["knn_n"] = np.array([len(kc)])
    for k, ((h, w), kern) in enumerate(kc):
        img = rng.random((h, w, 3))
        L = scipy.sparse.csr_matrix(pm.knn_laplacian(img, kernel=kern))
        L.sum_duplicates()
        L.sort_indices()
        out[f"knn{k}_image"], out[f"knn{k}_soft"] = img, np.array([kern == "soft"])
        out[f"knn{k}_indptr"] = L.indptr.astype(np.int64)
        out[f"knn{k}_indices"] = L.indices.astype(np.int64)
        out[f"knn{k}_data"] = L.data
    L = scipy.sparse.csr_matrix(pm.knn_laplacian(image))
    L.sum_duplicates()
    L.sort_indices()
    out["lemur_knn_indptr"], out["lemur_knn_indices"] = L.indptr.astype(np.int64), L.indices.astype(np.int64)
    out["lemur_knn_data"] = L.data
    for name, fn in (("knn", pm.estimate_alpha_knn), ("lbdm", pm.estimate_alpha_lbdm),
                     ("rw", pm.estimate_alpha_rw)):
        out[f"lemur_alpha_{name}"] = fn(image, trimap)
    out["lemur_image"], out["lemur_trimap"], out["lemur_good"] = image, trimap, good
    np.savez_compressed(os.path.join(HERE, "laplacians_small.npz"), **out)


def gen_layout(pm):
    """reference_layout.json: for every loaded pymatting module, which of its
    attributes are bound to a function the integration replaces, named by
    (defining module, name). Pins the re-export structure the integration
    stub has to rebind."""
    import json
    from pymatting_b200.integration import HOT_PATH, NEXT_ROWS
    targets = {}
    for mod, name in HOT_PATH + NEXT_ROWS:
        m = sys.modules.get(mod)
        if m is not None and hasattr(m, name):
            targets[id(getattr(m, name))] = [mod, name]
    layout = {}
    for mname in sorted(k for k in sys.modules if k == "pymatting" or k.startswith("pymatting.")):
        m = sys.modules[mname]
        if m is None:
            continue
        hits = {attr: targets[id(v)] for attr, v in vars(m).items() if id(v) in targets}
        if hits:
            layout[mname] = hits
    with open(os.path.join(HERE, "reference_layout.json"), "w") as f:
        json.dump(layout, f, indent=1, sort_keys=True)


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <pymatting source tree> [fixture names]")
    root = sys.argv[1]
    pm = import_reference(root)
    rng = np.random.default_rng(2024)
    only = sys.argv[2:]
    for name, fn in [("cf", lambda: gen_cf(pm, rng)), ("cg", lambda: gen_cg(pm)),
                     ("ichol", lambda: gen_ichol(pm, rng)), ("soft", lambda: gen_soft(pm)),
                     ("lemur", lambda: gen_lemur(pm, root)), ("c1", lambda: gen_c1(pm)),
                     ("alpha_r2", lambda: gen_alpha_r2(pm)),
                     ("lkm", lambda: gen_lkm(pm, root, np.random.default_rng(77))),
                     ("foreground", lambda: gen_foreground(pm, root, np.random.default_rng(91))),
                     ("cutout", lambda: gen_cutout(pm, root)),
                     ("laplacians", lambda: gen_laplacians(pm, root, np.random.default_rng(5))),
                     ("layout", lambda: gen_layout(pm))]:
        if not only or name in only:
            fn()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
