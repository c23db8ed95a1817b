"""Gradients of the soft-constraint alpha with respect to the image
(cf_alpha; no reference counterpart): the Laplacian VJP kernel against its
FP64 restatement, the full backward pass against the oracle's direct-solve
adjoint and against central differences of the oracle's forward solve, and
torch's gradcheck."""

import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _problem(h, w, seed):
    from pymatting_b200.synthetic import make_matting_problem
    img, tri, _a, _f = make_matting_problem(h, w, seed, sigma=2.0, band=3, unknown_fraction=0.25)
    return img, tri


def test_vjp_kernel_matches_restatement(gpu):
    import torch
    from pymatting_b200 import _ffi
    rng = np.random.default_rng(7)
    h, w = 37, 53
    img = rng.random((h, w, 3))
    x = rng.standard_normal(h * w)
    mu = rng.standard_normal(h * w)
    t = [torch.as_tensor(a, device=gpu) for a in (img, x, mu)]
    grad = torch.empty((h, w, 3), dtype=torch.float64, device=gpu)
    lib = _ffi.lib()
    rc = lib.pmb_cf_laplacian_vjp(ctypes.c_void_p(t[0].data_ptr()), None, h, w, 1e-7,
                                  ctypes.c_void_p(t[1].data_ptr()), ctypes.c_void_p(t[2].data_ptr()),
                                  ctypes.c_void_p(grad.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.pmb_last_error()
    ref = oracle.cf_laplacian_vjp(img, x, mu, 1e-7)   # d(mu' L x)/dI
    got = grad.cpu().numpy()
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-9 * scale


def test_backward_matches_oracle_adjoint(gpu):
    import torch
    from pymatting_b200.autograd import cf_alpha
    img, tri = _problem(40, 56, 11)
    g = np.random.default_rng(2).standard_normal(tri.shape)
    it = torch.as_tensor(img, device=gpu).requires_grad_(True)
    tt = torch.as_tensor(tri, device=gpu)
    alpha = cf_alpha(it, tt, rtol=1e-12)
    x_ref = oracle.soft_alpha_exact(img, tri)
    assert np.abs(alpha.detach().cpu().numpy().ravel() - x_ref).max() < 1e-9
    (alpha * torch.as_tensor(g, device=gpu)).sum().backward()
    ref = oracle.soft_alpha_grad(img, tri, g)
    got = it.grad.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_backward_matches_finite_differences_200(gpu):
    """Central differences (h = 1e-4) of the oracle's direct solve on 200
    random (pixel, channel) entries, cotangent N(0, 1)."""
    import torch
    from pymatting_b200.autograd import cf_alpha
    img, tri = _problem(48, 48, 5)
    rng = np.random.default_rng(9)
    g = rng.standard_normal(tri.shape)
    it = torch.as_tensor(img, device=gpu).requires_grad_(True)
    alpha = cf_alpha(it, torch.as_tensor(tri, device=gpu), rtol=1e-12)
    (alpha * torch.as_tensor(g, device=gpu)).sum().backward()
    got = it.grad.cpu().numpy()
    gf = g.ravel()
    picks = rng.choice(img.size, size=200, replace=False)
    step = 1e-4
    fd = np.empty(200)
    for n, flat in enumerate(picks):
        e = np.zeros(img.size)
        e[flat] = step
        e = e.reshape(img.shape)
        fp = gf @ oracle.soft_alpha_exact(img + e, tri)
        fm = gf @ oracle.soft_alpha_exact(img - e, tri)
        fd[n] = (fp - fm) / (2 * step)
    an = got.ravel()[picks]
    err = np.abs(an - fd)
    assert err.max() <= 1e-4 * max(1.0, np.abs(fd).max()), (err.max(), np.abs(fd).max())


def test_gradcheck_48(gpu):
    import torch
    from pymatting_b200.autograd import cf_alpha
    img, tri = _problem(48, 48, 3)
    it = torch.as_tensor(img, device=gpu).requires_grad_(True)
    tt = torch.as_tensor(tri, device=gpu)
    assert torch.autograd.gradcheck(lambda i: cf_alpha(i, tt, rtol=1e-13), (it,), eps=1e-6,
                                    atol=1e-5, rtol=1e-3, fast_mode=True)


def test_batched_gradients_equal_single(gpu):
    import torch
    from pymatting_b200.autograd import cf_alpha
    probs = [_problem(32, 40, s) for s in (21, 22, 23)]
    imgs = torch.stack([torch.as_tensor(p[0], device=gpu) for p in probs]).float()
    tris = torch.stack([torch.as_tensor(p[1], device=gpu) for p in probs]).float()
    g = torch.randn(3, 32, 40, device=gpu, generator=torch.Generator(device=gpu).manual_seed(1))
    ib = imgs.clone().requires_grad_(True)
    (cf_alpha(ib, tris) * g).sum().backward()
    for k in range(3):
        ik = imgs[k].clone().requires_grad_(True)
        (cf_alpha(ik, tris[k]) * g[k]).sum().backward()
        assert ik.grad.dtype == torch.float32
        assert torch.allclose(ib.grad[k], ik.grad, rtol=1e-4, atol=1e-6 * ik.grad.abs().max())
