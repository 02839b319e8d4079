"""The strong-NCC adjoint kernel (dpe_ncc_grad) against the FP64 oracle gradient and against
finite differences of the forward kernel, and its torch.autograd wrapper.

Checks, at 10,000 random (pixel, hypothesis, source) triples on the 160x120 scene:
  * plane gradient vs the FP64 forward-mode gradient of the oracle: relative error (max component
    over the gradient's largest component) <= 1e-3 on >= 99 % of the differentiable queries;
  * central finite differences of the GPU forward (step 1e-3 relative per plane component) agree
    with the adjoint as often as FP64 differences of the oracle agree with the exact FP64 gradient
    (the step crosses texel boundaries of the bilinear samples for some queries);
  * the source-image gradient of the summed cost vs the oracle's FP64 image gradient: relative L2
    error <= 1e-3.
"""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
import oracle_py as O
from test_oracle import _random_queries

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grad_inputs(small_scene):
    images = [np.ascontiguousarray(g.astype(np.float32)) for g in small_scene.gray]
    cams = [h.S.camera_struct(small_scene, i) for i in range(small_scene.n)]
    rng = np.random.default_rng(404)
    a = _random_queries(small_scene, 7000, rng)
    b = _random_queries(small_scene, 3000, rng, near_gt=False)
    q = tuple(np.concatenate([x, y]) for x, y in zip(a, b))
    return images, cams, D.default_params(), q


def _rel(a, b):
    scale = np.maximum(np.abs(b).max(axis=1), 1e-6)
    return np.abs(a - b).max(axis=1) / scale


def test_plane_gradient_matches_fp64(ctx, grad_inputs):
    images, cams, p, (px, py, src, planes) = grad_inputs
    cost, gp, gd, _ = ctx.ncc_grad(images, cams, p, px, py, src, planes)
    c64, g64, _ = O.ncc_strong_grad(images, cams, p, px, py, src, planes)
    assert np.abs(cost - c64).max() <= 1e-4
    live = (c64 > 0.01) & (c64 < 1.99) & (np.abs(g64).max(axis=1) > 0)
    rel = _rel(gp[live].astype(np.float64), g64[live])
    print(f"plane gradient vs FP64: {live.sum()} queries, median rel {np.median(rel):.2e}, "
          f"99% {np.quantile(rel, 0.99):.2e}")
    assert live.sum() > 5000
    assert (rel <= 1e-3).mean() >= 0.99
    # flat queries have zero gradient
    assert np.all(gp[c64 >= 2.0] == 0)


def test_plane_gradient_matches_finite_differences(ctx, grad_inputs):
    """Central differences with a 1e-3 relative step cross texel boundaries for some taps (the
    bilinear sample is only piecewise linear), so they disagree with any exact gradient on a
    share of the queries; FP32 differences add rounding noise on top.  The bar: the FP32 adjoint
    agrees with FP32 differences of the GPU forward nearly as often as the exact FP64 gradient
    agrees with FP64 differences of the oracle forward at the same step (within 5 points), and in
    the median within 3x + 5e-3."""
    images, cams, p, (px, py, src, planes) = grad_inputs

    def central(forward):
        fd = np.zeros((len(px), 4), np.float64)
        for i in range(4):
            step = (1e-3 * np.maximum(np.abs(planes[:, i]), 1e-2)).astype(np.float32)
            up, dn = planes.copy(), planes.copy()
            up[:, i] += step
            dn[:, i] -= step
            fd[:, i] = (forward(up) - forward(dn)) / (up[:, i].astype(np.float64) - dn[:, i].astype(np.float64))
        return fd

    cost, gp, _, _ = ctx.ncc_grad(images, cams, p, px, py, src, planes)
    fd32 = central(lambda pl: ctx.ncc_eval(images, cams, p, px, py, src, pl).astype(np.float64))
    c64, g64, _ = O.ncc_strong_grad(images, cams, p, px, py, src, planes)
    fd64 = central(lambda pl: O.ncc_strong(images, cams, p, px, py, src, pl, fp64=True))
    live = (c64 > 0.05) & (c64 < 1.95) & (np.abs(g64).max(axis=1) > 0) & (np.abs(gp).max(axis=1) > 0)
    r32 = _rel(fd32[live], gp[live].astype(np.float64))
    r64 = _rel(fd64[live], g64[live])
    f32, f64 = (r32 <= 5e-2).mean(), (r64 <= 5e-2).mean()
    print(f"finite differences (step 1e-3 rel), {live.sum()} queries: adjoint vs FP32 differences median "
          f"{np.median(r32):.2e}, within 5e-2 {f32:.3f}; exact FP64 gradient vs FP64 differences median "
          f"{np.median(r64):.2e}, within 5e-2 {f64:.3f}")
    assert f32 >= f64 - 0.05
    assert np.median(r32) <= 3 * np.median(r64) + 5e-3


def test_image_gradient_matches_fp64(ctx, grad_inputs):
    images, cams, p, (px, py, src, planes) = grad_inputs
    n = 2000
    q = (px[:n], py[:n], src[:n], planes[:n])
    _, _, _, gimg = ctx.ncc_grad(images, cams, p, *q, want_images=True)
    _, _, g64 = O.ncc_strong_grad(images, cams, p, *q, want_images=True)
    num = sum(np.sum((gimg[i].astype(np.float64) - g64[i]) ** 2) for i in range(1, len(images)))
    den = sum(np.sum(g64[i] ** 2) for i in range(1, len(images)))
    rel = np.sqrt(num / den)
    print(f"image gradient vs FP64: relative L2 {rel:.2e}")
    assert rel <= 1e-3


def _cuda_inputs(images, px, py, src, planes, n):
    import torch

    return (torch.from_numpy(np.stack(images)).cuda(), torch.from_numpy(np.ascontiguousarray(px[:n], np.int32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(py[:n], np.int32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(src[:n], np.int32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(planes[:n], np.float32)).cuda())


def _image_rel(gi, gi64):
    return np.sqrt(sum(np.sum((gi[i] - gi64[i]) ** 2) for i in range(1, len(gi64))) /
                   sum(np.sum(gi64[i] ** 2) for i in range(1, len(gi64))))


def test_autograd_function(grad_inputs):
    """NCCCost on CUDA tensors (no host round trip): plane and image gradients of the summed cost
    against the FP64 oracle."""
    import torch
    import ncc_autograd as AG

    images, cams, p, (px, py, src, planes) = grad_inputs
    n = 500
    imgs, tpx, tpy, tsrc, tpl = _cuda_inputs(images, px, py, src, planes, n)
    pl = tpl.clone().requires_grad_(True)
    imgs = imgs.requires_grad_(True)
    cost = AG.NCCCost.apply(pl, imgs, cams, p, tpx, tpy, tsrc)
    assert cost.is_cuda
    cost.sum().backward()
    assert pl.grad.is_cuda and imgs.grad.is_cuda
    c64, g64, gi64 = O.ncc_strong_grad(images, cams, p, px[:n], py[:n], src[:n], planes[:n], want_images=True)
    live = (c64 > 0.01) & (c64 < 1.99)
    assert (_rel(pl.grad.cpu().numpy()[live].astype(np.float64), g64[live]) <= 1e-3).mean() >= 0.99
    assert float(imgs.grad[0].abs().max()) == 0.0  # the reference image carries no gradient
    assert _image_rel(imgs.grad.cpu().numpy(), gi64) <= 1e-3


def test_autograd_weighted_image_gradient(grad_inputs):
    """Per-query upstream weights: the image gradient of sum_k w_k C_k (two query groups weighted 1
    and -2.5) against the FP64 oracle's gradients of the two groups' sums."""
    import torch
    import ncc_autograd as AG

    images, cams, p, (px, py, src, planes) = grad_inputs
    n = 600
    imgs, tpx, tpy, tsrc, tpl = _cuda_inputs(images, px, py, src, planes, n)
    imgs = imgs.requires_grad_(True)
    w = np.where(np.arange(n) < n // 2, 1.0, -2.5).astype(np.float32)
    cost = AG.NCCCost.apply(tpl, imgs, cams, p, tpx, tpy, tsrc)
    (cost * torch.from_numpy(w).cuda()).sum().backward()
    h = n // 2
    _, _, ga = O.ncc_strong_grad(images, cams, p, px[:h], py[:h], src[:h], planes[:h], want_images=True)
    _, _, gb = O.ncc_strong_grad(images, cams, p, px[h:n], py[h:n], src[h:n], planes[h:n], want_images=True)
    want = [None] + [ga[i] - 2.5 * gb[i] for i in range(1, len(images))]
    rel = _image_rel(imgs.grad.cpu().numpy(), want)
    print(f"weighted image gradient vs FP64: relative L2 {rel:.2e}")
    assert rel <= 1e-3


def test_autograd_depth_normal(ctx, grad_inputs):
    """d(NCC)/d(depth, normal) through autograd (planes built from depth and normal with torch ops)
    equals the kernel's own chain rule (dpe_ncc_grad's grad_depth_normal)."""
    import torch
    import ncc_autograd as AG

    images, cams, p, (px, py, src, planes) = grad_inputs
    n = 400
    imgs, tpx, tpy, tsrc, tpl = _cuda_inputs(images, px, py, src, planes, n)
    K = np.asarray(cams[0]["K"], np.float32).reshape(3, 3)
    ray = np.stack([(px[:n] - K[0, 2]) / K[0, 0], (py[:n] - K[1, 2]) / K[1, 1], np.ones(n)], 1).astype(np.float32)
    depth = (-planes[:n, 3] / np.sum(planes[:n, :3] * ray, 1)).astype(np.float32)
    d = torch.from_numpy(depth).cuda().requires_grad_(True)
    nrm = torch.from_numpy(np.ascontiguousarray(planes[:n, :3])).cuda().requires_grad_(True)
    AG.ncc_cost_depth_normal(d, nrm, imgs, cams, p, tpx, tpy, tsrc).sum().backward()
    c, _, gdn, _ = ctx.ncc_grad(images, cams, p, px[:n], py[:n], src[:n], planes[:n])
    live = (c > 0.01) & (c < 1.99)
    got = np.concatenate([d.grad.cpu().numpy()[:, None], nrm.grad.cpu().numpy()], 1)
    ok = (_rel(got[live].astype(np.float64), gdn[live].astype(np.float64)) <= 1e-2).mean()
    print(f"d/d(depth, normal) through autograd vs the kernel's chain rule: {ok:.4f} within 1e-2")
    assert ok >= 0.98
