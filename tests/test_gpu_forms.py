"""The precision and differentiation forms of the PatchMatch path (dpe_options).

Staging: source images stored as FP16 or BF16 pairs.  8-bit images are exact in both, so a call
on them computes the FP32 call's arithmetic (bit for bit in the exact build, test_gpu_exact.py).  On an interpolated pyramid level (non-integer
intensities) the staged costs differ by the rounding of the source texels: FP16 (11-bit
significand) keeps >= 98 % of the depths within 0.1 % of the FP32 run; BF16 (8-bit significand,
steps of 0.5-1 grey level at these intensities) moves many low-contrast decisions, so its bar is
accuracy against the ground truth no worse than FP32's by more than 2 points.

Gauss-Newton: the extra plane hypothesis from the NCC adjoint is kept only when it lowers the
pixel's cost.  The runs then propagate different planes, so the final maps are compared
statistically: mean cost no higher than the plain run's by more than 0.01, and depth accuracy
against ground truth no worse by more than 0.5 percentage points.
"""
import numpy as np
import pytest

import dpe_b200 as D
import helpers as h

pytestmark = pytest.mark.gpu


def _run(ctx, images, cams, p, seed, staging=D.STAGE_FP32, gn=0):
    ctx.set_options(staging=staging, gn_refine=gn)
    try:
        return ctx.pm_run(images, cams, p, seed=seed)
    finally:
        ctx.set_options()


@pytest.mark.parametrize("staging", [D.STAGE_FP16, D.STAGE_BF16])
def test_staging_on_8bit_images(ctx, small_scene, staging):
    """The staged texels equal the FP32 ones; each staging is its own kernel instance, and with
    multiply-add contraction the instances may round differently, so the default build is held
    to the parity bar here (test_gpu_exact.py holds the exact build to identical bits)."""
    images, cams, _ = h.view_inputs(small_scene, 1)
    p = h.first_init_params(small_scene, len(images))
    ref = _run(ctx, images, cams, p, 31)
    got = _run(ctx, images, cams, p, 31, staging=staging)
    assert h.rel_depth_agreement(got["plane"][..., 3], ref["plane"][..., 3], 1e-3) >= 0.995


@pytest.mark.parametrize("staging", [D.STAGE_FP16, D.STAGE_BF16])
def test_staging_on_interpolated_images(ctx, small_scene, staging):
    import cv2

    images, cams, srcs = h.view_inputs(small_scene, 1)
    H, W = images[0].shape
    w2, h2 = W // 2, H // 2
    small = [np.ascontiguousarray(cv2.resize(im, (w2, h2), interpolation=cv2.INTER_LINEAR)) for im in images]
    assert any(not np.array_equal(s, np.round(s)) for s in small)  # non-integer intensities
    cams2 = [h.S.camera_struct(small_scene, i, w2, h2) for i in [1] + list(srcs)]
    p = h.first_init_params(small_scene, len(images))
    ref = _run(ctx, small, cams2, p, 32)
    got = _run(ctx, small, cams2, p, 32, staging=staging)
    agree = h.rel_depth_agreement(got["plane"][..., 3], ref["plane"][..., 3], 1e-3)
    gt = cv2.resize(small_scene.depth[1].astype(np.float32), (w2, h2), interpolation=cv2.INTER_NEAREST)
    acc = lambda o: float((np.abs(o["plane"][..., 3] - gt) / gt < 0.01).mean())
    print(f"staging {staging} on interpolated images: depth agreement with FP32 {agree:.4f}; within 1% of GT "
          f"FP32 {acc(ref):.4f} staged {acc(got):.4f}")
    if staging == D.STAGE_FP16:
        assert agree >= 0.98  # 11-bit significand: the rounding rarely changes a decision
    assert acc(got) >= acc(ref) - 0.02


def test_gauss_newton_refinement(ctx, small_scene):
    images, cams, _ = h.view_inputs(small_scene, 2)
    p = h.first_init_params(small_scene, len(images))
    plain = _run(ctx, images, cams, p, 33)
    gn = _run(ctx, images, cams, p, 33, gn=1)
    gt = small_scene.depth[2]
    acc = lambda o: float((np.abs(o["plane"][..., 3] - gt) / gt < 0.01).mean())
    cp, cg = plain["costs"], gn["costs"]
    ok = np.isfinite(cp) & np.isfinite(cg)
    print(f"Gauss-Newton: within 1% of GT plain {acc(plain):.4f} gn {acc(gn):.4f}; "
          f"mean cost plain {cp[ok].mean():.4f} gn {cg[ok].mean():.4f}")
    assert acc(gn) >= acc(plain) - 0.005
    assert cg[ok].mean() <= cp[ok].mean() + 0.01
