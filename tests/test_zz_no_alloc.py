"""dpe_ncc_eval_noalloc, the NCC query entry point for callers that may not allocate device memory
(its scratch is a static device array), against dpe_ncc_eval on the same queries.  Collected last,
so that it also runs after every other GPU test in the same process; it passes alone as well."""
import ctypes as C

import numpy as np
import pytest

import dpe_b200 as D
import helpers as h
from test_oracle import _random_queries

pytestmark = pytest.mark.gpu

NCC_TOL = 1e-4  # absolute, the tolerance of the NCC parity tests


def _device_inputs(scene):
    import torch

    images = [np.ascontiguousarray(g.astype(np.float32)) for g in scene.gray]
    cams = [h.S.camera_struct(scene, i) for i in range(scene.n)]
    return images, cams, [torch.from_numpy(im).cuda() for im in images]


def _to_device(px, py, src, planes):
    import torch

    return (torch.from_numpy(np.ascontiguousarray(px, np.int32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(py, np.int32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(src, np.int32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(planes, np.float32)).cuda())


def test_noalloc_matches_ncc_eval_on_consecutive_calls(ctx, small_scene):
    import torch

    images, cams, d_images = _device_inputs(small_scene)
    p = D.default_params()
    rng = np.random.default_rng(31)
    batches = [_random_queries(small_scene, 6000, rng), _random_queries(small_scene, 6000, rng, near_gt=False)]
    outs = []
    for px, py, src, planes in batches:  # two calls in a row, different queries
        q = _to_device(px, py, src, planes)
        out = torch.full((len(px),), -7.0, dtype=torch.float32, device="cuda")
        D.ncc_eval_noalloc(d_images, cams, p, *q, out)
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    for (px, py, src, planes), got in zip(batches, outs):
        want = ctx.ncc_eval(images, cams, p, px, py, src, planes)
        err = np.abs(got.astype(np.float64) - want.astype(np.float64))
        print(f"noalloc vs dpe_ncc_eval: max |diff| {err.max():.3e}")
        assert np.isfinite(got).all()
        assert err.max() <= NCC_TOL
    # the same queries again give the same costs: nothing left over from the previous call matters
    px, py, src, planes = batches[0]
    again = torch.empty(len(px), dtype=torch.float32, device="cuda")
    D.ncc_eval_noalloc(d_images, cams, p, *_to_device(px, py, src, planes), again)
    torch.cuda.synchronize()
    assert np.array_equal(again.cpu().numpy(), outs[0])


def test_noalloc_out_of_range_queries_get_nan(small_scene):
    import torch

    _, cams, d_images = _device_inputs(small_scene)
    p = D.default_params()
    W, H = small_scene.spec.width, small_scene.spec.height
    px = np.array([0, W, 3, -1, 5], np.int32)
    py = np.array([0, 2, H, 4, 5], np.int32)
    src = np.array([1, 1, 1, 1, small_scene.n], np.int32)
    planes = np.tile(np.array([0, 0, -1, 5], np.float32), (5, 1))
    out = torch.zeros(5, dtype=torch.float32, device="cuda")
    D.ncc_eval_noalloc(d_images, cams, p, *_to_device(px, py, src, planes), out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.isfinite(got[0])
    assert np.isnan(got[1:]).all()


def test_noalloc_rejects_problems_beyond_the_static_scratch(small_scene):
    import torch

    lib = D.load_library()
    _, cams, d_images = _device_inputs(small_scene)
    q = D.NCCQuery()
    q.width, q.height, q.num_images = 1600, 1200, 3  # 3 x 1602 x 1202 x 4 B > 16 MiB
    for i in range(3):
        q.images[i] = d_images[0].data_ptr()  # never read: the size check comes first
        q.cameras[i] = D.make_camera(cams[i])
    q.params = D.default_params()
    px, py, src, planes = _to_device([0], [0], [1], np.zeros((1, 4), np.float32))
    out = torch.zeros(1, dtype=torch.float32, device="cuda")
    q.count = 1
    q.px, q.py, q.src, q.plane = px.data_ptr(), py.data_ptr(), src.data_ptr(), planes.data_ptr()
    st = lib.dpe_ncc_eval_noalloc(C.byref(q), C.c_void_p(out.data_ptr()), None)
    assert st == D.ERR_CAPACITY
    msg = lib.dpe_last_error().decode()
    print(msg)
    assert "16777216" in msg and "dpe_ncc_eval_noalloc" in msg
