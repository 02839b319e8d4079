"""torch.autograd wrappers of the strong NCC and its adjoint kernel (dpe_ncc_grad_device).

    cost = NCCCost.apply(planes, images, cameras, params, px, py, src)
    cost = ncc_cost_depth_normal(depth, normal, images, cameras, params, px, py, src)

`planes` (n, 4) float32 CUDA tensor: per query (nx, ny, nz, w) in reference-camera coordinates;
`images` a (N, H, W) float32 CUDA tensor, image 0 the reference; px, py, src (n,) int32 CUDA
tensors.  Every tensor stays on the device: the kernels read and write them in place on torch's
current stream.  Backward returns dC/dplane from the adjoint kernel and, for the images, the
gradient of sum_k gout[k] * C_k with respect to the source images' pixels, by one more adjoint pass
that recomputes the windows and weights each query's scatter by its gout[k] (the reference image
gets none: its pixels enter only through the bilateral weights, which the cost treats as fixed).

ncc_cost_depth_normal takes the hypothesis as the reference keeps it per pixel -- a depth and a
unit normal in reference-camera coordinates -- and builds the plane distance w = -depth * n . ray,
ray = Kr^-1 (x, y, 1), with torch operations, so autograd carries the adjoint to d(NCC)/d(depth,
normal).
"""
from __future__ import annotations

import ctypes as C

import torch

import dpe_b200 as D

_ctx = None


def _context():
    global _ctx
    if _ctx is None:
        _ctx = D.Context(torch.cuda.current_device())
    return _ctx


def _query(images, cameras, params, px, py, src, planes):
    q = D.NCCQuery()
    n_img, H, W = images.shape
    q.height, q.width, q.num_images = int(H), int(W), int(n_img)
    for i in range(n_img):
        q.images[i] = images[i].data_ptr()
        q.cameras[i] = D.make_camera(cameras[i])
    q.params = params
    q.count = int(px.numel())
    q.px, q.py, q.src, q.plane = px.data_ptr(), py.data_ptr(), src.data_ptr(), planes.data_ptr()
    return q


def _grad_device(images, cameras, params, px, py, src, planes, upstream=None, want_plane=True, want_images=False):
    for t, dt in ((images, torch.float32), (planes, torch.float32), (px, torch.int32), (py, torch.int32),
                  (src, torch.int32)):
        if not (t.is_cuda and t.dtype == dt):
            raise ValueError("images/planes float32 and px/py/src int32, all CUDA tensors")
    images, planes = images.contiguous(), planes.contiguous()
    px, py, src = px.contiguous(), py.contiguous(), src.contiguous()
    n = px.numel()
    if planes.shape != (n, 4) or py.numel() != n or src.numel() != n or images.dim() != 3:
        raise ValueError("planes (n, 4), px / py / src (n,), images (N, H, W)")
    dev = images.device
    cost = torch.empty(n, dtype=torch.float32, device=dev)
    gp = torch.empty((n, 4), dtype=torch.float32, device=dev) if want_plane else None
    gi = torch.empty((images.shape[0] - 1,) + tuple(images.shape[1:]), dtype=torch.float32, device=dev) \
        if want_images else None
    up = upstream.to(torch.float32).contiguous() if upstream is not None else None
    q = _query(images, cameras, params, px, py, src, planes)
    ctx = _context()
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = ctx.lib.dpe_ncc_grad_device(ctx.handle, C.byref(q), up.data_ptr() if up is not None else None,
                                     cost.data_ptr(), gp.data_ptr() if gp is not None else None, None,
                                     gi.data_ptr() if gi is not None else None, C.c_void_p(stream))
    if st != D.OK:
        raise D.DPEError(st, "dpe_ncc_grad_device")
    return cost, gp, gi


class NCCCost(torch.autograd.Function):
    @staticmethod
    def forward(fctx, planes, images, cameras, params, px, py, src):
        cost, gp, _ = _grad_device(images.detach(), cameras, params, px, py, src, planes.detach(),
                                   want_plane=planes.requires_grad)
        fctx.save_for_backward(images.detach(), planes.detach(), px, py, src)
        fctx.gp = gp
        fctx.cameras, fctx.params = cameras, params
        fctx.want_images = images.requires_grad
        return cost

    @staticmethod
    def backward(fctx, gout):
        images, planes, px, py, src = fctx.saved_tensors
        gout = gout.to(torch.float32).contiguous()
        gplanes = fctx.gp * gout[:, None] if fctx.gp is not None else None
        gimages = None
        if fctx.want_images:
            _, _, gi = _grad_device(images, fctx.cameras, fctx.params, px, py, src, planes, upstream=gout,
                                    want_plane=False, want_images=True)
            gimages = torch.cat([torch.zeros_like(images[:1]), gi], 0)
        return gplanes, gimages, None, None, None, None, None


def planes_from_depth_normal(depth, normal, camera, px, py):
    """(n, 4) planes (n, w) with w = -depth * n . Kr^-1 (x, y, 1) (DPE.cu:341-346), in torch ops."""
    K = torch.as_tensor(camera["K"], dtype=torch.float32, device=depth.device).reshape(3, 3)
    rx = (px.to(torch.float32) - K[0, 2]) / K[0, 0]
    ry = (py.to(torch.float32) - K[1, 2]) / K[1, 1]
    w = -depth * (normal[:, 0] * rx + normal[:, 1] * ry + normal[:, 2])
    return torch.cat([normal, w[:, None]], 1)


def ncc_cost_depth_normal(depth, normal, images, cameras, params, px, py, src):
    """The strong NCC of hypotheses given as (depth, normal); differentiable in both."""
    return NCCCost.apply(planes_from_depth_normal(depth, normal, cameras[0], px, py), images, cameras, params,
                         px, py, src)
