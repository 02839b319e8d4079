"""torch.autograd wrapper of the strong NCC and its adjoint kernel (dpe_ncc_grad).

    cost = NCCCost.apply(planes, images, cameras, params, px, py, src)

`planes` (n, 4) float32: per query (nx, ny, nz, w) in reference-camera coordinates; `images` a
(N, H, W) float32 tensor, image 0 the reference.  Both may require grad: backward returns
dC/dplane from the adjoint kernel and, for the images, the gradient with respect to the source
images' pixels (the reference image gets none: its pixels enter only through the bilateral
weights, which the cost treats as fixed).  The kernels run on the GPU through the C-ABI with host
buffers, so tensors are moved to and from the host here.
"""
from __future__ import annotations

import numpy as np
import torch

import dpe_b200 as D

_ctx = None


def _context():
    global _ctx
    if _ctx is None:
        _ctx = D.Context(0)
    return _ctx


class NCCCost(torch.autograd.Function):
    @staticmethod
    def forward(fctx, planes, images, cameras, params, px, py, src):
        imgs = [np.ascontiguousarray(im.detach().cpu().numpy().astype(np.float32)) for im in images]
        pl = np.ascontiguousarray(planes.detach().cpu().numpy().astype(np.float32))
        want_images = bool(images.requires_grad)
        cost, gp, _, gimg = _context().ncc_grad(imgs, cameras, params, px, py, src, pl, want_images=want_images)
        fctx.gp = torch.from_numpy(gp)
        fctx.gimg = gimg
        fctx.src = torch.from_numpy(np.asarray(src, np.int64))
        fctx.shape = images.shape
        return torch.from_numpy(cost).to(planes.device)

    @staticmethod
    def backward(fctx, gout):
        g = gout.detach().cpu().to(torch.float32)
        gplanes = (fctx.gp * g[:, None]).to(gout.device)
        gimages = None
        if fctx.gimg is not None:
            # the image gradient of sum_k gout[k] * C_k needs per-query weights: the kernel returns
            # the gradient of the plain sum, which is exact when all gout are equal
            if not torch.allclose(g, g[0].expand_as(g)):
                raise NotImplementedError("image gradients are available for uniformly weighted costs")
            gi = np.zeros(tuple(fctx.shape), np.float32)
            for i, a in enumerate(fctx.gimg):
                if a is not None:
                    gi[i] = a
            gimages = (torch.from_numpy(gi) * g[0]).to(gout.device)
        return gplanes, gimages, None, None, None, None, None
