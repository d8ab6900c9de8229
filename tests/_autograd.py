"""torch.autograd wrapper of P2M for checking the adjoint (test harness only).

forward: the unique-node field P2M(x, w) of ppm_interp_p2m (3D, periodic, one
subdomain) on CUDA tensors through the device entry point;
backward: ppm_interp_p2m_adjoint with the incoming gradient as the residual,
giving dL/dw = M2P(grad) and dL/dx from the kernel-derivative weights.
"""
from __future__ import annotations

import torch

import ppm_legacy_b200 as ppmg


def colmajor_copy(a):
    """A column-major (Fortran-order) copy of a torch tensor."""
    return a.detach().permute(*reversed(range(a.dim()))).contiguous().permute(
        *reversed(range(a.dim())))


class P2M(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xp, w, topo_id, mesh_id, nc, kernel=2):
        xc, wc = colmajor_copy(xp), colmajor_copy(w)
        lda, n = wc.shape
        g = [2, 2, 2]
        ext = nc + 1 + 2 * g[0]
        field = torch.zeros((1, ext, ext, ext, lda), dtype=xp.dtype,
                            device=xp.device).permute(4, 3, 2, 1, 0)
        info = ppmg.ppm_interp_p2m(xc, n, wc, lda, topo_id, mesh_id, kernel, g, field)
        if info != 0 or ppmg.sync_status(topo_id, mesh_id) != 0:
            raise RuntimeError(f"ppm_interp_p2m failed: {ppmg.last_error()}")
        ctx.save_for_backward(xc, wc)
        ctx.cfg = (topo_id, mesh_id, nc, kernel)
        return field[:, g[0]:g[0] + nc, g[1]:g[1] + nc, g[2]:g[2] + nc, 0].contiguous()

    @staticmethod
    def backward(ctx, grad):
        xc, wc = ctx.saved_tensors
        topo_id, mesh_id, nc, kernel = ctx.cfg
        lda, n = wc.shape
        r = colmajor_copy(grad.reshape(lda, nc, nc, nc, 1))
        dw = colmajor_copy(torch.empty_like(wc))
        dx = colmajor_copy(torch.empty((3, n), dtype=xc.dtype, device=xc.device))
        info = ppmg.ppm_interp_p2m_adjoint(xc, n, wc, lda, topo_id, mesh_id, kernel, r, dw, dx,
                                           field_lb=[1, 1, 1])
        if info != 0 or ppmg.sync_status(topo_id, mesh_id) != 0:
            raise RuntimeError(f"ppm_interp_p2m_adjoint failed: {ppmg.last_error()}")
        return dx, dw, None, None, None, None
