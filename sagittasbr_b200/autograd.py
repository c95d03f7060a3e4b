"""torch.autograd bridge of the sweep: the monostatic RCS sigma [n_angles, n_freqs]
as a differentiable function of the mesh vertices and the frequencies.

Forward builds the scene from the current vertices and runs the sweep through
sbr_run; backward turns the incoming gradient of sigma into the cotangent of every
sample's field (sigma = 4 pi |S|^2, so dLoss = sum Re(conj(8 pi w S) dS) for
w = dLoss/dsigma) and calls sbr_adjoint, which re-traces the rays and
differentiates along the frozen hit paths.  Torch only carries the tensors; all
work runs in libsbr.
"""
from __future__ import annotations

import numpy as np
import torch

from . import PREC_FP64, PREC_MIXED, JobSpec, Scene, adjoint, run


class RcsFunction(torch.autograd.Function):
    """sigma = RcsFunction.apply(verts, freqs, tris, theta, phi, nx, ny, grid, max_bounces, R, precision)."""

    @staticmethod
    def forward(ctx, verts, freqs, tris, theta, phi, nx, ny, grid, max_bounces, reflection_const, precision):
        v = verts.detach().to("cpu", torch.float64).numpy()
        f = freqs.detach().to("cpu", torch.float64).numpy().ravel()
        t = np.asarray(tris, dtype=np.uint32)
        job = JobSpec(np.asarray(theta, np.float64), np.asarray(phi, np.float64), f, nx, ny, grid, max_bounces,
                      reflection_const)
        scene = Scene(v, t, want_fp64=precision == PREC_FP64)
        try:
            res = run(scene, job, precision=precision)
        except Exception:
            scene.close()
            raise
        ctx.scene, ctx.job, ctx.field, ctx.precision = scene, job, res.field, precision
        ctx.shape = (job.n_angles, job.n_freqs)
        ctx.vdev, ctx.vdtype, ctx.fdev, ctx.fdtype = verts.device, verts.dtype, freqs.device, freqs.dtype
        return torch.from_numpy(res.sigma_m2.reshape(ctx.shape)).to(verts.device)

    @staticmethod
    def backward(ctx, gsigma):
        w = gsigma.detach().to("cpu", torch.float64).numpy().ravel()
        cot = 8.0 * np.pi * w * ctx.field
        try:
            gx, gf = adjoint(ctx.scene, ctx.job, cot, precision=ctx.precision)
        finally:
            ctx.scene.close()
        gverts = torch.from_numpy(gx).to(ctx.vdev, ctx.vdtype)
        gfreq = torch.from_numpy(gf.reshape(ctx.shape).sum(axis=0)).to(ctx.fdev, ctx.fdtype)
        return gverts, gfreq, None, None, None, None, None, None, None, None, None


def rcs(verts: torch.Tensor, tris, theta, phi, freqs: torch.Tensor, nx: int, ny: int, grid: float,
        max_bounces: int, reflection_const: float = 1.0, precision=PREC_MIXED) -> torch.Tensor:
    """Differentiable sigma [n_angles, n_freqs] (m^2) of the mesh (verts [V, 3])."""
    return RcsFunction.apply(verts, freqs, tris, theta, phi, nx, ny, grid, max_bounces, reflection_const,
                             precision)
