"""torch.autograd.Function over the hand-written colour + film adjoints.

`FilmModel.apply(cam_rgb, theta)` runs imops_param_forward; its backward
calls imops_param_backward with the upstream gradient dL/dout and returns
dL/dtheta (the 24 parameters of ImopsFilmGradParams, in that order).  The
camera RGB gets no gradient: demosaic decisions are held fixed and the
demosaic is upstream of every parameter.  The halation blur is recomputed
in the backward, not stored.
"""
from __future__ import annotations

import torch

import imops_b200 as im


class FilmModel(torch.autograd.Function):
    @staticmethod
    def forward(ctx, cam_rgb: torch.Tensor, theta: torch.Tensor, fixed=None):
        p = im.FilmGradParams.from_vector(theta.detach().cpu().tolist())
        out = im.param_forward(cam_rgb.contiguous(), p, fixed)
        ctx.save_for_backward(cam_rgb, theta)
        ctx.fixed = fixed
        return out

    @staticmethod
    def backward(ctx, g_out: torch.Tensor):
        cam_rgb, theta = ctx.saved_tensors
        p = im.FilmGradParams.from_vector(theta.detach().cpu().tolist())
        grad = torch.zeros(25, dtype=torch.float64, device=cam_rgb.device)
        im.param_backward(cam_rgb.contiguous(), p, grad, g_out=g_out.contiguous().float(), fixed=ctx.fixed)
        return None, grad[:24].to(theta.dtype).to(theta.device), None


def film_model(cam_rgb: torch.Tensor, theta: torch.Tensor, fixed=None) -> torch.Tensor:
    return FilmModel.apply(cam_rgb, theta, fixed)
