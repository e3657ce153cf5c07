"""The misfit as a differentiable torch function of (lambda, mu, rho).

`ElasticMisfit.apply(lam, mu, rho, prop, shot_ids, obs)` returns the misfit
J (float64 scalar) of the shots `shot_ids` against observed traces `obs`
(the engine's traces layout) on the engine `prop`; its backward is the exact
discrete adjoint of the forward scheme (EFWI_MODE_EXACT), so the gradients
are dJ/dlambda, dJ/dmu and dJ/drho of the returned J and compose with any
torch parametrisation of the model (for example lambda = (vp^2 - 2 vs^2) rho).

Like the reference's FWIFunction (FWI_ops_3d.py:34-44), the forward pass runs
the whole gradient computation once and the backward pass scales the stored
images by the incoming gradient.  The reference's FWIFunction returns the
reference algorithm's images regardless of the incoming gradient; this
function is the exact one.
"""
from __future__ import annotations

import torch


class ElasticMisfit(torch.autograd.Function):
    @staticmethod
    def forward(ctx, lam, mu, rho, prop, shot_ids, obs):
        prop.set_model(lam.detach(), mu.detach(), rho.detach())
        J, gl, gm, gr = prop.gradient(list(shot_ids), obs, mode="exact")
        ctx.save_for_backward(gl, gm, gr)
        ctx.devices = (lam.device, mu.device, rho.device)
        return torch.tensor(J, dtype=torch.float64, device=lam.device)

    @staticmethod
    def backward(ctx, grad_out):
        gl, gm, gr = ctx.saved_tensors
        s = grad_out.to(device=gl.device, dtype=torch.float32)
        out = [(g * s).to(d) if need else None
               for g, d, need in zip((gl, gm, gr), ctx.devices, ctx.needs_input_grad[:3])]
        return out[0], out[1], out[2], None, None, None


def misfit(lam, mu, rho, prop, shot_ids, obs) -> torch.Tensor:
    """J(lam, mu, rho) with exact gradients (see ElasticMisfit)."""
    return ElasticMisfit.apply(lam, mu, rho, prop, shot_ids, obs)
