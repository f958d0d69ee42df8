"""torch.autograd bridge of the opacity adjoint.

``Opacity.apply(hk, T, P, log_s, log_g, precision)`` returns the opacity K
(Nx, float64, CUDA) of one state (T, P) of the lines loaded in the hkb
Context ``hk``, with per-line strength multipliers exp(log_s) and Lorentz
width multipliers exp(log_g) (load order; None for 1).  Its backward is the
library's hand-written vector-Jacobian product (hk_opacity_vjp): gradients
for T, P, log_s and log_g; the forward is recomputed per grid tile inside the
adjoint kernel instead of being stored.  torch is plumbing here: every number
comes from libhkb's kernels.
"""
from __future__ import annotations

import torch

import hkb


def _scales(v):
    # a CUDA tensor stays on the GPU (hk_set_line_scales_device)
    if v is None:
        return None
    return torch.exp(v.detach().to(torch.float64)).contiguous()


class Opacity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, hk, T, P, log_s=None, log_g=None, precision=hkb.MIXED):
        s, g = _scales(log_s), _scales(log_g)
        Tf, Pf = float(T), float(P)
        hk.set_line_scales(s, g)
        K = torch.empty(hk.nx, dtype=torch.float64, device=torch.device("cuda", hk.device))
        hk.opacity([Tf], [Pf], precision, out=K.view(1, -1))
        ctx.hk = hk
        ctx.state = (Tf, Pf, precision)
        ctx.scales = (s, g)
        ctx.meta = [(v.dtype, v.device) if torch.is_tensor(v) else None
                    for v in (T, P, log_s, log_g)]
        return K

    @staticmethod
    def backward(ctx, gK):
        hk = ctx.hk
        Tf, Pf, prec = ctx.state
        s, g = ctx.scales
        hk.set_line_scales(s, g)  # the context may have served other calls since
        # per-line gradients per log S and per log gammaL, left on the GPU
        dT, dP, dS, dG = hk.opacity_vjp(Tf, Pf, gK.detach().to(torch.float64).contiguous(), prec,
                                        log_gamma=True, device_out=True)

        def like(v, meta):
            dt, dev = meta
            return torch.as_tensor(v, dtype=dt, device=dev)

        need = ctx.needs_input_grad
        m = ctx.meta
        gT = like(dT, m[0]) if need[1] else None
        gP = like(dP, m[1]) if need[2] else None
        gS = dS.to(dtype=m[2][0], device=m[2][1]) if need[3] else None
        gG = dG.to(dtype=m[3][0], device=m[3][1]) if need[4] else None
        return None, gT, gP, gS, gG, None
