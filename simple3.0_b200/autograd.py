"""torch.autograd.Function over the adjoint kernel.

``ShiftDefocusCorr.apply(x, pc, iref, iptcl, irot)`` returns, for every row
x[i] = (shift_x, shift_y, defocus offset [micron]) of a float64 tensor, the
reference-frame correlation of (iref[i], iptcl[i], irot[i]) with the particle's CTF
evaluated at its defocus plus the offset.  Forward and backward both come from one
pftcc_grad_batch call (the kernel returns the value and its three partial
derivatives together), so torch.autograd.gradcheck compares the hand-written
adjoint against finite differences of the same forward.
"""
from __future__ import annotations

import numpy as np
import torch


class ShiftDefocusCorr(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, pc, iref, iptcl, irot):
        xn = x.detach().cpu().numpy().astype(np.float64)
        f, g3 = pc.grad_batch(np.asarray(iref), np.asarray(iptcl), np.asarray(irot), xn[:, 0], xn[:, 1], xn[:, 2])
        ctx.save_for_backward(torch.as_tensor(g3, dtype=x.dtype, device=x.device))
        return torch.as_tensor(f, dtype=x.dtype, device=x.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g3,) = ctx.saved_tensors
        return grad_out[:, None] * g3, None, None, None, None


def shift_defocus_corr(x, pc, iref, iptcl, irot):
    return ShiftDefocusCorr.apply(x, pc, iref, iptcl, irot)
