"""torch.autograd binding of the evaluator and its hand-written adjoint.

``fmm_apply(f, den, trg)`` returns ``phi = A(trg) den`` ([n_trg, trgDOF]) for a
set-up ``fmmg.FMM3d`` handle ``f``.  Its backward pass calls the transposed
FMM (``fmmg_adjoint_device``): the density gradient is ``A^T dL/dphi`` and, when
``trg`` requires grad, the target-position gradient comes from the
kernel-gradient forms of the near-field, M2T and L2T sums (Laplace kernels 111
and 121).  ``trg`` must hold the positions the handle was set up with (the tree
and lists are built at setup); it only carries the gradient.
"""
import torch

import fmmg


class FMMEvaluate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, den, trg):
        ctx.den_shape = den.shape
        den = den.detach().contiguous().view(-1)
        if den.dtype != torch.float64 or not den.is_cuda:
            raise TypeError("den must be a float64 CUDA tensor")
        out = torch.empty(f.nt * f.td, dtype=torch.float64, device=den.device)
        f.evaluate_device(den, out)
        f.sync()
        ctx.f = f
        ctx.save_for_backward(den)
        return out.view(f.nt, f.td)

    @staticmethod
    def backward(ctx, gout):
        f = ctx.f
        (den,) = ctx.saved_tensors
        need_den, need_trg = ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        w = gout.detach().to(torch.float64).contiguous().view(-1)
        g = torch.empty(f.ns * f.sd, dtype=torch.float64, device=den.device) if need_den else None
        gt = torch.empty((f.nt, 3), dtype=torch.float64, device=den.device) if need_trg else None
        if need_den or need_trg:
            f.adjoint_device(den if need_trg else None, w, g, gt)
            f.sync()
        return None, (g.view(ctx.den_shape) if need_den else None), gt


def fmm_apply(f, den, trg=None):
    """phi = A(trg) den with gradients to den and (optionally) trg."""
    if trg is not None and tuple(trg.shape) != (f.nt, 3):
        raise ValueError("trg must be the (n_trg, 3) set-up target positions")
    return FMMEvaluate.apply(f, den, trg)
