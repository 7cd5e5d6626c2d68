"""torch.autograd binding of the evaluator and its hand-written adjoint.

``fmm_apply(f, den, trg, precision)`` returns ``phi = A(trg) den`` for a set-up
``fmmg.FMM3d`` handle ``f``: ``den`` holds one right-hand side
([n_src * srcDOF] or [n_src, srcDOF], giving [n_trg, trgDOF]) or k of them
([k, n_src * srcDOF] or [k, n_src, srcDOF], giving [k, n_trg, trgDOF]),
evaluated in one call in the given precision (``fmmg.PREC_FP64`` or
``fmmg.PREC_MIXED``).  The backward pass runs the transposed FMM
(``fmmg_adjoint_device``, FP64, on all k right-hand sides): the density
gradient is ``A^T dL/dphi`` and, when ``trg`` requires grad, the
target-position gradient comes from the kernel-gradient forms of the
near-field, M2T and L2T sums (Laplace kernels 111 and 121), summed over the k
right-hand sides.  ``trg`` must hold the positions the handle was set up with
(the tree and lists are built at setup); it only carries the gradient.
"""
import torch

import fmmg


class FMMEvaluate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f, den, trg, precision):
        ctx.den_shape = den.shape
        if den.dtype != torch.float64 or not den.is_cuda:
            raise TypeError("den must be a float64 CUDA tensor")
        per = f.ns * f.sd
        if den.numel() % per or den.numel() == 0:
            raise ValueError("den must hold k x n_src x srcDOF values")
        k = den.numel() // per
        batched = den.dim() >= 2 and den.numel() // den.shape[0] == per  # [k, ...] with k leading
        den = den.detach().contiguous().view(k, per)
        out = torch.empty(k, f.nt * f.td, dtype=torch.float64, device=den.device)
        f.evaluate_device(den, out, k, precision)
        f.sync()
        ctx.f, ctx.k = f, k
        ctx.save_for_backward(den)
        return out.view(k, f.nt, f.td) if batched else out.view(f.nt, f.td)

    @staticmethod
    def backward(ctx, gout):
        f, k = ctx.f, ctx.k
        (den,) = ctx.saved_tensors
        need_den, need_trg = ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        w = gout.detach().to(torch.float64).contiguous().view(k, -1)
        g = torch.empty(k, f.ns * f.sd, dtype=torch.float64, device=den.device) if need_den else None
        gt = torch.empty((k, f.nt, 3), dtype=torch.float64, device=den.device) if need_trg else None
        if need_den or need_trg:
            f.adjoint_device(den if need_trg else None, w, g, gt, k=k)
            f.sync()
        return (None, g.view(ctx.den_shape) if need_den else None, gt.sum(0) if need_trg else None, None)


def fmm_apply(f, den, trg=None, precision=fmmg.PREC_FP64):
    """phi = A(trg) den for one or k right-hand sides, with gradients to den
    and (optionally) trg."""
    if trg is not None and tuple(trg.shape) != (f.nt, 3):
        raise ValueError("trg must be the (n_trg, 3) set-up target positions")
    return FMMEvaluate.apply(f, den, trg, precision)
