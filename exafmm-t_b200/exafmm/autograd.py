"""Adjoint FMM as a torch.autograd.Function (no counterpart in the reference, whose FMM is not
differentiable).

Forward, for sources x_j with charges q_j and targets y_i, one FMM evaluate:
    phi_i = sum_j q_j G(y_i - x_j),   g_i = grad phi(y_i)            -> out[i] = (phi_i, g_i)
Backward, for a loss whose cotangent on the potentials is w (its cotangent on the gradient
components must be zero: second derivatives are not provided), one more FMM evaluate with the roles
of sources and targets swapped and the cotangent as charges:
    psi(x) = sum_i w_i G(x - y_i)
    dL/dq_j = psi(x_j)
    dL/dx_j = q_j grad psi(x_j)      (G is radial, so its gradient is odd)
    dL/dy_i = w_i g_i                (the forward's own gradient output)
Nothing of the forward pass is kept but its output: the swapped-role tree and lists are rebuilt
from the coordinates, and when the same tensor holds sources and targets the forward tree serves
both directions.  Real symmetric kernels: Laplace and modified Helmholtz.
"""
import torch

from . import _core


def _fmm_like(fmm):
    """A second Fmm object of the same kernel, order, ncrit, wavenumber and precision (it keeps its own
    operators, so the swapped-role tree does not invalidate the forward's)."""
    if fmm.kernel == "laplace":
        return _core.LaplaceFmm(fmm.p, fmm.ncrit, precision=fmm.precision)
    return _core.ModifiedHelmholtzFmm(fmm.p, fmm.ncrit, fmm.wavek, precision=fmm.precision)


def _evaluate(fmm, src_xyz, charges, trg_xyz, tree=None):
    if tree is None:
        tree = _core.setup(_core.init_sources(src_xyz, charges, fmm.kernel), _core.init_targets(trg_xyz), fmm)
    else:
        _core.update_charges(tree, charges)
    out = torch.empty((trg_xyz.shape[0], 4), dtype=torch.float64, device=trg_xyz.device)
    _core.evaluate(tree, fmm, out=out)
    return out, tree


class FmmFunction(torch.autograd.Function):
    """out = FmmFunction.apply(charges, src_xyz, trg_xyz, fmm, tree=None): (ntrg, 4) potential and gradient.

    charges (nsrc,), src_xyz (nsrc, 3), trg_xyz (ntrg, 3): float64 CUDA tensors.  Pass the same
    tensor as src_xyz and trg_xyz when sources and targets coincide.
    """

    @staticmethod
    def forward(ctx, charges, src_xyz, trg_xyz, fmm, tree=None):
        if fmm.kernel not in ("laplace", "modified_helmholtz"):
            raise NotImplementedError("the adjoint covers the real kernels (Laplace, modified Helmholtz)")
        for t in (charges, src_xyz, trg_xyz):
            if not (t.is_cuda and t.dtype == torch.float64):
                raise RuntimeError("charges and coordinates must be float64 CUDA tensors")
        q, x, y = charges.detach().contiguous(), src_xyz.detach().contiguous(), trg_xyz.detach().contiguous()
        same = src_xyz is trg_xyz or (src_xyz.data_ptr() == trg_xyz.data_ptr() and src_xyz.shape == trg_xyz.shape)
        out, tree = _evaluate(fmm, x, q, y, tree=tree)
        ctx.fmm, ctx.same = fmm, same
        ctx.tree = tree if same else None
        ctx.save_for_backward(q, x, y, out)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        q, x, y, out = ctx.saved_tensors
        grad_out = grad_out.contiguous()
        if bool((grad_out[:, 1:] != 0).any()):
            raise NotImplementedError("cotangents on the gradient components need second derivatives")
        w = grad_out[:, 0].contiguous()
        if ctx.same:
            psi, _ = _evaluate(ctx.fmm, x, w, x, tree=ctx.tree)  # same points: the forward tree
        else:
            fmm2 = getattr(ctx.fmm, "_adjoint_fmm", None)
            if fmm2 is None:
                fmm2 = _fmm_like(ctx.fmm)
                ctx.fmm._adjoint_fmm = fmm2
            psi, _ = _evaluate(fmm2, y, w, x)  # sources at the targets, targets at the sources
        dq = psi[:, 0] if ctx.needs_input_grad[0] else None
        dx = q[:, None] * psi[:, 1:4] if ctx.needs_input_grad[1] else None
        dy = w[:, None] * out[:, 1:4] if ctx.needs_input_grad[2] else None
        ctx.tree = None
        return dq, dx, dy, None, None


def fmm_apply(charges, src_xyz, trg_xyz, fmm, tree=None):
    """Differentiable FMM evaluate: (ntrg, 4) potential and gradient.

    tree: optional result of setup() on these same coordinates (e.g. across steps that change only the
    charges); without it the forward builds the tree, lists and operators from the coordinates.  The
    forward writes `charges` into the tree, and a backward with coinciding sources and targets writes
    the cotangent into it."""
    return FmmFunction.apply(charges, src_xyz, trg_xyz, fmm, tree)
