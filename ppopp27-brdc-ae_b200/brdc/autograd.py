"""torch.autograd.Function around the BR solve and its adjoint.

Forward: eigenvalues W (ascending) of the symmetric tridiagonal (D, E)
through brdc_dstebr with a checkpointing workspace.  Backward:
dL/dD, dL/dE through brdc_dstebr_backward on the same workspace, without
forming eigenvectors.
"""
from __future__ import annotations

import torch

from . import Solver


class TridiagEigvals(torch.autograd.Function):
    @staticmethod
    def forward(ctx, D, E, solver: Solver):
        n = D.shape[0]
        # A workspace of its own for every forward: the backward reads this
        # forward's checkpoints, which a later forward of the same order
        # (a second matrix in the same loss) would otherwise overwrite.
        ws = solver.new_checkpoint_workspace(n)
        W = solver.dstebr(D, E, workspace=ws)
        ctx.solver = solver
        ctx.ws = ws
        ctx.save_for_backward(D, E)
        return W

    @staticmethod
    def backward(ctx, G):
        D, E = ctx.saved_tensors
        solver = ctx.solver
        gD, gE = solver.dstebr_backward(D, E, G.contiguous(), workspace=ctx.ws,
                                        keep_forward=True)
        ctx.ws = None
        return gD, gE, None


def eigvalsh_tridiagonal(D, E, solver: Solver):
    """Differentiable eigenvalues of a symmetric tridiagonal matrix."""
    return TridiagEigvals.apply(D, E, solver)
