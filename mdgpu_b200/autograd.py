"""torch.autograd front-end of the adjoint: loss = log det A + b' A^-1 b.

The forward factors A in FP64 and solves through the C ABI; the backward
runs the selected inverse (mdgpu_selinv) and returns
d loss / d Ax = the gradient of the caller's lower-triangle values
(mdgpu_grad_lower) and d loss / d b = 2 A^-1 b.  The Solver's factor
generation is saved with the values: if another forward refactored the
Solver before this backward, the backward factors its own values again
rather than differentiate someone else's factor.  Only the front-end: all
arithmetic is in the library's kernels.
"""
import torch

import mdgpu_b200 as M


class LogdetQuad(torch.autograd.Function):
    @staticmethod
    def forward(ctx, S, Ax, b):
        """S: a Solver of A's pattern; Ax: CUDA float64 values of the lower
        triangle (the caller's order); b: CUDA float64 vector of length n."""
        vals = Ax.detach().contiguous()
        S.factor(vals, M.FP64)
        bb = b.detach().contiguous()
        x = S.solve(bb)
        loss = S.logdet() + float(torch.dot(bb, x))
        ctx.S = S
        ctx.generation = S.generation  # the factor this forward used
        ctx.save_for_backward(x, vals)
        return torch.tensor(loss, dtype=torch.float64, device=Ax.device)

    @staticmethod
    def backward(ctx, g):
        x, vals = ctx.saved_tensors
        if ctx.S.generation != ctx.generation:
            # another forward refactored the Solver since: factor these
            # values again (the factor is deterministic, bit for bit)
            ctx.S.factor(vals, M.FP64)
            ctx.generation = ctx.S.generation
        ctx.S.selinv()
        G = ctx.S.grad_lower(x.contiguous())
        return None, g * G, g * 2.0 * x


def logdet_quad(S, Ax, b):
    return LogdetQuad.apply(S, Ax, b)
