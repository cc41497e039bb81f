"""``torch.autograd.Function`` over the C ABI: the pseudo-likelihood as a
differentiable function of the single fields V and the couplings W.

The backward is the library's own gradient kernel, in the ``partial``
convention (true partial derivatives of f with respect to every entry, the
couplings untied and the self-edge blocks included), so that autograd and
finite differences agree.  The reference's optimizer uses the ``tied``
convention instead (src/evaluate_cpu.c:131-163); for a symmetric W the two are
related by  tied(b,k,a,j) = partial(b,k,a,j) + partial(a,j,b,k)  for k != j.

Tensor layouts:
  V  (L, 20)           V[j, a]        = single field of state a in column j
  W  (L, L, 21, 21)    W[k, j, b, a]  = coupling of state b in column k with
                                        state a in column j  (reference W(b,k,a,j))
"""
from __future__ import annotations

import torch

from . import Evaluator, nsingle_padded, nvar_padded

Q = 21
QPAD = 32


def pack(V: torch.Tensor, W: torch.Tensor) -> torch.Tensor:
    """(V, W) -> x in the reference's padded layout (differentiable)."""
    L = V.shape[0]
    nsp = nsingle_padded(L)
    head = torch.cat([V.transpose(0, 1).reshape(-1),
                      V.new_zeros(nsp - (Q - 1) * L)])
    x2 = W.permute(2, 0, 3, 1)                                     # [b, k, a, j]
    x2 = torch.cat([x2, W.new_zeros(Q, L, QPAD - Q, L)], dim=2)     # pad a to 32
    return torch.cat([head, x2.reshape(-1)])


def unpack(x: torch.Tensor, L: int):
    """x (padded layout) -> (V, W)."""
    nsp = nsingle_padded(L)
    V = x[: (Q - 1) * L].reshape(Q - 1, L).transpose(0, 1)
    W = x[nsp:].reshape(Q, L, QPAD, L)[:, :, :Q, :].permute(1, 3, 0, 2)
    return V, W


class PseudoLikelihoodFunction(torch.autograd.Function):
    """f(x) for a padded parameter vector x; backward = the CUDA gradient kernels."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, evaluator: Evaluator):
        if evaluator.gradient != "partial":
            raise ValueError("autograd needs an Evaluator with gradient='partial'")
        xc = x.detach().contiguous()
        g = torch.empty_like(xc)
        f = evaluator.evaluate(xc, g)
        ctx.save_for_backward(g)
        return torch.tensor(f, dtype=x.dtype, device=x.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None


def pseudo_likelihood(V: torch.Tensor, W: torch.Tensor, evaluator: Evaluator) -> torch.Tensor:
    """Differentiable f(V, W) (float32 on the tensor-core paths, float64 on simt_f64)."""
    x = pack(V, W)
    assert x.numel() == nvar_padded(V.shape[0])
    return PseudoLikelihoodFunction.apply(x, evaluator)
