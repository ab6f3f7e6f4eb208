"""torch.autograd binding: a batch's alignment scores as a differentiable function of the
substitution matrices and gap costs.

    batch = SeqPairBatch(seqs_a, seqs_b, params, grad_mode="soft")
    mats = torch.tensor(params.matrices, dtype=torch.float64, requires_grad=True)   # (K, N, N)
    gaps = torch.tensor(params.gaps, dtype=torch.float64, requires_grad=True)       # (K, 4)
    scores = align_scores(batch, mats, gaps)       # (n_pairs,) float64: soft log Z (or Viterbi)
    loss = scores[pos].sum() - scores[neg].sum()
    loss.backward()                                # mats.grad, gaps.grad

Forward: the parameters are handed to the batch (``set_params``, a copy) and the GPU runs
``score_and_grad`` -- the fused forward-backward kernel, which leaves every pair's
d score / d parameters (expected transition counts for soft, path counts for hard) in HBM.
Backward: the vector-Jacobian product sum_p grad_out[p] * d score_p / d params is the
batch's weighted gradient (``weighted_grad``: the fixed-order FP64 reduction kernel), so no
per-pair gradient leaves the device.  Gap costs enter the score with a minus sign, which the
per-pair gradients already carry (the reference's ``compute_grad`` convention).

A 2-D matrix (N, N) with gaps (4,) is one parameter set; (K, N, N) with (K, 4) is K sets.
If the batch is run again (by anything) between this forward and its backward, the backward
re-runs the forward with its own parameters first, so the gradient always belongs to them.
"""
from __future__ import annotations

import numpy as np
import torch

from .params import AlignParams

__all__ = ["align_scores", "AlignScores"]


class AlignScores(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mats, gaps, batch):
        squeeze = mats.dim() == 2
        m = mats.detach().to("cpu", torch.float64).numpy()
        g = gaps.detach().to("cpu", torch.float64).numpy()
        if squeeze:
            m, g = m[None], g[None]
        params = AlignParams.from_arrays(np.ascontiguousarray(m), np.ascontiguousarray(g),
                                         alphabet=batch._alpha)
        batch.set_params(params)
        batch.score_and_grad()
        ctx.batch = batch
        ctx.params = params
        ctx.run_id = batch._run_id
        ctx.squeeze = squeeze
        ctx.shapes = (mats.shape, gaps.shape, mats.dtype, gaps.dtype, mats.device, gaps.device)
        return torch.from_numpy(batch.scores()).to(mats.device)

    @staticmethod
    def backward(ctx, grad_out):
        batch = ctx.batch
        if batch._run_id != ctx.run_id:      # the batch ran since: recompute for these params
            batch.set_params(ctx.params)
            batch.score_and_grad()
        w = grad_out.detach().to("cpu", torch.float64).numpy()
        gp = batch.weighted_grad(np.ascontiguousarray(w))
        ms, gs, mdt, gdt, mdev, gdev = ctx.shapes
        gm = torch.from_numpy(np.ascontiguousarray(gp.matrices)).reshape(ms).to(mdev, mdt)
        gg = torch.from_numpy(np.ascontiguousarray(gp.gaps)).reshape(gs).to(gdev, gdt)
        return gm, gg, None


def align_scores(batch, mats: torch.Tensor, gaps: torch.Tensor) -> torch.Tensor:
    """Per-pair scores of ``batch`` under (mats, gaps), differentiable in both."""
    if batch._grad_mode == "none":
        raise ValueError("nwgrad: align_scores needs a batch with grad_mode \"soft\" or \"hard\"")
    return AlignScores.apply(mats, gaps, batch)
