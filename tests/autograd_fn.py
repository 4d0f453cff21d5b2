"""torch.autograd.Function over the C ABI's forward + adjoint pass (test harness only).

score = BPMaxScore.apply(weights, engine, pairs) gives one optimal score per pair; backward
returns d(sum of upstream grads * scores)/d(weights) from bpmax_gpu_grad_batch's exact pair-type
counts."""
import numpy as np
import torch


class BPMaxScore(torch.autograd.Function):
    @staticmethod
    def forward(ctx, weights, engine, pairs):
        w = weights.detach().cpu().numpy().astype(np.float32)
        engine.set_weights(w)
        scores, grads = engine.grad_batch(pairs)
        ctx.save_for_backward(torch.from_numpy(grads.copy()))
        return torch.from_numpy(scores.copy()).to(weights.dtype)

    @staticmethod
    def backward(ctx, g):
        (counts,) = ctx.saved_tensors
        return (g.to(counts.dtype) @ counts).to(g.dtype), None, None
