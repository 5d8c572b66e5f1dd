"""torch.autograd binding of one RK4 step of the dry dynamics.

`RK4Step.apply(model, t, u, v, w)` runs RungeKuttaJup on the model's device (atjup_gpu_rk4_step)
from the given state and returns the new t, u, v, w; its backward is the hand-written adjoint
(atjup_gpu_rk4_adjoint) about the step's input, which each step keeps as its checkpoint and from
which the adjoint recomputes the stages. The tensors are float64 CUDA tensors in the model's
padded layout, (im, jm, pitch) with pitch = model.field_ptr("t")[1]; lanes k >= km carry nothing.
Chaining K applications differentiates K RK4 steps: memory is the K checkpoints of four fields.
p_dyn, p_stat, rho_mix, wall_nue and the other inputs of the step are the model's, held fixed.
"""
from __future__ import annotations

import torch


class RK4Step(torch.autograd.Function):
    @staticmethod
    def forward(ctx, model, t, u, v, w):
        y = tuple(x.detach().contiguous() for x in (t, u, v, w))
        model.set_state_tensors(y, wait=False)   # ordered before the step on the library's stream
        model.runge_kutta()
        out = model.state_tensors()
        ctx.model = model
        ctx.save_for_backward(*y)
        return tuple(out)

    @staticmethod
    def backward(ctx, gt, gu, gv, gw):
        y = ctx.saved_tensors
        model = ctx.model
        model.set_state_tensors(y, wait=False)  # the linearisation point: the step's input
        grads = []
        for g, ref in zip((gt, gu, gv, gw), y):
            grads.append(torch.zeros_like(ref) if g is None else g.detach().clone().contiguous())
        model.rk4_adjoint(*grads)
        return (None, *grads)


def rk4_steps(model, t, u, v, w, steps: int):
    """K differentiable RK4 steps from (t, u, v, w)"""
    y = (t, u, v, w)
    for _ in range(steps):
        y = RK4Step.apply(model, *y)
    return y
