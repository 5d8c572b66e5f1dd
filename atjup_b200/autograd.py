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


class IterationStep(torch.autograd.Function):
    """One whole dry iteration of the reference's loop (atjup_gpu_step: the pressure pass and the
    mixture density on even iterations and the first, RK4, the boundary passes, the in-loop
    Shapiro filter and the column balance of v) on the nine fields one iteration hands the next
    (atjup_b200.params.LIN_FIELDS: t, u, v, w, p_dyn, aux_u, aux_v, aux_w, rho_mix). Its backward is
    atjup_gpu_iteration_adjoint_ckpt about the iteration's input: the step keeps its input and
    its RK stage inputs (X1, X2, X3 of t, u, v, w, written there by the forward step itself) as
    its checkpoint, and the adjoint recomputes only the pressure pass from it."""

    @staticmethod
    def forward(ctx, model, iter_n, first, chained, *x):
        from .params import LIN_FIELDS
        y = tuple(t.detach().contiguous() for t in x)
        if not chained:
            # chained: x are the outputs of the step just run, which the context still holds
            model.set_state_tensors(y, names=LIN_FIELDS, wait=False)
        stages = [torch.empty_like(y[0]) for _ in range(12)]
        model.set_stage_buffers(stages)
        try:
            model.step(iter_n, first)
        finally:
            model.set_stage_buffers(None)
        out = model.state_tensors(LIN_FIELDS)
        ctx.model, ctx.iter_n, ctx.first = model, iter_n, first
        ctx.save_for_backward(*y, *stages)
        return tuple(out)

    @staticmethod
    def backward(ctx, *grads):
        from .params import LIN_FIELDS
        saved = ctx.saved_tensors
        y, stages = saved[:len(LIN_FIELDS)], saved[len(LIN_FIELDS):]
        model = ctx.model
        model.set_state_tensors(y, names=LIN_FIELDS, wait=False)   # the linearisation point
        g = [torch.zeros_like(r) if gr is None else gr.detach().clone().contiguous()
             for gr, r in zip(grads, y)]
        model.iteration_adjoint_ckpt(g, stages, ctx.iter_n, ctx.first)
        return (None, None, None, None, *g)


def iterations(model, x, steps: int, start: int = 1):
    """`steps` differentiable dry iterations from the nine tensors x (LIN_FIELDS order), numbered
    start, start + 1, ... (the first of a run has first = True). Between the iterations of the
    chain the context keeps the state it just produced, so only the first input is copied in."""
    y = tuple(x)
    for n in range(start, start + steps):
        y = IterationStep.apply(model, n, n == 1, n > start, *y)
    return y
