"""The host logic of atjup_b200/autograd.py on the CPU: a fake model with the library model's
methods (set_state_tensors, runge_kutta, state_tensors, rk4_adjoint) runs a nonlinear map of
(t, u, v, w) with its hand-written adjoint, so chains of RK4Step must linearise each step about
that step's own input (its checkpoint) and leave the fields without a gradient at zero. The
gradients are compared with torch's autograd of the same map."""
import torch

from atjup_b200.autograd import RK4Step, rk4_steps


def step_map(t, u, v, w):
    return (t + 0.1 * u * v, u + 0.2 * torch.sin(t), v - 0.3 * w * t, w + 0.05 * u * u)


class FakeModel:
    """one 'RK4 step' is step_map; the adjoint is its transposed Jacobian at the state set last"""

    def __init__(self):
        self.state = None
        self.steps = 0
        self.adjoints = 0

    def set_state_tensors(self, y, wait=True):
        self.state = tuple(x.clone() for x in y)

    def runge_kutta(self):
        self.state = step_map(*self.state)
        self.steps += 1

    def state_tensors(self):
        return tuple(x.clone() for x in self.state)

    def rk4_adjoint(self, gt, gu, gv, gw):
        t, u, v, w = self.state
        at = gt + 0.2 * torch.cos(t) * gu - 0.3 * w * gv
        au = 0.1 * v * gt + gu + 0.1 * u * gw
        av = 0.1 * u * gt + gv
        aw = -0.3 * t * gv + gw
        for g, a in zip((gt, gu, gv, gw), (at, au, av, aw)):
            g.copy_(a)
        self.adjoints += 1


def inputs(seed):
    g = torch.Generator().manual_seed(seed)
    return [torch.randn(3, 5, 8, dtype=torch.float64, generator=g) for _ in range(4)]


def test_chain_gradient_matches_torch_autograd():
    x = inputs(1)
    wts = inputs(2)
    m = FakeModel()
    a = [xi.clone().requires_grad_(True) for xi in x]
    y = rk4_steps(m, *a, steps=3)
    loss = sum((wi * yi).sum() for wi, yi in zip(wts, y))
    loss.backward()
    b = [xi.clone().requires_grad_(True) for xi in x]
    z = b
    for _ in range(3):
        z = step_map(*z)
    ref = sum((wi * zi).sum() for wi, zi in zip(wts, z))
    ref.backward()
    assert m.steps == 3 and m.adjoints == 3        # the adjoint recomputes its stages itself
    assert abs(loss.item() - ref.item()) <= 1e-12 * abs(ref.item())
    for ga, gb in zip(a, b):
        assert torch.allclose(ga.grad, gb.grad, rtol=1e-13, atol=1e-13)


def test_fields_without_a_gradient_are_zero():
    """a loss that reads only u: the adjoint is seeded with zeros for t, v, w"""
    x = inputs(3)
    m = FakeModel()
    a = [xi.clone().requires_grad_(True) for xi in x]
    t1, u1, v1, w1 = RK4Step.apply(m, *a)
    u1.sum().backward()
    b = [xi.clone().requires_grad_(True) for xi in x]
    step_map(*b)[1].sum().backward()
    for ga, gb in zip(a, b):
        want = torch.zeros_like(ga) if gb.grad is None else gb.grad
        assert torch.allclose(ga.grad, want, rtol=1e-13, atol=1e-13)
    assert not a[2].grad.any() and not a[3].grad.any()
