"""Gradients of a Landau-Lifshitz trajectory by the discrete adjoint method.

The trajectory is integrated with the classical fixed-step RK4 scheme on the
device right-hand side (``mt_rhs``) under a piecewise-constant applied field
(one field per time segment, which the reference's interpolated field tables
cannot express), and the spatial average <m>(t) is sampled every few steps.
``mean_m_trajectory`` returns those samples as a torch tensor whose gradient
with respect to the segment fields and the per-cell Ms is computed by the
exact adjoint of the RK4 steps:

- the forward pass keeps m only every ``checkpoint_every`` steps;
- the backward pass recomputes the states of one checkpoint interval at a
  time and walks its steps in reverse, calling the hand-written
  vector-Jacobian product of the right-hand side (``mt_rhs_vjp``) four times
  per step.  The demag and exchange operators are symmetric, so their
  transposes run the forward kernels.

The gradient is that of the discrete computation, so it agrees with central
finite differences of the same forward pass.  Per-cell Ms follows the
reference's model: the demag field of cell i is -Ms_i (K m)_i (Ms at the
receiver), exchange and anisotropy use A0/(mu0 Ms_i) and K0/(mu0 Ms_i).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from .solver import Solver


@dataclass
class TrajectoryProblem:
    """A fixed-step RK4 trajectory of one grid.

    res, grid_L: the uniform grid; gamma, alpha: as in ``Solver.set_dynamics``
    (alpha is gamma * alpha_G); m0: (3n,) start state; t_seg: segment length
    (s); steps_per_segment: RK4 steps per field segment; sample_every: steps
    between samples of <m>; checkpoint_every: steps between stored states.
    """
    res: tuple
    grid_L: tuple
    gamma: float
    alpha: float
    m0: np.ndarray
    t_seg: float
    steps_per_segment: int
    sample_every: int
    checkpoint_every: int = 50
    A0: float = 1.3e-11
    K0: float = 0.0
    u_ea: np.ndarray | None = None
    solver: Solver | None = field(default=None, repr=False)

    def __post_init__(self):
        if self.solver is None:
            self.solver = Solver(self.res, self.grid_L, A0=self.A0, K0=self.K0, u_ea=self.u_ea)
            self.solver.assemble()
        self.n = self.solver.n

    @property
    def dt(self):
        return self.t_seg / self.steps_per_segment


class _Stepper:
    """RK4 steps of one problem for given segment fields and Ms."""

    def __init__(self, prob: TrajectoryProblem, hseg: np.ndarray, Ms: np.ndarray):
        self.p = prob
        self.s = prob.solver
        self.hseg = hseg
        self.seg = -1
        self.s.set_material(prob.A0, Ms, prob.K0, prob.u_ea)

    def set_segment(self, k):
        if k == self.seg:
            return
        p = self.p
        t0, t1 = k * p.t_seg, (k + 1) * p.t_seg
        h = self.hseg[k]
        self.s.set_dynamics(solver=2, gamma=p.gamma, alpha=p.alpha, hext=np.array([[t0, *h], [t1, *h]]))
        self.seg = k

    def step(self, k, m):
        """State after step k (t = k dt) from the state m at its start, and the stage inputs."""
        p = self.p
        self.set_segment(k // p.steps_per_segment)
        dt, t = p.dt, k * p.dt
        k1 = self.s.rhs(t, m)
        y2 = m + 0.5 * dt * k1
        k2 = self.s.rhs(t + 0.5 * dt, y2)
        y3 = m + 0.5 * dt * k2
        k3 = self.s.rhs(t + 0.5 * dt, y3)
        y4 = m + dt * k3
        k4 = self.s.rhs(t + dt, y4)
        return m + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4), (y2, y3, y4)

    def adjoint_step(self, k, m, lam, ghs, gms):
        """Cotangent of the state at the start of step k from lam at its end; adds the
        segment-field and Ms cotangents of the step to ghs and gms."""
        p = self.p
        n = p.n
        dt, t = p.dt, k * p.dt
        _, (y2, y3, y4) = self.step(k, m)
        mu4, he4, s4 = self.s.rhs_vjp(t + dt, y4, (dt / 6.0) * lam)
        mu3, he3, s3 = self.s.rhs_vjp(t + 0.5 * dt, y3, (dt / 3.0) * lam + dt * mu4)
        mu2, he2, s2 = self.s.rhs_vjp(t + 0.5 * dt, y2, (dt / 3.0) * lam + 0.5 * dt * mu3)
        mu1, he1, s1 = self.s.rhs_vjp(t, m, (dt / 6.0) * lam + 0.5 * dt * mu2)
        seg = k // p.steps_per_segment
        ghs[seg] -= (he1 + he2 + he3 + he4).reshape(3, n).sum(dim=1)
        gms += s1 + s2 + s3 + s4
        return lam + mu1 + mu2 + mu3 + mu4


class LLTrajectory(torch.autograd.Function):
    """<m>(t) samples of a fixed-step RK4 trajectory; differentiable in the segment
    fields (S, 3) [A/m] and the per-cell Ms (n,) [A/m]."""

    @staticmethod
    def forward(ctx, hseg, Ms, prob: TrajectoryProblem):
        S = hseg.shape[0]
        N = S * prob.steps_per_segment
        st = _Stepper(prob, hseg.detach().cpu().numpy(), Ms.detach().cpu().numpy())
        dev = prob.solver.device
        m = torch.as_tensor(np.asarray(prob.m0, dtype=np.float64).reshape(-1), device=dev).clone()
        n = prob.n
        ckpts = {}
        samples = []
        for k in range(N):
            if k % prob.checkpoint_every == 0:
                ckpts[k] = m.clone()
            m, _ = st.step(k, m)
            if (k + 1) % prob.sample_every == 0:
                samples.append(m.reshape(3, n).mean(dim=1))
        ctx.prob = prob
        ctx.ckpts = ckpts
        ctx.hseg = st.hseg
        ctx.Ms = Ms.detach().cpu().numpy()
        ctx.N = N
        return torch.stack(samples).to(hseg.device)

    @staticmethod
    def backward(ctx, gsamp):
        prob = ctx.prob
        n, N, C = prob.n, ctx.N, prob.checkpoint_every
        dev = prob.solver.device
        st = _Stepper(prob, ctx.hseg, ctx.Ms)
        g = gsamp.to(dev, torch.float64)
        lam = torch.zeros(3 * n, dtype=torch.float64, device=dev)
        ghs = torch.zeros((ctx.hseg.shape[0], 3), dtype=torch.float64, device=dev)
        gms = torch.zeros(n, dtype=torch.float64, device=dev)
        for k0 in sorted(ctx.ckpts, reverse=True):
            k1 = min(N, k0 + C)
            states = [ctx.ckpts[k0]]
            for k in range(k0, k1 - 1):
                states.append(st.step(k, states[-1])[0])
            for k in range(k1 - 1, k0 - 1, -1):
                if (k + 1) % prob.sample_every == 0:
                    j = (k + 1) // prob.sample_every - 1
                    lam = lam + (g[j][:, None] / n).expand(3, n).reshape(-1)
                lam = st.adjoint_step(k, states[k - k0], lam, ghs, gms)
        return ghs.to(gsamp.device), gms.to(gsamp.device), None


def mean_m_trajectory(hseg: torch.Tensor, Ms: torch.Tensor, prob: TrajectoryProblem) -> torch.Tensor:
    """Samples of <m>(t), shape (steps / sample_every, 3), differentiable in hseg and Ms."""
    return LLTrajectory.apply(hseg, Ms, prob)
