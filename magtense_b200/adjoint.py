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

Within a segment the right-hand side does not depend on time (the segment's
field is a constant table valid for every t), so one RK4 step, and one adjoint
step, is the same launch sequence for every step: with ``graphs=True`` each is
captured once into a CUDA graph and replayed, instead of being driven launch
by launch from Python.

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
    graphs: bool = True
    A0: float = 1.3e-11
    K0: float = 0.0
    u_ea: np.ndarray | None = None
    solver: Solver | None = field(default=None, repr=False)
    graph_cache: dict = field(default_factory=dict, repr=False)   # captured steps, reused across calls

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
        h = self.hseg[k]
        # constant over the whole time axis: the steps of the segment are time independent
        self.s.set_dynamics(solver=2, gamma=p.gamma, alpha=p.alpha, hext=np.array([[-1.0, *h], [1.0, *h]]))
        self.seg = k

    # -- one RK4 step and its adjoint, written once (the graphs capture these) --
    def _rk4(self, m):
        dt = self.p.dt
        k1 = self.s.rhs(0.0, m)
        y2 = m + 0.5 * dt * k1
        k2 = self.s.rhs(0.0, y2)
        y3 = m + 0.5 * dt * k2
        k3 = self.s.rhs(0.0, y3)
        y4 = m + dt * k3
        k4 = self.s.rhs(0.0, y4)
        return m + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4), (y2, y3, y4)

    def _adj(self, m, lam, ghe_acc, gms_acc):
        dt = self.p.dt
        _, (y2, y3, y4) = self._rk4(m)
        mu4, he4, s4 = self.s.rhs_vjp(0.0, y4, (dt / 6.0) * lam)
        mu3, he3, s3 = self.s.rhs_vjp(0.0, y3, (dt / 3.0) * lam + dt * mu4)
        mu2, he2, s2 = self.s.rhs_vjp(0.0, y2, (dt / 3.0) * lam + 0.5 * dt * mu3)
        mu1, he1, s1 = self.s.rhs_vjp(0.0, m, (dt / 6.0) * lam + 0.5 * dt * mu2)
        ghe_acc += he1 + he2 + he3 + he4
        gms_acc += s1 + s2 + s3 + s4
        return lam + mu1 + mu2 + mu3 + mu4

    def _capture(self, fn):
        """Warm up (allocations happen outside the capture), then capture fn into a graph."""
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            fn()
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            out = fn()
        return g, out

    def step(self, k, m):
        """State after step k from the state m at its start."""
        p = self.p
        self.set_segment(k // p.steps_per_segment)
        if not p.graphs:
            return self._rk4(m)[0]
        c = p.graph_cache
        if "fwd" not in c:
            f_in = m.clone()
            g, f_out = self._capture(lambda: self._rk4(f_in)[0])
            c["fwd"] = (g, f_in, f_out)
        g, f_in, f_out = c["fwd"]
        f_in.copy_(m)
        g.replay()
        return f_out.clone()

    def adjoint_step(self, k, m, lam, ghe_acc, gms_acc):
        """Cotangent of the state at the start of step k from lam at its end; adds the
        field cotangent of the step to ghe_acc (3n) and the Ms cotangent to gms_acc."""
        p = self.p
        self.set_segment(k // p.steps_per_segment)
        if not p.graphs:
            return self._adj(m, lam, ghe_acc, gms_acc)
        c = p.graph_cache
        if "adj" not in c:
            a_m, a_lam = m.clone(), lam.clone()
            a_he, a_ms = torch.zeros_like(ghe_acc), torch.zeros_like(gms_acc)
            g, a_out = self._capture(lambda: self._adj(a_m, a_lam, a_he, a_ms))
            c["adj"] = (g, a_m, a_lam, a_he, a_ms, a_out)
        g, a_m, a_lam, a_he, a_ms, a_out = c["adj"]
        a_he.zero_()
        a_ms.zero_()
        a_m.copy_(m)
        a_lam.copy_(lam)
        g.replay()
        ghe_acc += a_he
        gms_acc += a_ms
        return a_out.clone()


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
            m = st.step(k, m)
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
        ghe = torch.zeros(3 * n, dtype=torch.float64, device=dev)
        for k0 in sorted(ctx.ckpts, reverse=True):
            k1 = min(N, k0 + C)
            states = [ctx.ckpts[k0]]
            for k in range(k0, k1 - 1):
                states.append(st.step(k, states[-1]))
            for k in range(k1 - 1, k0 - 1, -1):
                if (k + 1) % prob.sample_every == 0:
                    j = (k + 1) // prob.sample_every - 1
                    lam = lam + (g[j][:, None] / n).expand(3, n).reshape(-1)
                lam = st.adjoint_step(k, states[k - k0], lam, ghe, gms)
                # the segment's field gradient: -sum over cells of its field cotangents
                if k % prob.steps_per_segment == 0:
                    ghs[k // prob.steps_per_segment] -= ghe.reshape(3, n).sum(dim=1)
                    ghe.zero_()
        return ghs.to(gsamp.device), gms.to(gsamp.device), None


def mean_m_trajectory(hseg: torch.Tensor, Ms: torch.Tensor, prob: TrajectoryProblem) -> torch.Tensor:
    """Samples of <m>(t), shape (steps / sample_every, 3), differentiable in hseg and Ms."""
    return LLTrajectory.apply(hseg, Ms, prob)
