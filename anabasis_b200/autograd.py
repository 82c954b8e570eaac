"""torch.autograd wrapper of the steady patch-force objective (used by the tests).

SteadyForce.apply(inlet, mu, problem) returns J = dir . F(U, p) on the converged state for the
inlet-face Dirichlet velocities `inlet` (3 x nInlet, float64) and viscosity `mu` (0-d float64).
The forward pass re-converges the library's SIMPLE state (SIMPLE steps, then Newton); the backward
pass is the library's discrete adjoint (anb_adjoint_force_grad), which needs only the converged
state kept in the context, not the iteration history.  torch is only the autograd host here:
every number comes from libanb.so.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import Solver


@dataclass
class SteadyForceProblem:
    solver: Solver
    bc: dict                      # boundary values as returned by HostMesh.evaluate_bc
    inlet_faces: np.ndarray       # face indices of the parameter (inlet) faces
    patch: int                    # patch of the force integral
    direction: tuple = (1.0, 0.0, 0.0)
    normal_sign: int = -1
    simple_steps: int = 200
    newton_tol: float = 1e-13
    last: dict = field(default_factory=dict)


class SteadyForce(torch.autograd.Function):
    @staticmethod
    def forward(ctx, inlet: torch.Tensor, mu: torch.Tensor, problem: SteadyForceProblem) -> torch.Tensor:
        s = problem.solver
        b = dict(problem.bc)
        vals = inlet.detach().cpu().numpy().astype(np.float64)
        for q, k in enumerate("uvw"):
            arr = np.array(problem.bc[k], np.float64)
            arr[problem.inlet_faces] = vals[q]
            b[k] = arr
        s.set_bc(b)
        s.set_viscosity(float(mu))
        s.iterate(problem.simple_steps, 1e-12, 1e-10)
        info = s.newton_solve(max_newton=10, tol=problem.newton_tol)
        J, _ = s.force_objective(problem.patch, problem.direction, problem.normal_sign)
        problem.last = dict(newton=info, J=J)
        ctx.problem = problem
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ: torch.Tensor):
        p = ctx.problem
        g, gmu, _, info = p.solver.adjoint_force_grad(p.patch, p.direction, p.normal_sign)
        F = p.solver.n_faces
        gi = np.stack([g[q * F + p.inlet_faces] for q in range(3)])
        p.last["adjoint"] = info
        scale = float(gJ)
        return torch.from_numpy(gi * scale), torch.tensor(gmu * scale, dtype=torch.float64), None
