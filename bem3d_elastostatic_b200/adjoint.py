"""Shape and material sensitivities by the adjoint method (no counterpart in the
reference).

``BEMSolve`` is a ``torch.autograd.Function``: its forward runs the FP64 GPU path
(geometry, ghmat8, FP64 LU) for node coordinates X (n, 3) and the material (mu, nu)
and returns the solution x of A(X) x = FI(X); its backward, given dL/dx, solves
A^T lambda = dL/dx with the same LU factors (``bem_solve_transposed``) and returns
lambda^T (dFI/dX - dA/dX x) and the same for mu and nu from the backward-assembly
kernels (``bem_adjoint_gradient``), without forming dA/dX.  Any scalar objective
written in torch on top of x gets its gradient through autograd, the explicit
dependence on X included.

``compliance`` is the objective of the hollow-sphere workload: J = integral of t . u
over a set of elements (6 x 6 Gauss points), with u and t reorganized from x as
reorganize_solution does (io_mod.f90:148-183).  ``compliance_gradient`` returns J and
its gradient.
"""
from __future__ import annotations

from typing import Iterable, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .api import Quadesth
from .mesh import Mesh

_GI = [0.238619186083197, -0.238619186083197, 0.661209386466265,
       -0.661209386466265, 0.932469514203152, -0.932469514203152]
_OME = [0.467913934572691, 0.467913934572691, 0.360761573048139,
        0.360761573048139, 0.171324492379170, 0.171324492379170]


def _shape9(g1: torch.Tensor, g2: torch.Tensor):
    f = torch.stack([0.25 * g1 * g2 * (g1 - 1) * (g2 - 1), 0.5 * (1 - g1 * g1) * g2 * (g2 - 1),
                     0.25 * g1 * g2 * (g1 + 1) * (g2 - 1), 0.5 * g1 * (g1 + 1) * (1 - g2 * g2),
                     0.25 * g1 * g2 * (g1 + 1) * (g2 + 1), 0.5 * (1 - g1 * g1) * g2 * (g2 + 1),
                     0.25 * g1 * g2 * (g1 - 1) * (g2 + 1), 0.5 * g1 * (g1 - 1) * (1 - g2 * g2),
                     (1 - g1 * g1) * (1 - g2 * g2)], -1)
    d1 = torch.stack([0.25 * g2 * (g2 - 1) * (2 * g1 - 1), -g1 * g2 * (g2 - 1),
                      0.25 * g2 * (g2 - 1) * (2 * g1 + 1), 0.5 * (1 - g2 * g2) * (2 * g1 + 1),
                      0.25 * g2 * (g2 + 1) * (2 * g1 + 1), -g1 * g2 * (g2 + 1),
                      0.25 * g2 * (g2 + 1) * (2 * g1 - 1), 0.5 * (1 - g2 * g2) * (2 * g1 - 1),
                      -2 * g1 * (1 - g2 * g2)], -1)
    d2 = torch.stack([0.25 * g1 * (g1 - 1) * (2 * g2 - 1), 0.5 * (1 - g1 * g1) * (2 * g2 - 1),
                      0.25 * g1 * (g1 + 1) * (2 * g2 - 1), -g1 * g2 * (g1 + 1),
                      0.25 * g1 * (g1 + 1) * (2 * g2 + 1), 0.5 * (1 - g1 * g1) * (2 * g2 + 1),
                      0.25 * g1 * (g1 - 1) * (2 * g2 + 1), -g1 * g2 * (g1 - 1),
                      -2 * g2 * (1 - g1 * g1)], -1)
    return f, d1, d2


class BEMSolve(torch.autograd.Function):
    """x = A(X, mu, nu)^{-1} FI(X, mu, nu) on the GPU, with the adjoint backward."""

    @staticmethod
    def forward(ctx, X: torch.Tensor, mu: torch.Tensor, nu: torch.Tensor, q: Quadesth):
        m = q.mesh
        Xn = X.detach().to("cpu", torch.float64).numpy()
        m.x[:] = Xn[:, 0]
        m.y[:] = Xn[:, 1]
        m.z[:] = Xn[:, 2]
        m.mu = float(mu)
        m.nu = float(nu)
        q.load_mesh()
        q.precompute_element_geometry()
        q.ghmat8()
        x = q.solve_linear_system("fp64")
        ctx.q = q
        return torch.as_tensor(x, dtype=torch.float64, device=X.device)

    @staticmethod
    def backward(ctx, gx: torch.Tensor):
        q = ctx.q
        L, h = q.ctx.L, q.ctx.h
        lam = np.ascontiguousarray(gx.detach().to("cpu", torch.float64).numpy())
        q.ctx.check(L.bem_solve_transposed(h, _lib.ptr(lam)), "solve_transposed")
        g = np.zeros(q.mesh.ndof)
        gm = np.zeros(2)
        q.ctx.check(L.bem_adjoint_gradient(h, _lib.ptr(lam), _lib.ptr(g), _lib.ptr(gm)), "adjoint_gradient")
        dev = gx.device
        gX = torch.as_tensor(g.reshape(-1, 3), dtype=torch.float64, device=dev)
        return gX, torch.tensor(gm[0], dtype=torch.float64, device=dev), \
            torch.tensor(gm[1], dtype=torch.float64, device=dev), None


def _known_values(mesh: Mesh):
    """u known per dof (first element prescribing it, as the column swap) and its value."""
    N = mesh.ndof
    uk = np.zeros(N, dtype=bool)
    vp = np.zeros(N)
    order = [[] for _ in range(mesh.n)]
    for e in range(mesh.ne):
        for k in range(int(mesh.nconec[e])):
            order[mesh.kconec[k, e] - 1].append((e, k))
    for i in range(mesh.n):
        for ld in range(3):
            for e, k in order[i][:8]:
                if mesh.kode[3 * e + ld] == 0:
                    uk[3 * i + ld] = True
                    vp[3 * i + ld] = mesh.bc[3 * k + ld, e]
                    break
    return uk, vp


def reorganize(mesh: Mesh, x: torch.Tensor, mu: torch.Tensor):
    """u (3n) and t (ne, 9, 3) from x as io_mod.f90:148-183, differentiable in x and mu."""
    uk, vp = _known_values(mesh)
    dev = x.device
    u = torch.where(torch.as_tensor(uk, device=dev), torch.as_tensor(vp, device=dev), x)
    kc = torch.as_tensor(np.asarray(mesh.kconec).T - 1, dtype=torch.long, device=dev)  # (ne, 9)
    xe = x.reshape(-1, 3)[kc]  # (ne, 9, 3)
    kode = torch.as_tensor(np.asarray(mesh.kode).reshape(mesh.ne, 1, 3) == 0, device=dev)
    bc = torch.as_tensor(np.asarray(mesh.bc).T.reshape(mesh.ne, 9, 3), dtype=torch.float64, device=dev)
    t = torch.where(kode, mu * xe, bc)
    return u, t


def compliance(mesh: Mesh, X: torch.Tensor, u: torch.Tensor, t: torch.Tensor, elements) -> torch.Tensor:
    """J = sum over `elements` of the integral of t . u (quad9, 6 x 6 Gauss points)."""
    dev = X.device
    g1 = torch.tensor([_GI[i] for i in range(6) for j in range(6)], dtype=torch.float64, device=dev)
    g2 = torch.tensor([_GI[j] for i in range(6) for j in range(6)], dtype=torch.float64, device=dev)
    w = torch.tensor([_OME[i] * _OME[j] for i in range(6) for j in range(6)], dtype=torch.float64, device=dev)
    f, d1, d2 = _shape9(g1, g2)
    el = torch.as_tensor(np.asarray(list(elements), dtype=np.int64), device=dev)
    kc = torch.as_tensor(np.asarray(mesh.kconec).T - 1, dtype=torch.long, device=dev)[el]
    Xe = X[kc]
    a1 = torch.einsum("qk,ekd->eqd", d1, Xe)
    a2 = torch.einsum("qk,ekd->eqd", d2, Xe)
    J = torch.linalg.norm(torch.cross(a1, a2, dim=-1), dim=-1)
    uq = torch.einsum("qk,ekd->eqd", f, u.reshape(-1, 3)[kc])
    tq = torch.einsum("qk,ekd->eqd", f, t[el])
    return ((uq * tq).sum(-1) * J * w).sum()


def compliance_gradient(mesh: Mesh, elements: Iterable[int], device: int = 0,
                        q: Optional[Quadesth] = None) -> Tuple[float, np.ndarray, float, float]:
    """J and dJ/dX (n, 3), dJ/dmu, dJ/dnu (mu and nu independent) at the mesh's state."""
    q = q or Quadesth(mesh, device=device)
    X = torch.tensor(np.stack([mesh.x, mesh.y, mesh.z], 1), dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(float(mesh.mu), dtype=torch.float64, requires_grad=True)
    nu = torch.tensor(float(mesh.nu), dtype=torch.float64, requires_grad=True)
    x = BEMSolve.apply(X, mu, nu, q)
    u, t = reorganize(mesh, x, mu)
    J = compliance(mesh, X, u, t, elements)
    J.backward()
    return float(J.detach()), X.grad.numpy().copy(), float(mu.grad), float(nu.grad)
