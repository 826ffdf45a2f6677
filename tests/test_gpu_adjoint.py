"""Adjoint shape and material gradients (bem3d_elastostatic_b200.adjoint) of the
inner-surface compliance of the hollow sphere: against autograd through the pure
PyTorch FP64 restatement of the discrete system (oracle/torch_bem.py) and against
central finite differences of the GPU solve; the GPU solution against the Lame
solution."""
import numpy as np
import pytest
import torch

import torch_bem as TB
from bem3d_elastostatic_b200.mesh import hollow_sphere, lame_sphere_displacement

pytestmark = pytest.mark.gpu


def _reference_gradient(mesh, inner):
    S = TB.System(mesh)
    X = torch.tensor(np.stack([mesh.x, mesh.y, mesh.z], 1), requires_grad=True)
    mu = torch.tensor(float(mesh.mu), dtype=torch.float64, requires_grad=True)
    nu = torch.tensor(float(mesh.nu), dtype=torch.float64, requires_grad=True)
    J, _ = S.objective(X, mu, nu, inner)
    J.backward()
    return float(J.detach()), X.grad.numpy(), float(mu.grad), float(nu.grad)


def test_adjoint_matches_autograd_reference():
    from bem3d_elastostatic_b200.adjoint import compliance_gradient

    mesh = hollow_sphere(1, nu=0.3)
    inner = list(range(mesh.ne // 2, mesh.ne))
    Jr, gXr, gmur, gnur = _reference_gradient(hollow_sphere(1, nu=0.3), inner)
    J, gX, gmu, gnu = compliance_gradient(mesh, inner)
    assert abs(J - Jr) <= 1e-10 * abs(Jr)
    scale = np.abs(gXr).max()
    assert np.abs(gX - gXr).max() <= 1e-8 * scale, np.abs(gX - gXr).max() / scale
    assert abs(gmu - gmur) <= 1e-8 * abs(gmur)
    assert abs(gnu - gnur) <= 1e-8 * abs(gnur)


def test_adjoint_matches_finite_differences():
    from bem3d_elastostatic_b200.adjoint import compliance_gradient
    from bem3d_elastostatic_b200.api import Quadesth

    mesh = hollow_sphere(2, nu=0.3)
    inner = list(range(mesh.ne // 2, mesh.ne))
    inner_nodes = np.unique(mesh.kconec[:, inner].ravel() - 1)
    q = Quadesth(mesh)
    J0, gX, gmu, gnu = compliance_gradient(mesh, inner, q=q)
    X0 = np.stack([mesh.x, mesh.y, mesh.z], 1).copy()
    mu0, nu0 = mesh.mu, mesh.nu

    def J_at(X=None, mu=None, nu=None):
        from bem3d_elastostatic_b200.adjoint import compliance, reorganize

        Xv = X0 if X is None else X
        mesh.x[:], mesh.y[:], mesh.z[:] = Xv[:, 0], Xv[:, 1], Xv[:, 2]
        mesh.mu = mu0 if mu is None else mu
        mesh.nu = nu0 if nu is None else nu
        q.load_mesh()
        q.precompute_element_geometry()
        q.ghmat8()
        # the objective from the refined FP64 solve (FP64 rounding of the stored system):
        # the central difference then carries ~1e-10 of rounding, not the LU's ~1e-13 / h
        x = torch.as_tensor(q.solve_linear_system("fp64-ir", tol=1e-15, max_iter=20))
        u, t = reorganize(mesh, x, torch.tensor(mesh.mu, dtype=torch.float64))
        return float(compliance(mesh, torch.as_tensor(Xv), u, t, inner))

    h = 1e-6
    rng = np.random.default_rng(3)
    for node in rng.choice(inner_nodes, size=6, replace=False):
        for d in range(3):
            Xp, Xm = X0.copy(), X0.copy()
            Xp[node, d] += h
            Xm[node, d] -= h
            fd = (J_at(X=Xp) - J_at(X=Xm)) / (2 * h)
            # per entry at 1e-6 (entries below 1e-3 of the largest at 1e-6 of the largest)
            assert abs(fd - gX[node, d]) <= 1e-6 * max(abs(gX[node, d]), 1e-3 * np.abs(gX).max()), (
                node, d, fd, gX[node, d])
    fd_nu = (J_at(nu=nu0 + h) - J_at(nu=nu0 - h)) / (2 * h)
    assert abs(fd_nu - gnu) <= 1e-6 * abs(gnu)
    fd_mu = (J_at(mu=mu0 + h) - J_at(mu=mu0 - h)) / (2 * h)
    assert abs(fd_mu - gmu) <= 1e-6 * abs(gmu)
    q.close()


def test_transposed_solve():
    """A^T y = g with the factors of the FP64 solve."""
    from bem3d_elastostatic_b200 import _lib
    from bem3d_elastostatic_b200.api import Quadesth

    mesh = hollow_sphere(2, nu=0.3)
    q = Quadesth(mesh)
    q.precompute_element_geometry()
    A, _ = q.ghmat8(return_system=True)
    q.solve_linear_system("fp64")
    g = np.random.default_rng(0).standard_normal(mesh.ndof)
    y = g.copy()
    q.ctx.check(q.ctx.L.bem_solve_transposed(q.ctx.h, _lib.ptr(y)), "solve_transposed")
    ref = np.linalg.solve(A.T, g)
    assert np.abs(y - ref).max() <= 1e-10 * np.abs(ref).max()
    q.close()


def test_lame_sphere_radial_displacement():
    """The GPU solution converges to the Lame solution: the discretisation error at
    4 x 4 elements per cube face is below half the one at 2 x 2, and below 0.3 %."""
    from bem3d_elastostatic_b200.api import Quadesth

    errs = []
    for m in (2, 4):
        mesh = hollow_sphere(m, nu=0.3)
        q = Quadesth(mesh)
        res = q.run("fp64")
        X = np.stack([mesh.x, mesh.y, mesh.z], 1)
        r = np.linalg.norm(X, axis=1)
        ur = (res["u"].reshape(-1, 3) * X).sum(1) / r
        young = 2 * mesh.mu * (1 + mesh.nu)
        exact = lame_sphere_displacement(r, 1.0, 2.0, 1.0, young, mesh.nu)
        errs.append(np.abs(ur - exact).max() / np.abs(exact).max())
        q.close()
    assert errs[1] < 0.5 * errs[0], errs
    assert errs[1] < 3e-3, errs
