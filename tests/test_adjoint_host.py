"""CPU checks of the Python layer around the adjoint solve.

`adjoint.reorganize` restates reorganize_solution (io_mod.f90:148-183) on torch tensors, and
`adjoint.compliance` is the objective of the hollow-sphere workload. Both run on whatever
device their inputs live on, so they are checked here on CPU tensors against the pure-PyTorch
FP64 restatement of the discrete system (oracle/torch_bem.py): values and autograd gradients.
"""
import numpy as np
import torch

import torch_bem as TB
from bem3d_elastostatic_b200.adjoint import compliance, reorganize
from bem3d_elastostatic_b200.mesh import hollow_sphere


def test_reorganize_and_compliance_match_torch_restatement():
    mesh = hollow_sphere(1, nu=0.3)
    S = TB.System(mesh)
    rng = np.random.default_rng(5)
    x = torch.tensor(rng.standard_normal(mesh.ndof), requires_grad=True)
    mu = torch.tensor(float(mesh.mu), dtype=torch.float64, requires_grad=True)
    X = torch.tensor(np.stack([mesh.x, mesh.y, mesh.z], 1), requires_grad=True)
    inner = list(range(mesh.ne // 2, mesh.ne))

    u1, t1 = reorganize(mesh, x, mu)
    u2, t2 = S.reorganize(x, mu)
    assert torch.equal(u1, u2)
    assert torch.equal(t1.reshape(-1), t2)  # (element, node, component) order

    J1 = compliance(mesh, X, u1, t1, inner)
    J2 = S.compliance(X, u2, t2, inner)
    assert abs(float(J1) - float(J2)) <= 1e-13 * abs(float(J2))

    # mu may not enter J (tractions prescribed on the integrated surface): unused -> 0
    ins = (X, x, mu)
    g1 = torch.autograd.grad(J1, ins, allow_unused=True)
    g2 = torch.autograd.grad(J2, ins, allow_unused=True)
    for a, b, v in zip(g1, g2, ins):
        a = torch.zeros_like(v) if a is None else a
        b = torch.zeros_like(v) if b is None else b
        scale = max(float(b.abs().max()), 1e-300)
        assert float((a - b).abs().max()) <= 1e-12 * scale
