"""Measure the adjoint on the hollow-sphere workload.

    python -m bem3d_elastostatic_b200.adjoint_bench --m 16 --fd 20

Thick sphere a = 1, b = 2 (cubed-sphere quad9 surfaces, m x m elements per cube face on
each surface: m = 16 gives 3,072 elements and 36,876 DOF), internal pressure 1, six
pinned DOFs.  Objective: the compliance J = integral over the inner surface of t . u.
Reports the time of the forward solve (geometry, assembly, FP64 LU) and of the
backward pass (transposed solve with the same factors, backward assembly), the
largest error of the radial displacement against Lame, and the relative error of the
adjoint gradient against FP64 central differences (step 1e-6) at --fd random
inner-surface coordinates and in nu.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from .adjoint import BEMSolve, compliance, reorganize
from .api import Quadesth
from .mesh import hollow_sphere, lame_sphere_displacement


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=16)
    ap.add_argument("--fd", type=int, default=20)
    ap.add_argument("--step", type=float, default=1e-6)
    args = ap.parse_args(argv)
    mesh = hollow_sphere(args.m, nu=0.3)
    inner = list(range(mesh.ne // 2, mesh.ne))
    q = Quadesth(mesh)
    X0 = np.stack([mesh.x, mesh.y, mesh.z], 1).copy()
    mu0, nu0 = float(mesh.mu), float(mesh.nu)

    def forward(Xv, mu, nu, grad=False):
        X = torch.tensor(Xv, dtype=torch.float64, requires_grad=grad)
        m_ = torch.tensor(mu, dtype=torch.float64, requires_grad=grad)
        n_ = torch.tensor(nu, dtype=torch.float64, requires_grad=grad)
        x = BEMSolve.apply(X, m_, n_, q)
        u, t = reorganize(mesh, x, m_)
        return compliance(mesh, X, u, t, inner), X, m_, n_, x

    forward(X0, mu0, nu0)  # warm-up
    t0 = time.perf_counter()
    J, X, mu, nu, x = forward(X0, mu0, nu0, grad=True)
    t1 = time.perf_counter()
    J.backward()
    t2 = time.perf_counter()
    g = X.grad.numpy().copy()
    gnu, gmu = float(nu.grad), float(mu.grad)
    r = np.linalg.norm(X0, axis=1)
    ur = (x.detach().numpy().reshape(-1, 3) * X0).sum(1) / r  # every node's dofs are unknown displacements
    exact = lame_sphere_displacement(r, 1.0, 2.0, 1.0, 2 * mu0 * (1 + nu0), nu0)
    res = {"workload": f"hollow sphere a=1 b=2, m={args.m}: {mesh.ne} quad9, {mesh.ndof} DOF",
           "J": float(J.detach()), "forward_s": t1 - t0, "backward_s": t2 - t1,
           "lame_ur_max_rel_err": float(np.abs(ur - exact).max() / np.abs(exact).max()),
           "dJ_dnu": gnu, "dJ_dmu": gmu}
    rng = np.random.default_rng(20261203)
    nodes = np.unique(mesh.kconec[:, inner].ravel() - 1)
    h = args.step
    errs = []
    with torch.no_grad():
        for _ in range(args.fd):
            i, d = int(rng.choice(nodes)), int(rng.integers(0, 3))
            Xp, Xm = X0.copy(), X0.copy()
            Xp[i, d] += h
            Xm[i, d] -= h
            fd = (float(forward(Xp, mu0, nu0)[0]) - float(forward(Xm, mu0, nu0)[0])) / (2 * h)
            errs.append(abs(fd - g[i, d]) / max(abs(fd), 1e-300))
        fdn = (float(forward(X0, mu0, nu0 + h)[0]) - float(forward(X0, mu0, nu0 - h)[0])) / (2 * h)
    res["fd_coordinates"] = args.fd
    res["fd_rel_err_max"] = float(max(errs)) if errs else None
    res["fd_rel_err_median"] = float(np.median(errs)) if errs else None
    res["fd_nu_rel_err"] = abs(fdn - gnu) / abs(fdn)
    print(json.dumps(res))
    q.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
