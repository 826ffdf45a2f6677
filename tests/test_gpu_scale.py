"""Parity at the benchmark configurations' full sizes, through the C ABI.

* 73,734-DOF unit cube (32 x 32 quad9 per face; A is 43.5 GB) at nu = 0.0, 0.3 and
  0.49: sampled row blocks of A and FI against the oracle's ghmat8 rows (the
  entrywise bar of test_gpu_parity: 1e-12 of the row scale); the solutions of both
  mixed modes (FP32 window-pivoted LU with refinement, the equilibrated LU with one
  BF16 tensor-core product and GMRES-IR; double-double residuals) against
  the FP64 solution of the same stored system at 1e-10, the FP64 reference being the
  FP64 LU with the same extra-precise refinement (the plain FP64 LU solution differs
  from it by up to ~kappa 1e-16, ~1e-10 at these conditions, and is checked at 1e-8);
  the nodal displacements against the analytic uniaxial-stress field
  u = (-nu x, -nu y, z) / E (the discretisation error of the 32 x 32 mesh, below 1e-5
  of the displacement scale).
* 46,086-DOF clamped plate (10 x 10 x 1, E = 210e3, nu = 0.3, 3,840 quad9): sampled
  rows of A against the oracle, the plain FP64 GPU solve against the mixed solve at
  1e-10 with a backward error at FP64 level, and 500 of the 200 x 200 x 5 internal
  points against the oracle's Somigliana quadrature applied to the GPU's u and t
  (1e-10 of the displacement and stress scales).
The oracle cannot factor these matrices in test time; its assembly and its internal
points are exact restatements of the reference and are compared where they apply.
"""
import numpy as np
import pytest

import oracle as O
from bem3d_elastostatic_b200.mesh import clamped_plate, plate_grid_points, uniaxial_cube

pytestmark = pytest.mark.gpu


def close_entrywise(got, ref, rowrel=1e-12, bigrel=1e-10):
    rowmax = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
    err = np.abs(got - ref)
    worst_row = float((err / (rowrel * rowmax)).max())
    big = np.abs(ref) > 1e-3 * rowmax
    worst_big = float((err[big] / (bigrel * np.abs(ref[big]))).max()) if big.any() else 0.0
    return max(worst_row, worst_big)


def _row_blocks(n):
    """Collocation-node blocks: the first nodes (the pinned origin among them), a block
    in the middle of the numbering and the last nodes."""
    return [(0, 96), (n // 2, n // 2 + 64), (n - 64, n)]


@pytest.mark.parametrize("nu", [0.0, 0.3, 0.49])
def test_cube32_rows_solution_and_analytic(nu):
    from bem3d_elastostatic_b200.api import Quadesth

    mesh = uniaxial_cube(32, young=1.0, nu=nu)
    orc = O.Oracle(mesh)
    q = Quadesth(mesh)
    try:
        q.precompute_element_geometry()
        q.ghmat8()
        for in0, in1 in _row_blocks(mesh.n):
            A, F = q.system_rows(in0, in1)
            Ar, Fr = orc.ghmat8(in0, in1)
            assert close_entrywise(A, Ar) <= 1.0, (in0, in1)
            assert np.abs(F - Fr).max() <= 1e-12 * max(np.abs(Fr).max(), 1e-300), (in0, in1)
        x = q.solve_linear_system("fp32-ir", tol=1e-15, max_iter=60)
        info = dict(q.solve_info)
        u, _ = q.reorganize_solution()
        xb = q.solve_linear_system("bf16-ir", tol=1e-12, max_iter=60)
        info_b = dict(q.solve_info)
        xref = q.solve_linear_system("fp64-ir", tol=1e-15, max_iter=20)
        q.ghmat8()
        x64 = q.solve_linear_system("fp64")
        err = np.abs(x - xref).max() / np.abs(xref).max()
        assert err <= 1e-10, (nu, err, info)
        assert info["rel_residual"] <= 1e-14
        errb = np.abs(xb - xref).max() / np.abs(xref).max()
        assert errb <= 1e-10, (nu, errb, info_b)
        # the one-product factorisation is a good preconditioner: 7-10 GMRES iterations
        # at these conditions (a wrong trailing update would still converge, slowly)
        assert info_b["iterations"] <= 20, (nu, info_b)
        err64 = np.abs(x64 - xref).max() / np.abs(xref).max()
        assert err64 <= 1e-8, (nu, err64)
        P = mesh.node_coords()
        ua = np.stack([-nu * P[:, 0], -nu * P[:, 1], P[:, 2]], 1) / mesh.young
        uerr = np.abs(u.reshape(-1, 3) - ua).max() / np.abs(ua).max()
        assert uerr <= 1e-5, (nu, uerr)
    finally:
        q.close()


def test_plate40_rows_solution_and_internal_points():
    from bem3d_elastostatic_b200.api import Quadesth

    pts = plate_grid_points()
    rng = np.random.default_rng(20261203)
    sample = pts[np.sort(rng.choice(pts.shape[0], size=500, replace=False))]
    mesh = clamped_plate(points=sample)
    orc = O.Oracle(mesh)
    q = Quadesth(mesh)
    try:
        q.precompute_element_geometry()
        q.ghmat8()
        for in0, in1 in _row_blocks(mesh.n):
            A, F = q.system_rows(in0, in1)
            Ar, Fr = orc.ghmat8(in0, in1)
            assert close_entrywise(A, Ar) <= 1.0, (in0, in1)
            assert np.abs(F - Fr).max() <= 1e-12 * max(np.abs(Fr).max(), 1e-300), (in0, in1)
        xm = q.solve_linear_system("fp32-ir", tol=1e-15, max_iter=60)
        q.ghmat8()
        x = q.solve_linear_system("fp64")
        assert np.abs(xm - x).max() <= 1e-10 * np.abs(x).max()
        u, t = q.reorganize_solution()
        ug, sg, pg, vg = q.compute_internal_points()
        ur, sr, pr, vr = orc.internal_points(u, t)
        assert np.abs(ug - ur).max() <= 1e-10 * np.abs(ur).max()
        assert np.abs(sg - sr).max() <= 1e-10 * np.abs(sr).max()
        assert np.abs(vg - vr).max() <= 1e-10 * np.abs(vr).max()
    finally:
        q.close()
