"""Pivoting modes and failure detection on the GPU, through the C ABI.

* Window pivoting (the default of the mixed-precision modes: each 32-wide sub-panel's
  pivot search restricted to its 32 x 32 diagonal block) and partial pivoting give
  solutions within 1e-10 of the oracle's LAPACK solve; the solve reports which one
  produced its solution.
* Failures the host can construct return a status and leave the context usable, with
  no GPU fault: a triangular sweep whose publication of one block is withheld runs
  into the context's wait limit (BEM_ERR_TIMEOUT); a node in more than 8 elements
  (io_mod.f90:125-135, BEM_ERR_MESH); a non-finite coordinate (BEM_ERR_ARG); a
  degenerate element whose Jacobian is zero, the division of assembly_mod.f90:331-334
  (BEM_ERR_MESH).
"""
import numpy as np
import pytest

import oracle as O
from bem3d_elastostatic_b200 import _lib
from bem3d_elastostatic_b200.mesh import Mesh, cube_grid_points, uniaxial_cube

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cube8_ref(cube8_mesh):
    return O.Oracle(cube8_mesh).run()


@pytest.mark.parametrize("panel_width", [0, 512, 1024])
@pytest.mark.parametrize("pivoting", [_lib.BEM_PIVOT_WINDOW, _lib.BEM_PIVOT_PARTIAL])
@pytest.mark.parametrize("precision", ["fp32-ir", "bf16-ir"])
def test_pivoting_modes_vs_oracle(pivoting, precision, panel_width, cube8_mesh, cube8_ref):
    """Both pivotings, both mixed modes, the modes' own panel widths and both explicit
    ones (4,614 DOF: 9 or 4 full panels and a partial last one)."""
    from bem3d_elastostatic_b200.api import Quadesth

    q = Quadesth(cube8_mesh)
    q.set_option(_lib.BEM_OPT_PIVOTING, pivoting)
    q.set_option(_lib.BEM_OPT_PANEL_WIDTH, panel_width)
    q.precompute_element_geometry()
    q.ghmat8()
    x = q.solve_linear_system(precision, tol=1e-15, max_iter=60)
    err = np.abs(x - cube8_ref["x"]).max() / np.abs(cube8_ref["x"]).max()
    assert err <= 1e-10, err
    assert q.solve_info["pivoting"] == pivoting
    assert q.solve_info["fallbacks"] == 0
    q.close()


def test_window_pivoting_falls_back_on_a_zero_window_pivot():
    """A nonsingular system whose leading 32 x 32 block is zero: the window-pivoted
    factorisation meets an exact zero pivot in its first window, the solve repeats with
    partial pivoting, reports the fallback, and still meets the FP64 bar."""
    from bem3d_elastostatic_b200.api import solve_system

    rng = np.random.default_rng(5)
    n = 300
    M = 0.1 * rng.standard_normal((n, n)) / np.sqrt(n) + np.eye(n)
    A = M.copy()
    A[[*range(32), *range(32, 64)]] = M[[*range(32, 64), *range(32)]]  # swap row blocks
    A[:32, :32] = 0.0
    b = rng.standard_normal(n)
    x_ref = np.linalg.solve(A, b)
    for precision in ("fp32-ir", "bf16-ir"):
        x, info = solve_system(A, b, precision, tol=1e-15, max_iter=60)
        assert info["pivoting"] == _lib.BEM_PIVOT_PARTIAL and info["fallbacks"] == 1
        assert np.abs(x - x_ref).max() <= 1e-10 * np.abs(x_ref).max()
    # the same system with partial pivoting requested: no fallback needed
    x, info = solve_system(A, b, "fp32-ir", tol=1e-15, max_iter=60, pivoting=_lib.BEM_PIVOT_PARTIAL)
    assert info["fallbacks"] == 0
    assert np.abs(x - x_ref).max() <= 1e-10 * np.abs(x_ref).max()


def test_wait_limit_runs_out_on_a_withheld_block(cube8_mesh, cube8_ref):
    from bem3d_elastostatic_b200.api import Quadesth

    q = Quadesth(cube8_mesh)
    q.precompute_element_geometry()
    q.ghmat8()
    q.set_option(_lib.BEM_OPT_WAIT_LIMIT_MS, 200)
    q.set_option(_lib.BEM_OPT_WITHHOLD_BLOCK, 0)
    with pytest.raises(_lib.BemError) as exc:
        q.solve_linear_system("fp32-ir", tol=1e-15, max_iter=60)
    assert exc.value.code == _lib.BEM_ERR_TIMEOUT
    # the context is still usable: the same solve without the injection succeeds
    q.set_option(_lib.BEM_OPT_WITHHOLD_BLOCK, -1)
    q.set_option(_lib.BEM_OPT_WAIT_LIMIT_MS, 2000)
    x = q.solve_linear_system("fp32-ir", tol=1e-15, max_iter=60)
    assert np.abs(x - cube8_ref["x"]).max() <= 1e-10 * np.abs(cube8_ref["x"]).max()
    q.close()


def test_set_option_rejects_bad_values():
    ctx = _lib.Context(0)
    L, h = ctx.L, ctx.h
    assert L.bem_set_option(h, _lib.BEM_OPT_PIVOTING, 7) == _lib.BEM_ERR_ARG
    assert L.bem_set_option(h, _lib.BEM_OPT_WAIT_LIMIT_MS, 0) == _lib.BEM_ERR_ARG
    assert L.bem_set_option(h, _lib.BEM_OPT_WAIT_LIMIT_MS, 60001) == _lib.BEM_ERR_ARG
    assert L.bem_set_option(h, 99, 0) == _lib.BEM_ERR_ARG
    for bad in (64, 100, 1152, -128):
        assert L.bem_set_option(h, _lib.BEM_OPT_PANEL_WIDTH, bad) == _lib.BEM_ERR_ARG
    assert L.bem_set_option(h, _lib.BEM_OPT_PANEL_WIDTH, 768) == 0
    assert L.bem_set_option(h, _lib.BEM_OPT_WAIT_LIMIT_MS, 500) == 0
    ctx.close()


def _raw_mesh(ctx, x, y, z, nconec, kconec):
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    nconec = np.ascontiguousarray(nconec, dtype=np.int32)
    kconec = np.asfortranarray(kconec, dtype=np.int32)
    return ctx.L.bem_set_mesh(ctx.h, x.size, nconec.size, _lib.ptr(x), _lib.ptr(y), _lib.ptr(z),
                              _lib.ptr(nconec), _lib.ptr(kconec))


def _solve_cube2_on(ctx):
    """The context still runs a whole small case correctly after a rejected input."""
    from bem3d_elastostatic_b200.api import Quadesth

    mesh = uniaxial_cube(2, young=1.0, nu=0.3, points=cube_grid_points([0.5]))
    ref = O.Oracle(mesh).run()
    res = Quadesth(mesh, ctx=ctx).run()
    assert np.abs(res["x"] - ref["x"]).max() <= 1e-10 * np.abs(ref["x"]).max()


def test_node_in_nine_elements_is_rejected():
    ctx = _lib.Context(0)
    # nine quad9 elements that all contain node 1 (a fan around it)
    n = 1 + 9 * 8
    rng = np.random.default_rng(3)
    xyz = rng.standard_normal((3, n))
    kconec = np.zeros((9, 9), dtype=np.int32)
    for e in range(9):
        kconec[0, e] = 1
        kconec[1:, e] = 2 + 8 * e + np.arange(8)
    rc = _raw_mesh(ctx, *xyz, np.full(9, 9), kconec)
    assert rc == _lib.BEM_ERR_MESH
    assert b"more than 8" in ctx.L.bem_last_error(ctx.h)
    _solve_cube2_on(ctx)
    ctx.close()


def test_non_finite_coordinate_is_rejected():
    ctx = _lib.Context(0)
    mesh = uniaxial_cube(2)
    x = mesh.x.copy()
    x[5] = np.nan
    rc = _raw_mesh(ctx, x, mesh.y, mesh.z, mesh.nconec, mesh.kconec)
    assert rc == _lib.BEM_ERR_ARG
    x[5] = np.inf
    assert _raw_mesh(ctx, x, mesh.y, mesh.z, mesh.nconec, mesh.kconec) == _lib.BEM_ERR_ARG
    _solve_cube2_on(ctx)
    ctx.close()


def test_zero_area_element_is_rejected():
    from bem3d_elastostatic_b200.api import Quadesth

    ctx = _lib.Context(0)
    mesh = uniaxial_cube(2)
    # collapse element 0 onto its first node: every Jacobian of it is zero
    x, y, z = mesh.x.copy(), mesh.y.copy(), mesh.z.copy()
    nodes = mesh.kconec[:, 0] - 1
    x[nodes], y[nodes], z[nodes] = x[nodes[0]], y[nodes[0]], z[nodes[0]]
    bad = Mesh(x, y, z, mesh.nconec, mesh.kconec, mesh.kode, mesh.bc, mesh.mu, mesh.nu, pins=mesh.pins)
    q = Quadesth(bad, ctx=ctx)
    with pytest.raises(_lib.BemError) as exc:
        q.precompute_element_geometry()
    assert exc.value.code == _lib.BEM_ERR_MESH
    with pytest.raises(_lib.BemError) as exc:  # and assembly refuses to run without geometry
        q.ghmat8()
    assert exc.value.code == _lib.BEM_ERR_STATE
    _solve_cube2_on(ctx)
    ctx.close()
