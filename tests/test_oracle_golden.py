"""Pins the CPU oracle to the reference's own shipped output.

internal_points.dat is the reference's result for cube8.dat (6 m cube, 866 nodes,
216 quad9, 1965 internal points), printed as E15.7 (stress_mod.f90:926-932).  The
oracle must reproduce every printed value to within half a unit of its last printed
digit, plus a noise floor of 1e-12 x the largest displacement (or stress) for entries
whose exact value is zero (shear stresses, lateral displacements: pure cancellation noise).
"""
import numpy as np
import pytest


def half_ulp_e15_7(v):
    e = np.floor(np.log10(np.maximum(np.abs(v), 1e-300))) + 1
    return 0.5 * 10.0 ** (e - 7)


def test_reader_cube8(cube8_mesh):
    m = cube8_mesh
    assert (m.n, m.ne, m.l, m.ntrack) == (866, 216, 1965, 770)
    assert m.mu == 1.0e6 and m.nu == 0.25
    assert m.max_elements_per_node() <= 8
    assert np.all(m.nconec == 9)
    # preproc.py:21-52: top face t_z = 100, bottom u_z prescribed
    assert np.isclose(m.bc.max(), 100.0)


def test_oracle_matches_reference_internal_points(cube8_oracle_solution, cube8_golden):
    _, res = cube8_oracle_solution
    got = np.concatenate([res["u_int"].T, res["sigma"].T, res["vm"][:, None], res["prin"].T], 1)
    ref = cube8_golden[:, 4:]
    assert got.shape == ref.shape
    # noise floor per quantity group: displacements by max |u|, stresses by max |sigma|
    scale = np.empty(13)
    scale[:3] = np.abs(ref[:, :3]).max()
    scale[3:] = np.abs(ref[:, 3:]).max()
    tol = half_ulp_e15_7(ref) + 1e-12 * scale[None, :]
    err = np.abs(got - ref)
    worst = (err / tol).max()
    assert worst <= 1.0, f"worst error / tolerance = {worst}"


def test_oracle_coordinates_roundtrip(cube8_mesh, cube8_golden):
    m = cube8_mesh
    pts = np.stack([m.cx, m.cy, m.cz], 1)
    assert np.all(np.abs(pts - cube8_golden[:, 1:4]) <= half_ulp_e15_7(cube8_golden[:, 1:4]) + 1e-15)


def test_oracle_readme_figures(cube8_oracle_solution, cube8_golden):
    """readme.md:271-301: node 770 u_z = 1.999998e-4 m, top traction 100."""
    orc, res = cube8_oracle_solution
    u770 = res["u"][3 * 769 + 2]
    assert abs(u770 - 1.999998e-4) < 1e-10
    # analytic uniaxial strain: u_z = p z / M, M = 3e6 (readme.md:186-204)
    assert abs(u770 - 100.0 * 6.0 / 3.0e6) / 2e-4 < 1e-5
    # central point 1880 sigma_zz ~ 99.9999 (readme.md:292)
    assert abs(res["sigma"][2, 1879] - 99.9999) < 1e-3


def test_gauss_legendre_40():
    import oracle as O

    x, w = O.gauss_legendre(40)
    assert abs(w.sum() - 2.0) < 1e-13
    # exact for x^78 over [-1,1]
    assert abs((w * x**78).sum() - 2.0 / 79.0) < 1e-13


def test_principal_closed_form():
    import oracle as O

    p, vm = O.principal([33.0, 33.0, 100.0, 0.0, 0.0, 0.0])
    assert np.allclose(p, [100.0, 33.0, 33.0])
    assert abs(vm - 67.0) < 1e-12
    p, vm = O.principal([5.0, 5.0, 5.0, 0.0, 0.0, 0.0])
    assert np.allclose(p, 5.0) and vm == 0.0
