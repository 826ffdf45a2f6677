"""Result files in the reference's formats, so its post-processing (posproc.py) and
plots read GPU results unchanged.

* ``write_internal_points``  internal_points.dat  (output_internal_points,
  stress_mod.f90:895-936)
* ``write_stresses``         stresses.dat         (output_boundary_stresses,
  stress_mod.f90:412-468)
* ``write_disp_trac``        disp_trac.dat        (save_disp_trac, io_mod.f90:232-255)
* ``write_output``           the main output file, e.g. cube8_out.dat: the input echo
  of input_data (io_mod.f90:36-146), output_data (:191-230), the boundary stress
  tables of output_boundary_stresses and the internal-point stress table of
  output_internal_points, in main.f90's order

Numbers are written with Fortran's E, G and I edit descriptors (``fortran_e``,
``fortran_g``, ``fortran_i``), as gfortran prints them.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .mesh import Mesh


def fortran_e(x: float, w: int, d: int) -> str:
    """Fortran ``Ew.d``: 0.ddd…E±xx, right-justified in w (asterisks if it does not fit)."""
    x = float(x)
    neg = math.copysign(1.0, x) < 0
    ax = abs(x)
    if ax == 0.0:
        digits, exp = "0" * d, 0
    elif not math.isfinite(ax):
        s = "Infinity" if math.isinf(ax) else "NaN"
        s = ("-" if neg and math.isinf(ax) else "") + s
        return s.rjust(w) if len(s) <= w else "*" * w
    else:
        m, e = f"{ax:.{d - 1}e}".split("e")
        digits, exp = m.replace(".", ""), int(e) + 1
    es = f"E{exp:+03d}" if -99 <= exp <= 99 else f"{exp:+04d}"
    s = ("-" if neg else "") + "0." + digits + es
    return s.rjust(w) if len(s) <= w else "*" * w


def fortran_g(x: float, w: int, d: int) -> str:
    """Fortran ``Gw.d`` (no exponent width): fixed notation with d significant digits
    and 4 trailing blanks when 0.1 <= |x| < 10**d after rounding, else ``Ew.d``."""
    x = float(x)
    ax = abs(x)
    if ax == 0.0:
        s = f"{0.0:.{d - 1}f}"
        s = ("-" if math.copysign(1.0, x) < 0 else "") + s
        return (s.rjust(w - 4) + "    ") if len(s) <= w - 4 else "*" * w
    if not math.isfinite(ax):
        return fortran_e(x, w, d)
    # the decimal exponent after rounding to d significant digits
    k = int(f"{ax:.{d - 1}e}".split("e")[1]) + 1
    if 0 <= k <= d:
        s = f"{x:.{d - k}f}"
        return (s.rjust(w - 4) + "    ") if len(s) <= w - 4 else "*" * w
    return fortran_e(x, w, d)


def fortran_i(v: int, w: int) -> str:
    s = str(int(v))
    return s.rjust(w) if len(s) <= w else "*" * w


def _e(vals, w, d, sep=" "):
    return "".join(sep + fortran_e(v, w, d) for v in vals)


def write_internal_points(path: str, cx, cy, cz, u_int, sigma, vm, prin) -> None:
    """internal_points.dat: id, x, y, z, u(3), sigma(6), von Mises, principal(3)."""
    u_int, sigma, prin = (np.asarray(a, dtype=np.float64) for a in (u_int, sigma, prin))
    l = len(cx)
    with open(path, "w") as f:
        f.write("# INTERNAL POINTS DISPLACEMENTS AND STRESSES (QUADESTH 3D ELASTOSTATICS)\n")
        f.write("# Total Internal Points: " + fortran_i(l, 6) + "\n")
        f.write("# Col 1: Point ID\n")
        f.write("# Col 2-4: X, Y, Z coordinates\n")
        f.write("# Col 5-7: u_x, u_y, u_z displacements\n")
        f.write("# Col 8-13: Sigma_xx, Sigma_yy, Sigma_zz, Sigma_xy, Sigma_yz, Sigma_zx\n")
        f.write("# Col 14: Von Mises Equivalent Stress\n")
        f.write("# Col 15-17: Principal Stresses (Sigma_1 >= Sigma_2 >= Sigma_3)\n")
        f.write("# " + "-" * 140 + "\n")
        for i in range(l):
            row = [cx[i], cy[i], cz[i], *u_int[:, i], *sigma[:, i], vm[i], *prin[:, i]]
            f.write(fortran_i(i + 1, 6) + _e(row, 15, 7) + "\n")


def write_stresses(path: str, mesh: Mesh, sigma_node, vm, prin) -> None:
    """stresses.dat: node id, x, y, z, sigma(6), von Mises, principal(3)."""
    sigma_node, prin = np.asarray(sigma_node), np.asarray(prin)
    with open(path, "w") as f:
        f.write("# BOUNDARY NODES STRESSES (QUADESTH 3D ELASTOSTATICS)\n")
        f.write("# Col 1: Node ID\n")
        f.write("# Col 2-4: X, Y, Z coordinates\n")
        f.write("# Col 5-10: Sigma_xx, Sigma_yy, Sigma_zz, Sigma_xy, Sigma_yz, Sigma_zx\n")
        f.write("# Col 11: Von Mises Equivalent Stress\n")
        f.write("# Col 12-14: Principal Stresses (Sigma_1 >= Sigma_2 >= Sigma_3)\n")
        f.write("# " + "-" * 140 + "\n")
        for i in range(mesh.n):
            row = [mesh.x[i], mesh.y[i], mesh.z[i], *sigma_node[:, i], vm[i], *prin[:, i]]
            f.write(fortran_i(i + 1, 6) + _e(row, 15, 7) + "\n")


def _tracked(mesh: Mesh):
    """ke(1, ntrack) and the tracked node's local number in it (io_mod.f90:235-242)."""
    nt = int(mesh.ntrack)
    for e in range(mesh.ne):
        for k in range(int(mesh.nconec[e])):
            if int(mesh.kconec[k, e]) == nt:
                return e, k
    raise ValueError(f"tracked node {nt} is in no element")


def write_disp_trac(path: str, mesh: Mesh, u, dfi, append: bool = False) -> None:
    """disp_trac.dat: u and t of the tracked node (one line per call, 6(2X, E18.8))."""
    e, k = _tracked(mesh)
    nt = int(mesh.ntrack) - 1
    vals = [u[3 * nt], u[3 * nt + 1], u[3 * nt + 2], dfi[3 * k, e], dfi[3 * k + 1, e], dfi[3 * k + 2, e]]
    with open(path, "a" if append else "w") as f:
        f.write(_e(vals, 18, 8, "  ") + "\n")


def write_output(path: str, mesh: Mesh, u, dfi, sigma_node=None, vm=None, prin=None, sigma_elem=None,
                 u_int=None, sigma_int=None, vm_int=None, prin_int=None) -> None:
    """The main output file (unit ipr): input echo, boundary displacements and
    tractions, internal displacements, boundary stresses, internal stresses."""
    n, ne, l = mesh.n, mesh.ne, mesh.l
    young = 2.0 * mesh.mu * (1.0 + mesh.nu)
    stars = " " + "*" * 79
    out = []
    w = out.append
    # input_data echo
    w(stars)
    w(mesh.title.rstrip())
    w("")
    w("")
    w("  DATA")
    w("")
    w("  NUMBER OF BOUNDARY NODES    =" + fortran_i(n, 5))
    w("  NUMBER OF BOUNDARY ELEMENTS =" + fortran_i(ne, 5))
    w("  NUMBER OF INTERNAL POINTS   =" + fortran_i(l, 5))
    w("  SHEAR MODULUS (MU)          =" + fortran_g(mesh.mu, 14, 7))
    w("  YOUNG MODULUS (E)           =" + fortran_g(young, 14, 7))
    w("  POISSON RATIO (NU)          =" + fortran_g(mesh.nu, 14, 7))
    w("")
    w("")
    w("  BOUNDARY NODES COORDINATES")
    w("")
    w("")
    w("    NODE" + " " * 12 + "X" + " " * 18 + "Y" + " " * 18 + "Z")
    w("")
    for i in range(n):
        w(" " * 5 + fortran_i(i + 1, 5) + _e([mesh.x[i], mesh.y[i], mesh.z[i]], 14, 7, " " * 5))
    w("")
    w("")
    w("  ELEMENT CONNECTIVITIES")
    w("")
    w("")
    w("  ELEMENT NO.CON." + " " * 24 + "NODES")
    w("")
    for e in range(ne):
        nc = int(mesh.nconec[e])
        w(" " * 4 + fortran_i(e + 1, 5) + " " * 4 + fortran_i(nc, 2) + "  "
          + "".join("   " + fortran_i(mesh.kconec[j, e], 5) for j in range(nc)))
    w("")
    w("")
    w("  BOUNDARY CONDITIONS")
    w("")
    w(" ELEMEN CODE" + " " * 22 + "PRESCRIBED VALUES")
    w("")
    for e in range(ne):
        nc = int(mesh.nconec[e])
        for ld, axis in enumerate("XYZ"):
            vals = "".join(" " + fortran_g(mesh.bc[3 * j + ld, e], 12, 5) for j in range(nc))
            head = (" " + fortran_i(e + 1, 5) + " " * 4) if ld == 0 else " " * 8
            w(head + fortran_i(mesh.kode[3 * e + ld], 2) + " " + axis + vals)
    if l > 0:
        w("")
        w("")
        w("  COORDINATES OF INTERNAL POINTS")
        w("")
        w("    POINT" + " " * 11 + "X" + " " * 18 + "Y" + " " * 17 + " Z")
        w("")
        for i in range(l):
            w(" " * 5 + fortran_i(i + 1, 5) + _e([mesh.cx[i], mesh.cy[i], mesh.cz[i]], 14, 7, " " * 5))
    w(" TRACKED NODE = " + fortran_i(mesh.ntrack, 6))
    # output_data
    w(stars)
    w(" QUADESTH: 3D ELASTOSTATIC ANALYSIS RESULTS")
    w(stars)
    w(" BOUNDARY NODES DISPLACEMENTS")
    w(" NODE           DISPLACEMENT X          DISPLACEMENT Y          DISPLACEMENT Z")
    for i in range(n):
        w(" " + fortran_i(i + 1, 5) + _e(u[3 * i:3 * i + 3], 18, 8, " " * 5))
    w("")
    w("")
    w("  BOUNDARY ELEMENTS TRACTIONS")
    w("")
    w(" ELEMENT  NODE" + " " * 8 + "TRACTION X" + " " * 14 + "TRACTION Y" + " " * 14 + "TRACTION Z")
    w("")
    for e in range(ne):
        w(" " + fortran_i(e + 1, 5))
        for k in range(int(mesh.nconec[e])):
            w(" " * 10 + fortran_i(mesh.kconec[k, e], 5) + _e(dfi[3 * k:3 * k + 3, e], 18, 8, " " * 5))
    if l > 0 and u_int is not None:
        w("")
        w("")
        w("  INTERNAL POINTS DISPLACEMENTS")
        w("")
        w("POINT" + " " * 7 + "DISPLACEMENT X" + " " * 10 + "DISPLACEMENT Y" + " " * 10 + "DISPLACEMENT Z")
        w("")
        for i in range(l):
            w(" " + fortran_i(i + 1, 5) + _e(u_int[:, i], 18, 8, " " * 5))
    w(stars)
    # output_boundary_stresses
    if sigma_node is not None:
        w(stars)
        w(" BOUNDARY NODES STRESSES (NODAL AVERAGED)")
        w(stars)
        w(" NODE      SIGMA_XX        SIGMA_YY        SIGMA_ZZ        SIGMA_XY        SIGMA_YZ"
          "        SIGMA_ZX       VON_MISES         SIGMA_1         SIGMA_2         SIGMA_3")
        w("")
        for i in range(n):
            w(" " + fortran_i(i + 1, 5) + _e([*sigma_node[:, i], vm[i], *prin[:, i]], 15, 7))
        if sigma_elem is not None:
            w("")
            w("")
            w(stars)
            w(" BOUNDARY ELEMENTS NODAL STRESSES")
            w(stars)
            w(" ELEMENT  NODE      SIGMA_XX        SIGMA_YY        SIGMA_ZZ        SIGMA_XY"
              "        SIGMA_YZ        SIGMA_ZX")
            w("")
            for e in range(ne):
                w(" " + fortran_i(e + 1, 5))
                for k in range(int(mesh.nconec[e])):
                    w(" " * 10 + fortran_i(mesh.kconec[k, e], 5) + _e(sigma_elem[:, k, e], 15, 7))
    # output_internal_points (the table written to unit ipr)
    if l > 0 and sigma_int is not None:
        w("")
        w("")
        w(stars)
        w(" INTERNAL POINTS STRESSES")
        w(stars)
        w(" POINT     SIGMA_XX        SIGMA_YY        SIGMA_ZZ        SIGMA_XY        SIGMA_YZ"
          "        SIGMA_ZX       VON_MISES         SIGMA_1         SIGMA_2         SIGMA_3")
        w("")
        for i in range(l):
            w(" " + fortran_i(i + 1, 5) + _e([*sigma_int[:, i], vm_int[i], *prin_int[:, i]], 15, 7))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def write_all(prefix: str, mesh: Mesh, res: dict) -> dict:
    """Every result file of one run from ``Quadesth.run()``'s dictionary; returns the
    paths.  ``prefix`` is a directory (the reference writes into its working one)."""
    import os

    os.makedirs(prefix, exist_ok=True)
    paths = {k: os.path.join(prefix, v) for k, v in (
        ("output", "cube8_out.dat"), ("stresses", "stresses.dat"),
        ("internal_points", "internal_points.dat"), ("disp_trac", "disp_trac.dat"))}
    write_output(paths["output"], mesh, res["u"], res["t"], res.get("sigma_node"), res.get("sigma_node_vm"),
                 res.get("sigma_node_prin"), res.get("sigma_elem"), res.get("u_int"), res.get("sigma"),
                 res.get("vm"), res.get("prin"))
    if "sigma_node" in res:
        write_stresses(paths["stresses"], mesh, res["sigma_node"], res["sigma_node_vm"], res["sigma_node_prin"])
    if mesh.l > 0 and "u_int" in res:
        write_internal_points(paths["internal_points"], mesh.cx, mesh.cy, mesh.cz, res["u_int"], res["sigma"],
                              res["vm"], res["prin"])
    write_disp_trac(paths["disp_trac"], mesh, res["u"], res["t"])
    return paths
