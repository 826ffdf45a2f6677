"""Run the hot path once on a generated cube and print phase timings.

    python -m bem3d_elastostatic_b200.profile_case --cube 16 --precision fp32-ir

Geometry, ghmat8 assembly and the solve of the uniaxially loaded unit cube with
m x m quad9 elements per face (--cube m; 16 gives 18,438 DOF).  Meant as a small,
self-contained case for profilers (every kernel of the path runs, a few GB on the
device at most for m <= 16).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .api import Quadesth
from .mesh import cube_grid_points, uniaxial_cube


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cube", type=int, default=16)
    ap.add_argument("--precision", default="fp32-ir", choices=["fp64", "fp32-ir", "bf16-ir"])
    ap.add_argument("--points", action="store_true", help="also evaluate 27 internal points")
    args = ap.parse_args(argv)
    mesh = uniaxial_cube(args.cube, young=1.0, nu=0.3,
                         points=cube_grid_points([0.25, 0.5, 0.75]) if args.points else None)
    q = Quadesth(mesh)
    t0 = time.perf_counter()
    q.precompute_element_geometry()
    q.ghmat8()
    q.ctx.sync()
    t1 = time.perf_counter()
    x = q.solve_linear_system(args.precision, tol=1e-15, max_iter=60)
    t2 = time.perf_counter()
    out = {"dof": mesh.ndof, "precision": args.precision, "assembly_s": t1 - t0,
           "solve_s": t2 - t1, "solve_info": q.solve_info,
           "max_u": float(np.abs(x).max())}
    if args.points:
        q.reorganize_solution()
        u, s, _, _ = q.compute_internal_points()
        out["sigma_zz_range"] = [float(s[2].min()), float(s[2].max())]
    print(json.dumps(out))
    q.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
