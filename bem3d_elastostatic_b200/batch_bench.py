"""Measure the batched path on the box workload.

    python -m bem3d_elastostatic_b200.batch_bench --systems 512 --loads 8

512 boxes (sides uniform in [0.5, 2], k in {1..6} quad9 elements per edge, nu uniform
in [0.05, 0.45], E = 1), 8 random top-face traction vectors each; supports as the
uniaxial cube.  Times (CUDA events on the batch's stream, after one warm-up): assembly
of every system, the FP32 LU + FP64 refinement solve and the plain FP64 solve; reports
systems/s, the largest backward error and the largest difference between the refined
and the FP64 solutions (relative to each solution's maximum).  --check k also solves k
systems with the CPU oracle (LAPACK dgesv) and reports the largest relative error.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .api import Batch
from .mesh import box_batch


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=512)
    ap.add_argument("--loads", type=int, default=8)
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--check", type=int, default=0)
    args = ap.parse_args(argv)
    systems = box_batch(args.systems, loads=args.loads)
    N = np.array([m.ndof for m, _ in systems])
    b = Batch()
    t0 = time.perf_counter()
    for m, bcs in systems:
        b.add(m, bcs)
    t_add = time.perf_counter() - t0
    import torch

    b.assemble()  # warm-up (allocations, constants)
    stream = None
    res = {"systems": args.systems, "loads": args.loads, "dof_min": int(N.min()), "dof_max": int(N.max()),
           "dof_mean": float(N.mean()), "host_add_s": t_add}
    t0 = time.perf_counter()
    b.assemble()
    res["assemble_s"] = time.perf_counter() - t0
    b.solve("fp32-ir", tol=1e-15, max_iter=args.sweeps)  # warm-up: autotune + graph capture
    info = b.solve("fp32-ir", tol=1e-15, max_iter=args.sweeps)
    res["fp32_ir"] = info
    x_ir = [b.solution(i) for i in range(args.systems)]
    b.solve("fp64")
    info64 = b.solve("fp64")
    res["fp64"] = info64
    x64 = [b.solution(i) for i in range(args.systems)]
    diff = max(float(np.abs(a - c).max() / np.abs(c).max()) for a, c in zip(x_ir, x64))
    res["rel_diff_ir_vs_fp64"] = diff
    res["systems_per_s_fp32_ir"] = args.systems / info["solve_seconds"]
    res["systems_per_s_fp64"] = args.systems / info64["solve_seconds"]
    res["speedup_fp32_ir_vs_fp64"] = info64["solve_seconds"] / info["solve_seconds"]
    res["kernel_launches"] = b.launches()
    if args.check:
        import os
        import sys

        sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
        import oracle as O

        worst = 0.0
        rng = np.random.default_rng(1)
        for i in rng.choice(args.systems, size=min(args.check, args.systems), replace=False):
            m, bcs = systems[i]
            m.bc = np.asfortranarray(bcs[-1])
            A, F = O.Oracle(m).ghmat8()
            xr, _ = O.Oracle.solve(A, F)
            worst = max(worst, float(np.abs(x_ir[i][:, -1] - xr).max() / np.abs(xr).max()))
        res["oracle_checked_systems"] = int(min(args.check, args.systems))
        res["rel_err_vs_oracle_max"] = worst
    print(json.dumps(res))
    b.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
