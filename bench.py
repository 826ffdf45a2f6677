#!/usr/bin/env python
"""Benchmark: assembly + solve of the 73,734-DOF unit cube on one B200.

Workload (BASELINE config "mixed precision"): unit cube [0,1]^3, 32 x 32 quad9
elements per face (6,144 elements, 24,578 nodes, 73,734 DOF; the FP64 matrix is
43.5 GB), E = 1, nu = 0.3, u_z = 0 on z = 0 with three pinned DOFs, t_z = 1 on z = 1.

A step is one pass of the hot path on that mesh with the inputs resident in HBM:
element geometry, ghmat8 assembly of A x = FI (FP64), and the mixed-precision solve
(FP32 LU whose trailing updates run on the tensor cores as a three-term BF16 split,
FP64 iterative refinement against the FP64 A).  ``value`` is seconds per solved
system (lower is better).  The same step with the plain FP64 LU is timed once for
the "vs plain FP64" comparison, and its solution is the accuracy reference.

``e2e`` times the same work through the public API from pinned host buffers: mesh,
material, supports and pins copied in, then geometry, assembly, solve, and the
solution copied back.

``cpu_baseline`` / ``--impl reference``: the reference's algorithm restated in C++
(oracle/, OpenMP on every host core) with LAPACK dgesv from scipy's OpenBLAS, on a
bounded sample: assembly of a slice of collocation rows and dgesv at a reduced
order, extrapolated linearly in rows and cubically in order (labelled so).

Multi-GPU: the dense LU does not shard; --gpus N runs N independent replicas (one
process per GPU under torchrun) and value = max-over-ranks step time / N.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "assembly+solve s at 73.7k DOF: mixed-prec+IR vs plain FP64, rel err<=1e-10"
WORKLOAD = ("unit cube [0,1]^3, 32x32 quad9 per face: 6,144 elements, 24,578 nodes, "
            "73,734 DOF, E=1, nu=0.3, u_z=0 on z=0 + 3 pins, t_z=1 on z=1")


def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        rows = getattr(self, "rows", [])
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [v for v in sm if v > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows)}


def dist_setup(n_gpus: int):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def allreduce_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------------------------------
# CPU leg (oracle: the reference's algorithm restated in C++, OpenMP, + OpenBLAS dgesv)
# ------------------------------------------------------------------------------------

def cpu_sample(mesh, rows: int = 256, n_lu: int = 10240):
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import oracle as O
    from scipy.linalg import lapack

    orc = O.Oracle(mesh)
    t0 = time.perf_counter()
    orc.geometry()
    orc.ghmat8(0, rows, pins=False)
    t_asm = time.perf_counter() - t0
    rng = np.random.default_rng(20261203)
    A = np.asfortranarray(rng.standard_normal((n_lu, n_lu)))
    A[np.diag_indices(n_lu)] += n_lu ** 0.5
    b = rng.standard_normal(n_lu)
    t0 = time.perf_counter()
    lapack.dgesv(A, b, overwrite_a=True, overwrite_b=True)
    t_lu = time.perf_counter() - t0
    N = mesh.ndof
    est = t_asm * (mesh.n / rows) + t_lu * (N / n_lu) ** 3
    sample = (f"assembly of collocation rows 0..{rows} of {mesh.n} (x{mesh.n / rows:.1f}) and "
              f"dgesv at N={n_lu} (x(N/{n_lu})^3 = {(N / n_lu) ** 3:.0f}); extrapolated")
    return est, sample, {"assembly_sample_s": t_asm, "dgesv_sample_s": t_lu}


def host_cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    from bem3d_elastostatic_b200.mesh import uniaxial_cube

    mesh = uniaxial_cube(32, young=1.0, nu=0.3)
    for _ in range(args.warmup):
        cpu_sample(mesh, rows=64, n_lu=4096)
    vals, extra = [], {}
    for _ in range(args.steps):
        v, sample, extra = cpu_sample(mesh)
        vals.append(v)
    value = float(statistics.median(vals))
    cores = host_cores()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "path": "CPU restatement of the reference (oracle/)"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "extra": extra,
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------
# GPU arm
# ------------------------------------------------------------------------------------

def run_gpu(args, ws, rank, local):
    import torch
    import torch.cuda.profiler

    from bem3d_elastostatic_b200 import _lib
    from bem3d_elastostatic_b200.api import Quadesth
    from bem3d_elastostatic_b200.mesh import uniaxial_cube

    torch.cuda.set_device(local)
    mesh = uniaxial_cube(32, young=1.0, nu=0.3)
    q = Quadesth(mesh, device=local)
    stream = torch.cuda.ExternalStream(q.ctx.stream(), device=local)

    def step(precision):
        q.precompute_element_geometry()
        q.ghmat8()
        return q.solve_linear_system(precision, tol=args.tol, max_iter=60)

    for _ in range(args.warmup):
        step(args.precision)
    # one more untimed step in the timed region's profile mode: the factorisation's
    # launch sequence is captured per profile mode, so that capture happens here
    q.ctx.profile_begin(timing=_lib.BEM_PROF_TRAILING)
    step(args.precision)
    q.ctx.profile_end()
    barrier(ws)
    torch.cuda.synchronize()
    q.ctx.sync()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    infos = []
    with ClockSampler(local) as clk:
        # inside the timed region only the trailing updates carry events (two per panel)
        q.ctx.profile_begin(timing=_lib.BEM_PROF_TRAILING)
        # the timed region is the profiler range (ncu --profile-from-start off)
        torch.cuda.profiler.start()
        ev0.record(stream)
        marks = [ev0]
        for _ in range(args.steps):
            x_mixed = step(args.precision)
            infos.append(q.solve_info)
            e = torch.cuda.Event(enable_timing=True)
            e.record(stream)
            marks.append(e)
        ev1.record(stream)
        torch.cuda.profiler.stop()
        prof = q.ctx.profile_end()
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier(ws)
    t_step = ev0.elapsed_time(ev1) / 1e3 / args.steps
    step_ms = [marks[i].elapsed_time(marks[i + 1]) for i in range(args.steps)]
    t_step = allreduce_max(t_step, ws)

    # one more step, outside the timed region, with every LU phase timed
    q.ctx.profile_begin(timing=_lib.BEM_PROF_PHASES)
    step(args.precision)
    phases = q.ctx.profile_end()

    # the assembly alone (geometry + ghmat8, regular and singular pairs), untimed step:
    # regular quad9 pairs at 36 Gauss points x ~470 flops = 16,920 flops each
    # (assembly_mod.f90:356-383, 618-650), against the nominal FP64 peak of a B200
    assembly = None
    try:
        q.ctx.sync()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        q.precompute_element_geometry()
        q.ghmat8()
        a1.record(stream)
        a1.synchronize()
        t_asm = a0.elapsed_time(a1) / 1e3
        pairs = int(mesh.n) * int(mesh.ne) - int(np.sum(mesh.nconec))
        tflops = pairs * 16920.0 / t_asm / 1e12
        assembly = {"seconds": t_asm, "regular_pairs": pairs, "pairs_per_s": pairs / t_asm,
                    "fp64_tflops": tflops, "fp64_peak_tflops_nominal": 37.0, "frac": tflops / 37.0}
    except Exception as ex:  # a measurement of the report only: never lose the bench line
        assembly = {"error": str(ex)[:200]}

    # plain FP64 comparison step (also the accuracy reference at this size)
    fp64_s = None
    rel_err = None
    if not args.skip_fp64:
        q.ctx.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        x64 = step("fp64")
        e1.record(stream)
        e1.synchronize()
        fp64_s = allreduce_max(e0.elapsed_time(e1) / 1e3, ws)
        rel_err = float(np.abs(x_mixed - x64).max() / np.abs(x64).max())

    # end to end through the public API from pinned host memory
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    hx, hy, hz = pin(mesh.x), pin(mesh.y), pin(mesh.z)
    hnc, hkc = pin(mesh.nconec), pin(mesh.kconec.ravel(order="F"))
    hkode, hbc = pin(mesh.kode), pin(mesh.bc.ravel(order="F"))
    hpins = pin(mesh.pins)
    hsol = torch.empty(mesh.ndof, dtype=torch.float64).pin_memory().numpy()
    h2d = sum(a.nbytes for a in (hx, hy, hz, hnc, hkc, hkode, hbc, hpins))
    d2h = hsol.nbytes
    L, h = q.ctx.L, q.ctx.h
    info = _lib.C.c_int(0)
    st = _lib.SolveInfo()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    q.ctx.sync()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        ck = q.ctx.check
        ck(L.bem_set_mesh(h, mesh.n, mesh.ne, _lib.ptr(hx), _lib.ptr(hy), _lib.ptr(hz),
                          _lib.ptr(hnc), _lib.ptr(hkc)), "set_mesh")
        ck(L.bem_set_material(h, float(mesh.mu), float(mesh.nu)), "set_material")
        ck(L.bem_set_bc(h, _lib.ptr(hkode), _lib.ptr(hbc)), "set_bc")
        ck(L.bem_set_pins(h, int(hpins.size), _lib.ptr(hpins)), "set_pins")
        ck(L.bem_precompute_geometry(h), "geometry")
        ck(L.bem_ghmat8(h, _lib.BEM_ASM_FP64, None, 0, None), "ghmat8")
        ck(L.bem_solve(h, _lib.BEM_PREC_FP32_IR if args.precision == "fp32-ir" else _lib.BEM_PREC_BF16_IR,
                       args.tol, 60, _lib.ptr(hsol), _lib.C.byref(info), _lib.C.byref(st)), "solve")
    e1.record(stream)
    e1.synchronize()
    e2e_s = allreduce_max(e0.elapsed_time(e1) / 1e3 / e2e_steps, ws)
    e2e_err = float(np.abs(hsol - x_mixed).max() / np.abs(x_mixed).max())

    if rank != 0:
        q.close()
        return 0

    peaks, src = measured_peaks()
    t_ms = prof["lu_trailing_ms"]
    gbs = prof["lu_trailing_bytes"] / (t_ms * 1e-3) / 1e9 if t_ms > 0 else 0.0
    fp32_tflops = prof["lu_trailing_flops"] / (t_ms * 1e-3) / 1e12 if t_ms > 0 else 0.0
    # the BF16x3 split executes three BF16 products (hi.hi, hi.lo, lo.hi) per FP32
    # multiply-add of the update; the plain BF16 mode one
    products = 3 if args.precision == "fp32-ir" else 1
    bf16_tflops = products * fp32_tflops
    # a kernel timed inside a seconds-long step: the sustained BF16 figure
    tpeak = peaks.get("bf16_tflops_sustained") or peaks["bf16_tflops"]
    hbm_frac, tensor_frac = gbs / peaks["hbm_gbs"], bf16_tflops / tpeak
    n_launch = max(1, prof["lu_trailing_launches"])
    roofline = {
        "kernel": ("umma_update_kernel + its BF16 split kernels (LU trailing update: C -= A B, "
                   "tcgen05 BF16x3 into TMEM, TMA-reduce epilogue)" if args.precision == "fp32-ir" else
                   "sgemm_bf16_kernel<0,1> (LU trailing update, BF16 mma.sync)"),
        "traffic": None,
        "algorithmic_bytes_per_launch": prof["lu_trailing_bytes"] / n_launch,
        "algorithmic_fp32_flops_per_launch": prof["lu_trailing_flops"] / n_launch,
        "avg_launch_ms": t_ms / n_launch,
        "hbm": {"achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": hbm_frac,
                "peak_source": f"{src} hbm_gbs"},
        "tensor": {"achieved": bf16_tflops, "peak": tpeak, "unit": "TFLOP/s", "frac": tensor_frac,
                   "peak_source": f"{src} bf16_tflops_sustained", "bf16_products_per_fp32_fma": products,
                   "fp32_equivalent_tflops": fp32_tflops},
    }
    # the bound is the resource the kernel runs closer to
    b = roofline["tensor"] if tensor_frac >= hbm_frac else roofline["hbm"]
    roofline.update({"bound": "tensor" if tensor_frac >= hbm_frac else "hbm", "achieved": b["achieved"],
                     "peak": b["peak"], "unit": b["unit"], "frac": b["frac"], "peak_source": b["peak_source"]})
    tf = os.path.join(HERE, "profiles", "trailing_gemm_traffic.json")
    if os.path.exists(tf):
        with open(tf) as f:
            ratio = json.load(f).get("dram_bytes_over_algorithmic")
        if ratio:
            roofline["traffic"] = ratio * roofline["algorithmic_bytes_per_launch"]
            roofline["traffic_source"] = "ncu dram__bytes ratio, profiles/trailing_gemm_traffic.json"

    cpu = None
    if ws == 1 and not args.skip_cpu:
        v, sample, extra = cpu_sample(mesh)
        cpu = {"value": v, "unit": "s", "cores": host_cores(), "kind": "port", "sample": sample}

    it = [i["iterations"] for i in infos]
    line = {
        "metric": METRIC, "value": t_step / ws, "unit": "s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 assembly + residual, f32 LU on bf16x3 tensor cores",
        "data": "synthetic",
        "config": {
            "workload": WORKLOAD, "precision": args.precision,
            "parallelism": "replicas" if ws > 1 else "single GPU",
            "l2": "inputs larger than L2 (A is 43.5 GB FP64 + 21.7 GB FP32)",
            "fp64_plain_s": fp64_s,
            "speedup_vs_fp64": (fp64_s / t_step) if fp64_s else None,
            "rel_err_vs_fp64": rel_err,
            "step_ms": step_ms,
            "refine_iterations": it, "backward_error": infos[-1]["rel_residual"],
            "factor_s": infos[-1]["factor_seconds"], "refine_s": infos[-1]["refine_seconds"],
            "assembly_untimed_step": assembly,
            "lu_phase_ms_untimed_step": {k: phases[k] for k in (
                "lu_panel_ms", "lu_swap_ms", "lu_panel_update_ms", "lu_trsm_ms", "lu_trailing_ms")},
        },
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_s / ws, "unit": "s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "rel_diff_vs_value_path": e2e_err},
        "gpu_launches": int(prof["kernel_launches"]),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    q.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--precision", default="fp32-ir", choices=["fp32-ir", "bf16-ir"])
    ap.add_argument("--tol", type=float, default=1e-15)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            return run_reference(args, ws, rank)
        return run_gpu(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
