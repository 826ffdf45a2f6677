"""CPU checks of bench.py's host-side logic (no device calls): the fitted CPU
baseline's least-squares fits and extrapolation, and that a failing extra leg is
recorded instead of ending the bench line."""
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_cpu_fit_recovers_exact_models():
    b = _bench()
    a0, a2, c0, c3 = 0.05, 3e-8, 0.01, 2e-12
    times = {N: (a0 + a2 * N ** 2, c0 + c3 * float(N) ** 3) for N in (4614, 10374, 18438)}
    est, det = b.cpu_fit(times, 73734)
    want = a0 + a2 * 73734 ** 2 + c0 + c3 * 73734.0 ** 3
    assert abs(est - want) <= 1e-9 * want
    assert max(abs(r) for r in det["assembly_fit_rel_residuals"]) < 1e-9
    assert max(abs(r) for r in det["dgesv_fit_rel_residuals"]) < 1e-9
    assert det["sizes_dof"] == [4614, 10374, 18438]


def test_failing_leg_is_recorded():
    b = _bench()
    out = {}
    b._leg("ok", lambda: {"x": 1}, out)
    b._leg("bad", lambda: 1 / 0, out)
    assert out["ok"]["x"] == 1 and "leg_wall_s" in out["ok"]
    assert out["bad"]["error"].startswith("ZeroDivisionError")
    assert np.isfinite(out["bad"]["leg_wall_s"])
