"""Reference-shaped interface to the B200 hot path.

``Quadesth`` mirrors the phase sequence of the reference's driver (main.f90:30-79)
and the names of the module procedures it calls, each running on the GPU through the
C ABI:

    input_data                  -> Quadesth(mesh)                 (io_mod.f90:36)
    precompute_element_geometry -> .precompute_element_geometry() (assembly_mod.f90:28)
    ghmat8                      -> .ghmat8()                      (assembly_mod.f90:53)
    solve_linear_system         -> .solve_linear_system()         (solver_mod.f90:17)
    reorganize_solution         -> .reorganize_solution()         (io_mod.f90:148)
    compute_internal_points     -> .compute_internal_points()     (stress_mod.f90:511)

Errors follow the reference: a singular system stops the run with the DGESV message
(solver_mod.f90:30-33), raised here as ``SolverFailure`` carrying ``info``.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import _lib
from .mesh import Mesh

PRECISIONS = {"fp64": _lib.BEM_PREC_FP64, "fp32-ir": _lib.BEM_PREC_FP32_IR,
              "bf16-ir": _lib.BEM_PREC_BF16_IR, "fp64-ir": _lib.BEM_PREC_FP64_IR}
ASSEMBLY = {"fp64": _lib.BEM_ASM_FP64, "fp32-far": _lib.BEM_ASM_FP32_FAR}


class SolverFailure(RuntimeError):
    def __init__(self, info: int):
        super().__init__(f" *** ERROR in LAPACK DGESV: info = {info:6d}\n"
                         "Solver failure: Singular matrix or bad arguments in LAPACK DGESV.")
        self.info = info


class Quadesth:
    def __init__(self, mesh: Mesh, device: int = 0, ctx: Optional[_lib.Context] = None):
        mesh.validate()
        self.mesh = mesh
        self.ctx = ctx or _lib.Context(device)
        self.load_mesh()
        self.solve_info: Optional[dict] = None

    # input_data (io_mod.f90:36-146): the mesh's current arrays to the device
    def load_mesh(self) -> None:
        mesh = self.mesh
        L, h = self.ctx.L, self.ctx.h
        self._keep = [mesh.x, mesh.y, mesh.z, mesh.nconec, mesh.kconec, mesh.kode, mesh.bc, mesh.pins]
        c = self.ctx.check
        c(L.bem_set_mesh(h, mesh.n, mesh.ne, _lib.ptr(mesh.x), _lib.ptr(mesh.y), _lib.ptr(mesh.z),
                         _lib.ptr(mesh.nconec), _lib.ptr(mesh.kconec)), "set_mesh")
        c(L.bem_set_material(h, float(mesh.mu), float(mesh.nu)), "set_material")
        c(L.bem_set_bc(h, _lib.ptr(mesh.kode), _lib.ptr(mesh.bc)), "set_bc")
        c(L.bem_set_pins(h, int(mesh.pins.size), _lib.ptr(mesh.pins) if mesh.pins.size else None),
          "set_pins")

    # assembly_mod.f90:28
    def precompute_element_geometry(self) -> None:
        self.ctx.check(self.ctx.L.bem_precompute_geometry(self.ctx.h), "precompute_geometry")

    def geometry_tables(self) -> dict:
        ne = self.mesh.ne
        arrs = [np.zeros((36, ne), order="F") for _ in range(7)] + [np.zeros((9, 36, ne), order="F")]
        self.ctx.check(self.ctx.L.bem_get_geometry(self.ctx.h, *[_lib.ptr(a) for a in arrs]),
                       "get_geometry")
        return dict(zip(("eta1", "eta2", "eta3", "xja", "xg1", "xg2", "xg3", "ff"), arrs))

    # assembly_mod.f90:53
    def ghmat8(self, precision: str = "fp64", return_system: bool = False):
        N = self.mesh.ndof
        A = np.zeros((N, N), order="F") if return_system else None
        FI = np.zeros(N) if return_system else None
        self.ctx.check(self.ctx.L.bem_ghmat8(self.ctx.h, ASSEMBLY[precision], _lib.ptr(A), N,
                                             _lib.ptr(FI)), "ghmat8")
        return (A, FI) if return_system else None

    def system_rows(self, in0: int, in1: int):
        """Rows of A and FI for collocation nodes [in0, in1) (3 rows per node), read from
        the device after ghmat8 (before an FP64 factorisation overwrites A)."""
        r0, r1 = 3 * in0, 3 * in1
        A = np.zeros((r1 - r0, self.mesh.ndof), order="F")
        FI = np.zeros(r1 - r0)
        self.ctx.check(self.ctx.L.bem_get_rows(self.ctx.h, r0, r1, _lib.ptr(A), r1 - r0, _lib.ptr(FI)),
                       "get_rows")
        return A, FI

    def set_option(self, option: int, value: int) -> None:
        self.ctx.set_option(option, value)

    def hg(self, in0: int = 0, in1: Optional[int] = None):
        in1 = self.mesh.n if in1 is None else in1
        nr = 3 * (in1 - in0)
        H = np.zeros((nr, self.mesh.ndof), order="F")
        G = np.zeros((nr, 27 * self.mesh.ne), order="F")
        self.ctx.check(self.ctx.L.bem_get_hg(self.ctx.h, in0, in1, _lib.ptr(H), nr, _lib.ptr(G), nr),
                       "get_hg")
        return H, G

    # solver_mod.f90:17
    def solve_linear_system(self, precision: str = "fp64", tol: float = 1e-13,
                            max_iter: int = 50) -> np.ndarray:
        x = np.zeros(self.mesh.ndof)
        info = _lib.C.c_int(0)
        st = _lib.SolveInfo()
        rc = self.ctx.L.bem_solve(self.ctx.h, PRECISIONS[precision], tol, max_iter, _lib.ptr(x),
                                  _lib.C.byref(info), _lib.C.byref(st))
        self.solve_info = st.as_dict()
        if rc > 0 or info.value != 0:
            raise SolverFailure(info.value or rc)
        self.ctx.check(rc, "solve")
        return x

    # io_mod.f90:148
    def reorganize_solution(self):
        u = np.zeros(self.mesh.ndof)
        t = np.zeros((27, self.mesh.ne), order="F")
        self.ctx.check(self.ctx.L.bem_reorganize(self.ctx.h, _lib.ptr(u), _lib.ptr(t)), "reorganize")
        return u, t

    # stress_mod.f90:365
    def compute_boundary_stresses(self, element_nodal: bool = True):
        """Traction-recovery boundary stresses: (sigma_elem (6, 9, ne) or None,
        sigma_node (6, n), principal (3, n), von Mises (n))."""
        m = self.mesh
        se = np.zeros((6, 9, m.ne), order="F") if element_nodal else None
        sn = np.zeros((6, m.n), order="F")
        pr = np.zeros((3, m.n), order="F")
        vm = np.zeros(m.n)
        self.ctx.check(self.ctx.L.bem_boundary_stresses(self.ctx.h, _lib.ptr(se), _lib.ptr(sn), _lib.ptr(pr),
                                                        _lib.ptr(vm)), "boundary_stresses")
        return se, sn, pr, vm

    # stress_mod.f90:511
    def compute_internal_points(self, points: Optional[np.ndarray] = None,
                                kelvin_consistent: bool = False):
        m = self.mesh
        if points is None:
            cx, cy, cz = m.cx, m.cy, m.cz
        else:
            p = np.asarray(points, dtype=np.float64)
            cx, cy, cz = (np.ascontiguousarray(p[:, i]) for i in range(3))
        l = int(cx.shape[0])
        u = np.zeros((3, l), order="F")
        s = np.zeros((6, l), order="F")
        pr = np.zeros((3, l), order="F")
        vm = np.zeros(l)
        flags = _lib.BEM_IP_KELVIN_CONSISTENT if kelvin_consistent else 0
        self.ctx.check(self.ctx.L.bem_internal_points(self.ctx.h, l, _lib.ptr(cx), _lib.ptr(cy),
                                                      _lib.ptr(cz), _lib.ptr(u), _lib.ptr(s),
                                                      _lib.ptr(pr), _lib.ptr(vm), flags),
                       "internal_points")
        return u, s, pr, vm

    def run(self, precision: str = "fp64", kelvin_consistent: bool = False, tol: float = 1e-13):
        """main.f90:38-68 on the GPU."""
        self.precompute_element_geometry()
        self.ghmat8()
        x = self.solve_linear_system(precision, tol=tol)
        u, t = self.reorganize_solution()
        res = {"x": x, "u": u, "t": t, "solve_info": self.solve_info}
        (res["sigma_elem"], res["sigma_node"], res["sigma_node_prin"],
         res["sigma_node_vm"]) = self.compute_boundary_stresses()
        if self.mesh.l > 0:
            res["u_int"], res["sigma"], res["prin"], res["vm"] = self.compute_internal_points(
                kelvin_consistent=kelvin_consistent)
        return res

    def close(self):
        self.ctx.close()


class Batch:
    """Many independent systems solved together (no counterpart in the reference).

    ``add(mesh, bcs)`` registers a mesh with its load cases: ``bcs`` is a list of
    (27, ne) prescribed-value arrays for the mesh's ``kode`` (every system of a batch
    has the same number of load cases, at most 8).  ``assemble()`` builds every A and
    FI; ``solve(precision)`` factors and solves all of them ("fp32-ir": FP32 LU + FP64
    refinement; "fp64": FP64 LU); ``solution(i)`` returns system i's (3n, nrhs)
    solution.
    """

    def __init__(self, device: int = 0):
        self.L = _lib.load()
        h = _lib.C.c_void_p()
        rc = self.L.bem_batch_create(_lib.C.byref(h), device)
        if rc != 0:
            raise _lib.BemError(rc, "bem_batch_create failed")
        self.h = h
        self.meshes = []
        self.nrhs = []
        self.info: Optional[dict] = None

    def _check(self, rc: int, what: str) -> int:
        if rc < 0:
            msg = self.L.bem_batch_last_error(self.h)
            raise _lib.BemError(rc, f"{what}: {msg.decode() if msg else ''}")
        return rc

    def add(self, mesh: Mesh, bcs=None) -> int:
        mesh.validate()
        bcs = [mesh.bc] if bcs is None else list(bcs)
        bc = np.ascontiguousarray(np.stack([np.asfortranarray(b, dtype=np.float64).ravel(order="F") for b in bcs]))
        pins = np.ascontiguousarray(mesh.pins, dtype=np.int32)
        keep = [mesh.x, mesh.y, mesh.z, mesh.nconec, mesh.kconec, mesh.kode, bc, pins]
        idx = self._check(self.L.bem_batch_add(
            self.h, mesh.n, mesh.ne, _lib.ptr(mesh.x), _lib.ptr(mesh.y), _lib.ptr(mesh.z),
            _lib.ptr(mesh.nconec), _lib.ptr(mesh.kconec), float(mesh.mu), float(mesh.nu),
            _lib.ptr(mesh.kode), len(bcs), _lib.ptr(bc), int(pins.size), _lib.ptr(pins)), "batch_add")
        del keep
        self.meshes.append(mesh)
        self.nrhs.append(len(bcs))
        return idx

    def assemble(self):
        self._check(self.L.bem_batch_assemble(self.h), "batch_assemble")

    def solve(self, precision: str = "fp32-ir", tol: float = 1e-15, max_iter: int = 10) -> dict:
        st = _lib.BatchInfo()
        rc = self.L.bem_batch_solve(self.h, PRECISIONS[precision], tol, max_iter, _lib.C.byref(st))
        self.info = st.as_dict()
        if rc == _lib.BEM_ERR_NOCONV:
            raise SolverFailure(0)
        self._check(rc, "batch_solve")
        return self.info

    def solution(self, i: int) -> np.ndarray:
        m = self.meshes[i]
        x = np.zeros((m.ndof, self.nrhs[i]), order="F")
        self._check(self.L.bem_batch_get_solution(self.h, i, _lib.ptr(x)), "batch_get_solution")
        return x

    def system(self, i: int):
        m = self.meshes[i]
        A = np.zeros((m.ndof, m.ndof), order="F")
        F = np.zeros((m.ndof, self.nrhs[i]), order="F")
        self._check(self.L.bem_batch_get_system(self.h, i, _lib.ptr(A), _lib.ptr(F)), "batch_get_system")
        return A, F

    def launches(self) -> int:
        return int(self.L.bem_batch_launches(self.h))

    def close(self):
        if self.h:
            self.L.bem_batch_destroy(self.h)
            self.h = None


def solve_system(A: np.ndarray, FI: np.ndarray, precision: str = "fp32-ir", tol: float = 1e-13,
                 max_iter: int = 50, ctx: Optional[_lib.Context] = None,
                 pivoting: Optional[int] = None):
    """solve_linear_system (solver_mod.f90:17) for any dense system in any precision
    mode: A (n x n) and FI (n) go to the device (bem_set_system), bem_solve solves.
    Returns (x, solve_info)."""
    ctx = ctx or _lib.Context(0)
    A = np.asfortranarray(A, dtype=np.float64)
    FI = np.ascontiguousarray(FI, dtype=np.float64)
    n = A.shape[0]
    if pivoting is not None:
        ctx.set_option(_lib.BEM_OPT_PIVOTING, pivoting)
    ctx.check(ctx.L.bem_set_system(ctx.h, n, _lib.ptr(A), n, _lib.ptr(FI)), "set_system")
    x = np.zeros(n)
    info = _lib.C.c_int(0)
    st = _lib.SolveInfo()
    rc = ctx.L.bem_solve(ctx.h, PRECISIONS[precision], tol, max_iter, _lib.ptr(x), _lib.C.byref(info),
                         _lib.C.byref(st))
    if rc > 0 or info.value != 0:
        raise SolverFailure(info.value or rc)
    ctx.check(rc, "solve")
    return x, st.as_dict()


def dgesv(A: np.ndarray, B: np.ndarray, ctx: Optional[_lib.Context] = None):
    """LAPACK dgesv on the GPU (solver_mod.f90:28).  Returns (LU, ipiv, X, info); the
    factors are those of the column-pivoted form documented in csrc/lu.cuh."""
    ctx = ctx or _lib.Context(0)
    A = np.array(A, dtype=np.float64, order="F", copy=True)
    B = np.array(B, dtype=np.float64, order="F", copy=True)
    if B.ndim == 1:
        B = B.reshape(-1, 1, order="F")
    n, nrhs = A.shape[0], B.shape[1]
    ipiv = np.zeros(n, dtype=np.int32)
    info = _lib.C.c_int(0)
    rc = ctx.L.bem_dgesv(ctx.h, n, nrhs, _lib.ptr(A), n, _lib.ptr(ipiv), _lib.ptr(B), n,
                         _lib.C.byref(info))
    if rc < 0:
        ctx.check(rc, "dgesv")
    return A, ipiv, B, info.value
