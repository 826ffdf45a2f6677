"""ctypes front-end of the CPU oracle (test infrastructure only).

Loads ``oracle/libbem_oracle.so`` (built by ``oracle/Makefile``) and exposes the
reference's phases on a :class:`bem3d_elastostatic_b200.mesh.Mesh`:

* ``geometry``            precompute_element_geometry / etaxja  (assembly_mod.f90:28-51, 225-337)
* ``ghmat8``              A and FI                              (assembly_mod.f90:53-223)
* ``hg``                  H and G as separate products          (blocks combined by ghmat8)
* ``solve``               LAPACK dgesv                          (solver_mod.f90:17-36)
* ``reorganize``          un-swap into u and t                  (io_mod.f90:148-183)
* ``boundary_stresses``   traction-recovery boundary stresses   (stress_mod.f90:119-406)
* ``internal_points``     Somigliana displacement and stress    (stress_mod.f90:511-886)
* ``principal``           principal and von Mises stress        (stress_mod.f90:299-359)

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbem_oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Mesh(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("ne", C.c_int),
        ("x", _dp), ("y", _dp), ("z", _dp),
        ("nconec", _ip), ("kconec", _ip), ("kode", _ip), ("bc", _dp),
        ("mu", C.c_double), ("nu", C.c_double),
    ]


class _Geo(C.Structure):
    _fields_ = [(k, _dp) for k in ("eta1", "eta2", "eta3", "xja", "xg1", "xg2", "xg3", "ff")]


def build() -> str:
    """Compile the oracle if it is missing or older than its source."""
    src = os.path.join(HERE, "bem_oracle.cpp")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.orc_adjacency.argtypes = [P(_Mesh), _ip, _ip]
        L.orc_geometry.argtypes = [P(_Mesh)] + [_dp] * 8
        L.orc_ghmat8.argtypes = [P(_Mesh), P(_Geo), C.c_int, C.c_int, _dp, C.c_int64, _dp]
        L.orc_hg.argtypes = [P(_Mesh), P(_Geo), C.c_int, C.c_int, _dp, C.c_int64, _dp, C.c_int64]
        L.orc_reorganize.argtypes = [P(_Mesh), _dp, _dp]
        L.orc_boundary_stresses.argtypes = [P(_Mesh), _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_gauss_legendre.argtypes = [C.c_int, _dp, _dp]
        L.orc_gauss_legendre.restype = None
        L.orc_principal.argtypes = [_dp, _dp, _dp]
        L.orc_principal.restype = None
        L.orc_internal_points.argtypes = [P(_Mesh), P(_Geo), _dp, _dp, C.c_int, _dp, _dp, _dp,
                                          C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_int]
        _lib = L
    return _lib


def _d(a: np.ndarray):
    assert a.dtype == np.float64
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    assert a.dtype == np.int32
    return a.ctypes.data_as(_ip)


class Oracle:
    """Holds one mesh, its geometry tables and (after ``solve``) its solution."""

    def __init__(self, mesh):
        mesh.validate()
        self.mesh = mesh
        self._keep = [mesh.x, mesh.y, mesh.z, mesh.nconec, mesh.kconec, mesh.kode, mesh.bc]
        self.cm = _Mesh(mesh.n, mesh.ne, _d(mesh.x), _d(mesh.y), _d(mesh.z), _i(mesh.nconec),
                        _i(mesh.kconec), _i(mesh.kode), _d(mesh.bc), float(mesh.mu),
                        float(mesh.nu))
        self.geo_arrays = None

    # precompute_element_geometry
    def geometry(self):
        ne = self.mesh.ne
        arrs = [np.zeros((36, ne), order="F") for _ in range(7)] + [np.zeros((9, 36, ne), order="F")]
        rc = lib().orc_geometry(C.byref(self.cm), *[_d(a) for a in arrs])
        assert rc == 0
        self.geo_arrays = dict(zip(("eta1", "eta2", "eta3", "xja", "xg1", "xg2", "xg3", "ff"), arrs))
        self.cg = _Geo(*[_d(a) for a in arrs])
        return self.geo_arrays

    def _need_geo(self):
        if self.geo_arrays is None:
            self.geometry()

    # ghmat8 (rows of collocation nodes [in0, in1))
    def ghmat8(self, in0: int = 0, in1: Optional[int] = None, pins: bool = True
               ) -> Tuple[np.ndarray, np.ndarray]:
        self._need_geo()
        n = self.mesh.n
        in1 = n if in1 is None else in1
        nrow = 3 * (in1 - in0)
        A = np.zeros((nrow, 3 * n), order="F")
        FI = np.zeros(nrow)
        rc = lib().orc_ghmat8(C.byref(self.cm), C.byref(self.cg), in0, in1, _d(A), nrow, _d(FI))
        if rc != 0:
            raise ValueError("a node lies in more than 8 elements")
        if pins:
            apply_pins(A, FI, self.mesh.pins, row0=3 * in0)
        return A, FI

    def hg(self, in0: int = 0, in1: Optional[int] = None):
        self._need_geo()
        n, ne = self.mesh.n, self.mesh.ne
        in1 = n if in1 is None else in1
        nrow = 3 * (in1 - in0)
        H = np.zeros((nrow, 3 * n), order="F")
        G = np.zeros((nrow, 27 * ne), order="F")
        rc = lib().orc_hg(C.byref(self.cm), C.byref(self.cg), in0, in1, _d(H), nrow, _d(G), nrow)
        assert rc == 0
        return H, G

    @staticmethod
    def solve(A: np.ndarray, FI: np.ndarray) -> Tuple[np.ndarray, int]:
        """LAPACK dgesv (solver_mod.f90:28) through scipy's bundled OpenBLAS."""
        from scipy.linalg import lapack
        lu, piv, x, info = lapack.dgesv(A, FI, overwrite_a=True, overwrite_b=False)
        return x, int(info)

    def reorganize(self, x: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        FI = np.array(x, dtype=np.float64, copy=True)
        DFI = np.zeros((27, self.mesh.ne), order="F")
        rc = lib().orc_reorganize(C.byref(self.cm), _d(FI), _d(DFI))
        assert rc == 0
        return FI, DFI

    def internal_points(self, FI: np.ndarray, DFI: np.ndarray, p0: int = 0,
                        p1: Optional[int] = None, kelvin_consistent: bool = False):
        self._need_geo()
        m = self.mesh
        p1 = m.l if p1 is None else p1
        cnt = p1 - p0
        u = np.zeros((3, cnt), order="F")
        s = np.zeros((6, cnt), order="F")
        pr = np.zeros((3, cnt), order="F")
        vm = np.zeros(cnt)
        FI = np.ascontiguousarray(FI, dtype=np.float64)
        DFI = np.asfortranarray(DFI, dtype=np.float64)
        rc = lib().orc_internal_points(C.byref(self.cm), C.byref(self.cg), _d(FI), _d(DFI), m.l,
                                       _d(m.cx), _d(m.cy), _d(m.cz), p0, p1, _d(u), _d(s),
                                       _d(pr), _d(vm), 1 if kelvin_consistent else 0)
        assert rc == 0
        return u, s, pr, vm

    def boundary_stresses(self, FI: np.ndarray, DFI: np.ndarray):
        """compute_boundary_stresses (stress_mod.f90:174-297, 365-406): element-nodal
        stresses (6, 9, ne), nodal averages (6, n), principal (3, n), von Mises (n)."""
        m = self.mesh
        se = np.zeros((6, 9, m.ne), order="F")
        sn = np.zeros((6, m.n), order="F")
        pr = np.zeros((3, m.n), order="F")
        vm = np.zeros(m.n)
        FI = np.ascontiguousarray(FI, dtype=np.float64)
        DFI = np.asfortranarray(DFI, dtype=np.float64)
        rc = lib().orc_boundary_stresses(C.byref(self.cm), _d(FI), _d(DFI), _d(se), _d(sn), _d(pr),
                                         _d(vm))
        assert rc == 0
        return se, sn, pr, vm

    def run(self, kelvin_consistent: bool = False):
        """The whole reference sequence (main.f90:38-68) on this mesh."""
        self.geometry()
        A, FI = self.ghmat8()
        x, info = self.solve(A, FI)
        if info != 0:
            raise RuntimeError(f"dgesv info = {info}")
        u, t = self.reorganize(x)
        res = {"x": x, "u": u, "t": t}
        (res["sigma_elem"], res["sigma_node"], res["sigma_node_prin"],
         res["sigma_node_vm"]) = self.boundary_stresses(u, t)
        if self.mesh.l > 0:
            res["u_int"], res["sigma"], res["prin"], res["vm"] = self.internal_points(
                u, t, kelvin_consistent=kelvin_consistent)
        return res


def apply_pins(A: np.ndarray, FI: np.ndarray, pins: np.ndarray, row0: int = 0) -> None:
    """Pinned displacement DOFs (value 0): equation row := unit row, rhs := 0."""
    for dof in np.asarray(pins, dtype=np.int64):
        r = int(dof) - row0
        if 0 <= r < A.shape[0]:
            A[r, :] = 0.0
            A[r, dof] = 1.0
            FI[r] = 0.0


def gauss_legendre(n: int):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss_legendre(n, _d(x), _d(w))
    return x, w


def principal(sig6) -> Tuple[np.ndarray, float]:
    s = np.ascontiguousarray(sig6, dtype=np.float64)
    p = np.zeros(3)
    vm = np.zeros(1)
    lib().orc_principal(_d(s), _d(p), _d(vm))
    return p, float(vm[0])
