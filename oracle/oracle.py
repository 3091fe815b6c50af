"""TEST INFRASTRUCTURE ONLY: Python access to the parity checker.

* ``Oracle``   -- the CPU restatement (oracle/_build/liboracle.so);
* ``Reference`` -- the unmodified reference compiled from its own sources
  (oracle/_ref/libacfd_ref.so, built here by oracle/Makefile and shipped
  prebuilt).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from artracfd_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libacfd_ref.so")
REF_BIN = os.path.join(HERE, "_ref", "artracfd")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_PP = ctypes.POINTER(abi.Partition)
_MP = ctypes.POINTER(abi.Model)
_GP = ctypes.POINTER(abi.Polyhedron)


def build(ref: bool = True) -> None:
    """Compile the restatement (and, when the reference tree exists, the
    reference harness) with oracle/Makefile."""
    targets = ["oracle", "ref"] if ref else ["oracle"]
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        lib = ctypes.CDLL(path)
        d, i = ctypes.c_double, ctypes.c_int
        sig = {
            "orc_symmetric_average": (None, [i, d, _dp, _dp, _dp]),
            "orc_eigenvectors": (None, [i, d, _dp, _dp, _dp]),
            "orc_weno5": (None, [_vp, _dp]),
            "orc_weno3": (None, [_vp, _dp]),
            "orc_fhat_stencil": (None, [_MP, i, _vp, _dp]),
            "orc_compute_fhat": (None, [i, i, i, i, i, _PP, _vp, _MP, _dp]),
            "orc_compute_fvhat": (None, [i, i, i, i, i, _PP, _vp, _MP, _dp]),
            "orc_lllu": (None, [d, d, d, i, i, i, i, _vp, _PP, _MP]),
            "orc_treat_domain_boundary": (None, [i, _vp, _PP, _MP]),
            "orc_treat_boundary": (None, [i, _vp, _PP, _MP, _GP, i]),
            "orc_discretize_time": (None, [d, i, _vp, _PP, _MP, _GP, i]),
            "orc_evolve_fluid": (None, [d, _vp, _PP, _MP, _GP, i]),
            "orc_cfl": (None, [_vp, _PP, _MP, _dp]),
            "orc_time_step": (d, [d, _vp, _PP, _MP, _GP, i]),
            "orc_compute_geometric_field": (None, [_vp, _PP, _MP, _GP, i]),
            "orc_treat_ib": (None, [i, _vp, _PP, _MP, _GP, i]),
            "orc_point_in_polyhedron": (i, [_dp, _GP, _ip]),
            "orc_integrate_surface_force": (None, [_vp, _PP, _MP, _GP, i, _dp]),
            "orc_collision_scan": (i, [_vp, _PP, _GP, i, i, _ip, _ip]),
            "orc_transform_polyhedron": (None, [_dp, _dp, _dp, _dp, i, i, i, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_set_node_number": (None, [_PP, _MP]),
            "orc_partition_domain": (None, [_PP]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        self.lib = lib

    # convenience wrappers -------------------------------------------------
    def weno5(self, F: np.ndarray) -> np.ndarray:
        F = np.ascontiguousarray(F, dtype=np.float64).reshape(5, 5)
        out = np.zeros(5)
        self.lib.orc_weno5(_ptr(F), out.ctypes.data_as(_dp))
        return out

    def eigenvectors(self, s, gamma, Uo):
        """(L, R) of direction s at the averaged state Uo (u, v, w, h_T, c
        after the unused first entry)."""
        Uo = np.ascontiguousarray(np.array(Uo, dtype=np.float64).reshape(6))
        L, R = np.zeros((5, 5)), np.zeros((5, 5))
        self.lib.orc_eigenvectors(s, gamma, Uo.ctypes.data_as(_dp), L.ctypes.data_as(_dp), R.ctypes.data_as(_dp))
        return L, R

    def weno3(self, F: np.ndarray) -> np.ndarray:
        F = np.ascontiguousarray(F, dtype=np.float64).reshape(3, 5)
        out = np.zeros(5)
        self.lib.orc_weno3(_ptr(F), out.ctypes.data_as(_dp))
        return out

    def fhat_stencil(self, model, s, Ust: np.ndarray) -> np.ndarray:
        U = np.zeros((6, 5))
        Ust = np.asarray(Ust, dtype=np.float64)
        U[: Ust.shape[0]] = Ust
        out = np.zeros(5)
        self.lib.orc_fhat_stencil(ctypes.byref(model), s, _ptr(U), out.ctypes.data_as(_dp))
        return out

    def evolve_fluid(self, node, part, model, dt, geo=None):
        g, n = _geo(geo)
        self.lib.orc_evolve_fluid(dt, _ptr(node), ctypes.byref(part), ctypes.byref(model), g, n)

    def lllu(self, node, part, model, dt, coeA, coeB, to, tn, tm, p):
        self.lib.orc_lllu(dt, coeA, coeB, to, tn, tm, p, _ptr(node), ctypes.byref(part),
                          ctypes.byref(model))

    def treat_boundary(self, node, part, model, tn, geo=None):
        g, n = _geo(geo)
        self.lib.orc_treat_boundary(tn, _ptr(node), ctypes.byref(part), ctypes.byref(model), g, n)

    def treat_domain_boundary(self, node, part, model, tn):
        self.lib.orc_treat_domain_boundary(tn, _ptr(node), ctypes.byref(part), ctypes.byref(model))

    def cfl(self, node, part, model) -> np.ndarray:
        v = np.zeros(3)
        self.lib.orc_cfl(_ptr(node), ctypes.byref(part), ctypes.byref(model), v.ctypes.data_as(_dp))
        return v

    def time_step(self, node, part, model, numCFL, geo=None) -> float:
        g, n = _geo(geo)
        return self.lib.orc_time_step(numCFL, _ptr(node), ctypes.byref(part), ctypes.byref(model), g, n)

    def compute_geometric_field(self, node, part, model, geo):
        g, n = _geo(geo)
        self.lib.orc_compute_geometric_field(_ptr(node), ctypes.byref(part), ctypes.byref(model), g, n)

    def treat_ib(self, node, part, model, tn, geo):
        g, n = _geo(geo)
        self.lib.orc_treat_ib(tn, _ptr(node), ctypes.byref(part), ctypes.byref(model), g, n)


    def integrate_surface_force(self, node, part, model, geo, force=None):
        """IntegrateSurfaceForce: (totN, 9) array of Fp, Fv, Tt per body; rows
        of bodies with state > 0 keep ``force`` (zeros when not given)."""
        g, n = _geo(geo)
        out = np.zeros((n, 9)) if force is None else np.array(force, dtype=np.float64).reshape(n, 9)
        self.lib.orc_integrate_surface_force(_ptr(node), ctypes.byref(part), ctypes.byref(model), g, n,
                                             out.ctypes.data_as(_dp))
        return out

    def collision_scan(self, node, part, geo):
        """Contact list of every body: [(body id, line of impact)] in the
        reference's list order."""
        g, n = _geo(geo)
        res = []
        for p in range(n):
            gid = np.zeros(max(n, 1), dtype=np.int32)
            N = np.zeros(3 * max(n, 1), dtype=np.int32)
            c = self.lib.orc_collision_scan(_ptr(node), ctypes.byref(part), g, n, p, gid.ctypes.data_as(_ip),
                                            N.ctypes.data_as(_ip))
            res.append([(int(gid[q]), tuple(int(v) for v in N[3 * q:3 * q + 3])) for q in range(c)])
        return res

    def transform_polyhedron(self, O, scale, angle, offset, surface, centroid, inertia):
        """TransformPolyhedron on copies: returns (surface dict of v, Nf, Ne,
        Nv; centroid; inertia (3, 3); box (3, 2))."""
        vec = lambda a, k: np.ascontiguousarray(np.array(a, dtype=np.float64).reshape(k))
        surf = {k: np.ascontiguousarray(np.array(surface[k], dtype=np.float64)) for k in ("v", "Nf", "Ne", "Nv")}
        c, inert, box = vec(centroid, 3).copy(), vec(inertia, 9).copy(), np.zeros(6)
        p = lambda a: a.ctypes.data_as(_dp)
        self.lib.orc_transform_polyhedron(p(vec(O, 3)), p(vec(scale, 3)), p(vec(angle, 3)), p(vec(offset, 3)),
                                          len(surf["v"]), len(surf["Nf"]), len(surf["Ne"]),
                                          *[p(surf[k]) for k in ("v", "Nf", "Ne", "Nv")], p(c), p(inert), p(box))
        return surf, c, inert.reshape(3, 3), box.reshape(3, 2)


def _geo(geo):
    if not geo:
        return None, 0
    arr = (abi.Polyhedron * len(geo))(*geo)
    return ctypes.cast(arr, _GP), len(geo)


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class Reference:
    """The reference program's own functions on a loaded case directory.
    One instance per process (the reference keeps its state in globals of
    the harness)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run make -C oracle ref where the reference exists)")
        lib = ctypes.CDLL(path)
        d, i = ctypes.c_double, ctypes.c_int
        sig = {
            "ref_load": (i, [ctypes.c_char_p]),
            "ref_get_partition": (None, [_PP]),
            "ref_get_model": (None, [_MP]),
            "ref_get_time": (None, [_dp, _dp, _dp, _ip, _ip]),
            "ref_set_numerics": (None, [i, i, i, i]),
            "ref_node_count": (i, []),
            "ref_get_nodes": (None, [_vp]),
            "ref_set_nodes": (None, [_vp]),
            "ref_geo_count": (i, []),
            "ref_get_poly": (None, [i, _GP]),
            "ref_compute_time_step": (d, []),
            "ref_evolve_fluid": (None, [d]),
            "ref_treat_boundary": (None, [i]),
            "ref_compute_geometric_field": (None, []),
            "ref_treat_ib": (None, [i]),
            "ref_evolve_solid": (None, [d, d]),
            "ref_integrate_surface_force": (None, [_dp]),
            "ref_collision_scan": (i, [i, _ip, _ip]),
            "ref_eigenvectors": (None, [i, ctypes.c_double, _dp, _dp, _dp]),
            "ref_transform_polyhedron": (None, [i, _dp, _dp, _dp, _dp]),
            "ref_get_inertia": (None, [i, _dp]),
            "ref_step": (d, []),
            "ref_weno5": (None, [_vp, _dp]),
            "ref_weno3": (None, [_vp, _dp]),
            "ref_compute_fhat": (None, [i, i, i, i, i, _dp]),
            "ref_compute_fvhat": (None, [i, i, i, i, i, _dp]),
            "ref_point_in_polyhedron": (i, [i, _dp, _ip]),
            "ref_close": (None, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        self.lib = lib

    def load(self, case_dir: str) -> None:
        cwd = os.getcwd()
        try:
            if self.lib.ref_load(os.path.abspath(case_dir).encode()) != 0:
                raise RuntimeError(f"cannot load {case_dir}")
        finally:
            os.chdir(cwd)

    def partition(self) -> abi.Partition:
        p = abi.Partition()
        self.lib.ref_get_partition(ctypes.byref(p))
        return p

    def model(self) -> abi.Model:
        m = abi.Model()
        self.lib.ref_get_model(ctypes.byref(m))
        return m

    def time(self):
        end, now, cfl = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        stepN, stepC = ctypes.c_int(), ctypes.c_int()
        self.lib.ref_get_time(ctypes.byref(end), ctypes.byref(now), ctypes.byref(cfl),
                              ctypes.byref(stepN), ctypes.byref(stepC))
        return dict(end=end.value, now=now.value, cfl=cfl.value, stepN=stepN.value, stepC=stepC.value)

    def nodes(self) -> np.ndarray:
        out = np.zeros(self.lib.ref_node_count(), dtype=abi.NODE_DTYPE)
        self.lib.ref_get_nodes(_ptr(out))
        return out

    def set_nodes(self, node: np.ndarray) -> None:
        node = np.ascontiguousarray(node)
        assert node.size == self.lib.ref_node_count()
        self.lib.ref_set_nodes(_ptr(node))

    def geometry(self):
        out = []
        for q in range(self.lib.ref_geo_count()):
            p = abi.Polyhedron()
            self.lib.ref_get_poly(q, ctypes.byref(p))
            out.append(p)
        return out

    def weno5(self, F) -> np.ndarray:
        F = np.ascontiguousarray(F, dtype=np.float64).reshape(5, 5)
        out = np.zeros(5)
        self.lib.ref_weno5(_ptr(F), out.ctypes.data_as(_dp))
        return out

    def weno3(self, F) -> np.ndarray:
        F = np.ascontiguousarray(F, dtype=np.float64).reshape(3, 5)
        out = np.zeros(5)
        self.lib.ref_weno3(_ptr(F), out.ctypes.data_as(_dp))
        return out

    def compute_fhat(self, tn, s, k, j, i) -> np.ndarray:
        out = np.zeros(5)
        self.lib.ref_compute_fhat(tn, s, k, j, i, out.ctypes.data_as(_dp))
        return out

    def compute_fvhat(self, tn, s, k, j, i) -> np.ndarray:
        out = np.zeros(5)
        self.lib.ref_compute_fvhat(tn, s, k, j, i, out.ctypes.data_as(_dp))
        return out

    def time_step(self) -> float:
        return self.lib.ref_compute_time_step()

    def evolve_fluid(self, dt: float) -> None:
        self.lib.ref_evolve_fluid(dt)

    def treat_boundary(self, tn: int) -> None:
        self.lib.ref_treat_boundary(tn)

    def integrate_surface_force(self) -> np.ndarray:
        out = np.zeros((self.lib.ref_geo_count(), 9))
        self.lib.ref_integrate_surface_force(out.ctypes.data_as(_dp))
        return out

    def collision_scan(self):
        n = self.lib.ref_geo_count()
        res = []
        for p in range(n):
            gid = np.zeros(max(n, 1), dtype=np.int32)
            N = np.zeros(3 * max(n, 1), dtype=np.int32)
            c = self.lib.ref_collision_scan(p, gid.ctypes.data_as(_ip), N.ctypes.data_as(_ip))
            res.append([(int(gid[q]), tuple(int(v) for v in N[3 * q:3 * q + 3])) for q in range(c)])
        return res

    def eigenvectors(self, s, gamma, Uo):
        Uo = np.ascontiguousarray(np.array(Uo, dtype=np.float64).reshape(6))
        L, R = np.zeros((5, 5)), np.zeros((5, 5))
        self.lib.ref_eigenvectors(s, gamma, Uo.ctypes.data_as(_dp), L.ctypes.data_as(_dp), R.ctypes.data_as(_dp))
        return L, R

    def transform_polyhedron(self, n, O, scale, angle, offset) -> None:
        args = [np.ascontiguousarray(np.array(a, dtype=np.float64).reshape(3)) for a in (O, scale, angle, offset)]
        self.lib.ref_transform_polyhedron(n, *[a.ctypes.data_as(_dp) for a in args])

    def inertia(self, n) -> np.ndarray:
        out = np.zeros(9)
        self.lib.ref_get_inertia(n, out.ctypes.data_as(_dp))
        return out.reshape(3, 3)

    def surface(self, n):
        """Copies of body n's vertices and normals: dict of v, Nf, Ne, Nv."""
        p = self.geometry()[n]
        rows = {"v": p.vertN, "Nf": p.faceN, "Ne": p.edgeN, "Nv": p.vertN}
        return {k: np.ctypeslib.as_array(getattr(p, k), shape=(rows[k] * 3,)).reshape(rows[k], 3).copy()
                for k in rows}

    def compute_geometric_field(self) -> None:
        self.lib.ref_compute_geometric_field()

    def treat_ib(self, tn: int) -> None:
        self.lib.ref_treat_ib(tn)

    def step(self) -> float:
        return self.lib.ref_step()

    def close(self) -> None:
        self.lib.ref_close()
