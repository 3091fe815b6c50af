"""Host-side driver of libacfd_gpu through its C ABI (ctypes).

``Solver`` mirrors the reference's per-stage interface for one case
(Solve / EvolveSolution / ComputeTimeStep in solve.c, EvolveFluidDynamics in
fluid_dynamics.c, TreatBoundary in boundary_treatment.c, ComputeGeometricField
and TreatImmersedBoundary in immersed_boundary.c): same names, same level
indices, same meaning of dt.  Errors from the library raise ``AcfdError``;
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi
from .abi import AcfdError, check, load_library


class Solver:
    def __init__(self, part: abi.Partition, model: abi.Model, mode: int = abi.FP64, lib=None):
        self.lib = lib or load_library()
        self.part = part
        self.model = model
        self._geo_keep = None
        self.geo = []
        h = ctypes.c_void_p()
        check(self.lib.acfd_init(ctypes.byref(part), ctypes.byref(model), ctypes.byref(h)), self.lib)
        self.h = h
        self.set_precision(mode)

    # life cycle ---------------------------------------------------------
    def close(self):
        if self.h:
            self.lib.acfd_finalize(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_precision(self, mode: int):
        check(self.lib.acfd_set_precision(self.h, mode), self.lib)
        self.mode = mode

    def set_stream(self, stream_ptr: int | None):
        check(self.lib.acfd_set_stream(self.h, ctypes.c_void_p(stream_ptr) if stream_ptr else None), self.lib)

    def autotune(self):
        """Pick the fastest stage-kernel variant per sweep axis on this case
        for the current arithmetic form (acfd_autotune); returns the chosen
        variant per axis."""
        t = (ctypes.c_int * 3)()
        check(self.lib.acfd_autotune(self.h, t), self.lib)
        return list(t)

    def set_tiles(self, tiles):
        """Select the stage-kernel variant per sweep axis for the current
        arithmetic form (acfd_set_tiles): below BRICK_VARIANTS the brick
        kernels, from there the line-march kernels."""
        t = (ctypes.c_int * 3)(*[int(v) for v in tiles])
        check(self.lib.acfd_set_tiles(self.h, t), self.lib)

    def set_wait_limit(self, polls: int):
        """Polls of the plane-march kernels' bounded device waits before they
        give up and report through the status word (acfd_set_wait_limit);
        a negative value restores the default."""
        check(self.lib.acfd_set_wait_limit(self.h, int(polls)), self.lib)

    # learned sensor -------------------------------------------------------
    def sensor_load(self, params: np.ndarray, threshold: float):
        """Trained sensor parameters and the probability threshold above which
        a node keeps the full WENO5 reconstruction (acfd_sensor_load)."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        check(self.lib.acfd_sensor_load(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(threshold)),
              self.lib)

    def sensor_load_file(self, path: str):
        """The sensor from a weights file (acfd_sensor_load_file)."""
        check(self.lib.acfd_sensor_load_file(self.h, path.encode()), self.lib)

    def sensor_update(self) -> int:
        """Evaluate the sensor on U[TO]; returns the number of flags set."""
        n = ctypes.c_ulonglong()
        check(self.lib.acfd_sensor_update(self.h, ctypes.byref(n)), self.lib)
        return n.value

    def launches(self) -> int:
        """Kernels launched by this case so far (graph replays included)."""
        n = ctypes.c_longlong()
        check(self.lib.acfd_stats(self.h, ctypes.byref(n)), self.lib)
        return n.value

    @property
    def node_count(self) -> int:
        n = self.part.n
        return n[0] * n[1] * n[2]

    # coherence ----------------------------------------------------------
    def upload(self, node: np.ndarray, mask: int = abi.SYNC_ALL):
        node = np.ascontiguousarray(node, dtype=abi.NODE_DTYPE)
        if node.size != self.node_count:
            raise AcfdError(f"node array has {node.size} records, case needs {self.node_count}")
        check(self.lib.acfd_sync_to_device(self.h, node.ctypes.data_as(ctypes.c_void_p), mask), self.lib)

    def download(self, node: np.ndarray | None = None, mask: int = abi.SYNC_ALL) -> np.ndarray:
        if node is None:
            node = np.zeros(self.node_count, dtype=abi.NODE_DTYPE)
        check(self.lib.acfd_sync_to_host(self.h, node.ctypes.data_as(ctypes.c_void_p), mask), self.lib)
        return node

    # snapshots and FP64 checkpoints ----------------------------------
    def snapshot_begin(self):
        """Queue a copy of the node records (returns at once; later work
        overlaps the copy)."""
        check(self.lib.acfd_snapshot_begin(self.h), self.lib)

    def snapshot_nodes(self) -> np.ndarray:
        node = np.zeros(self.node_count, dtype=abi.NODE_DTYPE)
        check(self.lib.acfd_snapshot_nodes(self.h, node.ctypes.data_as(ctypes.c_void_p)), self.lib)
        return node

    def snapshot_save(self, path: str, user: bytes = b""):
        buf = ctypes.create_string_buffer(user, len(user)) if user else None
        check(self.lib.acfd_snapshot_save(self.h, path.encode(), buf, len(user)), self.lib)

    def checkpoint_save(self, path: str, user: bytes = b""):
        buf = ctypes.create_string_buffer(user, len(user)) if user else None
        check(self.lib.acfd_checkpoint_save(self.h, path.encode(), buf, len(user)), self.lib)

    def checkpoint_load(self, path: str, user_cap: int = 1 << 20) -> bytes:
        buf = ctypes.create_string_buffer(max(user_cap, 1))
        n = ctypes.c_size_t()
        check(self.lib.acfd_checkpoint_load(self.h, path.encode(), buf, user_cap, ctypes.byref(n)), self.lib)
        return buf.raw[:n.value]

    def device_state(self):
        U = ctypes.POINTER(ctypes.c_double)()
        F = ctypes.POINTER(ctypes.c_int)()
        pitch = ctypes.c_int()
        plane = ctypes.c_size_t()
        check(self.lib.acfd_device_state(self.h, ctypes.byref(U), ctypes.byref(F), ctypes.byref(pitch),
                                         ctypes.byref(plane)), self.lib)
        return (ctypes.cast(U, ctypes.c_void_p).value, ctypes.cast(F, ctypes.c_void_p).value,
                pitch.value, plane.value)

    # the time step ------------------------------------------------------
    def cfl(self) -> np.ndarray:
        v = np.zeros(3)
        check(self.lib.acfd_cfl(self.h, v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), self.lib)
        return v

    def time_step(self, numCFL: float) -> float:
        """ComputeTimeStep (solve.c:108-153): body speeds on the host, fluid
        wave speeds on the device, dt = CFL * min_s(d_s / Vmax_s)."""
        vmax = [0.0, 0.0, 0.0]
        for P in self.geo:
            V = [abs(P.V[0]) + max(abs(P.W[1]), abs(P.W[2])) * P.r,
                 abs(P.V[1]) + max(abs(P.W[2]), abs(P.W[0])) * P.r,
                 abs(P.V[2]) + max(abs(P.W[0]), abs(P.W[1])) * P.r]
            for s in range(3):
                if vmax[s] < V[s]:
                    vmax[s] = V[s]
        vf = self.cfl()
        for s in range(3):
            if vmax[s] < vf[s]:
                vmax[s] = vf[s]
        d = self.part.d
        a = d[1] / vmax[1]
        b = d[2] / vmax[2]
        inner = a if a < b else b
        c = d[0] / vmax[0]
        return numCFL * (c if c < inner else inner)

    def evolve(self, dt: float, graph: bool = False):
        fn = self.lib.acfd_evolve_fluid_graph if graph else self.lib.acfd_evolve_fluid
        check(fn(self.h, dt), self.lib)

    def profile_step(self, dt: float):
        """One time step (acfd_evolve_fluid) with CUDA events around each
        piece (acfd_profile_step): a list of (kind, axis, stage, ms), kind
        one of abi.PIECE_*."""
        cap = 256
        kind, axis, stage = ((ctypes.c_int * cap)() for _ in range(3))
        ms = (ctypes.c_float * cap)()
        n = ctypes.c_int()
        check(self.lib.acfd_profile_step(self.h, dt, cap, kind, axis, stage, ms, ctypes.byref(n)), self.lib)
        return [(kind[k], axis[k], stage[k], ms[k]) for k in range(min(n.value, cap))]

    def discretize_time(self, dt: float, s: int):
        check(self.lib.acfd_discretize_time(self.h, dt, s), self.lib)

    def lllu(self, dt, coeA, coeB, to, tn, tm, s):
        check(self.lib.acfd_lllu(self.h, dt, coeA, coeB, to, tn, tm, s), self.lib)

    def treat_boundary(self, tn: int):
        check(self.lib.acfd_treat_boundary(self.h, tn), self.lib)

    # immersed bodies ---------------------------------------------------
    def geo_upload(self, polys):
        self.geo = list(polys)
        arr = (abi.Polyhedron * len(self.geo))(*self.geo) if self.geo else None
        self._geo_keep = arr
        check(self.lib.acfd_geo_upload(self.h, arr, len(self.geo)), self.lib)

    def compute_geometric_field(self):
        check(self.lib.acfd_compute_geometric_field(self.h), self.lib)

    def treat_ib(self, tn: int):
        check(self.lib.acfd_treat_ib(self.h, tn), self.lib)

    def integrate_surface_force(self, force=None):
        """IntegrateSurfaceForce (solid_dynamics.c:51-171) on the device:
        (totN, 9) array of Fp, Fv, Tt per body; rows of bodies with state > 0
        keep the values of ``force`` (zeros when not given)."""
        n = len(self.geo)
        out = np.zeros((n, 9)) if force is None else np.array(force, dtype=np.float64).reshape(n, 9)
        if n:
            check(self.lib.acfd_integrate_surface_force(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                  self.lib)
        return out

    def collision_scan(self):
        """Contact lists of ApplyCollision's node scan: for each body a list of
        (body id, line of impact (3 ints)) in the reference's list order."""
        n = len(self.geo)
        if n == 0:
            return []
        counts = np.zeros(n, dtype=np.int32)
        gid = np.zeros(n * n, dtype=np.int32)
        N = np.zeros(n * n * 3, dtype=np.int32)
        check(self.lib.acfd_collision_scan(self.h, counts.ctypes.data, gid.ctypes.data, N.ctypes.data), self.lib)
        return [[(int(gid[p * n + c]), tuple(int(v) for v in N[3 * (p * n + c):3 * (p * n + c) + 3]))
                 for c in range(counts[p])] for p in range(n)]


    def transform_polyhedron(self, n, O, scale, angle, offset, centroid, inertia):
        """TransformPolyhedron (computational_geometry.c:162-208) of
        triangulated body n with its surface on the device.  Returns the moved
        centroid (3), the rotated inertia tensor (3, 3) and the box (3, 2) of
        the moved vertices and centroid."""
        def vec(x, k):
            return np.ascontiguousarray(np.array(x, dtype=np.float64).reshape(k))
        args = [vec(O, 3), vec(scale, 3), vec(angle, 3), vec(offset, 3)]
        c = vec(centroid, 3).copy()
        inert = vec(inertia, 9).copy()
        box = np.zeros(6)
        ptr = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        check(self.lib.acfd_transform_polyhedron(self.h, n, *[ptr(a) for a in args], ptr(c), ptr(inert), ptr(box)),
              self.lib)
        return c, inert.reshape(3, 3), box.reshape(3, 2)

    def geo_fetch(self, n):
        """The device surface of triangulated body n: dict of v, Nf, Ne, Nv
        as (rows, 3) arrays."""
        g = self.geo[n]
        out = {"v": np.zeros((g.vertN, 3)), "Nf": np.zeros((g.faceN, 3)), "Ne": np.zeros((g.edgeN, 3)),
               "Nv": np.zeros((g.vertN, 3))}
        check(self.lib.acfd_geo_fetch(self.h, n, out["v"].ctypes.data, out["Nf"].ctypes.data, out["Ne"].ctypes.data,
                                      out["Nv"].ctypes.data), self.lib)
        return out


def run(solver: Solver, numCFL: float, end: float, steps: int, now: float = 0.0):
    """The fluid part of EvolveSolution's loop (solve.c:65-89) without output
    or solid dynamics: dt from the CFL condition, rectified to end exactly at
    ``end``.  Returns (now, list of dt)."""
    dts = []
    for _ in range(steps):
        if not now < end:
            break
        dt = solver.time_step(numCFL)
        now = now + dt
        if now > end:
            dt = end - (now - dt)
            now = end
        solver.evolve(dt)
        dts.append(dt)
    return now, dts


def weno_batch(F: np.ndarray, scheme: int = 1, mode: int = abi.FP64_EXACT, lib=None) -> np.ndarray:
    """Device twins of WENO5/WENO3 on stencils F (count x 5 x 5)."""
    lib = lib or load_library()
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(-1, 5, 5)
    out = np.zeros((F.shape[0], 5))
    check(lib.acfd_weno_batch(scheme, mode, F.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p),
                              F.shape[0]), lib)
    return out


def fhat_batch(model: abi.Model, s: int, Ust: np.ndarray, mode: int = abi.FP64_EXACT, lib=None) -> np.ndarray:
    """Device twin of ComputeFhat on stencils Ust (count x 6 x 5)."""
    lib = lib or load_library()
    Ust = np.ascontiguousarray(Ust, dtype=np.float64).reshape(-1, 6, 5)
    out = np.zeros((Ust.shape[0], 5))
    check(lib.acfd_fhat_batch(ctypes.byref(model), s, mode, Ust.ctypes.data_as(ctypes.c_void_p),
                              out.ctypes.data_as(ctypes.c_void_p), Ust.shape[0]), lib)
    return out
