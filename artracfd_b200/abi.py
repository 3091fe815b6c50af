"""ctypes mirror of include/acfd.h and the loader of libacfd_gpu.so.

The structures here have the exact layout of the C ABI.  ``NODE_DTYPE`` is
the numpy view of ``acfd_node_t``, which has the same layout as the reference
``Node`` record (commons.h:128-134): four int32 flags and U[3][5] doubles,
136 bytes per node.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libacfd_gpu.so")

# status codes
ACFD_OK = 0
ACFD_ERR_ARG = 1
ACFD_ERR_CUDA = 2
ACFD_ERR_STATE = 3
ACFD_ERR_DEVICE = 4
ACFD_ERR_NOMEM = 5
ACFD_ERR_NOT_FOUND = 6
ACFD_ERR_IO = 7
# levels / operators
TO, TN, TM = 0, 1, 2
# pieces of a profiled step (acfd_profile_step)
PIECE_STAGE, PIECE_STAGE_XT, PIECE_FILL, PIECE_TRANSPOSE, PIECE_SENSOR = 0, 1, 2, 3, 4
X, Y, Z, DIMS, PHI = 0, 1, 2, 3, 4
# arithmetic forms
FP64_EXACT, FP64, FP32_BULK, FP32_HYBRID = 0, 1, 2, 3
# stage-kernel variants (acfd_set_tiles): bricks below BRICK_VARIANTS, then
# the line-march kernels with 1, 2, 4 waves, then from PLANE_VARIANT the
# plane-march kernels with 1, 2, 4 waves (lines cut into segments per tile)
BRICK_VARIANTS, PLANE_VARIANT, STAGE_VARIANTS = 2, 5, 11
# the plane march with equal shares of all tiles' planes per block
PLANE_SHARE_VARIANT = PLANE_VARIANT + 3
# stage kernel of a batch (acfd_batch_set_kernel)
BATCH_BRICK, BATCH_PLANE, BATCH_PERSISTENT = 0, 1, 2
# sync masks
SYNC_TO, SYNC_TN, SYNC_TM, SYNC_U, SYNC_FLAGS, SYNC_ALL = 0x1, 0x2, 0x4, 0x7, 0x8, 0xF
# boundary kinds (commons.h:83-87)
INFLOW, OUTFLOW, SLIPWALL, NOSLIPWALL, PERIODIC = 0, 1, 2, 3, 4

NODE_DTYPE = np.dtype(
    [("did", "<i4"), ("fid", "<i4"), ("lid", "<i4"), ("gst", "<i4"), ("U", "<f8", (3, 5))]
)
assert NODE_DTYPE.itemsize == 136


class Partition(ctypes.Structure):
    _fields_ = [
        ("m", ctypes.c_int * 3),
        ("n", ctypes.c_int * 3),
        ("ng", ctypes.c_int * 3),
        ("gl", ctypes.c_int),
        ("collapse", ctypes.c_int),
        ("d", ctypes.c_double * 3),
        ("dd", ctypes.c_double * 3),
        ("tinyL", ctypes.c_double),
        ("ns", ((ctypes.c_int * 2) * 3) * 15),
        ("np", ((ctypes.c_int * 2) * 3) * 3),
        ("path", (ctypes.c_int * 3) * 30),
        ("pathSep", ctypes.c_int * 4),
        ("typeBC", ctypes.c_int * 7),
        ("N", (ctypes.c_int * 3) * 7),
        ("varBC", (ctypes.c_double * 6) * 7),
        ("domain", (ctypes.c_double * 2) * 3),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = np.ctypeslib.as_array(v).copy() if hasattr(v, "_length_") else v
        return out


class Model(ctypes.Structure):
    _fields_ = [
        ("tScheme", ctypes.c_int),
        ("sScheme", ctypes.c_int),
        ("sL", ctypes.c_int),
        ("sR", ctypes.c_int),
        ("multidim", ctypes.c_int),
        ("jacobMean", ctypes.c_int),
        ("fluxSplit", ctypes.c_int),
        ("psi", ctypes.c_int),
        ("ibmLayer", ctypes.c_int),
        ("gState", ctypes.c_int),
        ("sState", ctypes.c_int),
        ("refMa", ctypes.c_double),
        ("refMu", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("gasR", ctypes.c_double),
        ("cv", ctypes.c_double),
        ("refL", ctypes.c_double),
        ("refRho", ctypes.c_double),
        ("refV", ctypes.c_double),
        ("refT", ctypes.c_double),
        ("g", ctypes.c_double * 3),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "_length_") else v
        return out


class Polyhedron(ctypes.Structure):
    _fields_ = [
        ("faceN", ctypes.c_int),
        ("edgeN", ctypes.c_int),
        ("vertN", ctypes.c_int),
        ("state", ctypes.c_int),
        ("r", ctypes.c_double),
        ("O", ctypes.c_double * 3),
        ("V", ctypes.c_double * 3),
        ("W", ctypes.c_double * 3),
        ("T", ctypes.c_double),
        ("cf", ctypes.c_double),
        ("box", (ctypes.c_double * 2) * 3),
        ("f", ctypes.POINTER(ctypes.c_int)),
        ("Nf", ctypes.POINTER(ctypes.c_double)),
        ("e", ctypes.POINTER(ctypes.c_int)),
        ("Ne", ctypes.POINTER(ctypes.c_double)),
        ("v", ctypes.POINTER(ctypes.c_double)),
        ("Nv", ctypes.POINTER(ctypes.c_double)),
        ("area", ctypes.c_double),
    ]


def copy_struct(src, cls):
    dst = cls()
    ctypes.memmove(ctypes.byref(dst), ctypes.byref(src), ctypes.sizeof(cls))
    return dst


_LIB = None


class AcfdError(RuntimeError):
    pass


def load_library(path: str | None = None):
    """Load libacfd_gpu.so.  Raises if it has not been built: there is no
    CPU fallback for the product path."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise AcfdError(
            f"libacfd_gpu.so not found at {p}; build it with "
            "`python -m artracfd_b200.build` (there is no CPU fallback)"
        )
    lib = ctypes.CDLL(p)
    vp = ctypes.c_void_p
    pp = ctypes.POINTER(ctypes.c_void_p)
    i, d, u, sz = ctypes.c_int, ctypes.c_double, ctypes.c_uint, ctypes.c_size_t
    dp = ctypes.POINTER(ctypes.c_double)
    sigs = {
        "acfd_init": [ctypes.POINTER(Partition), ctypes.POINTER(Model), pp],
        "acfd_finalize": [vp],
        "acfd_last_error": [ctypes.c_char_p, sz],
        "acfd_abi_version": [],
        "acfd_set_stream": [vp, vp],
        "acfd_set_precision": [vp, i],
        "acfd_stats": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "acfd_synchronize": [vp],
        "acfd_autotune": [vp, ctypes.POINTER(ctypes.c_int)],
        "acfd_set_tiles": [vp, ctypes.POINTER(ctypes.c_int)],
        "acfd_set_wait_limit": [vp, ctypes.c_longlong],
        "acfd_mlp_param_count": [],
        "acfd_sensor_load": [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_float],
        "acfd_sensor_load_file": [vp, ctypes.c_char_p],
        "acfd_sensor_update": [vp, ctypes.POINTER(ctypes.c_ulonglong)],
        "acfd_sensor_flags": [vp, ctypes.POINTER(vp)],
        "acfd_sensor_features": [vp, i, vp, vp],
        "acfd_mlp_forward": [vp, vp, i, vp, vp],
        "acfd_mlp_grad": [vp, vp, vp, i, ctypes.c_float, vp, vp, vp],
        "acfd_mlp_adam": [vp, vp, vp, vp, i, ctypes.c_float, ctypes.c_float, vp],
        "acfd_sync_to_device": [vp, vp, u],
        "acfd_sync_to_host": [vp, vp, u],
        "acfd_device_state": [vp, ctypes.POINTER(dp), ctypes.POINTER(ctypes.POINTER(ctypes.c_int)),
                              ctypes.POINTER(i), ctypes.POINTER(sz)],
        "acfd_cfl": [vp, dp],
        "acfd_cfl_noalloc": [ctypes.POINTER(Partition), ctypes.POINTER(Model), vp, vp, i, vp, vp],
        "acfd_evolve_fluid": [vp, d],
        "acfd_evolve_fluid_graph": [vp, d],
        "acfd_profile_step": [vp, d, i, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(i),
                              ctypes.POINTER(ctypes.c_float), ctypes.POINTER(i)],
        "acfd_discretize_time": [vp, d, i],
        "acfd_lllu": [vp, d, d, d, i, i, i, i],
        "acfd_treat_boundary": [vp, i],
        "acfd_geo_upload": [vp, ctypes.POINTER(Polyhedron), i],
        "acfd_compute_geometric_field": [vp],
        "acfd_treat_ib": [vp, i],
        "acfd_integrate_surface_force": [vp, dp],
        "acfd_snapshot_begin": [vp],
        "acfd_snapshot_nodes": [vp, vp],
        "acfd_snapshot_save": [vp, ctypes.c_char_p, vp, sz],
        "acfd_checkpoint_save": [vp, ctypes.c_char_p, vp, sz],
        "acfd_checkpoint_load": [vp, ctypes.c_char_p, vp, sz, ctypes.POINTER(sz)],
        "acfd_collision_scan": [vp, vp, vp, vp],
        "acfd_transform_polyhedron": [vp, i, dp, dp, dp, dp, dp, dp, dp],
        "acfd_geo_fetch": [vp, i, vp, vp, vp, vp],
        "acfd_weno_batch": [i, i, vp, vp, i],
        "acfd_fhat_batch": [ctypes.POINTER(Model), i, i, vp, vp, i],
        "acfd_batch_init": [i, ctypes.POINTER(Partition), ctypes.POINTER(Model), pp],
        "acfd_batch_finalize": [vp],
        "acfd_batch_case": [vp, i, pp],
        "acfd_batch_set_precision": [vp, i],
        "acfd_batch_sensor_load": [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_float],
        "acfd_batch_advance": [vp, dp, i, dp],
        "acfd_batch_stats": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "acfd_batch_set_stream": [vp, vp],
        "acfd_batch_set_kernel": [vp, i],
    }
    for name, args in sigs.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    _LIB = lib
    return lib


def last_error(lib=None) -> str:
    lib = lib or load_library()
    buf = ctypes.create_string_buffer(1024)
    lib.acfd_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int, lib=None):
    if status != ACFD_OK:
        raise AcfdError(f"libacfd_gpu status {status}: {last_error(lib)}")
