"""Load the golden fixtures (tests/golden/*.npz) into ABI objects."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from artracfd_b200 import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
JUNK = np.frombuffer(b"\x01" * 8, dtype="<f8")[0]  # the reference's memset(U, 1) value


def names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def _struct(cls, raw):
    obj = cls()
    assert raw.size == ctypes.sizeof(cls)
    ctypes.memmove(ctypes.byref(obj), raw.tobytes(), raw.size)
    return obj


def _geo(z, prefix):
    keep = []
    geo = []
    if prefix + "count" not in z:
        return geo, keep
    for q in range(int(z[prefix + "count"])):
        p = f"{prefix}{q}_"
        P = abi.Polyhedron()
        P.faceN, P.edgeN, P.vertN, P.state = (int(v) for v in z[p + "scal"])
        real = z[p + "real"]
        P.r = real[0]
        for s in range(3):
            P.O[s] = real[1 + s]
            P.V[s] = real[4 + s]
            P.W[s] = real[7 + s]
        P.T = real[10]
        P.cf = real[11]
        for s in range(3):
            for m in range(2):
                P.box[s][m] = real[12 + 2 * s + m]
        if P.faceN > 0:
            arrs = {}
            for key, ct in (("f", ctypes.c_int), ("Nf", ctypes.c_double), ("e", ctypes.c_int),
                            ("Ne", ctypes.c_double), ("v", ctypes.c_double), ("Nv", ctypes.c_double)):
                a = np.ascontiguousarray(z[p + key], dtype=np.int32 if ct is ctypes.c_int else np.float64)
                arrs[key] = a
                setattr(P, key, a.ctypes.data_as(ctypes.POINTER(ct)))
            keep.append(arrs)
        geo.append(P)
    return geo, keep


def nodes_from(U, flags):
    node = np.zeros(U.shape[0], dtype=abi.NODE_DTYPE)
    node["U"][:] = JUNK
    node["U"][:, 0, :] = U
    for q, f in enumerate(("did", "fid", "lid", "gst")):
        node[f] = flags[:, q]
    return node


class Bundle:
    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.name = name
        self.z = z
        self.part = _struct(abi.Partition, z["part"])
        self.model = _struct(abi.Model, z["model"])
        self.cfl = float(z["cfl"])
        self.end = float(z["end"])
        self.dt = z["dt"]
        self.geo, self._keep = _geo(z, "geo_")
        self.geo_moved, self._keep2 = _geo(z, "geos_")

    def initial_nodes(self):
        return nodes_from(self.z["U0"], self.z["flags0"])

    def U_after(self, k):
        return self.z[f"U{k}"]

    @property
    def has_motion(self):
        return "Us" in self.z
