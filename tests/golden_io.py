"""Load the golden fixtures (tests/golden/*.npz) into ABI objects."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from artracfd_b200 import abi
from artracfd_b200.case import load_polyhedra

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
JUNK = np.frombuffer(b"\x01" * 8, dtype="<f8")[0]  # the reference's memset(U, 1) value


def names():
    """The golden cases (bodies_*.npz hold preprocessed bodies, not cases)."""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and not f.startswith("bodies_"))


def _struct(cls, raw):
    obj = cls()
    assert raw.size == ctypes.sizeof(cls)
    ctypes.memmove(ctypes.byref(obj), raw.tobytes(), raw.size)
    return obj


def _geo(z, prefix):
    return load_polyhedra(z, prefix)


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

    def nodes_after(self, k):
        """The reference's own state after k fluid steps (k = 0: the initial
        state); the bodies do not move in these steps, so the flags are the
        initial ones."""
        if k == 0:
            return self.initial_nodes()
        return nodes_from(self.U_after(k), self.z["flags0"])

    @property
    def has_motion(self):
        return "Us" in self.z
