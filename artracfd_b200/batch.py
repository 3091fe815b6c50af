"""A batch of independent cases advanced together (acfd_batch_*).

Every RK stage of every case is one launch over the tiles of all cases (the
plane-march kernel, or the persistent brick kernel); each case keeps its own
grid, model, boundary conditions and time step (dt from its own CFL maximum,
on the device); one time step of the batch is a CUDA graph.

    from artracfd_b200 import configs
    from artracfd_b200.batch import Batch

    specs = configs.batch_cases(count=48, seed=42)
    with Batch([s.descriptors() for s in specs]) as b:
        for c, spec in enumerate(specs):
            b.upload(c, spec.initial_nodes(*b.descriptors(c)))
            b.treat_boundary(c)
        dts = b.advance([s.cfl for s in specs], steps=100)
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import abi
from .abi import check, load_library
from .solver import Solver


class _CaseView(Solver):
    """A case of a batch seen through the single-case API (the batch owns
    the handle: closing the view does nothing)."""

    def __init__(self, lib, h, part, model):  # noqa: D401 - no acfd_init here
        self.lib = lib
        self.h = h
        self.part = part
        self.model = model
        self._geo_keep = None
        self.geo = []
        self.mode = abi.FP32_BULK

    def close(self):
        self.h = None

    def __del__(self):
        pass


class Batch:
    def __init__(self, descriptors, lib=None):
        """descriptors: list of (Partition, Model), one per case."""
        self.lib = lib or load_library()
        self.parts = [p for p, _ in descriptors]
        self.models = [m for _, m in descriptors]
        n = len(descriptors)
        P = (abi.Partition * n)(*self.parts)
        M = (abi.Model * n)(*self.models)
        h = ctypes.c_void_p()
        check(self.lib.acfd_batch_init(n, P, M, ctypes.byref(h)), self.lib)
        self.h = h
        self.n = n
        self.views = []
        for c in range(n):
            ch = ctypes.c_void_p()
            check(self.lib.acfd_batch_case(self.h, c, ctypes.byref(ch)), self.lib)
            self.views.append(_CaseView(self.lib, ch, self.parts[c], self.models[c]))

    def close(self):
        if self.h:
            for v in self.views:
                v.close()
            self.lib.acfd_batch_finalize(self.h)
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

    def descriptors(self, c):
        return self.parts[c], self.models[c]

    def case(self, c) -> Solver:
        return self.views[c]

    def upload(self, c, node):
        self.views[c].upload(node)

    def download(self, c):
        return self.views[c].download()

    def treat_boundary(self, c, tn=abi.TO):
        self.views[c].treat_boundary(tn)

    def set_stream(self, stream_ptr: int):
        check(self.lib.acfd_batch_set_stream(self.h, ctypes.c_void_p(stream_ptr)), self.lib)

    def set_precision(self, mode: int):
        check(self.lib.acfd_batch_set_precision(self.h, mode), self.lib)

    def set_kernel(self, kernel: int):
        """abi.BATCH_PLANE (one plane-march launch per RK stage; the default
        when the cases allow it), abi.BATCH_PERSISTENT (the RK stages of each
        directional half step of every case in one persistent launch) or
        abi.BATCH_BRICK (persistent brick kernel, one launch per RK stage)."""
        check(self.lib.acfd_batch_set_kernel(self.h, kernel), self.lib)

    def sensor_load(self, params: np.ndarray, threshold: float):
        p = np.ascontiguousarray(params, dtype=np.float32)
        check(self.lib.acfd_batch_sensor_load(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                              float(threshold)), self.lib)

    def advance(self, cfl, steps: int) -> np.ndarray:
        """Advance every case `steps` time steps; returns dt[steps, case]."""
        c = np.ascontiguousarray(cfl, dtype=np.float64)
        if c.size != self.n:
            raise ValueError(f"{c.size} CFL numbers for {self.n} cases")
        dts = np.zeros((max(steps, 1), self.n))
        check(self.lib.acfd_batch_advance(self.h, c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(steps),
                                          dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), self.lib)
        return dts[:steps]

    def launches(self) -> int:
        n = ctypes.c_longlong()
        check(self.lib.acfd_batch_stats(self.h, ctypes.byref(n)), self.lib)
        return n.value
