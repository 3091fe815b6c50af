"""acfd_cfl_noalloc: the CFL maximum for callers that cannot allocate device
memory (a pool allocator owns all device memory, or the memory budget is fixed
before the time loop).  It must give the same result as acfd_cfl while
allocating nothing itself: the caller passes the device state and a device
output; the only scratch is the library's fixed device array.

The file is named to be collected last, so that a run stopping at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

from artracfd_b200 import abi, configs
from artracfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _noalloc(lib, s, out_ptr):
    U, F, pitch, plane = s.device_state()
    st = lib.acfd_cfl_noalloc(ctypes.byref(s.part), ctypes.byref(s.model), ctypes.c_void_p(U),
                              ctypes.c_void_p(F), pitch, ctypes.c_void_p(out_ptr), None)
    assert st == abi.ACFD_OK, abi.last_error(lib)


def test_cfl_noalloc_matches_cfl_on_two_calls():
    import torch

    spec = configs.tgv(n=32)
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    with Solver(part, model, abi.FP64) as s:
        lib = s.lib
        s.upload(node)
        s.treat_boundary(abi.TO)
        for call in range(2):
            expect = s.cfl()  # existing entry point (synchronizes its stream)
            _noalloc(lib, s, out.data_ptr())
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            # same reduction of the same values: equal bit for bit (tolerance 0)
            assert np.array_equal(got, expect), (call, got, expect)
            assert np.all(got > 0)
            # change the state between the two calls
            s.evolve(s.time_step(spec.cfl))
            s.download()


def test_cfl_noalloc_rejects_cases_beyond_its_scratch():
    lib = abi.load_library()
    part, model = configs.tgv(n=16).descriptors()
    big = abi.copy_struct(part, abi.Partition)
    for s in range(3):
        big.n[s] = 400
        big.ns[0][s][0] = 0
        big.ns[0][s][1] = 400  # 64 M computed nodes > 33.5 M
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.acfd_cfl_noalloc(ctypes.byref(big), ctypes.byref(model), dummy, dummy, 400, dummy, None)
    assert st == abi.ACFD_ERR_ARG
    assert "scratch limit" in abi.last_error(lib)
