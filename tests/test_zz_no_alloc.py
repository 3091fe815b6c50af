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


def _noalloc(lib, s, out_ptr, stream=None):
    U, F, pitch, plane = s.device_state()
    st = lib.acfd_cfl_noalloc(ctypes.byref(s.part), ctypes.byref(s.model), ctypes.c_void_p(U),
                              ctypes.c_void_p(F), pitch, ctypes.c_void_p(out_ptr),
                              ctypes.c_void_p(stream) if stream else None)
    assert st == abi.ACFD_OK, abi.last_error(lib)


def _two_calls_equal(spec, stream=None, steps_between=1):
    """acfd_cfl_noalloc against acfd_cfl on two calls in a row, with the state
    advanced between them; returns the last result."""
    import torch

    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    with Solver(part, model, abi.FP64) as s:
        lib = s.lib
        s.upload(node)
        if spec.bodies:
            s.compute_geometric_field()
        s.treat_boundary(abi.TO)
        got = None
        for call in range(2):
            expect = s.cfl()  # existing entry point (synchronizes its stream)
            _noalloc(lib, s, out.data_ptr(), stream.cuda_stream if stream is not None else None)
            if stream is not None:
                stream.synchronize()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            # same reduction of the same values: equal bit for bit (tolerance 0)
            assert np.array_equal(got, expect), (call, got, expect)
            assert np.all(got > 0)
            for _ in range(steps_between):
                s.evolve(s.time_step(spec.cfl))
            s.download()
        return got


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


def test_cfl_noalloc_skips_solid_nodes_like_cfl():
    """Immersed bodies: nodes inside them (did != 0) are left out of the
    maximum by both entry points."""
    spec = configs.ib_spheres(n=32, count=2, analytic=1, level=2, stepN=0)
    _two_calls_equal(spec)


def test_cfl_noalloc_many_blocks_on_a_side_stream():
    """TGV 128^3 (2.1 M computed nodes, over 2,000 blocks of partial maxima)
    on a caller's stream that is not the default one."""
    import torch

    side = torch.cuda.Stream()
    _two_calls_equal(configs.tgv(n=128), stream=side, steps_between=1)


def test_cfl_noalloc_reports_a_non_finite_state_as_nan():
    """A NaN planted in one fluid node's energy: acfd_cfl returns
    ACFD_ERR_DEVICE; the allocation-free call, which does not wait for its
    kernels, writes NaN to all three outputs instead.  The next call on a
    clean state gives acfd_cfl's maxima again (the shared scratch keeps no
    stale flag)."""
    import torch

    spec = configs.tgv(n=16)
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    with Solver(part, model, abi.FP64) as s:
        s.upload(node)
        s.treat_boundary(abi.TO)
        good = s.cfl()
        bad = s.download()
        fluid = np.flatnonzero(bad["did"] == 0)
        bad["U"][fluid[len(fluid) // 3], 0, 4] = np.nan
        s.upload(bad)
        _noalloc(s.lib, s, out.data_ptr())
        torch.cuda.synchronize()
        assert np.all(np.isnan(out.cpu().numpy()))
        s.upload(node)
        s.treat_boundary(abi.TO)
        _noalloc(s.lib, s, out.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), good)


def test_cfl_noalloc_rejects_an_inverted_pin_range():
    lib = abi.load_library()
    part, model = configs.tgv(n=16).descriptors()
    bad = abi.copy_struct(part, abi.Partition)
    bad.ns[0][0][0], bad.ns[0][0][1] = bad.ns[0][0][1], bad.ns[0][0][0]
    bad.ns[0][1][0], bad.ns[0][1][1] = bad.ns[0][1][1], bad.ns[0][1][0]
    dummy = ctypes.c_void_p(16)  # never dereferenced: the range check comes first
    st = lib.acfd_cfl_noalloc(ctypes.byref(bad), ctypes.byref(model), dummy, dummy, part.n[0], dummy, None)
    assert st == abi.ACFD_ERR_ARG
    assert "not inside" in abi.last_error(lib)


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
