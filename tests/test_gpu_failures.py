"""Failure detection without a GPU fault: the failures are made on the host
(a NaN planted in the node array before upload, a case too large for the
device, a device wait limited to zero polls) and the library reports them
through its status codes, leaving the device context usable for the next
call."""
import numpy as np
import pytest

from artracfd_b200 import abi, configs
from artracfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def test_non_finite_state_is_reported_and_the_case_stays_usable():
    spec = configs.tgv(n=16)
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    with Solver(part, model, abi.FP64) as s:
        s.upload(node)
        s.treat_boundary(abi.TO)
        dt = s.time_step(spec.cfl)
        bad = s.download()
        fluid = np.flatnonzero(bad["did"] == 0)
        bad["U"][fluid[len(fluid) // 2], 0, 4] = np.nan  # energy of one fluid node
        s.upload(bad)
        with pytest.raises(abi.AcfdError) as err:
            s.time_step(spec.cfl)
        assert "non-finite" in str(err.value)
        s.upload(node)
        s.treat_boundary(abi.TO)
        assert s.time_step(spec.cfl) == dt


def test_device_allocation_failure_is_reported():
    """A case whose state needs terabytes: acfd_init fails with a status and a
    message, and the next case on the same device works."""
    big = configs.tgv(n=3000)
    part, model = big.descriptors()
    with pytest.raises(abi.AcfdError):
        Solver(part, model, abi.FP64)
    spec = configs.tgv(n=8)
    part, model = spec.descriptors()
    with Solver(part, model, abi.FP64) as s:
        s.upload(spec.initial_nodes(part, model))
        s.treat_boundary(abi.TO)
        assert s.time_step(spec.cfl) > 0.0


def test_device_wait_that_runs_out_is_reported_and_the_case_stays_usable():
    """The plane-march stage kernels' waits for their TMA planes limited to zero
    polls (acfd_set_wait_limit): every consumer warp gives up at its first
    plane, the kernel writes the case's status word and leaves (the producer
    still waits for its own copies in flight); the host reports
    ACFD_ERR_DEVICE with the message and clears the word.  With the default
    limit restored the same case steps again, bit for bit as a case that
    never failed."""
    spec = configs.tgv(n=32)
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    plane = [7, 7, 7]  # plane march on every sweep axis

    def step(s):
        s.upload(node)
        s.treat_boundary(abi.TO)
        s.evolve(s.time_step(spec.cfl))
        return s.download()["U"][:, 0, :].copy()

    with Solver(part, model, abi.FP64) as s:
        s.set_tiles(plane)
        clean = step(s)
    with Solver(part, model, abi.FP64) as s:
        s.set_tiles(plane)
        s.upload(node)
        s.treat_boundary(abi.TO)
        dt = s.time_step(spec.cfl)
        s.set_wait_limit(0)
        with pytest.raises(abi.AcfdError) as err:
            s.evolve(dt)
            s.download()
        assert "wait limit" in str(err.value)
        s.set_wait_limit(-1)
        again = step(s)
    assert np.array_equal(again, clean)


def test_debug_mode_names_the_stage_that_made_a_non_finite_value(monkeypatch):
    """ACFD_DEBUG=1 (the stand-in for a sanitizer run): every stage and ghost
    fill is followed by a scan of its level for non-finite values, checked at
    once.  A NaN planted in one fluid node of U[TO] is reported by the x-sweep
    stage that reads it, naming the sweep axis; the same case stepped in
    debug mode without the NaN gives the bits of a normal run."""
    spec = configs.tgv(n=16)
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)

    def two_steps():
        with Solver(part, model, abi.FP64) as s:
            s.upload(node)
            s.treat_boundary(abi.TO)
            for _ in range(2):
                s.evolve(s.time_step(spec.cfl), graph=True)
            return s.download()["U"][:, 0, :].copy()

    plain = two_steps()
    monkeypatch.setenv("ACFD_DEBUG", "1")
    assert np.array_equal(two_steps(), plain)
    with Solver(part, model, abi.FP64) as s:
        s.upload(node)
        s.treat_boundary(abi.TO)
        bad = s.download()
        fluid = np.flatnonzero(bad["did"] == 0)
        bad["U"][fluid[len(fluid) // 2], 0, 4] = np.nan
        s.upload(bad)
        with pytest.raises(abi.AcfdError) as err:
            s.lllu(0.01, 0.0, 1.0, abi.TO, abi.TO, abi.TN, 0)
        assert "not finite after the stage of sweep axis 0" in str(err.value)
