"""Failure detection without a GPU fault: the failures are made on the host
(a NaN planted in the node array before upload, a case too large for the
device) and the library reports them through its status codes, leaving the
device context usable for the next call."""
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
