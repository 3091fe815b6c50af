"""FP64 checkpoints and asynchronous snapshots (acfd_checkpoint_*,
acfd_snapshot_*): a checkpoint holds every node record in FP64, so a case
restored from it continues bit for bit; a snapshot taken before more steps
are queued gives the state of that moment while the steps run on."""
import numpy as np
import pytest

from artracfd_b200 import abi, configs
from artracfd_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _steps(s, spec, k, dts=None):
    out = []
    for q in range(k):
        dt = s.time_step(spec.cfl) if dts is None else dts[q]
        s.evolve(dt)
        out.append(dt)
    return out


@pytest.mark.parametrize("mode", [abi.FP64, abi.FP32_BULK])
def test_checkpoint_restart_continues_bit_for_bit(tmp_path, mode):
    spec = configs.tgv(n=16)
    part, model = spec.descriptors()
    path = str(tmp_path / "tgv.ckpt")
    with Solver(part, model, mode) as s:
        s.upload(spec.initial_nodes(part, model))
        s.treat_boundary(abi.TO)
        _steps(s, spec, 2)
        s.checkpoint_save(path, b"time and bodies")
        dts = _steps(s, spec, 3)
        want = s.download()
    with Solver(part, model, mode) as s:
        assert s.checkpoint_load(path) == b"time and bodies"
        _steps(s, spec, 3, dts)
        got = s.download()
    assert np.array_equal(got, want)


def test_snapshot_is_the_state_when_taken(tmp_path):
    spec = configs.tgv(n=24)
    part, model = spec.descriptors()
    with Solver(part, model, abi.FP64) as s:
        s.upload(spec.initial_nodes(part, model))
        s.treat_boundary(abi.TO)
        _steps(s, spec, 1)
        then = s.download()
        s.snapshot_begin()
        for _ in range(3):
            s.evolve(s.time_step(spec.cfl), graph=True)
        snap = s.snapshot_nodes()
        now = s.download()
        s.snapshot_save(str(tmp_path / "snap.ckpt"))
    assert np.array_equal(snap, then)
    assert not np.array_equal(now["U"], then["U"])
    with Solver(part, model, abi.FP64) as s:
        s.checkpoint_load(str(tmp_path / "snap.ckpt"))
        assert np.array_equal(s.download(), then)


def test_checkpoint_of_another_case_is_refused(tmp_path):
    a, b = configs.tgv(n=16), configs.tgv(n=20)
    path = str(tmp_path / "a.ckpt")
    pa, ma = a.descriptors()
    with Solver(pa, ma, abi.FP64) as s:
        s.upload(a.initial_nodes(pa, ma))
        s.checkpoint_save(path, b"x" * 100)
    pb, mb = b.descriptors()
    with Solver(pb, mb, abi.FP64) as s:
        with pytest.raises(abi.AcfdError):
            s.checkpoint_load(path)
    with Solver(pa, ma, abi.FP64) as s:
        with pytest.raises(abi.AcfdError):
            s.checkpoint_load(path, user_cap=10)  # the caller's block does not fit
        with pytest.raises(abi.AcfdError):
            s.checkpoint_load(str(tmp_path / "missing.ckpt"))
