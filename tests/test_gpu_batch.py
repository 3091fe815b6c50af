"""The batch of independent cases (acfd_batch_*) against the same cases run one
at a time through the single-case API.

Each RK stage of the batch is one launch over the tiles of all cases, with
the plane-march kernel (the single-case plane variants) or the persistent
brick kernel (the single-case brick variant 0), or one persistent launch
runs every stage of a step; a case of the batch computes every interface
with the single-case kernel's block code, and its dt comes from its own CFL
maximum in the reference's expression.  The batch kernels are other kernels
than the single-case ones, in which the compiler may contract a different
set of FP32 (and FP64) multiply-adds into FMAs, so a case agrees with its
single-case run to FP32 round-off, its first dt (computed before any stage)
bit for bit.  The cases
mix periodic (TGV), outflow (Riemann), outflow + periodic (Sod) and
inflow/outflow/wall/periodic boundaries (channel, the ordered ghost fill).
"""
import numpy as np
import pytest

from artracfd_b200 import abi, configs, sensor
from artracfd_b200.batch import Batch
from artracfd_b200.solver import Solver

import cases
from test_gpu_march import TOL_FP32_ORDER
from test_gpu_parity import rel_err

pytestmark = pytest.mark.gpu

STEPS = 3


def _specs(inviscid=True):
    rng = np.random.default_rng(7)
    out = [configs.tgv(n=16, Re=800.0, Ma=0.2, stepN=0),
           configs.riemann_viscous(n=16, Re=1000.0, Ma=0.3, rng=rng),
           configs.tgv(n=24, Re=1200.0, Ma=0.4, stepN=0),
           cases.channel()]
    if inviscid:
        out.insert(3, configs.sod(m=(32, 4, 4)))
    return out


BRICK = [0, 0, 0]
PLANE = [abi.PLANE_VARIANT] * 3


def _single(spec, part, model, mode, steps, params=None, thr=0.5, tiles=BRICK):
    node = spec.initial_nodes(part, model)
    dts, out = [], None
    with Solver(part, model, abi.FP64 if params is not None else mode) as s:
        s.upload(node)
        s.treat_boundary(abi.TO)
        if params is not None:
            s.sensor_load(params, thr)
            s.set_precision(abi.FP32_HYBRID)
        s.set_tiles(tiles)
        for _ in range(steps):
            dt = s.time_step(spec.cfl)
            s.evolve(dt)
            dts.append(dt)
        out = s.download()["U"][:, 0, :].copy()
    return np.array(dts), out


def _batch(specs, descs, mode, steps, params=None, thr=0.5, kernel=None):
    with Batch(descs) as b:
        if kernel is not None:
            b.set_kernel(kernel)
        for c, spec in enumerate(specs):
            b.upload(c, spec.initial_nodes(*descs[c]))
            b.treat_boundary(c)
        if params is not None:
            b.sensor_load(params, thr)
        b.set_precision(mode)
        dts = b.advance([s.cfl for s in specs], steps)
        outs = [b.download(c)["U"][:, 0, :].copy() for c in range(len(specs))]
        launches = b.launches()
    return dts, outs, launches


def _agree(dts, outs, c, sdt, sout):
    assert dts[0, c] == sdt[0], (c, dts[0, c], sdt[0])
    assert np.all(np.abs(dts[:, c] - sdt) <= 1e-6 * sdt), (c, dts[:, c], sdt)
    assert rel_err(outs[c], sout) <= TOL_FP32_ORDER, (c, rel_err(outs[c], sout))


def test_batch_equals_single_cases_fp32():
    specs = _specs()
    descs = [s.descriptors() for s in specs]
    dts, outs, launches = _batch(specs, descs, abi.FP32_BULK, STEPS)
    assert launches > 0
    for c, spec in enumerate(specs):
        sdt, sout = _single(spec, *descs[c], abi.FP32_BULK, STEPS)
        _agree(dts, outs, c, sdt, sout)


@pytest.mark.skipif(not __import__("os").path.exists(sensor.WEIGHTS), reason="no trained sensor weights")
def test_batch_equals_single_cases_hybrid():
    specs = _specs()
    descs = [s.descriptors() for s in specs]
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    dts, outs, _ = _batch(specs, descs, abi.FP32_HYBRID, STEPS, params, thr)
    for c, spec in enumerate(specs):
        sdt, sout = _single(spec, *descs[c], abi.FP32_HYBRID, STEPS, params, thr)
        _agree(dts, outs, c, sdt, sout)


def test_batch_brick_viscous_cases_equal_single_cases():
    """All cases viscous, the persistent brick batch against brick variant 0."""
    specs = _specs(inviscid=False)
    descs = [s.descriptors() for s in specs]
    dts, outs, _ = _batch(specs, descs, abi.FP32_BULK, STEPS, kernel=abi.BATCH_BRICK)
    for c, spec in enumerate(specs):
        sdt, sout = _single(spec, *descs[c], abi.FP32_BULK, STEPS, tiles=BRICK)
        _agree(dts, outs, c, sdt, sout)


@pytest.mark.parametrize("form", ["fp32", "hybrid"])
def test_batch_plane_matches_single_cases(form):
    """The plane-march batch (the default for all-viscous batches) runs the
    single-case plane kernels' block code inside another kernel, where the
    compiler may contract a different set of FP32 multiply-adds into FMAs:
    the two agree to FP32 round-off (the first dt, computed before any FP32
    stage, bit for bit)."""
    specs = _specs(inviscid=False)
    descs = [s.descriptors() for s in specs]
    if form == "hybrid":
        if not __import__("os").path.exists(sensor.WEIGHTS):
            pytest.skip("no trained sensor weights")
        params, thr, _ = sensor.load(sensor.WEIGHTS)
        mode = abi.FP32_HYBRID
    else:
        params, thr, mode = None, 0.5, abi.FP32_BULK
    dts, outs, _ = _batch(specs, descs, mode, STEPS, params, thr, kernel=abi.BATCH_PLANE)
    for c, spec in enumerate(specs):
        sdt, sout = _single(spec, *descs[c], mode, STEPS, params, thr, tiles=PLANE)
        assert dts[0, c] == sdt[0], c
        assert np.all(np.abs(dts[:, c] - sdt) <= 1e-6 * sdt), (c, dts[:, c], sdt)
        assert rel_err(outs[c], sout) <= TOL_FP32_ORDER, (c, rel_err(outs[c], sout))


def test_batch_mixed_viscosity_has_no_plane_kernel():
    specs = _specs(inviscid=True)
    with Batch([s.descriptors() for s in specs]) as b:
        with pytest.raises(abi.AcfdError):
            b.set_kernel(abi.BATCH_PLANE)


def test_batch_rejects_unsupported_cases():
    spec = configs.tgv(n=10, sScheme=0, stepN=0)  # WENO3
    with pytest.raises(abi.AcfdError):
        Batch([spec.descriptors()])


def _copy_only_specs():
    rng = np.random.default_rng(11)
    return [configs.tgv(n=16, Re=800.0, Ma=0.2, stepN=0),
            configs.riemann_viscous(n=16, Re=1000.0, Ma=0.3, rng=rng),
            configs.tgv(n=24, Re=1200.0, Ma=0.4, stepN=0),
            configs.riemann_viscous(n=20, Re=2000.0, Ma=0.2, rng=rng)]


@pytest.mark.parametrize("form", ["fp32", "hybrid"])
def test_batch_persistent_step_matches_single_cases(form):
    """The persistent step (for all-viscous batches whose ghost fills are
    copies): the RK stages of each directional half step of every
    case in one launch (six per time step), the plane-march blocks and the
    ghost fills linked by per-case counters.  Each case agrees with the
    single-case plane kernels to FP32 round-off (the first dt bit for bit)
    and with the per-stage plane batch to the same bound, and the launch
    count per step is the CFL, dt, sensor and six persistent launches."""
    specs = _copy_only_specs()
    descs = [s.descriptors() for s in specs]
    if form == "hybrid":
        if not __import__("os").path.exists(sensor.WEIGHTS):
            pytest.skip("no trained sensor weights")
        params, thr, mode = (*sensor.load(sensor.WEIGHTS)[:2], abi.FP32_HYBRID)
    else:
        params, thr, mode = None, 0.5, abi.FP32_BULK
    dts, outs, launches = _batch(specs, descs, mode, STEPS, params, thr, kernel=abi.BATCH_PERSISTENT)
    pdts, pouts, _ = _batch(specs, descs, mode, STEPS, params, thr, kernel=abi.BATCH_PLANE)
    for c, spec in enumerate(specs):
        sdt, sout = _single(spec, *descs[c], mode, STEPS, params, thr, tiles=PLANE)
        assert dts[0, c] == sdt[0], c
        assert np.all(np.abs(dts[:, c] - sdt) <= 1e-6 * sdt), (c, dts[:, c], sdt)
        assert rel_err(outs[c], sout) <= TOL_FP32_ORDER, (c, rel_err(outs[c], sout))
        assert rel_err(outs[c], pouts[c]) <= TOL_FP32_ORDER, (c, rel_err(outs[c], pouts[c]))
    per_case = 1 + (2 if form == "hybrid" else 0)  # CFL; the sensor's two kernels
    assert launches == STEPS * (len(specs) * per_case + 1 + 6), launches


def test_batch_persistent_step_is_offered_for_copy_only_viscous_cases():
    specs = _copy_only_specs()
    with Batch([s.descriptors() for s in specs]) as b:
        b.set_kernel(abi.BATCH_PERSISTENT)  # accepted
    specs = _specs(inviscid=False)  # the channel needs formulas in its fill
    with Batch([s.descriptors() for s in specs]) as b:
        with pytest.raises(abi.AcfdError):
            b.set_kernel(abi.BATCH_PERSISTENT)
