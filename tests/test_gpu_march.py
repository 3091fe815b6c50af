"""Line-march and plane-march stage kernels against the brick kernels and the
oracle, through the C ABI (acfd_set_tiles selects the kernel of each sweep
axis).

* fast FP64 form on the line-march and plane-march kernels: within the plain
  path's tolerance of the reference on every golden case (all option
  variants: WENO3/RK2, Steger-Warming, arithmetic mean, walls, inflow,
  gravity with the operator-by-operator form, 2D-collapsed, immersed bodies);
* FP32 and hybrid forms: the march and brick kernels compute the same
  discretisation in a different FP32 operation order; they agree to FP32
  round-off (tolerance below);
* the launch size of one kernel (segments per line, or equal shares of the
  tiles' planes) does not change a single bit, on the golden cases and at the
  benchmark size (TGV 128^3, FP64 and FP32 forms), where the lines are cut
  into many segments and the share variants march several items per block.
"""
import ctypes

import numpy as np
import pytest

from artracfd_b200 import abi, configs, sensor
from artracfd_b200.solver import Solver

import golden_io
from test_gpu_parity import TOL_STEP, rel_err

pytestmark = pytest.mark.gpu

CASES = golden_io.names()
BRICK = [0, 0, 0]
MARCH = [abi.BRICK_VARIANTS] * 3
PLANE = [abi.PLANE_VARIANT] * 3
SHARE = [abi.PLANE_SHARE_VARIANT] * 3
FAMILIES = {"march": MARCH, "plane": PLANE, "share": SHARE}
# FP32 stencil arithmetic in two operation orders, after two steps (relative
# to the magnitude of each conservative variable)
TOL_FP32_ORDER = 2e-5


def _const_sensor(value):
    p = np.zeros(sensor.param_count(), dtype=np.float32)
    p[-1] = value
    return p


def run(b, mode, tiles, steps, dts=None, params=None, thr=0.5):
    out = []
    with Solver(b.part, b.model, abi.FP64 if params is not None else mode) as s:
        s.upload(b.initial_nodes())
        if b.geo:
            s.geo_upload(b.geo)
        if params is not None:
            abi.check(s.lib.acfd_sensor_load(s.h, params.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), thr), s.lib)
            s.set_precision(abi.FP32_HYBRID)
        s.set_tiles(tiles)
        for k in range(steps):
            dt = s.time_step(b.cfl) if dts is None else dts[k]
            s.evolve(dt)
            out.append(s.download()["U"][:, 0, :].copy())
    return out


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("name", CASES)
def test_march_fp64_within_tolerance_per_step(name, family):
    """Each golden step from the reference's own state of the step before:
    the bound holds per step, not accumulated."""
    b = golden_io.Bundle(name)
    with Solver(b.part, b.model, abi.FP64) as s:
        if b.geo:
            s.geo_upload(b.geo)
        s.set_tiles(FAMILIES[family])
        for k in range(len(b.dt)):
            s.upload(b.nodes_after(k))
            s.evolve(b.dt[k])
            got = s.download()["U"][:, 0, :]
            assert rel_err(got, b.U_after(k + 1)) <= TOL_STEP, (k + 1, rel_err(got, b.U_after(k + 1)))


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("name", CASES)
def test_march_fp32_matches_brick(name, family):
    b = golden_io.Bundle(name)
    a = run(b, abi.FP32_BULK, FAMILIES[family], len(b.dt), dts=b.dt)
    c = run(b, abi.FP32_BULK, BRICK, len(b.dt), dts=b.dt)
    for k in range(len(b.dt)):
        assert rel_err(a[k], c[k]) <= TOL_FP32_ORDER, (k, rel_err(a[k], c[k]))


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("value", [-50.0, 50.0])
def test_march_hybrid_matches_brick(value, family):
    """Constant sensors: every interface smooth (linear weights) or every
    interface flagged (full WENO5)."""
    b = golden_io.Bundle("tgv")
    dts = [b.dt[0]] * 3
    a = run(b, None, FAMILIES[family], 3, dts=dts, params=_const_sensor(value))
    c = run(b, None, BRICK, 3, dts=dts, params=_const_sensor(value))
    assert rel_err(a[-1], c[-1]) <= TOL_FP32_ORDER


@pytest.mark.skipif(not __import__("os").path.exists(sensor.WEIGHTS), reason="no trained sensor weights")
def test_march_hybrid_trained_sensor_matches_brick():
    """The trained sensor on the shock-cylinder state (flagged and smooth
    interfaces side by side in the same warps)."""
    spec = configs.shock_cylinder(m=(64, 32, 4), segments=24)
    spec.bodies = []
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    res = []
    for tiles in (MARCH, PLANE, BRICK):
        with Solver(part, model, abi.FP64) as s:
            s.upload(node)
            s.treat_boundary(abi.TO)
            dt = 0.5 * s.time_step(spec.cfl)
            s.sensor_load(params, thr)
            s.set_precision(abi.FP32_HYBRID)
            s.set_tiles(tiles)
            for _ in range(5):
                s.evolve(dt)
            res.append(s.download()["U"][:, 0, :].copy())
    assert rel_err(res[0], res[2]) <= TOL_FP32_ORDER
    assert rel_err(res[1], res[2]) <= TOL_FP32_ORDER


@pytest.mark.parametrize("family", FAMILIES)
@pytest.mark.parametrize("mode", [abi.FP64, abi.FP32_BULK])
def test_march_launch_size_does_not_change_results(mode, family):
    """One kernel launched for 1, 2 or 4 waves gives the same bits; the share
    kernel of the plane march against its segment kernel: bit for bit in the
    FP64 form, to round-off in the FP32 form (two compiled kernels)."""
    b = golden_io.Bundle("tgv")
    dts = [b.dt[0]] * 2
    first = FAMILIES[family][0]
    ref = run(b, mode, [first] * 3, 2, dts=dts)[-1]
    for v in (first + 1, first + 2):
        assert np.array_equal(run(b, mode, [v] * 3, 2, dts=dts)[-1], ref), v
    if family == "plane":
        got = run(b, mode, SHARE, 2, dts=dts)[-1]
        if mode == abi.FP64:
            assert np.array_equal(got, ref)
        else:
            assert rel_err(got, ref) <= TOL_FP32_ORDER


@pytest.mark.parametrize("mode", [abi.FP64, abi.FP32_BULK])
def test_march_full_size_tgv_one_step(mode):
    """TGV 128^3, one step.  The line-march and plane-march kernels agree with
    the brick kernels to the form's round-off, and one kernel's launch size
    does not change a single bit: lines cut into segments for 1, 2 or 4 waves,
    or equal shares of all tiles' planes, where every block marches two or
    three items of different tiles through one ring.  A segment's first
    interface takes the viscous terms of the node left of it from the same
    arithmetic as the segment before it, which carries them from its march,
    so that both sides of the interface see the same flux.  The segment and
    share variants of the plane march are two compiled kernels: the assembler
    may fuse their multiply-adds differently, so they agree bit for bit in the
    FP64 form (as measured) and to round-off in the FP32 form."""
    spec = configs.tgv(n=128)
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)

    def one(tiles):
        with Solver(part, model, mode) as s:
            s.upload(node)
            s.treat_boundary(abi.TO)
            s.set_tiles(tiles)
            s.evolve(s.time_step(spec.cfl))
            return s.download()["U"][:, 0, :].copy()

    tol = TOL_FP32_ORDER if mode == abi.FP32_BULK else TOL_STEP
    brick = one(BRICK)
    # kernel families: line march, plane march by segments, plane march by shares
    refs = []
    for first in (abi.BRICK_VARIANTS, abi.PLANE_VARIANT, abi.PLANE_SHARE_VARIANT):
        ref = one([first] * 3)
        assert rel_err(ref, brick) <= tol
        for v in (first + 1, first + 2):
            assert np.array_equal(one([v] * 3), ref), v
        refs.append(ref)
    if mode == abi.FP64:
        assert np.array_equal(refs[2], refs[1])
    else:
        assert rel_err(refs[2], refs[1]) <= TOL_FP32_ORDER
