"""The FP32 forms' X half steps as Y sweeps of the transposed state.

For a case whose ghost fill is copies only (periodic and outflow faces) and
that has no bodies, the learned-sensor hybrid and the FP32-bulk forms run
the X half steps of a time step on
a copy of U[TO] with x and y exchanged (and the x and y momenta with them):
the Y plane-march kernel sweeps it, the copy-only fill of the transposed grid
fills its ghosts, and the state is transposed back after the last X half
step of a run.  The discretisation is the same; the Y kernel is another
compiled kernel than the X kernel, so the two agree to FP32 round-off
(relative to each variable's magnitude), on grids whose x, y and z extents
all differ.  ACFD_X_TRANSPOSE=0 at case creation keeps the X sweep.
"""
import ctypes
import dataclasses

import numpy as np
import pytest

from artracfd_b200 import abi, configs, sensor
from artracfd_b200.solver import Solver

from test_gpu_march import PLANE, SHARE, TOL_FP32_ORDER, _const_sensor
from test_gpu_parity import rel_err

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not __import__("os").path.exists(sensor.WEIGHTS),
                                 reason="no trained sensor weights")]

# transposes per time step: U[TO] in and out around the one run of X half
# steps of a 3D step (sweep order z y x x y z), and (hybrid) the x flags
XT_LAUNCHES = {"all": 3, "none": 3, "fp32": 2}


def _cases():
    tgv = configs.tgv(n=16, stepN=0)
    tgv = dataclasses.replace(tgv, m=(40, 28, 20))
    rv = configs.riemann_viscous(n=16, rng=np.random.default_rng(5))
    rv = dataclasses.replace(rv, m=(36, 24, 20))
    return {"tgv_40x28x20": tgv, "riemann_36x24x20": rv}


CASES = _cases()


def _steps(spec, params, thr, tiles, steps, transpose, monkeypatch, dts=None, graph=False, geo=None):
    """U after each step, the dts, and the launches of each step."""
    monkeypatch.setenv("ACFD_X_TRANSPOSE", "1" if transpose else "0")
    part, model = spec.descriptors()
    outs, used, per_step = [], [], []
    with Solver(part, model, abi.FP64) as s:
        s.upload(spec.initial_nodes(part, model))
        if geo is not None:
            s.geo_upload(geo)
            s.compute_geometric_field()
        s.treat_boundary(abi.TO)
        if params is None:
            s.set_precision(abi.FP32_BULK)
        else:
            s.sensor_load(params, thr)
            s.set_precision(abi.FP32_HYBRID)
        s.set_tiles(tiles)
        for k in range(steps):
            dt = s.time_step(spec.cfl) if dts is None else dts[k]
            n0 = s.launches()
            s.evolve(dt, graph=graph)
            per_step.append(s.launches() - n0)
            used.append(dt)
            outs.append(s.download()["U"][:, 0, :].copy())
    return outs, used, per_step


@pytest.mark.parametrize("flags", ["all", "none", "fp32"])
@pytest.mark.parametrize("name", CASES)
def test_transposed_x_matches_x_sweep(name, flags, monkeypatch):
    """The hybrid form with every node flagged (WENO5) or none (linear
    weights), and the FP32-bulk form: the flags do not depend on the state,
    so three steps stay within FP32 round-off."""
    spec = CASES[name]
    params = None if flags == "fp32" else _const_sensor(50.0 if flags == "all" else -50.0)
    ref, dts, lref = _steps(spec, params, 0.5, PLANE, 3, False, monkeypatch)
    got, _, lgot = _steps(spec, params, 0.5, PLANE, 3, True, monkeypatch, dts=dts)
    for k in range(3):
        assert rel_err(got[k], ref[k]) <= TOL_FP32_ORDER, (k, rel_err(got[k], ref[k]))
        assert lgot[k] == lref[k] + XT_LAUNCHES[flags], (lgot, lref)


@pytest.mark.parametrize("name", CASES)
def test_transposed_x_trained_sensor_one_step(name, monkeypatch):
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    spec = CASES[name]
    ref, dts, _ = _steps(spec, params, thr, SHARE, 1, False, monkeypatch)
    got, _, _ = _steps(spec, params, thr, SHARE, 1, True, monkeypatch, dts=dts)
    assert rel_err(got[0], ref[0]) <= TOL_FP32_ORDER, rel_err(got[0], ref[0])


def test_transposed_x_full_size_tgv(monkeypatch):
    """TGV 128^3, the benchmark's case: one step, and the captured step graph
    gives the same bits as the step launched kernel by kernel."""
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    spec = configs.tgv(n=128)
    ref, dts, _ = _steps(spec, params, thr, SHARE, 1, False, monkeypatch)
    got, _, _ = _steps(spec, params, thr, SHARE, 1, True, monkeypatch, dts=dts)
    assert rel_err(got[0], ref[0]) <= TOL_FP32_ORDER, rel_err(got[0], ref[0])
    gra, _, _ = _steps(spec, params, thr, SHARE, 1, True, monkeypatch, dts=dts, graph=True)
    assert np.array_equal(gra[0], got[0])


def test_autotune_times_the_transposed_x(monkeypatch):
    """An eligible hybrid case: acfd_autotune times the X half steps as they
    would run, transposed, and so picks a plane-march variant for them."""
    monkeypatch.setenv("ACFD_X_TRANSPOSE", "1")
    spec = CASES["tgv_40x28x20"]
    part, model = spec.descriptors()
    with Solver(part, model, abi.FP64) as s:
        s.upload(spec.initial_nodes(part, model))
        s.treat_boundary(abi.TO)
        sensor.attach(s)
        tiles = s.autotune()
        assert abi.PLANE_VARIANT <= tiles[0] < abi.STAGE_VARIANTS, tiles
        for _ in range(2):
            s.evolve(s.time_step(spec.cfl))


def test_brick_x_variant_keeps_the_x_sweep(monkeypatch):
    """A brick variant chosen for X keeps the X kernel: the same bits and
    launches with and without the transposed path."""
    spec = CASES["riemann_36x24x20"]
    params = _const_sensor(50.0)
    tiles = [0, abi.PLANE_VARIANT, abi.PLANE_VARIANT]
    ref, dts, lref = _steps(spec, params, 0.5, tiles, 2, False, monkeypatch)
    got, _, lgot = _steps(spec, params, 0.5, tiles, 2, True, monkeypatch, dts=dts)
    for k in range(2):
        assert np.array_equal(got[k], ref[k])
    assert lgot == lref


def _sphere(O, r):
    P = abi.Polyhedron()
    P.faceN = P.edgeN = P.vertN = 0
    P.state = 0
    P.r = r
    for s in range(3):
        P.O[s] = O[s]
        P.V[s] = P.W[s] = 0.0
        P.box[s][0] = O[s] - r
        P.box[s][1] = O[s] + r
    P.T = -1.0
    P.cf = 0.0
    return P


def test_bodies_keep_the_x_sweep(monkeypatch):
    """Bodies treat their ghost nodes after the fill, which the transposed
    fill does not: a case with a body keeps the X sweep (same bits and
    launches as without the transposed path), and a step graph captured
    before the body list arrived is released and captured again."""
    spec = configs.tgv(n=24, stepN=0)
    params = _const_sensor(50.0)
    geo = [_sphere((np.pi, np.pi, np.pi), 0.9)]
    ref, dts, lref = _steps(spec, params, 0.5, PLANE, 2, False, monkeypatch, geo=geo)
    got, _, lgot = _steps(spec, params, 0.5, PLANE, 2, True, monkeypatch, dts=dts, geo=geo)
    for k in range(2):
        assert np.array_equal(got[k], ref[k])
    assert lgot == lref

    def graph_then_body(transpose):
        monkeypatch.setenv("ACFD_X_TRANSPOSE", "1" if transpose else "0")
        part, model = spec.descriptors()
        with Solver(part, model, abi.FP64) as s:
            s.upload(spec.initial_nodes(part, model))
            s.treat_boundary(abi.TO)
            s.sensor_load(params, 0.5)
            s.set_precision(abi.FP32_HYBRID)
            s.set_tiles(PLANE)
            s.evolve(dts[0], graph=True)
            s.geo_upload(geo)
            s.compute_geometric_field()
            s.treat_boundary(abi.TO)
            n0 = s.launches()
            s.evolve(dts[1], graph=True)
            return s.launches() - n0, s.download()["U"][:, 0, :].copy()

    na, ua = graph_then_body(True)
    nb, ub = graph_then_body(False)
    assert na == nb
    assert rel_err(ua, ub) <= TOL_FP32_ORDER


@pytest.mark.parametrize("form", ["fp64", "fp32", "hybrid"])
def test_profile_step_lists_the_pieces_of_a_step(form, monkeypatch):
    """acfd_profile_step is acfd_evolve_fluid with events around its pieces:
    the same bits, and the pieces in step order -- per half step (sweep
    order z y x x y z) three RK stages each followed by its ghost fill; in
    the FP32 forms the X half steps on the transposed state between the two
    transposes of U[TO], and in the hybrid form first the sensor's flags and
    the x flags' transpose."""
    monkeypatch.setenv("ACFD_X_TRANSPOSE", "1")
    spec = CASES["tgv_40x28x20"]
    part, model = spec.descriptors()

    def start(s):
        s.upload(spec.initial_nodes(part, model))
        s.treat_boundary(abi.TO)
        if form == "hybrid":
            s.sensor_load(_const_sensor(50.0), 0.5)
            s.set_precision(abi.FP32_HYBRID)
        elif form == "fp32":
            s.set_precision(abi.FP32_BULK)
        s.set_tiles(SHARE)

    with Solver(part, model, abi.FP64) as a, Solver(part, model, abi.FP64) as b:
        start(a)
        start(b)
        dt = a.time_step(spec.cfl)
        pieces = a.profile_step(dt)
        b.evolve(dt)
        assert np.array_equal(a.download()["U"], b.download()["U"])
    kinds = [p[0] for p in pieces]
    half = []
    for ax in (2, 1, 0, 0, 1, 2):
        st = abi.PIECE_STAGE_XT if (form != "fp64" and ax == 0) else abi.PIECE_STAGE
        for q in range(3):
            half += [(st, ax, q), (abi.PIECE_FILL, ax, q)]
    T = (abi.PIECE_TRANSPOSE, -1, 0)
    if form == "hybrid":
        want = [(abi.PIECE_SENSOR, -1, 0), T] + half[:12] + [T] + half[12:24] + [T] + half[24:]
    elif form == "fp32":
        want = half[:12] + [T] + half[12:24] + [T] + half[24:]
    else:
        want = half
    assert [p[:3] for p in pieces] == want, kinds
    assert all(p[3] > 0.0 for p in pieces)
