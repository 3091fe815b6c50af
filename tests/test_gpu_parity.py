"""Parity of the CUDA path with the reference, through the C ABI.

* exact FP64 form: bitwise equal to the reference's own results (golden
  fixtures made by the reference) for inviscid cases; viscous cases differ
  only through pow() in Sutherland's law and are held to 1e-13 relative;
* fast FP64 form (the plain GPU path): within 1e-12 relative per step
  (each step taken from the reference's own state of the step before, so
  the bound holds for every step's increment and is not accumulated) and
  1e-10 after 100 steps, against the oracle on the same inputs;
* FP32 bulk form: L1/Linf error of density, momentum and pressure stated
  against the FP64 oracle;
* per-point device twins (WENO5/WENO3, ComputeFhat) against the oracle;
* full-size properties at the benchmark size (TGV 128^3): conservation on
  the periodic torus and free-stream preservation.
"""
import numpy as np
import pytest

from artracfd_b200 import abi, configs
from artracfd_b200.solver import Solver, fhat_batch, weno_batch
from oracle.oracle import Oracle

import golden_io

pytestmark = pytest.mark.gpu

CASES = golden_io.names()
# tolerance of the FP64 forms (relative to the largest magnitude of each
# conservative variable)
TOL_STEP = 1e-12
TOL_100 = 1e-10
TOL_EXACT_VISCOUS = 1e-13


def scales(b):
    """Magnitude of each conservative variable: density, the momentum vector
    (shared by its three components, so that a component that is zero up to
    round-off is not divided by its own round-off) and total energy."""
    b = np.abs(np.asarray(b, dtype=np.float64))
    mom = max(b[..., 1].max(), b[..., 2].max(), b[..., 3].max())
    return np.array([b[..., 0].max(), mom, mom, mom, b[..., 4].max()])


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    sc = np.maximum(scales(b), 1e-300)
    return max(np.max(np.abs(a[..., v] - b[..., v])) / sc[v] for v in range(5))


@pytest.fixture(scope="module")
def orc():
    return Oracle()


def gpu_run(b, mode, steps, graph=False, dts=None):
    out = []
    times = []
    with Solver(b.part, b.model, mode) as s:
        s.upload(b.initial_nodes())
        if b.geo:
            s.geo_upload(b.geo)
        for k in range(steps):
            dt = s.time_step(b.cfl) if dts is None else dts[k]
            s.evolve(dt, graph=graph)
            times.append(dt)
            out.append(s.download()["U"][:, 0, :].copy())
    return out, times


@pytest.mark.parametrize("name", CASES)
def test_exact_form_matches_reference(name):
    b = golden_io.Bundle(name)
    outs, dts = gpu_run(b, abi.FP64_EXACT, len(b.dt))
    viscous = b.model.refMu > 0.0
    for k, (got, dt) in enumerate(zip(outs, dts)):
        ref = b.U_after(k + 1)
        if viscous:
            assert abs(dt - b.dt[k]) <= 1e-14 * b.dt[k]
            assert rel_err(got, ref) <= TOL_EXACT_VISCOUS
        else:
            assert dt == b.dt[k]
            assert np.array_equal(got, ref), f"step {k + 1}: max|diff| {np.nanmax(np.abs(got - ref))}"


def gpu_each_step(b, mode, tiles=None):
    """Every golden step taken on the GPU from the reference's own state of
    the step before, with the reference's dt: U[TO] after each step."""
    out = []
    with Solver(b.part, b.model, mode) as s:
        if b.geo:
            s.geo_upload(b.geo)
        if tiles is not None:
            s.set_tiles(tiles)
        for k in range(len(b.dt)):
            s.upload(b.nodes_after(k))
            s.evolve(b.dt[k])
            out.append(s.download()["U"][:, 0, :].copy())
    return out


@pytest.mark.parametrize("name", CASES)
def test_fast_form_within_tolerance_per_step(name, orc):
    b = golden_io.Bundle(name)
    for k, got in enumerate(gpu_each_step(b, abi.FP64)):
        assert rel_err(got, b.U_after(k + 1)) <= TOL_STEP, (k + 1, rel_err(got, b.U_after(k + 1)))


@pytest.mark.parametrize("name", ["tgv", "channel", "sod"])
def test_fast_form_after_100_steps(name, orc):
    b = golden_io.Bundle(name)
    node = b.initial_nodes()
    with Solver(b.part, b.model, abi.FP64) as s:
        s.upload(node)
        for _ in range(100):
            dt = orc.time_step(node, b.part, b.model, b.cfl, b.geo)
            orc.evolve_fluid(node, b.part, b.model, dt, b.geo)
            s.evolve(dt)
        got = s.download()["U"][:, 0, :]
    assert rel_err(got, node["U"][:, 0, :]) <= TOL_100


def test_graph_replay_equals_eager():
    b = golden_io.Bundle("tgv")
    eager, _ = gpu_run(b, abi.FP64, 3, dts=[b.dt[0]] * 3)
    graph, _ = gpu_run(b, abi.FP64, 3, graph=True, dts=[b.dt[0]] * 3)
    for a, c in zip(eager, graph):
        assert np.array_equal(a, c)


@pytest.mark.parametrize("name", ["sod", "channel", "gravity_box", "cylinder2d"])
def test_treat_boundary_and_cfl_bitwise(name, orc):
    b = golden_io.Bundle(name)
    node = b.initial_nodes()
    rng = np.random.default_rng(3)
    node["U"][:, :, :] *= 1.0 + 1e-3 * rng.standard_normal(node["U"].shape)
    node["U"][:, 1, :] = node["U"][:, 0, :] * 1.01
    with Solver(b.part, b.model, abi.FP64_EXACT) as s:
        s.upload(node)
        assert np.array_equal(s.cfl(), orc.cfl(node, b.part, b.model))
        for tn in (abi.TN, abi.TO):
            s.treat_boundary(tn)
            orc.treat_domain_boundary(node, b.part, b.model, tn)
        got = s.download()
    assert np.array_equal(got["U"], node["U"])


@pytest.mark.parametrize("name", ["channel", "gravity_box", "tgv", "spheres"])
def test_fused_ghost_fill_equals_phase_launches(name, monkeypatch):
    """The single cooperative ghost-fill launch (grid barriers between the
    ordered phases) gives the same bits as one launch per phase."""
    b = golden_io.Bundle(name)
    outs = []
    for fused in (False, True):
        if fused:
            monkeypatch.setenv("ACFD_BC_FUSED", "1")
        else:
            monkeypatch.delenv("ACFD_BC_FUSED", raising=False)
        o, _ = gpu_run(b, abi.FP64, 2, dts=list(b.dt))
        outs.append(o)
    for a, c in zip(*outs):
        assert np.array_equal(a, c)


@pytest.mark.parametrize("name", ["tgv", "sod", "tgv_weno3_rk2", "channel", "gravity_box", "cylinder2d", "spheres"])
def test_gather_ghost_fill_equals_phase_launches(name, monkeypatch):
    """The domain ghost fill in one launch, built from a replay of the ordered
    fill on formulas (copies for periodic and outflow faces, the inflow state,
    the wall formula of boundary nodes, the image of wall ghosts), gives the
    same bits as the ordered per-phase launches: copy-only cases, inflow /
    outflow / slip / no-slip walls, an all-wall box with gravity, a 2D
    collapsed case with a body."""
    b = golden_io.Bundle(name)
    outs = []
    for phases in (True, False):
        if phases:
            monkeypatch.setenv("ACFD_BC_PHASES", "1")
        else:
            monkeypatch.delenv("ACFD_BC_PHASES", raising=False)
        o, _ = gpu_run(b, abi.FP64, 2, dts=list(b.dt))
        outs.append(o)
    for a, c in zip(*outs):
        assert np.array_equal(a, c)
    if b.geo:
        return  # the body's ghost values add their own launches
    with Solver(b.part, b.model, abi.FP64) as s:
        s.upload(b.initial_nodes())
        n0 = s.launches()
        s.treat_boundary(abi.TO)
        assert s.launches() - n0 == 1


@pytest.mark.parametrize("s_dir", [0, 1, 2])
def test_single_stage_lllu(s_dir, orc):
    b = golden_io.Bundle("channel")
    node = b.initial_nodes()
    with Solver(b.part, b.model, abi.FP64_EXACT) as s:
        s.upload(node)
        s.lllu(0.01, 0.0, 1.0, abi.TO, abi.TO, abi.TN, s_dir)
        orc.lllu(node, b.part, b.model, 0.01, 0.0, 1.0, abi.TO, abi.TO, abi.TN, s_dir)
        got = s.download()
    assert rel_err(got["U"][:, 1, :], node["U"][:, 1, :]) <= TOL_EXACT_VISCOUS


def test_geometric_field_bit_exact():
    b = golden_io.Bundle("spheres")
    with Solver(b.part, b.model, abi.FP64_EXACT) as s:
        s.upload(b.initial_nodes())
        s.geo_upload(b.geo_moved)
        s.compute_geometric_field()
        s.treat_ib(abi.TO)
        got = s.download()
    flags = np.stack([got[f] for f in ("did", "fid", "lid", "gst")], 1)
    assert np.array_equal(flags, b.z["flagss"])
    assert np.array_equal(got["U"][:, 0, :], b.z["Us"])


def _stencils(rng, count):
    rho = rng.uniform(0.1, 10.0, size=(count, 6))
    vel = rng.uniform(-2.0, 2.0, size=(count, 6, 3))
    p = rng.uniform(0.1, 100.0, size=(count, 6))
    U = np.empty((count, 6, 5))
    U[..., 0] = rho
    U[..., 1:4] = rho[..., None] * vel
    U[..., 4] = 0.5 * rho * (vel ** 2).sum(-1) + p / 0.4
    return U


def test_per_point_twins(orc):
    rng = np.random.default_rng(11)
    F = rng.normal(size=(512, 5, 5)) * 10.0 ** rng.integers(-3, 3, size=(512, 1, 1))
    ex5 = weno_batch(F, 1, abi.FP64_EXACT)
    ex3 = weno_batch(F, 0, abi.FP64_EXACT)
    fa5 = weno_batch(F, 1, abi.FP64)
    for q in range(F.shape[0]):
        assert np.array_equal(ex5[q], orc.weno5(F[q]))
        assert np.array_equal(ex3[q], orc.weno3(F[q, :3]))
    assert np.allclose(fa5, ex5, rtol=1e-12, atol=1e-12 * np.abs(F).max())
    U = _stencils(rng, 256)
    for sS, jm, fs in [(1, 1, 0), (1, 0, 1), (0, 1, 1), (0, 0, 0)]:
        model = abi.Model()
        model.sScheme, model.jacobMean, model.fluxSplit = sS, jm, fs
        model.sL, model.sR = (-2, 3) if sS == 1 else (-1, 2)
        model.gamma = 1.4
        for s_dir in range(3):
            npt = 6 if sS == 1 else 4
            ex = fhat_batch(model, s_dir, U, abi.FP64_EXACT)
            fa = fhat_batch(model, s_dir, U, abi.FP64)
            f32 = fhat_batch(model, s_dir, U, abi.FP32_BULK)
            for q in range(U.shape[0]):
                assert np.array_equal(ex[q], orc.fhat_stencil(model, s_dir, U[q, :npt])), (sS, jm, fs, s_dir, q)
            scale = np.abs(ex).max(axis=0)
            assert np.all(np.abs(fa - ex).max(axis=0) <= 1e-12 * scale)
            assert np.all(np.abs(f32 - ex).max(axis=0) <= 2e-5 * scale)


def test_fp32_bulk_error_stated():
    """FP32 stencil arithmetic with FP64 accumulation: error of density,
    momentum and pressure against the FP64 exact form after 20 TGV steps."""
    b = golden_io.Bundle("tgv")
    dts = [b.dt[0]] * 20
    ref, _ = gpu_run(b, abi.FP64_EXACT, 20, dts=dts)
    f32, _ = gpu_run(b, abi.FP32_BULK, 20, dts=dts)
    a, r = f32[-1], ref[-1]
    l1 = np.abs(a[:, 0] - r[:, 0]).mean() / np.abs(r[:, 0]).mean()
    linf = np.abs(a[:, 0] - r[:, 0]).max() / np.abs(r[:, 0]).max()
    assert l1 < 1e-5 and linf < 1e-4, (l1, linf)


def _tgv_full():
    spec = configs.tgv(n=128)
    part, model = spec.descriptors()
    return spec, part, model


def test_full_size_tgv_conservation():
    """TGV 128^3 (the benchmark size): on the periodic torus the sums of the
    conservative variables over one period are conserved to round-off."""
    spec, part, model = _tgv_full()
    node = spec.initial_nodes(part, model)
    n = list(part.n)
    ns = np.array(part.ns)
    lo, hi = ns[0, :, 0], ns[0, :, 1] - 1  # one period: drop the duplicated end node

    def sums(nd):
        U = nd["U"][:, 0, :].reshape(n[2], n[1], n[0], 5)
        return U[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]].sum(axis=(0, 1, 2))

    with Solver(part, model, abi.FP64) as s:
        s.upload(node)
        s.treat_boundary(abi.TO)
        before = sums(s.download())
        for _ in range(2):
            s.evolve(s.time_step(spec.cfl))
        after = sums(s.download())
    pin = np.zeros((n[2], n[1], n[0]), dtype=bool)
    pin[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = True
    scale = scales(node["U"][pin.ravel(), 0, :]) * np.prod(hi - lo)
    assert np.all(np.abs(after - before) <= 1e-12 * scale), (after - before) / scale


def test_full_size_free_stream_preservation():
    spec, part, model = _tgv_full()
    spec.init = ("1", "0.3", "-0.2", "0.1", "%.17g" % (1 / (1.4 * 0.01)))
    node = spec.initial_nodes(part, model)
    with Solver(part, model, abi.FP64) as s:
        s.upload(node)
        s.treat_boundary(abi.TO)
        u0 = s.download()["U"][:, 0, :].copy()
        for _ in range(2):
            s.evolve(s.time_step(spec.cfl))
        u1 = s.download()["U"][:, 0, :]
    assert rel_err(u1, u0) <= 1e-13
