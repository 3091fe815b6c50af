"""FP64 parity at the named sizes against the unmodified reference itself
(the harness in oracle/_ref, compiled from the reference's own sources).

* Sod shock tube at 128 x 8 x 8 cells to t = 0.2 (92 steps): every step of
  the plain FP64 path taken from the reference's own state of the step
  before equals the reference's step within 1e-12 relative (the per-step
  tolerance is checked on each step's increment, not accumulated), dt
  bitwise; the free-running GPU run ends within 1e-10 of the reference with
  the same dt sequence to 1e-12; the learned-sensor hybrid form (its plane
  kernels) ends within L1 density error 1e-3.
* Viscous Taylor-Green vortex at 128^3 cells: two steps, each from the
  reference's own state, with the stage-kernel variants the benchmark runs
  (FP64 [0, 8, 8]: brick X sweep, plane-march Y and Z; hybrid [7, 8, 7] and
  [10, 8, 7]), against the reference within 1e-12 relative per step
  (FP64) and L1 density 1e-3 (hybrid).
* Eight moving 1280-facet spheres at 192^3 cells: three full time steps
  of the drop-in program (reference sources + libacfd_gpu, exact mode,
  rigid-body step's node scans, collisions and surface motion on the
  device, an FP64 checkpoint after every step) against three passes of the
  reference's own EvolveSolution loop body (solid half step, fluid step,
  solid half step): node flags did/fid/lid/gst bit-exact after every step,
  the state (ghost values included) within 1e-12 relative per step
  (cumulative bound k * 1e-12 after k steps; the viscous flux's pow() is the
  only non-bitwise operation of the exact form), body centroids within
  1e-12.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from artracfd_b200 import abi, configs, sensor
from artracfd_b200.solver import Solver
from oracle.oracle import Reference, reference_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference_available(), reason="reference harness oracle/_ref not built")]

TOL_STEP = 1e-12   # relative, one step from the reference's own state
TOL_RUN = 1e-10    # relative, after a whole run
TOL_L1_HYBRID = 1e-3

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "artracfd_b200", "shim", "_build", "artracfd_gpu")
INT_MAX = 2147483647


def scales(b):
    b = np.abs(np.asarray(b, dtype=np.float64))
    mom = max(b[..., 1].max(), b[..., 2].max(), b[..., 3].max())
    return np.array([b[..., 0].max(), mom, mom, mom, b[..., 4].max()])


def rel_err(a, b):
    sc = np.maximum(scales(b), 1e-300)
    return max(float(np.max(np.abs(a[..., v] - b[..., v]))) / sc[v] for v in range(5))


def pin_of(part):
    n = list(part.n)
    ns = np.array(part.ns)[0]
    m = np.zeros((n[2], n[1], n[0]), dtype=bool)
    m[ns[2, 0]:ns[2, 1], ns[1, 0]:ns[1, 1], ns[0, 0]:ns[0, 1]] = True
    return m.ravel()


def l1_rho(got, want, mask):
    return float(np.abs(got[mask, 0] - want[mask, 0]).sum() / np.abs(want[mask, 0]).sum())


def _compact(node):
    """U[TO] and the four flags of a node array (a quarter of its bytes)."""
    out = np.zeros(node.size, dtype=[("U", "<f8", (5,)), ("did", "<i4"), ("fid", "<i4"), ("lid", "<i4"),
                                     ("gst", "<i4")])
    out["U"] = node["U"][:, 0, :]
    for f in ("did", "fid", "lid", "gst"):
        out[f] = node[f]
    return out


def reference_run(spec, path, steps, compact=False):
    """Load the case in the reference and take `steps` passes of its
    EvolveSolution loop body; returns descriptors, the node arrays before
    and after every step (compact: U[TO] and flags only), the dt sequence
    and the body centroids after every step."""
    spec.write(path)
    ref = Reference()
    ref.load(path)
    part, model = ref.partition(), ref.model()
    keep = _compact if compact else (lambda a: a)
    states = [keep(ref.nodes())]
    dts, bodies = [], []
    for _ in range(steps):
        dt = ref.step()
        if dt < 0.0:
            break
        dts.append(dt)
        states.append(keep(ref.nodes()))
        bodies.append([np.array(g.O[:]) for g in ref.geometry()])
    geo = ref.geometry()
    return dict(part=part, model=model, states=states, dts=dts, bodies=bodies, geo=geo, ref=ref)


def one_step_each(run, mode, tiles=None, params=None, thr=0.5):
    """Every step taken on the GPU from the reference's own state of the step
    before; yields (k, dt on the GPU, U[TO] after the step)."""
    with Solver(run["part"], run["model"], abi.FP64) as s:
        if params is not None:
            s.sensor_load(params, thr)
        s.set_precision(mode)
        if tiles is not None:
            s.set_tiles(tiles)
        for k in range(len(run["dts"])):
            s.upload(run["states"][k])
            dt = s.time_step(run["cfl"])
            s.evolve(dt)
            yield k, dt, s.download()["U"][:, 0, :]


# --------------------------------------------------------------------------
# Sod shock tube, 128 x 8 x 8 cells, t = 0.2
# --------------------------------------------------------------------------

@pytest.fixture(scope="module")
def sod_run(tmp_path_factory):
    spec = configs.sod()
    run = reference_run(spec, str(tmp_path_factory.mktemp("sod") / "sod"), 1000)
    run["cfl"] = spec.cfl
    run["end"] = spec.end_time
    assert len(run["dts"]) == 92 and sum(run["dts"]) == pytest.approx(0.2, rel=1e-14)
    return run


def test_sod_full_run_every_step_within_1e12_of_the_reference(sod_run):
    worst = 0.0
    for k, dt, got in one_step_each(sod_run, abi.FP64):
        want = sod_run["states"][k + 1]["U"][:, 0, :]
        if k < len(sod_run["dts"]) - 1:  # the last dt is rectified to end at t = 0.2
            assert dt == sod_run["dts"][k], (k, dt, sod_run["dts"][k])
        else:
            assert dt >= sod_run["dts"][k]
        if dt != sod_run["dts"][k]:
            continue
        e = rel_err(got, want)
        worst = max(worst, e)
        assert e <= TOL_STEP, (k + 1, e)
    print(f"Sod 128x8x8: worst per-step relative error over 91 steps {worst:.3g}")


def test_sod_free_run_to_t02_within_1e10(sod_run):
    from artracfd_b200.solver import run as run_steps

    with Solver(sod_run["part"], sod_run["model"], abi.FP64) as s:
        s.upload(sod_run["states"][0])
        s.autotune()
        s.upload(sod_run["states"][0])
        now, dts = run_steps(s, sod_run["cfl"], sod_run["end"], 1000)
        got = s.download()["U"][:, 0, :]
    assert len(dts) == len(sod_run["dts"])
    assert now == sod_run["end"]
    np.testing.assert_allclose(dts, sod_run["dts"], rtol=1e-12, atol=0)
    e = rel_err(got, sod_run["states"][-1]["U"][:, 0, :])
    print(f"Sod 128x8x8 free run to t=0.2 ({len(dts)} steps): relative error {e:.3g}")
    assert e <= TOL_RUN, e


def test_sod_hybrid_plane_kernels_within_stated_error(sod_run):
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    with Solver(sod_run["part"], sod_run["model"], abi.FP64) as s:
        s.sensor_load(params, thr)
        s.set_precision(abi.FP32_HYBRID)
        s.set_tiles([7, 8, 7])
        s.upload(sod_run["states"][0])
        for dt in sod_run["dts"]:
            s.evolve(dt, graph=True)
        got = s.download()["U"][:, 0, :]
    pin = pin_of(sod_run["part"])
    want = sod_run["states"][-1]["U"][:, 0, :]
    e = l1_rho(got, want, pin)
    print(f"Sod 128x8x8 hybrid [7,8,7] at t=0.2: L1 rho {e:.3g}")
    assert e <= TOL_L1_HYBRID, e


# --------------------------------------------------------------------------
# viscous TGV, 128^3 cells
# --------------------------------------------------------------------------

@pytest.fixture(scope="module")
def tgv_run(tmp_path_factory):
    spec = configs.tgv(n=128)
    run = reference_run(spec, str(tmp_path_factory.mktemp("tgv") / "tgv"), 2)
    run["cfl"] = spec.cfl
    assert len(run["dts"]) == 2
    return run


@pytest.mark.parametrize("tiles", [[0, 8, 8], None], ids=["bench_tiles", "default_tiles"])
def test_tgv128_fp64_each_step_within_1e12_of_the_reference(tgv_run, tiles):
    for k, dt, got in one_step_each(tgv_run, abi.FP64, tiles=tiles):
        assert dt == tgv_run["dts"][k]
        e = rel_err(got, tgv_run["states"][k + 1]["U"][:, 0, :])
        print(f"TGV 128^3 step {k + 1}, FP64 tiles {tiles}: relative error {e:.3g}")
        assert e <= TOL_STEP, (k + 1, e)


@pytest.mark.parametrize("tiles", [[7, 8, 7], [10, 8, 7]])
def test_tgv128_hybrid_plane_kernels_within_stated_error(tgv_run, tiles):
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    pin = pin_of(tgv_run["part"])
    for k, dt, got in one_step_each(tgv_run, abi.FP32_HYBRID, tiles=tiles, params=params, thr=thr):
        e = l1_rho(got, tgv_run["states"][k + 1]["U"][:, 0, :], pin)
        print(f"TGV 128^3 step {k + 1}, hybrid tiles {tiles}: L1 rho {e:.3g}")
        assert e <= TOL_L1_HYBRID, e


# --------------------------------------------------------------------------
# eight moving spheres, 192^3 cells, through the drop-in program
# --------------------------------------------------------------------------

STEPS_IB = 3


def _checkpoint_state(part, model, path, geo):
    """Node records and body centroids of a drop-in checkpoint (the user block
    holds now, stepC, dataC, the bodies' count and states, then per body 64
    doubles starting with its centroid O, then its surface arrays)."""
    with Solver(part, model, abi.FP64) as s:
        user = s.checkpoint_load(path, user_cap=1 << 26)
        node = s.download()
    off = 3 * 8 + 4 * (1 + len(geo))
    centroids = []
    for g in geo:
        centroids.append(np.frombuffer(user, dtype=np.float64, count=3, offset=off).copy())
        off += 64 * 8
        if g.faceN > 0:
            off += 3 * 8 * (2 * g.vertN + g.faceN + g.edgeN)
    assert off == len(user)
    return node, centroids


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in program not built")
def test_ib_spheres_192_three_steps_flags_bit_exact_every_step(tmp_path):
    spec = configs.ib_spheres(n=192)
    spec.stepN = STEPS_IB
    spec.dataW = INT_MAX  # space data (and a checkpoint) after every step, no dt rectification
    gpu_dir = str(tmp_path / "gpu")
    spec.write(gpu_dir)
    env = dict(os.environ, ACFD_MODE="exact", ACFD_CHECKPOINT="1")
    proc = subprocess.Popen([DROPIN, "-m", "gpu"], cwd=gpu_dir, env=env, stdout=subprocess.PIPE,
                            stderr=subprocess.STDOUT, text=True)
    # the reference's own steps run meanwhile on the host
    run = reference_run(configs.ib_spheres(n=192), str(tmp_path / "ref"), STEPS_IB, compact=True)
    out, _ = proc.communicate(timeout=900)
    assert proc.returncode == 0, out[-3000:]
    assert len(run["dts"]) == STEPS_IB
    part, model, geo = run["part"], run["model"], run["geo"]
    assert len(geo) == 8 and all(g.faceN == 1280 for g in geo)
    for k in range(STEPS_IB):
        ckpt = os.path.join(gpu_dir, "artracfd.ckpt.%05d" % (k + 1))
        got, cents = _checkpoint_state(part, model, ckpt, geo)
        os.unlink(ckpt)
        want = run["states"][k + 1]
        for f in ("did", "fid", "lid", "gst"):
            bad = np.flatnonzero(got[f] != want[f])
            assert bad.size == 0, (k + 1, f, bad[:10], got[f][bad[:10]], want[f][bad[:10]])
        e = rel_err(got["U"][:, 0, :], want["U"])
        ghosts = want["gst"] > 0
        eg = rel_err(got["U"][ghosts, 0, :], want["U"][ghosts])
        for n in range(8):
            np.testing.assert_allclose(cents[n], run["bodies"][k][n], rtol=TOL_STEP, atol=0)
        print(f"spheres 192^3 step {k + 1}: flags bit-exact ({int(ghosts.sum())} ghost nodes); "
              f"relative error all nodes {e:.3g}, ghost nodes {eg:.3g}")
        assert e <= TOL_STEP * (k + 1), (k + 1, e)
    shutil.rmtree(gpu_dir, ignore_errors=True)
