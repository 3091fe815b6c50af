"""The learned smoothness sensor: training kernels against the CPU oracle,
labels and features, and the hybrid form that uses it."""
import ctypes
import os

import numpy as np
import pytest

from artracfd_b200 import abi, configs, sensor
from artracfd_b200.solver import Solver
from oracle import mlp_oracle

import golden_io

pytestmark = pytest.mark.gpu
vp = ctypes.c_void_p


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def _batch(torch, n=3000, seed=4):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 10)).astype(np.float32) * 2
    y = (rng.uniform(size=n) < 0.3).astype(np.float32)
    p = sensor.init_params(seed) + rng.normal(size=sensor.param_count()).astype(np.float32) * 0.05
    return X, y, p.astype(np.float32)


def test_mlp_forward_matches_oracle(torch):
    X, _, p = _batch(torch)
    got = sensor.predict(p, torch.tensor(X, device="cuda")).cpu().numpy()
    z, _ = mlp_oracle.forward(p, X)
    assert np.allclose(got, 1 / (1 + np.exp(-z)), rtol=1e-5, atol=1e-6)


def test_mlp_gradient_matches_oracle(torch):
    """Back-propagation by the library's kernel against the float64 oracle."""
    lib = abi.load_library()
    X, y, p = _batch(torch)
    dp = torch.tensor(p, device="cuda")
    dx = torch.tensor(X, device="cuda")
    dy = torch.tensor(y, device="cuda")
    g = torch.zeros(p.size, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    abi.check(lib.acfd_mlp_grad(vp(dp.data_ptr()), vp(dx.data_ptr()), vp(dy.data_ptr()), X.shape[0], 2.5,
                                vp(g.data_ptr()), vp(loss.data_ptr()), None), lib)
    torch.cuda.synchronize()
    l_ref, g_ref = mlp_oracle.loss_and_grad(p, X, y, 2.5)
    assert abs(loss.item() - l_ref) <= 1e-4 * abs(l_ref)
    gg = g.cpu().numpy()
    assert np.max(np.abs(gg - g_ref)) <= 2e-4 * np.max(np.abs(g_ref))


def test_mlp_adam_matches_oracle(torch):
    lib = abi.load_library()
    _, _, p = _batch(torch)
    rng = np.random.default_rng(9)
    gr = rng.normal(size=p.size).astype(np.float32)
    m = rng.normal(size=p.size).astype(np.float32) * 0.1
    v = np.abs(rng.normal(size=p.size)).astype(np.float32) * 0.1
    dp, dg, dm, dv = (torch.tensor(a, device="cuda") for a in (p, gr, m, v))
    abi.check(lib.acfd_mlp_adam(vp(dp.data_ptr()), vp(dg.data_ptr()), vp(dm.data_ptr()), vp(dv.data_ptr()), 7,
                                1e-3, 0.5, None), lib)
    pr, mr, vr = mlp_oracle.adam(p.astype(np.float64), gr, m, v, 7, 1e-3, 0.5)
    assert np.allclose(dp.cpu().numpy(), pr, rtol=1e-5, atol=1e-7)
    assert np.allclose(dm.cpu().numpy(), mr, rtol=1e-5, atol=1e-7)


def test_labels_and_features(torch):
    """Departure of the WENO5 weights: ~0 in uniform flow, large at the Sod
    contact/shock; features are the normalised rho/p stencils."""
    b = golden_io.Bundle("sod")
    with Solver(b.part, b.model, abi.FP64) as s:
        s.upload(b.initial_nodes())
        ns = np.array(b.part.ns)
        L = ns[0, :, 1] - ns[0, :, 0]
        n = int(np.prod(L))
        f = torch.empty((n, 10), dtype=torch.float32, device="cuda")
        d = torch.empty(n, dtype=torch.float32, device="cuda")
        abi.check(s.lib.acfd_sensor_features(s.h, 0, vp(f.data_ptr()), vp(d.data_ptr())), s.lib)
        d = d.cpu().numpy().reshape(L[2], L[1], L[0])[0, 0]
        f = f.cpu().numpy().reshape(L[2], L[1], L[0], 10)[0, 0]
    x = b.part.domain[0][0] + (np.arange(L[0]) + ns[0, 0, 0] - b.part.ng[0]) * b.part.d[0]
    jump = np.argmin(np.abs(x - 0.5))
    assert d[jump] > 0.02
    assert np.all(d[np.abs(x - 0.5) > 0.2] < 1e-6)
    assert np.all(np.abs(f[np.abs(x - 0.5) > 0.2]) < 1e-6)
    assert np.abs(f[jump]).max() > 1.0


class _DeviceBytes:
    """A device allocation owned by the library, seen by torch as uint8."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def test_tensor_core_flags_match_the_network(torch):
    """The hybrid step's flag pass (f16 tensor-core MMAs, f32 accumulation,
    features from float density and pressure) against the oracle of the same
    arithmetic on the features of the same state, for the three sweep axes of
    a seeded 3D Riemann problem after two steps: a flag differs only where the
    logit lies within the rounding of the features of the threshold."""
    spec = sensor.riemann_3d(3, n=24)
    part, model = spec.descriptors()
    rng = np.random.default_rng(3)
    p = (sensor.init_params(2) + rng.normal(size=sensor.param_count()) * 0.2).astype(np.float32)
    with Solver(part, model, abi.FP64) as s:
        s.upload(spec.initial_nodes(part, model))
        s.treat_boundary(abi.TO)
        for _ in range(2):
            s.evolve(0.5 * s.time_step(spec.cfl))
        ns = np.array(part.ns)
        lo, hi = ns[0, :, 0], ns[0, :, 1]
        n = int(np.prod(hi - lo))
        logits, scales, fluid = [], [], None
        for ax in range(3):
            f = torch.empty((n, 10), dtype=torch.float32, device="cuda")
            d = torch.empty(n, dtype=torch.float32, device="cuda")
            abi.check(s.lib.acfd_sensor_features(s.h, ax, vp(f.data_ptr()), vp(d.data_ptr())), s.lib)
            z, sc = mlp_oracle.forward_f16(p, f.cpu().numpy())
            logits.append(z)
            scales.append(sc)
            fluid = d.cpu().numpy() >= 0
        z_all, sc_all = np.stack(logits), np.stack(scales)
        # threshold in a gap of the logits wider than four times the rounding
        # bound below, nearest to the median (many nodes of the constant
        # states share one logit, which must stay clear of the threshold)
        tol = 1e-3 * float(np.max(sc_all))
        zs = np.unique(z_all[:, fluid])
        gaps = np.nonzero(zs[1:] - zs[:-1] > 4 * tol)[0]
        mids = 0.5 * (zs[gaps] + zs[gaps + 1])
        thr_logit = float(mids[np.argmin(np.abs(mids - np.median(z_all[:, fluid])))])
        thr = 1.0 / (1.0 + np.exp(-thr_logit))
        s.sensor_load(p, thr)
        count = s.sensor_update()
        fp = vp()
        abi.check(s.lib.acfd_sensor_flags(s.h, ctypes.byref(fp)), s.lib)
        _, _, pitch, plane = s.device_state()
        torch.cuda.synchronize()
        flags = torch.as_tensor(_DeviceBytes(fp.value, 3 * plane), device="cuda").cpu().numpy()
    flags = flags.reshape(3, -1)
    k, j, i = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]), indexing="ij")
    node = ((k * part.n[1] + j) * pitch + i).ravel()
    got = flags[:, node].astype(bool)
    want = (z_all > np.float32(np.log(np.float32(thr) / (1 - np.float32(thr))))) | ~fluid[None, :]
    assert count == got.sum()
    assert 0.01 < want[:, fluid].mean() < 0.99
    bad = got != want
    # f32 features and accumulation against the exact ones: a few 1e-4 of the
    # logit scale at most
    assert not bad.any(), (bad.mean(), np.abs(z_all[bad] - thr_logit).min())


def _const_sensor(value):
    """Parameters whose logit is `value` everywhere (all weights zero)."""
    p = np.zeros(sensor.param_count(), dtype=np.float32)
    p[-1] = value
    return p


def _run(b_part, b_model, node, mode, steps, dt, params=None, thr=0.5):
    with Solver(b_part, b_model, abi.FP64 if params is not None else mode) as s:
        s.upload(node)
        if params is not None:
            abi.check(s.lib.acfd_sensor_load(s.h, params.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), thr), s.lib)
            s.set_precision(abi.FP32_HYBRID)
        for _ in range(steps):
            s.evolve(dt)
        return s.download()["U"][:, 0, :].copy()


def test_hybrid_all_flagged_is_the_fp32_form():
    """Every node flagged: the hybrid form is the FP32-bulk form.  A warp whose
    flagged lanes are few (tile edges) shares their WENO5 evaluations out over
    the warp through shared memory, where the split eigenvalue times the
    characteristic variable is rounded to FP32 before the reconstruction
    (inline, the compiler may fuse it), so the two agree to FP32 rounding
    relative to each variable's magnitude."""
    from test_gpu_march import TOL_FP32_ORDER
    from test_gpu_parity import rel_err
    b = golden_io.Bundle("tgv")
    node = b.initial_nodes()
    full = _run(b.part, b.model, node, abi.FP32_BULK, 3, b.dt[0])
    hyb = _run(b.part, b.model, node, None, 3, b.dt[0], params=_const_sensor(50.0))
    assert rel_err(hyb, full) <= TOL_FP32_ORDER / 10, rel_err(hyb, full)


def test_hybrid_smooth_path_is_linear_weight_weno():
    """With no flag the hybrid form is WENO5 with the linear weights: on the
    smooth TGV it differs from full WENO5 only by the small weight
    departure, and it differs from it at all (the smooth path is taken)."""
    b = golden_io.Bundle("tgv")
    node = b.initial_nodes()
    full = _run(b.part, b.model, node, abi.FP64, 3, b.dt[0])
    lin = _run(b.part, b.model, node, None, 3, b.dt[0], params=_const_sensor(-50.0))
    rel = np.abs(lin[:, 0] - full[:, 0]).max() / np.abs(full[:, 0]).max()
    assert 0 < rel < 1e-3


WEIGHTS = sensor.WEIGHTS


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained sensor weights")
def test_trained_sensor_gain_on_shock_cylinder():
    """What the trained network gains over the method without it, on the
    shock-cylinder case (128 x 64 x 4): the hybrid form stays within the
    stated L1 density error of the FP64 path where the linear scheme alone
    (no sensor) does not, while skipping the nonlinear weights on the
    interfaces the network finds smooth."""
    spec = configs.shock_cylinder(m=(128, 64, 4), segments=24)
    spec.bodies = []  # the domain path; the immersed cylinder is covered elsewhere
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    steps = 40
    with Solver(part, model, abi.FP64) as s:
        s.upload(node)
        s.treat_boundary(abi.TO)
        node = s.download()
        dt = 0.5 * s.time_step(spec.cfl)
    ref = _run(part, model, node, abi.FP64, steps, dt)
    params, thr, meta = sensor.load(WEIGHTS)
    hyb = _run(part, model, node, None, steps, dt, params=params, thr=thr)
    lin = _run(part, model, node, None, steps, dt, params=_const_sensor(-50.0))

    def l1(a):
        finite = np.isfinite(a[:, 0])
        if not finite.all():
            return np.inf
        return np.abs(a[:, 0] - ref[:, 0]).sum() / np.abs(ref[:, 0]).sum()

    e_hyb, e_lin = l1(hyb), l1(lin)
    assert e_hyb <= 1e-3, e_hyb
    assert e_lin > 3 * e_hyb, (e_lin, e_hyb)


@pytest.mark.skipif(not os.path.exists(sensor.WEIGHTS_BIN), reason="no trained sensor weights")
def test_sensor_file_is_the_trained_sensor(tmp_path):
    """acfd_sensor_load_file reads the shipped weights file: the same flags as
    the parameters given directly; a damaged file is refused."""
    spec = configs.shock_cylinder(m=(64, 32, 4), segments=24)
    spec.bodies = []
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    counts = []
    for how in ("params", "file"):
        with Solver(part, model, abi.FP64) as s:
            s.upload(node)
            s.treat_boundary(abi.TO)
            if how == "params":
                s.sensor_load(params, thr)
            else:
                s.sensor_load_file(sensor.WEIGHTS_BIN)
            counts.append(s.sensor_update())
    assert counts[0] == counts[1] > 0
    bad = tmp_path / "bad.bin"
    bad.write_bytes(open(sensor.WEIGHTS_BIN, "rb").read()[:100])
    with Solver(part, model, abi.FP64) as s:
        with pytest.raises(abi.AcfdError):
            s.sensor_load_file(str(bad))
