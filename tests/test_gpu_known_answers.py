"""Known answer of the viscous Taylor-Green vortex: at early times the
kinetic energy of u = sin x cos y cos z, v = -cos x sin y cos z, w = 0
decays at the viscous rate.  Every velocity component satisfies
-Laplace(u) = 3u, so the dissipation <|grad u|^2> is 6 nu times the kinetic
energy <|u|^2>/2 and E(t) = E0 exp(-6 nu t) until the nonlinear transfer to
smaller scales starts.  The case sets mu(T0) = 1/1600 at rho0 = 1, so
nu = 1/1600.  The GPU runs the plain FP64 path at 64^3 and 128^3 (the
numerical dissipation of WENO5 shrinks with the cell size) and the
learned-sensor hybrid form at 128^3."""
import numpy as np
import pytest

from artracfd_b200 import abi, configs, sensor
from artracfd_b200.solver import Solver

pytestmark = pytest.mark.gpu

NU = 1.0 / 1600.0
T_END = 0.1


def _kinetic_energy(node, part):
    n = list(part.n)
    ns = np.array(part.ns)
    U = node["U"][:, 0, :].reshape(n[2], n[1], n[0], 5)
    # one period: the last node of each periodic axis repeats the first
    c = U[ns[0, 2, 0]:ns[0, 2, 1] - 1, ns[0, 1, 0]:ns[0, 1, 1] - 1, ns[0, 0, 0]:ns[0, 0, 1] - 1]
    return float((0.5 * (c[..., 1] ** 2 + c[..., 2] ** 2 + c[..., 3] ** 2) / c[..., 0]).mean())


def _decay_rate(n, hybrid=False):
    spec = configs.tgv(n=n)
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    with Solver(part, model, abi.FP64) as s:
        s.upload(node)
        s.treat_boundary(abi.TO)
        if hybrid:
            s.sensor_load_file(sensor.WEIGHTS_BIN)
            s.set_precision(abi.FP32_HYBRID)
        e0 = _kinetic_energy(s.download(), part)
        t = 0.0
        while t < T_END:
            dt = s.time_step(spec.cfl)
            s.evolve(dt, graph=True)
            t += dt
        e = _kinetic_energy(s.download(), part)
    assert e0 == pytest.approx(0.125, rel=1e-12)
    return -np.log(e / e0) / t


def test_tgv_kinetic_energy_decays_at_the_viscous_rate():
    r64, r128 = _decay_rate(64), _decay_rate(128)
    err64, err128 = abs(r64 / (6 * NU) - 1), abs(r128 / (6 * NU) - 1)
    assert err64 < 0.05, r64
    assert err128 < 0.02, r128
    assert err128 < err64  # the numerical dissipation shrinks with the cell size


@pytest.mark.skipif(not __import__("os").path.exists(sensor.WEIGHTS_BIN), reason="no trained sensor weights")
def test_tgv_hybrid_form_decays_at_the_fp64_rate():
    assert _decay_rate(128, hybrid=True) == pytest.approx(_decay_rate(128), rel=0.01)
