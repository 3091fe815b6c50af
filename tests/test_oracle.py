"""The oracle (CPU restatement) pinned against the reference: committed golden
fixtures made by the reference itself, the reference's own per-point
functions (when oracle/_ref is built), and analytic known answers."""
import numpy as np
import pytest

from artracfd_b200 import abi
from oracle.oracle import Oracle, Reference, reference_available

import golden_io

CASES = golden_io.names()


@pytest.fixture(scope="module")
def orc():
    return Oracle()


@pytest.mark.parametrize("name", CASES)
def test_oracle_steps_match_reference_bitwise(orc, name):
    b = golden_io.Bundle(name)
    node = b.initial_nodes()
    for k in range(len(b.dt)):
        dt = orc.time_step(node, b.part, b.model, b.cfl, b.geo)
        assert dt == b.dt[k], f"step {k + 1}: dt {dt!r} != reference {b.dt[k]!r}"
        orc.evolve_fluid(node, b.part, b.model, dt, b.geo)
        got = node["U"][:, 0, :]
        ref = b.U_after(k + 1)
        assert np.array_equal(got, ref), f"step {k + 1}: max |diff| {np.nanmax(np.abs(got - ref))}"


@pytest.mark.parametrize("name", [n for n in CASES if golden_io.Bundle(n).has_motion])
def test_oracle_geometric_field_matches_reference(orc, name):
    """ComputeGeometricField + TreatImmersedBoundary after a body motion:
    flags bit-exact, reconstructed values bitwise."""
    b = golden_io.Bundle(name)
    node = b.initial_nodes()
    orc.compute_geometric_field(node, b.part, b.model, b.geo_moved)
    orc.treat_ib(node, b.part, b.model, abi.TO, b.geo_moved)
    flags = np.stack([node[f] for f in ("did", "fid", "lid", "gst")], 1)
    assert np.array_equal(flags, b.z["flagss"])
    assert np.array_equal(node["U"][:, 0, :], b.z["Us"])


def test_weno5_reduces_to_linear_scheme_on_smooth_data(orc):
    """Known answer: for smooth data the WENO5 weights tend to (0.1, 0.6, 0.3),
    so the reconstruction tends to the linear fifth-order upwind value."""
    x = np.arange(5) * 1e-3
    F = np.stack([np.sin(1.0 + x + 0.1 * r) for r in range(5)], axis=1)
    lin = (2 * F[0] - 13 * F[1] + 47 * F[2] + 27 * F[3] - 3 * F[4]) / 60.0
    got = orc.weno5(F)
    assert np.allclose(got, lin, rtol=0, atol=1e-9)


def test_weno5_is_non_oscillatory_at_a_jump(orc):
    F = np.zeros((5, 5))
    F[3:, :] = 1.0
    got = orc.weno5(F)
    assert np.all(got < 1e-5)  # the stencil across the jump gets ~zero weight


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
def test_per_point_functions_match_reference():
    orc = Oracle()
    ref = Reference()
    rng = np.random.default_rng(7)
    for _ in range(200):
        F = rng.normal(size=(5, 5)) * 10.0 ** rng.integers(-3, 3)
        assert np.array_equal(orc.weno5(F), ref.weno5(F))
        assert np.array_equal(orc.weno3(F[:3]), ref.weno3(F[:3]))


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("motion", ["rotate", "scale", "shift"])
def test_oracle_transform_polyhedron_matches_reference(tmp_path, motion):
    """The restated TransformPolyhedron against the reference's on every
    triangulated body of the contact case: surface, centroid, inertia tensor
    and box bitwise."""
    import cases
    scale, angle, offset = cases.MOTIONS[motion]
    spec = cases.contact_spheres()
    spec.stepN = 1
    path = str(tmp_path / "case")
    spec.write(path)
    ref = Reference()
    ref.load(path)
    orc = Oracle()
    bodies = [n for n, g in enumerate(ref.geometry()) if g.faceN > 0]
    assert bodies
    for n in bodies:
        O = list(ref.geometry()[n].O)
        surf, c, inertia, box = orc.transform_polyhedron(O, scale, angle, offset, ref.surface(n), O, ref.inertia(n))
        ref.transform_polyhedron(n, O, scale, angle, offset)
        want, moved = ref.surface(n), ref.geometry()[n]
        for k in want:
            assert np.array_equal(surf[k], want[k]), (n, k)
        assert np.array_equal(c, np.array(list(moved.O)))
        assert np.array_equal(inertia, ref.inertia(n))
        assert np.array_equal(box, np.array([list(b) for b in moved.box]))


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["spheres48", "contact_spheres", "contact_spheres_inviscid"])
def test_oracle_surface_force_matches_reference(tmp_path, name):
    """The restated IntegrateSurfaceForce against the reference's on the
    state the reference reaches after three of its own steps (moving spheres
    in a crossflow, viscous and inviscid, some resting on one another):
    pressure force, shear force and torque of every body, bitwise."""
    import cases
    spec = dict(cases.SMALL, **cases.SOLID)[name]()
    spec.stepN = 4
    path = str(tmp_path / name)
    spec.write(path)
    ref = Reference()
    ref.load(path)
    for _ in range(3):
        assert ref.lib.ref_step() > 0.0
    node, part, model, geo = ref.nodes(), ref.partition(), ref.model(), ref.geometry()
    got = Oracle().integrate_surface_force(node, part, model, geo)
    want = ref.integrate_surface_force()
    moving = [n for n, g in enumerate(geo) if g.state <= 0]
    assert moving and np.any(want[moving] != 0.0)
    assert np.array_equal(got[moving], want[moving])


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("steps", [0, 2])
def test_oracle_collision_scan_matches_reference(tmp_path, steps):
    """The restated contact scan against the reference's DetectColState
    lists on the touching-spheres case: same bodies, same order, same lines
    of impact."""
    import cases
    spec = cases.contact_spheres(viscous=False)
    spec.stepN = steps + 1
    path = str(tmp_path / "case")
    spec.write(path)
    ref = Reference()
    ref.load(path)
    for _ in range(steps):
        assert ref.lib.ref_step() > 0.0
    got = Oracle().collision_scan(ref.nodes(), ref.partition(), ref.geometry())
    want = ref.collision_scan()
    assert any(want), "the case has no contact"
    assert got == want


def _roe_states(count, seed):
    """Roe-averaged interface states of random left/right states drawn from
    the sensor-training ranges (rho in [0.1, 10], |u_i| <= 2, p in [0.1, 100])."""
    import ctypes
    orc = Oracle()
    rng = np.random.default_rng(seed)
    gamma = 1.4
    out = []
    for _ in range(count):
        sides = []
        for _side in range(2):
            rho, p = rng.uniform(0.1, 10.0), rng.uniform(0.1, 100.0)
            vel = rng.uniform(-2.0, 2.0, size=3)
            sides.append(np.array([rho, *(rho * vel), p / (gamma - 1.0) + 0.5 * rho * vel @ vel]))
        Uo = np.zeros(6)
        dp = ctypes.POINTER(ctypes.c_double)
        orc.lib.orc_symmetric_average(1, gamma, sides[0].ctypes.data_as(dp), sides[1].ctypes.data_as(dp),
                                      Uo.ctypes.data_as(dp))
        out.append(Uo)
    return gamma, out


def test_eigenvectors_are_inverse_to_each_other():
    """Known answer: the left eigenvectors are the inverse of the right ones,
    L R = I, in every direction, to the rounding bound of a 5x5 product."""
    orc = Oracle()
    gamma, states = _roe_states(300, 3)
    eps = np.finfo(np.float64).eps
    for Uo in states:
        for s in range(3):
            L, R = orc.eigenvectors(s, gamma, Uo)
            bound = 10 * eps * (np.abs(L) @ np.abs(R)) + 1e-300
            assert np.all(np.abs(L @ R - np.eye(5)) <= bound), (s, Uo)


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
def test_oracle_eigenvectors_match_reference():
    orc, ref = Oracle(), Reference()
    gamma, states = _roe_states(100, 5)
    for Uo in states:
        for s in range(3):
            for a, b in zip(orc.eigenvectors(s, gamma, Uo), ref.eigenvectors(s, gamma, Uo)):
                assert np.array_equal(a, b), s


def _sod_exact_plateaus():
    # exact Riemann solution of the Sod problem (gamma = 1.4)
    return 0.42632, 0.26557


@pytest.mark.slow
def test_sod_density_plateaus_known_answer(orc):
    """Known answer: the oracle run of the Sod case (128x8x8, t = 0.2) has the
    exact Riemann density plateaus behind the rarefaction and the shock."""
    from artracfd_b200 import configs
    spec = configs.sod()
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    orc.treat_boundary(node, part, model, abi.TO)
    now, end = 0.0, spec.end_time
    while now < end:
        dt = orc.time_step(node, part, model, spec.cfl)
        now += dt
        if now > end:
            dt = end - (now - dt)
            now = end
        orc.evolve_fluid(node, part, model, dt)
    n = list(part.n)
    rho = node["U"][:, 0, 0].reshape(n[2], n[1], n[0])[n[2] // 2, n[1] // 2]
    x = part.domain[0][0] + (np.arange(n[0]) - part.ng[0]) * part.d[0]
    p3, p4 = _sod_exact_plateaus()
    assert abs(rho[(x > 0.52) & (x < 0.62)].mean() - p3) < 2e-3
    assert abs(rho[(x > 0.72) & (x < 0.82)].mean() - p4) < 2e-3
