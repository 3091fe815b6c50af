"""Immersed boundaries at the named size: crossflow over 8 moving
1280-facet icospheres in [0,4]^3 at 192^3 cells (197 x 199 x 199 nodes).

The unmodified reference (the harness in oracle/_ref) loads the case, which
includes its own ComputeGeometricField at start-up, and takes one rigid-body
half step (EvolveSolidDynamics, solid_dynamics.c:38-49: surface forces,
kinematics, collisions, motion, then the node remapping of
ComputeGeometricField and the ghost values of TreatImmersedBoundary).  The
GPU path starts from the reference's state before the motion, receives the
moved bodies and redoes the remapping: the node flags did/fid/lid/gst (body
ids, closest-facet indices, interfacial and ghost layers) must be bit-exact
and the reconstructed values bitwise equal on every node.
"""
import os

import numpy as np
import pytest

from artracfd_b200 import abi, configs
from artracfd_b200.solver import Solver
from oracle.oracle import Reference, reference_available

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not reference_available(), reason="reference harness oracle/_ref not built")
def test_ib_spheres_192_remap_bit_exact(tmp_path):
    spec = configs.ib_spheres(n=192)
    path = os.path.join(str(tmp_path), "ib192")
    spec.write(path)
    ref = Reference()
    ref.load(path)
    part, model = ref.partition(), ref.model()
    node0 = ref.nodes()
    dt = ref.lib.ref_compute_time_step()
    ref.lib.ref_evolve_solid(0.0, 0.5 * dt)
    geo = ref.geometry()
    assert len(geo) == 8 and all(g.faceN == 1280 for g in geo)
    want = ref.nodes()
    with Solver(part, model, abi.FP64_EXACT) as s:
        s.upload(node0)
        s.geo_upload(geo)
        s.compute_geometric_field()
        s.treat_ib(abi.TO)
        got = s.download()
    for f in ("did", "fid", "lid", "gst"):
        bad = np.flatnonzero(got[f] != want[f])
        assert bad.size == 0, (f, bad[:10], got[f][bad[:10]], want[f][bad[:10]])
    assert (want["gst"] > 0).sum() > 5000  # the ghost layers of all eight spheres
    assert np.array_equal(got["U"][:, 0, :], want["U"][:, 0, :])


@pytest.mark.skipif(not reference_available(), reason="reference harness oracle/_ref not built")
def test_ib_spheres_192_surface_force(tmp_path):
    """IntegrateSurfaceForce of the eight spheres on a perturbed state (the
    loaded state is uniform, whose forces the variance test zeroes): pressure
    forces bitwise, shear forces and torques (pow() in the viscosity) to
    1e-13."""
    spec = configs.ib_spheres(n=192)
    path = os.path.join(str(tmp_path), "ib192")
    spec.write(path)
    ref = Reference()
    ref.load(path)
    part, model = ref.partition(), ref.model()
    node = ref.nodes()
    rng = np.random.default_rng(3)
    U = node["U"][:, 0, :]
    U[:, 4] *= 1.0 + 0.01 * rng.standard_normal(U.shape[0])
    U[:, 1] += 0.05 * rng.standard_normal(U.shape[0]) * U[:, 0]
    node["U"][:, 0, :] = U
    ref.set_nodes(node)
    geo = ref.geometry()
    want = ref.integrate_surface_force()
    with Solver(part, model, abi.FP64_EXACT) as s:
        s.upload(node)
        s.geo_upload(geo)
        got = s.integrate_surface_force()
    assert np.abs(want[:, 0:6]).min() > 0.0
    assert np.array_equal(got[:, 0:3], want[:, 0:3])
    scale = np.abs(want).max(axis=0)
    assert np.all(np.abs(got - want) <= 1e-13 * scale), np.abs(got - want) / scale
