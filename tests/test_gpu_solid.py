"""The node scans of the rigid-body step on the device against the
reference's own functions on the same state (the harness in oracle/_ref):

* IntegrateSurfaceForce (solid_dynamics.c:51-171): pressure force, shear
  force and torque of every body, summed over its ghost nodes of layer 2 in
  the reference's node order and calibrated by area / interfacial node
  count.  The pressure force takes IEEE +, -, *, / only and is bitwise equal;
  the shear force (and the torque it enters) of no-slip bodies in a viscous
  fluid goes through pow() in Sutherland's law, whose last bit the device
  library may round differently, so those agree to 1e-13;
* the contact scan of ApplyCollision (DetectColState / AddColObject,
  solid_dynamics.c:242-256, 327-357): the same contact lists, in the same
  order, with the same lines of impact.
* TransformPolyhedron (computational_geometry.c:162-208), the surface motion
  of ApplyMotion: vertices, normals, centroid, inertia tensor and box
  bitwise; a moved surface kept on the device through a new body list.

The states are those of the reference after a few of its own time steps
(moving spheres in a crossflow, three of them resting on one another).
"""
import os

import numpy as np
import pytest

from artracfd_b200 import abi
from artracfd_b200.solver import Solver
from oracle.oracle import Reference, reference_available

import cases

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference_available(), reason="reference harness oracle/_ref not built")]

BUILDERS = dict(cases.SMALL, **cases.SOLID)


def _load(tmp_path, name, steps):
    spec = BUILDERS[name]()
    spec.stepN = steps + 1
    path = os.path.join(str(tmp_path), name)
    spec.write(path)
    ref = Reference()
    ref.load(path)
    for _ in range(steps):
        assert ref.lib.ref_step() > 0.0
    return ref


def _device(ref):
    s = Solver(ref.partition(), ref.model(), abi.FP64_EXACT)
    s.upload(ref.nodes())
    s.geo_upload(ref.geometry())
    return s


@pytest.mark.parametrize("name", ["spheres48", "contact_spheres", "contact_spheres_inviscid"])
def test_surface_force_matches_reference(tmp_path, name):
    ref = _load(tmp_path, name, 3)
    model, geo = ref.model(), ref.geometry()
    with _device(ref) as s:
        got = s.integrate_surface_force()
    want = ref.integrate_surface_force()
    assert np.abs(want[:, 0:3]).max() > 0.0
    assert np.array_equal(got[:, 0:3], want[:, 0:3]), np.abs(got - want).max()
    if model.refMu > 0.0 and any(g.cf > 0.0 for g in geo):
        assert np.abs(want[:, 3:6]).max() > 0.0
        scale = np.abs(want).max(axis=0)
        assert np.all(np.abs(got - want) <= 1e-13 * scale), np.abs(got - want) / scale
    else:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("steps", [0, 3])
def test_collision_scan_matches_reference(tmp_path, steps):
    ref = _load(tmp_path, "contact_spheres", steps)
    with _device(ref) as s:
        got = s.collision_scan()
    want = ref.collision_scan()
    assert all(len(c) == 2 for c in want), want  # every sphere touches the other two
    assert got == want


def test_collision_scan_skips_stationary_bodies(tmp_path):
    ref = _load(tmp_path, "contact_spheres", 0)
    geo = ref.geometry()
    geo[0].state = 1
    with Solver(ref.partition(), ref.model(), abi.FP64_EXACT) as s:
        s.upload(ref.nodes())
        s.geo_upload(geo)
        got = s.collision_scan()
    assert got[0] == []
    assert got[1] == ref.collision_scan()[1]


def test_moved_bodies_update_in_place(tmp_path):
    """A moved body list of the same bodies is written into the device
    buffers in place (no new allocation, a captured step stays valid): the
    node mapping and ghost values afterwards equal those of a case given the
    moved bodies as a new list."""
    ref = _load(tmp_path, "contact_spheres", 0)
    part, model, node = ref.partition(), ref.model(), ref.nodes()
    before = ref.geometry()
    before_copy = [abi.copy_struct(g, abi.Polyhedron) for g in before]
    ref.lib.ref_step()  # moves the bodies (the arrays behind `before` are the reference's own)
    after = ref.geometry()
    outs = []
    for lists in ([before_copy, after], [after]):
        with Solver(part, model, abi.FP64_EXACT) as s:
            s.upload(node)
            for geo in lists:
                s.geo_upload(geo)
            s.compute_geometric_field()
            s.treat_ib(abi.TO)
            outs.append(s.download())
    for f in ("did", "fid", "lid", "gst"):
        assert np.array_equal(outs[0][f], outs[1][f]), f
    assert np.array_equal(outs[0]["U"], outs[1]["U"])
    assert not np.array_equal(np.array([g.O[0] for g in before_copy]), np.array([g.O[0] for g in after]))


MOTIONS = cases.MOTIONS


def _rows(box):
    return np.array([list(b) for b in box])


@pytest.mark.parametrize("motion", MOTIONS)
def test_transform_polyhedron_matches_reference(tmp_path, motion):
    """The device transform of each triangulated body against the
    reference's TransformPolyhedron on the same body: moved vertices, rotated
    face, edge and vertex normals, centroid, inertia tensor and box."""
    scale, angle, offset = MOTIONS[motion]
    ref = _load(tmp_path, "contact_spheres", 0)
    tri = [n for n, g in enumerate(ref.geometry()) if g.faceN > 0]
    assert tri
    with _device(ref) as s:
        for n in tri:
            g = ref.geometry()[n]
            O = list(g.O)
            c, inertia, box = s.transform_polyhedron(n, O, scale, angle, offset, O, ref.inertia(n))
            got = s.geo_fetch(n)
            ref.transform_polyhedron(n, O, scale, angle, offset)
            want = ref.surface(n)
            moved = ref.geometry()[n]
            for k in ("v", "Nf", "Ne", "Nv"):
                assert np.array_equal(got[k], want[k]), (n, k)
            assert np.array_equal(c, np.array(list(moved.O))), n
            assert np.array_equal(inertia, ref.inertia(n)), n
            assert np.array_equal(box, _rows(moved.box)), n


@pytest.mark.parametrize("motion", ["rotate", "scale"])
def test_transformed_surface_stays_on_device(tmp_path, motion):
    """Bodies moved on the device and listed again without surface arrays
    (the drop-in program's device motion) map the nodes and fill the ghost
    nodes as a case given the reference's moved bodies.  The anisotropic
    scale grows the node boxes past the ghost lists, so the list takes a new
    layout, which brings the kept surfaces along."""
    scale, angle, offset = MOTIONS[motion]
    ref = _load(tmp_path, "contact_spheres", 0)
    with _device(ref) as s:
        for n, g in enumerate(ref.geometry()):
            if g.faceN > 0:
                O = list(g.O)
                s.transform_polyhedron(n, O, scale, angle, offset, O, ref.inertia(n))
                ref.transform_polyhedron(n, O, scale, angle, offset)
        moved = ref.geometry()
        kept = []
        for g in moved:
            p = abi.copy_struct(g, abi.Polyhedron)
            if p.faceN > 0:
                p.f, p.Nf, p.e, p.Ne, p.v, p.Nv = None, None, None, None, None, None
            kept.append(p)
        s.geo_upload(kept)
        s.compute_geometric_field()
        s.treat_ib(abi.TO)
        got = s.download()
        for n, g in enumerate(moved):
            if g.faceN > 0:
                surf, want = s.geo_fetch(n), ref.surface(n)
                for k in want:
                    assert np.array_equal(surf[k], want[k]), (n, k)
    with _device(ref) as s:
        s.compute_geometric_field()
        s.treat_ib(abi.TO)
        want = s.download()
    for f in ("did", "fid", "lid", "gst"):
        assert np.array_equal(got[f], want[f]), f
    assert np.array_equal(got["U"], want["U"])


def test_transform_rejects_analytical_and_missing_bodies(tmp_path):
    ref = _load(tmp_path, "contact_spheres", 0)
    sphere = [n for n, g in enumerate(ref.geometry()) if g.faceN <= 0][0]
    with _device(ref) as s:
        one = [1.0, 1.0, 1.0]
        for n in (sphere, len(ref.geometry()), -1):
            with pytest.raises(abi.AcfdError):
                s.transform_polyhedron(n, [0.0] * 3, one, [0.0] * 3, [0.0] * 3, [0.0] * 3, np.eye(3))
