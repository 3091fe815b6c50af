"""Small versions of the named workloads and extra option variants, used by
the parity tests and by tests/golden/make_golden.py.  Each builder returns a
CaseSpec; the reference loads it from a case directory written by
CaseSpec.write."""
from __future__ import annotations

import os
import tempfile

import numpy as np

from artracfd_b200 import abi, configs
from artracfd_b200.case import Body, Boundary, CaseSpec, Region, icosphere


def channel(m=(16, 8, 4)) -> CaseSpec:
    """Inflow/outflow channel between a no-slip wall with given temperature
    (south) and an adiabatic slip wall (north); periodic front/back; viscous."""
    refT = 1.0 / (0.3 * 0.3 * 1.4 * 287.058)
    p0 = 1.0 / (1.4 * 0.09)
    return CaseSpec(
        domain_lo=(0.0, 0.0, 0.0), domain_hi=(2.0, 1.0, 0.5), m=m, end=1.0e6, cfl=0.5, stepN=0,
        refMu=(1.0 / 100.0) / configs.sutherland(refT), refT=refT,
        init=("1", "0.5+0.1*sin(3*x)", "0.05*cos(2*x)", "0.02", "%.17g" % p0),
        boundaries=[Boundary(abi.INFLOW, (1.2, 0.6, 0.0, 0.0, p0 * 1.1)), Boundary(abi.OUTFLOW),
                    Boundary(abi.NOSLIPWALL, (1.05,)), Boundary(abi.SLIPWALL, (-1.0,)),
                    Boundary(abi.PERIODIC), Boundary(abi.PERIODIC)],
        regions=[Region("sphere", p1=(1.0, 0.5, 0.25), r=0.3, exprs=("1.5", "0.2", "0", "0", "%.17g" % (p0 * 1.5)))])


def gravity_box(m=(8, 8, 8), multidim=1) -> CaseSpec:
    """All-wall box with gravity on and the operator-by-operator form."""
    spec = configs.sod(m=m)
    spec.domain_hi = (1.0, 1.0, 1.0)
    spec.multidim = multidim
    spec.gState = 1
    spec.g = (0.0, -0.5, 0.1)
    spec.boundaries = [Boundary(abi.SLIPWALL, (-1.0,))] * 2 + [Boundary(abi.NOSLIPWALL, (-1.0,))] * 2 + [
        Boundary(abi.OUTFLOW)] * 2
    spec.regions = [Region("box", p1=(0.2, 0.2, 0.2), p2=(0.6, 0.5, 0.7), exprs=("2", "0", "0", "0", "2"))]
    return spec


def spheres(n=24, count=2, analytic=1, level=2) -> CaseSpec:
    return configs.ib_spheres(n=n, count=count, analytic=analytic, level=level, stepN=0)


def contact_spheres(n=32, viscous=True) -> CaseSpec:
    """Three moving spheres (one analytical, two 320-facet icospheres) of
    radius 0.15 in the unit cube, closing on one another with surface gaps
    below a cell, in a crossflow: their nodes meet on the collision search
    paths of the rigid-body step."""
    d = 1.0 / n
    c0 = (0.3, 0.5, 0.5)
    c1 = (0.6 + 0.3 * d, 0.5, 0.5)
    # the third sphere rests on the first two, 0.3 cells from each
    c2 = (0.45 + 0.15 * d, 0.5 + float(np.sqrt((0.3 + 0.3 * d) ** 2 - (0.15 + 0.15 * d) ** 2)), 0.5)
    refT = 1.0 / (0.3 * 0.3 * 1.4 * 287.058)
    p0 = 1.0 / (1.4 * 0.09)
    bodies = [Body(O=c0, r=0.15, V=(0.2, 0.01, 0.0), W=(0.0, 0.0, 0.5), rho=2.0, T=-1.0, cf=1.0),
              Body(O=c1, r=0.15, V=(-0.2, 0.0, 0.02), rho=3.0, T=-1.0, cf=1.0, stl="s1.stl",
                   triangles=icosphere(c1, 0.15, level=2)),
              Body(O=c2, r=0.15, V=(0.0, -0.2, 0.0), W=(0.3, 0.0, 0.0), rho=2.5, T=-1.0, cf=0.0, stl="s2.stl",
                   triangles=icosphere(c2, 0.15, level=2))]
    P = Boundary(abi.PERIODIC)
    return CaseSpec(
        domain_lo=(0.0, 0.0, 0.0), domain_hi=(1.0, 1.0, 1.0), m=(n, n, n), end=1.0e6, cfl=0.5, stepN=0,
        psi=2, ibmLayer=1, refMu=((0.3 / 200.0) / configs.sutherland(refT)) if viscous else 0.0, refT=refT,
        init=("1", "0.6", "0.1*sin(6*y)", "0", "%.17g" % p0),
        boundaries=[Boundary(abi.INFLOW, (1.0, 0.6, 0.0, 0.0, p0)), Boundary(abi.OUTFLOW), P, P, P, P],
        bodies=bodies)


def cylinder2d(m=(64, 32, 1)) -> CaseSpec:
    spec = configs.shock_cylinder(m=m, segments=24)
    return spec


SMALL = {
    "sod": lambda: configs.sod(m=(32, 4, 4)),
    "sod_variants": lambda: configs.sod(m=(32, 4, 4), tScheme=0, sScheme=0, jacobMean=0, fluxSplit=1),
    "tgv": lambda: configs.tgv(n=12),
    "tgv_weno3_rk2": lambda: configs.tgv(n=10, tScheme=0, sScheme=0, fluxSplit=1, jacobMean=0),
    "channel": channel,
    "gravity_box": gravity_box,
    "cylinder2d": cylinder2d,
    "spheres": spheres,
}

SOLID = {
    "spheres48": lambda: configs.ib_spheres(n=48, count=2, analytic=1, level=2, stepN=0),
    "contact_spheres": contact_spheres,
    "contact_spheres_inviscid": lambda: contact_spheres(viscous=False),
}


def load(ref, name: str, workdir: str | None = None):
    """Write case ``name`` and load it in the reference; returns a bundle with
    the reference's own descriptors, initial nodes and geometry."""
    spec = SMALL[name]()
    d = workdir or tempfile.mkdtemp(prefix=f"acfd_{name}_")
    path = os.path.join(d, name)
    spec.write(path)
    ref.load(path)
    return dict(spec=spec, part=ref.partition(), model=ref.model(), nodes=ref.nodes(), geo=ref.geometry(),
                time=ref.time(), path=path)


def pin_mask(part) -> np.ndarray:
    n = list(part.n)
    mask = np.zeros((n[2], n[1], n[0]), dtype=bool)
    ns = np.array(part.ns)
    mask[ns[0, 2, 0]:ns[0, 2, 1], ns[0, 1, 0]:ns[0, 1, 1], ns[0, 0, 0]:ns[0, 0, 1]] = True
    return mask.ravel()


# rigid motions of a triangulated body (scale, angle, offset) for the
# TransformPolyhedron parity tests: a rotation with a shift, an anisotropic
# scale with a small rotation, a pure shift towards negative coordinates
MOTIONS = {"rotate": ((1.0, 1.0, 1.0), (0.3, -0.2, 0.7), (0.01, -0.02, 0.005)),
           "scale": ((1.5, 0.75, 2.0), (1e-3, 2e-3, -5e-4), (0.0, 0.0, 0.0)),
           "shift": ((1.0, 1.0, 1.0), (0.0, 0.0, 0.0), (-0.5, -0.5, -0.5))}
