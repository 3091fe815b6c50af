"""The named workloads, as reference cases (synthetic inputs of the stated
shapes; no external data set is involved).

Each builder takes the mesh size so that tests can run the same physics on
small grids:

* ``sod``            inviscid 3D Sod shock tube (WENO5/LLF/RK3, CFL 0.6, t=0.2)
* ``tgv``            viscous Taylor-Green vortex, Re 1600, Ma 0.1 (CFL 0.5)
* ``ib_spheres``     crossflow Ma 0.3, Re 200 over seeded moving icospheres
* ``shock_cylinder`` Ma 2.81 planar shock over an extruded cylinder
"""
from __future__ import annotations

import math

import numpy as np

from . import abi
from .case import Body, Boundary, CaseSpec, Region, extruded_cylinder, icosphere

GAS_R = 287.058
GAMMA = 1.4


def sutherland(T: float) -> float:
    """Sutherland's law as the reference evaluates it (cfd_commons.c:288-291)."""
    return 1.458e-6 * T ** 1.5 / (T + 110.4)


def sod(m=(128, 8, 8), end=0.2, cfl=0.6, stepN=0, tScheme=1, sScheme=1, jacobMean=1,
        fluxSplit=0) -> CaseSpec:
    P = Boundary(abi.PERIODIC)
    O = Boundary(abi.OUTFLOW)
    return CaseSpec(
        domain_lo=(0.0, 0.0, 0.0), domain_hi=(1.0, 0.0625, 0.0625), m=m, end=end, cfl=cfl,
        stepN=stepN, tScheme=tScheme, sScheme=sScheme, jacobMean=jacobMean, fluxSplit=fluxSplit,
        refMu=0.0, init=("1", "0", "0", "0", "1"), boundaries=[O, O, P, P, P, P],
        regions=[Region("plane", p1=(0.5, 0.0, 0.0), p2=(1.0, 0.0, 0.0),
                        exprs=("0.125", "0", "0", "0", "0.1"))])


def tgv(n=128, Re=1600.0, Ma=0.1, cfl=0.5, stepN=200, tScheme=1, sScheme=1,
        jacobMean=1, fluxSplit=0) -> CaseSpec:
    """Viscous TGV on [0,2pi]^3 with rho0 = 1, T0 = 1: refT makes refMa = Ma
    (cfd_parameters.c:175) and refMu makes mu(T0) = 1/Re (cfd_parameters.c:177
    with the Sutherland law).  The reference fixes Pr = 0.71."""
    refT = 1.0 / (Ma * Ma * GAMMA * GAS_R)
    refMu = (1.0 / Re) / sutherland(refT)
    p0 = 1.0 / (GAMMA * Ma * Ma)
    P = Boundary(abi.PERIODIC)
    L = 2.0 * math.pi
    return CaseSpec(
        domain_lo=(0.0, 0.0, 0.0), domain_hi=(L, L, L), m=(n, n, n), end=1.0e6, cfl=cfl,
        stepN=stepN, tScheme=tScheme, sScheme=sScheme, jacobMean=jacobMean, fluxSplit=fluxSplit,
        refMu=refMu, refT=refT,
        init=("1", "sin(x)*cos(y)*cos(z)", "-cos(x)*sin(y)*cos(z)", "0",
              "%.17g+(1/16)*(cos(2*x)+cos(2*y))*(cos(2*z)+2)" % p0),
        boundaries=[P] * 6)


def sphere_centres(count=8, radius=0.15, lo=0.35, hi=3.65, gap=0.1, seed=1):
    """Seeded centres, uniform in [lo,hi]^3, rejection-sampled for a surface
    gap >= gap; velocities uniform in [-0.05, 0.05]^3 from the same stream."""
    rng = np.random.default_rng(seed)
    centres = []
    while len(centres) < count:
        c = rng.uniform(lo, hi, size=3)
        if all(np.linalg.norm(c - q) >= 2 * radius + gap for q in centres):
            centres.append(c)
    vel = rng.uniform(-0.05, 0.05, size=(count, 3))
    return np.array(centres), vel


def ib_spheres(n=192, count=8, Re=200.0, Ma=0.3, stepN=100, level=3, analytic=0,
               moving=True, psi=2) -> CaseSpec:
    """Crossflow over ``count`` spheres of radius 0.15 in [0,4]^3: west inflow
    (rho 1, u 1), east outflow, periodic y/z; the first ``analytic`` bodies are
    analytical spheres, the rest 1280-facet icospheres (level 3)."""
    refT = 1.0 / (Ma * Ma * GAMMA * GAS_R)
    D = 0.3
    refMu = (1.0 * 1.0 * D / Re) / sutherland(refT)
    p0 = 1.0 / (GAMMA * Ma * Ma)
    centres, vel = sphere_centres(count)
    bodies = []
    for q in range(count):
        V = tuple(vel[q]) if moving else (0.0, 0.0, 0.0)
        rho = 10.0 if moving else 1.0e40
        if q < analytic:
            bodies.append(Body(O=tuple(centres[q]), r=0.15, V=V, rho=rho, T=-1.0, cf=1.0))
        else:
            tris = icosphere(centres[q], 0.15, level=level)
            bodies.append(Body(O=tuple(centres[q]), r=0.15, V=V, rho=rho, T=-1.0, cf=1.0,
                               stl=f"sphere{q}.stl", triangles=tris))
    P = Boundary(abi.PERIODIC)
    return CaseSpec(
        domain_lo=(0.0, 0.0, 0.0), domain_hi=(4.0, 4.0, 4.0), m=(n, n, n), end=1.0e6, cfl=0.5,
        stepN=stepN, psi=psi if moving else 0, ibmLayer=1, refMu=refMu, refT=refT,
        init=("1", "1", "0", "0", "%.17g" % p0),
        boundaries=[Boundary(abi.INFLOW, (1.0, 1.0, 0.0, 0.0, p0)), Boundary(abi.OUTFLOW), P, P, P, P],
        bodies=bodies)


POST_SHOCK = (3.67372, 2.41981, 0.0, 0.0, 9.04545)  # Rankine-Hugoniot state, Ma 2.81


def shock_cylinder(m=(1024, 512, 4), stepN=100, segments=64) -> CaseSpec:
    P = Boundary(abi.PERIODIC)
    W = Boundary(abi.SLIPWALL, (-1.0,))
    tris = extruded_cylinder((4.0, 4.0), 0.5, -0.25, 0.3125, segments=segments)
    body = Body(O=(4.0, 4.0, 0.03125), r=0.5, rho=1.0e40, T=-1.0, cf=0.0, stl="cylinder.stl",
                triangles=tris)
    return CaseSpec(
        domain_lo=(0.0, 0.0, 0.0), domain_hi=(16.0, 8.0, 0.0625), m=m, end=1.0e6, cfl=0.5,
        stepN=stepN, refMu=0.0, init=("1", "0", "0", "0", "1"),
        boundaries=[Boundary(abi.INFLOW, POST_SHOCK), Boundary(abi.OUTFLOW), W, W, P, P],
        regions=[Region("plane", p1=(2.0, 0.0, 0.0), p2=(-1.0, 0.0, 0.0),
                        exprs=tuple("%.17g" % v for v in POST_SHOCK))],
        bodies=[body])


def riemann_viscous(n=64, Re=1600.0, Ma=0.3, rng=None, cfl=0.5) -> CaseSpec:
    """Viscous 3D Riemann problem on the unit cube: eight seeded constant
    states in the octants, outflow on all faces.  As for the TGV, rho0 = 1 and
    T0 = 1 define the reference state (refT from Ma, refMu from Re with the
    unit cube's edge as length scale).  The octant states are drawn in
    rho in [0.5, 2], p in [0.5, 2] * p0 (p0 = 1/(gamma Ma^2)), each velocity
    component in [-0.5, 0.5]: the reference's time step has no viscous limit,
    and Sutherland's law at the temperatures of wider draws (rho in [0.1, 10],
    p in [0.1, 100]) would make the explicit viscous update unstable."""
    rng = rng if rng is not None else np.random.default_rng(0)
    refT = 1.0 / (Ma * Ma * GAMMA * GAS_R)
    refMu = (1.0 / Re) / sutherland(refT)
    p0 = 1.0 / (GAMMA * Ma * Ma)
    O = Boundary(abi.OUTFLOW)

    def state():
        rho = rng.uniform(0.5, 2.0)
        u, v, w = rng.uniform(-0.5, 0.5, size=3)
        p = p0 * rng.uniform(0.5, 2.0)
        return tuple("%.17g" % x for x in (rho, u, v, w, p))

    first = state()
    regions = []
    for a in range(2):
        for b in range(2):
            for c in range(2):
                if a == 0 and b == 0 and c == 0:
                    continue
                regions.append(Region("box", p1=(0.5 * a, 0.5 * b, 0.5 * c),
                                      p2=(0.5 * a + 0.5, 0.5 * b + 0.5, 0.5 * c + 0.5), exprs=state()))
    return CaseSpec(domain_lo=(0.0, 0.0, 0.0), domain_hi=(1.0, 1.0, 1.0), m=(n, n, n), end=1.0e6, cfl=cfl,
                    stepN=0, refMu=refMu, refT=refT, init=first, boundaries=[O] * 6, regions=regions)


def batch_cases(count=48, seed=42, sizes=range(64, 161, 16)):
    """The batched sweep: `count` independent cases, each a viscous TGV or a
    viscous 3D Riemann problem (equal odds), grid n^3 with n drawn uniformly
    from `sizes`, Ma uniform in [0.1, 0.5], Re uniform in [400, 3200], all
    from one seeded generator.  Returns a list of CaseSpec; spec.kind, spec.n,
    spec.Ma and spec.Re describe each case."""
    rng = np.random.default_rng(seed)
    sizes = list(sizes)
    out = []
    for _ in range(count):
        n = int(sizes[rng.integers(len(sizes))])
        kind = "tgv" if rng.random() < 0.5 else "riemann"
        Ma = float(rng.uniform(0.1, 0.5))
        Re = float(rng.uniform(400.0, 3200.0))
        spec = tgv(n=n, Re=Re, Ma=Ma, stepN=0) if kind == "tgv" else riemann_viscous(n=n, Re=Re, Ma=Ma, rng=rng)
        spec.kind, spec.n, spec.Ma, spec.Re = kind, n, Ma, Re
        out.append(spec)
    return out
