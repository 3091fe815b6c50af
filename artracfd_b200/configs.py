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
