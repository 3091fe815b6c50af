"""Whole time steps of a named configuration, for launch lists.

    python -m artracfd_b200.step_probe --case shock_cylinder --form hybrid [--steps 3] [--warmup 2]

Builds the case as the benchmark does (TGV 128^3, or the shock-cylinder at
1024x512x4 with the extruded cylinder of tests/golden/bodies_shock_cylinder.npz
uploaded and mapped onto the nodes), selects the arithmetic form, autotunes
the stage-kernel variants after a few steps, runs `warmup` steps and then
`steps` steps -- CFL read back, host dt, EvolveFluidDynamics replayed as one
CUDA graph -- inside the NVTX range "timed", so that a profiler can list
exactly the kernels of those steps:

    ncu --nvtx --nvtx-include "timed/" --metrics gpu__time_duration.sum ...
"""
from __future__ import annotations

import argparse
import os

import numpy as np

from . import abi, configs, sensor
from .case import load_polyhedra
from .solver import Solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="shock_cylinder", choices=["tgv", "shock_cylinder"])
    ap.add_argument("--form", default="hybrid", choices=["fp64", "fp32", "hybrid"])
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=2)
    args = ap.parse_args(argv)
    import torch

    geo, keep = None, None
    if args.case == "tgv":
        spec = configs.tgv(n=128)
    else:
        spec = configs.shock_cylinder()
        z = np.load(os.path.join(ROOT, "tests", "golden", "bodies_shock_cylinder.npz"))
        geo, keep = load_polyhedra(z)
    part, model = spec.descriptors()
    mode = {"fp64": abi.FP64, "fp32": abi.FP32_BULK, "hybrid": abi.FP64}[args.form]
    with Solver(part, model, mode) as s:
        if args.form == "hybrid":
            sensor.attach(s)
        s.upload(spec.initial_nodes(part, model))
        if geo:
            s.geo_upload(geo)
            s.compute_geometric_field()
        s.treat_boundary(abi.TO)
        for _ in range(3):
            s.evolve(s.time_step(spec.cfl))
        tiles = s.autotune()
        for _ in range(args.warmup):
            s.evolve(s.time_step(spec.cfl), graph=True)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")
        for _ in range(args.steps):
            s.evolve(s.time_step(spec.cfl), graph=True)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    del keep
    print("step_probe", args.case, args.form, "tiles", tiles)


if __name__ == "__main__":
    main()
