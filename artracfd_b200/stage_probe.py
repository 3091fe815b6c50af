"""One RK stage per sweep axis on the TGV 128^3 workload, for profilers.

    python -m artracfd_b200.stage_probe --form hybrid --tiles 7,7,7 [--n 128]

Builds the viscous Taylor-Green case, fills the ghosts, selects the
arithmetic form and the stage-kernel variant of each axis (acfd_set_tiles;
"auto" runs the autotuner), updates the sensor flags (hybrid form) and runs
RK stage 2 (U[TO], U[TN] -> U[TM]) once along x, y and z, so that a profiler
captures exactly one launch of each axis' stage kernel after the set-up.

With --step (and tiles given, so that the set-up launches no stage kernel)
it runs one time step (acfd_evolve_fluid) instead: the stage kernels then
launch in step order, three per half step (sweep order z y x x y z), and the
hybrid form's X half steps run as they do in a step, as Y sweeps of the
transposed state.  The X half step's RK stage 2 is then the eighth
stage-kernel launch:

    ncu -k regex:stage_plane -s 7 -c 1 ... python -m artracfd_b200.stage_probe --form hybrid --tiles 8,8,8 --step
"""
from __future__ import annotations

import argparse

from . import abi, configs, sensor
from .solver import Solver


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--form", default="hybrid", choices=["fp64", "fp32", "hybrid"])
    ap.add_argument("--tiles", default="auto", help="variant per axis, e.g. 0,7,7, or auto")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--step", action="store_true", help="one time step instead of one stage per axis")
    args = ap.parse_args(argv)
    spec = configs.tgv(n=args.n)
    part, model = spec.descriptors()
    node = spec.initial_nodes(part, model)
    mode = {"fp64": abi.FP64, "fp32": abi.FP32_BULK, "hybrid": abi.FP64}[args.form]
    with Solver(part, model, mode) as s:
        if args.form == "hybrid":
            sensor.attach(s)
        s.upload(node)
        s.treat_boundary(abi.TO)
        if args.tiles == "auto":
            tiles = s.autotune()
        else:
            tiles = [int(t) for t in args.tiles.split(",")]
            s.set_tiles(tiles)
        dt = s.time_step(spec.cfl)
        if args.step:
            s.evolve(dt)
        else:
            if args.form == "hybrid":
                s.sensor_update()
            for sd in (0, 1, 2):
                s.lllu(0.5 * dt, 0.0, 1.0, abi.TO, abi.TO, abi.TN, sd)
            for sd in (0, 1, 2):
                s.lllu(0.5 * dt, 0.75, 0.25, abi.TO, abi.TN, abi.TM, sd)
        s.download()
    print("stage_probe", args.form, "tiles", tiles)


if __name__ == "__main__":
    main()
