"""The learned-sensor configuration at its named size: a Ma 2.81 planar shock
passing an extruded cylinder (diameter 1, 256 facets) in [0,16]x[0,8]x[0,0.0625]
at 1024 x 512 x 4 cells (1023 x 511 x 5 computed nodes), inviscid, WENO5/LLF/
Roe, RK3, CFL 0.5.

The unmodified reference (the harness in oracle/_ref) loads the case: its
initial field, node flags and cylinder geometry are the start of three GPU
runs over the same 100 time steps (the dt sequence of the plain FP64 path):
the plain FP64 path, the learned-sensor hybrid form and the linear-weight
scheme alone (a sensor that flags nothing).  The hybrid form stays within
L1 density error 1e-3 of the FP64 path; the linear scheme alone does not
stay as close, which is what the sensor buys.
"""
import os

import numpy as np
import pytest

from artracfd_b200 import abi, configs, sensor
from artracfd_b200.solver import Solver
from oracle.oracle import Reference, reference_available

pytestmark = pytest.mark.gpu

STEPS = 100


def _run(part, model, node0, geo, mode, dts=None, cfl=0.5, params=None, thr=0.5):
    import torch

    out_dts = []
    stream = torch.cuda.Stream()
    with Solver(part, model, abi.FP64) as s:
        s.set_stream(stream.cuda_stream)
        s.upload(node0)
        s.geo_upload(geo)
        if mode == abi.FP32_HYBRID:
            s.sensor_load(params, thr)
        s.set_precision(mode)
        s.autotune()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(STEPS):
            dt = s.time_step(cfl) if dts is None else dts[k]
            s.evolve(dt, graph=True)
            out_dts.append(dt)
        e1.record(stream)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        node = s.download()
    return node, out_dts, sec


@pytest.mark.skipif(not reference_available() or not os.path.exists(sensor.WEIGHTS),
                    reason="reference harness or sensor weights missing")
def test_shock_cylinder_full_size_hybrid_within_stated_error(tmp_path):
    spec = configs.shock_cylinder()
    path = os.path.join(str(tmp_path), "shock_cylinder")
    spec.write(path)
    ref = Reference()
    ref.load(path)
    part, model, node0, geo = ref.partition(), ref.model(), ref.nodes(), ref.geometry()
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    _, dts, _ = _run(part, model, node0, geo, abi.FP64)
    # every timed run replays the same dt sequence (no host dt in the loop)
    ref64, _, t64 = _run(part, model, node0, geo, abi.FP64, dts)
    hyb, _, thyb = _run(part, model, node0, geo, abi.FP32_HYBRID, dts, params=params, thr=thr)
    lin, _, _ = _run(part, model, node0, geo, abi.FP32_HYBRID, dts, params=np.r_[np.zeros(params.size - 1),
                                                                                  -50.0].astype(np.float32))
    fluid = ref64["did"] == 0
    r = ref64["U"][fluid, 0, 0]

    def l1(a):
        d = a["U"][fluid, 0, 0]
        return float(np.abs(d - r).sum() / np.abs(r).sum()) if np.isfinite(d).all() else float("inf")

    e_hyb, e_lin = l1(hyb), l1(lin)
    pin = int(np.prod(np.array(part.ns)[0, :, 1] - np.array(part.ns)[0, :, 0]))
    print(f"shock-cylinder 1024x512x4, {STEPS} steps: FP64 {pin * STEPS / t64 / 1e6:.1f} Mcell-steps/s, "
          f"hybrid {pin * STEPS / thyb / 1e6:.1f} Mcell-steps/s; L1 rho hybrid {e_hyb:.3g}, linear alone {e_lin:.3g}")
    assert e_hyb <= 1e-3, e_hyb
    assert e_lin > e_hyb, (e_lin, e_hyb)
