"""Generate the golden fixtures in this directory from the reference itself.

For every small case of tests/cases.py the unmodified reference (built by
oracle/Makefile into oracle/_ref/libacfd_ref.so) loads the case directory and
records:

* its own partition and model descriptors (raw acfd_partition_t/acfd_model_t
  bytes), the CFL number and end time;
* the initial node field after InitializeComputeDomain (U[TO] and the four
  flags; U[TN], U[TM] are the reference's memset(1) junk everywhere);
* the body list with the reference's preprocessed geometry arrays;
* dt and U[TO] after each of two fluid steps (ComputeTimeStep +
  EvolveFluidDynamics, no solid dynamics);
* for cases with moving bodies: the bodies and node field after one
  EvolveSolidDynamics (motion, ComputeGeometricField, TreatImmersedBoundary).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import cases  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

STEPS = 2


def geo_arrays(prefix: str, geo) -> dict:
    out = {prefix + "count": np.array(len(geo))}
    for q, P in enumerate(geo):
        p = f"{prefix}{q}_"
        out[p + "scal"] = np.array([P.faceN, P.edgeN, P.vertN, P.state], dtype=np.int64)
        out[p + "real"] = np.array([P.r, *P.O, *P.V, *P.W, P.T, P.cf] + [P.box[s][m] for s in range(3) for m in range(2)])
        if P.faceN > 0:
            out[p + "f"] = np.ctypeslib.as_array(P.f, (P.faceN * 3,)).copy()
            out[p + "Nf"] = np.ctypeslib.as_array(P.Nf, (P.faceN * 3,)).copy()
            out[p + "e"] = np.ctypeslib.as_array(P.e, (P.edgeN * 4,)).copy()
            out[p + "Ne"] = np.ctypeslib.as_array(P.Ne, (P.edgeN * 3,)).copy()
            out[p + "v"] = np.ctypeslib.as_array(P.v, (P.vertN * 3,)).copy()
            out[p + "Nv"] = np.ctypeslib.as_array(P.Nv, (P.vertN * 3,)).copy()
    return out


def field(node) -> dict:
    return {"U": node["U"][:, 0, :].copy(), "flags": np.stack([node[f] for f in ("did", "fid", "lid", "gst")], 1)}


def main():
    ref = Reference()
    work = tempfile.mkdtemp(prefix="acfd_golden_")
    for name in cases.SMALL:
        b = cases.load(ref, name, work)
        rec = {
            "part": np.frombuffer(bytes(b["part"]), dtype=np.uint8).copy(),
            "model": np.frombuffer(bytes(b["model"]), dtype=np.uint8).copy(),
            "cfl": np.array(b["time"]["cfl"]),
            "end": np.array(b["time"]["end"]),
        }
        f0 = field(b["nodes"])
        rec["U0"], rec["flags0"] = f0["U"], f0["flags"]
        rec.update(geo_arrays("geo_", b["geo"]))
        dts = []
        for k in range(STEPS):
            dt = ref.time_step()
            ref.evolve_fluid(dt)
            dts.append(dt)
            rec[f"U{k + 1}"] = ref.nodes()["U"][:, 0, :].copy()
        rec["dt"] = np.array(dts)
        if b["model"].psi != 0 and b["geo"]:
            # one solid half step from the initial state: motion + remapping
            ref.load(b["path"])
            ref.lib.ref_evolve_solid(0.0, 0.5 * dts[0])
            fs = field(ref.nodes())
            rec["Us"], rec["flagss"] = fs["U"], fs["flags"]
            rec.update(geo_arrays("geos_", ref.geometry()))
        out = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(out, **rec)
        print(f"{name}: {os.path.getsize(out) / 1024:.0f} KiB, dt={dts}")


if __name__ == "__main__":
    main()
