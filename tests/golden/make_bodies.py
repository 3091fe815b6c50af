"""Generate the preprocessed bodies of the named workloads from the reference
itself, for callers that build those cases without the reference program
(bench.py's shock-cylinder block).

The unmodified reference (oracle/_ref/libacfd_ref.so) loads the case written
by artracfd_b200.configs and preprocesses its bodies as the program does
(ReadStlFile, ConvertPolyhedron, the polyhedron transform and
ComputeGeometryParameters: initialization.c:164-205, computational_geometry.c);
the body descriptors and surface arrays are saved with the key prefix
``geo_`` (artracfd_b200.case.load_polyhedra reads them back), together with
the reference's partition and model bytes for a consistency check.

Run from the repository root:  python tests/golden/make_bodies.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from artracfd_b200 import configs  # noqa: E402
from make_golden import geo_arrays  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

BODIES = {"shock_cylinder": configs.shock_cylinder}


def main():
    ref = Reference()
    work = tempfile.mkdtemp(prefix="acfd_bodies_")
    for name, make in BODIES.items():
        path = os.path.join(work, name)
        make().write(path)
        ref.load(path)
        rec = {"part": np.frombuffer(bytes(ref.partition()), dtype=np.uint8).copy(),
               "model": np.frombuffer(bytes(ref.model()), dtype=np.uint8).copy()}
        rec.update(geo_arrays("geo_", ref.geometry()))
        out = os.path.join(HERE, f"bodies_{name}.npz")
        np.savez_compressed(out, **rec)
        print(f"{name}: {int(rec['geo_count'])} bodies, {os.path.getsize(out) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
