"""Host-side logic without a GPU: descriptors restated from the reference's
set-up code, the C ABI surface, and the node record layout."""
import ctypes
import os
import re

import numpy as np
import pytest

from artracfd_b200 import abi, configs
from artracfd_b200.abi import load_library

import cases
import golden_io

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name", golden_io.names())
def test_python_descriptors_equal_reference(name):
    """CaseSpec.descriptors restates ComputeParameters/PartitionDomain: the
    partition and model must equal the reference's bytes."""
    b = golden_io.Bundle(name)
    part, model = cases.SMALL[name]().descriptors()
    assert bytes(part) == bytes(b.part)
    assert bytes(model) == bytes(b.model)


def test_node_record_layout():
    # acfd_node_t has the reference Node layout: 4 ints, U[3][5] doubles
    assert abi.NODE_DTYPE.itemsize == 136
    assert abi.NODE_DTYPE.fields["U"][1] == 16
    assert ctypes.sizeof(abi.Partition) == len(golden_io.Bundle("sod").z["part"])


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "acfd.h")).read()
    declared = sorted(set(re.findall(r"^int\s+(acfd_\w+)\s*\(", header, re.M)))
    assert len(declared) >= 20
    lib = load_library()
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_library_reports_errors_without_crashing():
    lib = load_library()
    assert lib.acfd_abi_version() == 1
    buf = ctypes.create_string_buffer(64)
    assert lib.acfd_last_error(buf, 64) == 0
    assert lib.acfd_last_error(None, 0) == abi.ACFD_ERR_ARG
    # a null handle is an argument error, not a crash
    assert lib.acfd_cfl(None, None) == abi.ACFD_ERR_ARG
    assert lib.acfd_evolve_fluid(None, 1.0) == abi.ACFD_ERR_ARG


def test_initial_field_matches_reference_on_pin_nodes():
    """The numpy initializer reproduces the reference's initial PIN field to
    rounding (the reference evaluates expressions with its own calculator)."""
    b = golden_io.Bundle("tgv")
    spec = cases.SMALL["tgv"]()
    mine = spec.initial_nodes(b.part, b.model)
    pin = cases.pin_mask(b.part)
    ref = b.z["U0"]
    assert np.allclose(mine["U"][pin, 0, :], ref[pin], rtol=1e-13, atol=1e-13)
    for q, f in enumerate(("did", "fid", "lid", "gst")):
        assert np.array_equal(mine[f][pin], b.z["flags0"][pin, q])


def test_batch_cases_are_seeded_and_cover_the_stated_ranges():
    a = configs.batch_cases(count=48, seed=42)
    b = configs.batch_cases(count=48, seed=42)
    assert len(a) == 48
    assert [(s.kind, s.n, s.Ma, s.Re) for s in a] == [(s.kind, s.n, s.Ma, s.Re) for s in b]
    assert {s.kind for s in a} == {"tgv", "riemann"}
    assert all(s.n in range(64, 161, 16) for s in a)
    assert all(0.1 <= s.Ma <= 0.5 and 400.0 <= s.Re <= 3200.0 for s in a)
    for s in a[:4]:
        part, model = s.descriptors()
        assert model.refMu > 0.0 and part.collapse == 0
