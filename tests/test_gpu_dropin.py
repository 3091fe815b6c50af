"""The drop-in program: the reference program linked with libacfd_gpu
(artracfd_b200/shim), run with `-m gpu`, against the unmodified reference
program (oracle/_ref/artracfd) on the same case directory.  Both write their
fields as EnSight float32 files, which are compared."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from artracfd_b200 import configs

import cases

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "artracfd_b200", "shim", "_build", "artracfd_gpu")
REFBIN = os.path.join(ROOT, "oracle", "_ref", "artracfd")
FIELDS = ("rho", "u", "v", "w", "p", "T", "did")


def _run(binary, mode, case_dir, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    r = subprocess.run([binary, "-m", mode], cwd=case_dir, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (binary, r.stdout[-2000:], r.stderr[-2000:])
    return r


def _field(path):
    # EnSight Gold binary variable file: 3 x 80-byte strings, part id, 80-byte
    # "block" line, then float32 values
    raw = open(path, "rb").read()
    return np.frombuffer(raw[80 + 80 + 4 + 80:], dtype=np.float32)


def _last_fields(case_dir):
    names = sorted(f for f in os.listdir(case_dir) if f.startswith("field0") and f.endswith(".rho"))
    stem = names[-1][:-4]
    return stem, {f: _field(os.path.join(case_dir, f"{stem}.{f}")) for f in FIELDS}


def _pair(tmp_path, spec):
    a = tmp_path / "ref"
    b = tmp_path / "gpu"
    spec.write(str(a))
    shutil.copytree(a, b)
    return str(a), str(b)


needs = pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFBIN)),
                           reason="drop-in or reference program not built")


@needs
def test_dropin_exact_mode_reproduces_reference_files(tmp_path):
    spec = configs.sod(m=(32, 4, 4), stepN=6)
    a, b = _pair(tmp_path, spec)
    _run(REFBIN, "serial", a)
    _run(DROPIN, "gpu", b, {"ACFD_MODE": "exact"})
    sa, fa = _last_fields(a)
    sb, fb = _last_fields(b)
    assert sa == sb
    for f in FIELDS:
        assert np.array_equal(fa[f], fb[f]), f


@needs
@pytest.mark.parametrize("name", ["tgv", "channel", "spheres"])
def test_dropin_fast_mode_close_to_reference(tmp_path, name):
    spec = cases.SMALL[name]()
    spec.stepN = 4
    a, b = _pair(tmp_path, spec)
    _run(REFBIN, "serial", a)
    _run(DROPIN, "gpu", b, {"ACFD_MODE": "fp64"})
    sa, fa = _last_fields(a)
    sb, fb = _last_fields(b)
    assert sa == sb
    assert np.array_equal(fa["did"], fb["did"])
    for f in FIELDS[:-1]:
        scale = max(np.abs(fa[f]).max(), np.abs(fa["rho"]).max() * 1e-3)
        assert np.abs(fa[f] - fb[f]).max() <= 1e-5 * scale, f


@needs
@pytest.mark.parametrize("solid", ["device", "device_host_motion", "host"])
def test_dropin_exact_mode_moving_bodies_with_contacts(tmp_path, solid):
    """Three inviscid moving spheres resting on one another in a crossflow:
    with the rigid-body step's node scans on the device (surface forces,
    contact lists, remapping and ghost values; the node array stays on the
    GPU) and the surfaces moved there too (default) or on the host
    (ACFD_MOTION=host), or with the whole step on the host, the exact mode
    writes the reference's files."""
    spec = cases.contact_spheres(viscous=False)
    spec.stepN = 5
    a, b = _pair(tmp_path, spec)
    _run(REFBIN, "serial", a)
    env = {"ACFD_MODE": "exact", "ACFD_SOLID": "host" if solid == "host" else "device"}
    if solid == "device_host_motion":
        env["ACFD_MOTION"] = "host"
    _run(DROPIN, "gpu", b, env)
    sa, fa = _last_fields(a)
    sb, fb = _last_fields(b)
    assert sa == sb
    for f in FIELDS:
        assert np.array_equal(fa[f], fb[f]), (f, np.abs(fa[f] - fb[f]).max())


@needs
def test_dropin_viscous_contacts_close_to_reference(tmp_path):
    spec = cases.contact_spheres(viscous=True)
    spec.stepN = 5
    a, b = _pair(tmp_path, spec)
    _run(REFBIN, "serial", a)
    _run(DROPIN, "gpu", b, {"ACFD_MODE": "fp64"})
    sa, fa = _last_fields(a)
    sb, fb = _last_fields(b)
    assert sa == sb
    assert np.array_equal(fa["did"], fb["did"])
    for f in FIELDS[:-1]:
        scale = max(np.abs(fa[f]).max(), np.abs(fa["rho"]).max() * 1e-3)
        assert np.abs(fa[f] - fb[f]).max() <= 1e-5 * scale, f


def _fields_of(case_dir, index):
    stem = "field%05d" % index
    return {f: _field(os.path.join(case_dir, f"{stem}.{f}")) for f in FIELDS}


@needs
@pytest.mark.parametrize("name", ["sod", "contact_spheres"])
def test_dropin_fp64_checkpoint_restart_continues_bit_for_bit(tmp_path, name):
    """Two space data outputs; the run restarted from the first one (restart
    tag 1) with its FP64 checkpoint writes the second one exactly as the
    uninterrupted run (the reference restarts from its float32 files).  With
    moving, touching bodies the checkpoint also carries their motion state
    and transformed surfaces."""
    if name == "sod":
        spec = configs.sod(m=(32, 4, 4))
    else:
        spec = cases.contact_spheres(viscous=False)
        spec.end = 0.03
    spec.stepN = 0
    spec.dataW = 2
    a = tmp_path / "a"
    spec.write(str(a))
    _run(DROPIN, "gpu", str(a), {"ACFD_MODE": "exact", "ACFD_CHECKPOINT": "1"})
    assert (a / "artracfd.ckpt.00001").exists() and (a / "artracfd.ckpt.00002").exists()
    b = tmp_path / "b"
    shutil.copytree(a, b)
    for f in b.glob("field00002.*"):
        f.unlink()
    spec.restart = 1
    spec.write(str(b))
    r = _run(DROPIN, "gpu", str(b), {"ACFD_MODE": "exact"})
    assert "restarted from the FP64 checkpoint" in r.stdout
    fa, fb = _fields_of(str(a), 2), _fields_of(str(b), 2)
    for f in FIELDS:
        assert np.array_equal(fa[f], fb[f]), f


@needs
def test_dropin_async_output_equals_synchronous_output(tmp_path):
    """Outputs written from a device snapshot while the next step runs are
    the outputs of a synchronous download."""
    spec = configs.sod(m=(32, 4, 4))
    spec.stepN = 0
    spec.dataW = 4
    a, b = _pair(tmp_path, spec)
    _run(DROPIN, "gpu", a, {"ACFD_MODE": "fp64", "ACFD_ASYNC_OUTPUT": "0"})
    _run(DROPIN, "gpu", b, {"ACFD_MODE": "fp64"})
    for q in range(5):
        fa, fb = _fields_of(a, q), _fields_of(b, q)
        for f in FIELDS:
            assert np.array_equal(fa[f], fb[f]), (q, f)


@needs
def test_dropin_hybrid_mode_within_stated_error(tmp_path):
    """ACFD_MODE=hybrid: the learned-sensor form through the drop-in program
    (the shipped sensor weights) on a reduced shock-cylinder case stays within
    L1 density error 1e-3 of the unmodified reference program."""
    spec = configs.shock_cylinder(m=(128, 64, 4), segments=48)
    spec.stepN = 20
    a, b = _pair(tmp_path, spec)
    _run(REFBIN, "serial", a)
    r = _run(DROPIN, "gpu", b, {"ACFD_MODE": "hybrid", "ACFD_AUTOTUNE": "1"})
    assert "autotuned" in r.stdout
    sa, fa = _last_fields(a)
    sb, fb = _last_fields(b)
    assert sa == sb
    assert np.array_equal(fa["did"], fb["did"])
    fluid = fa["did"] == 0
    l1 = np.abs(fb["rho"][fluid] - fa["rho"][fluid]).sum() / np.abs(fa["rho"][fluid]).sum()
    assert l1 <= 1e-3, l1


@needs
def test_dropin_serial_mode_is_the_reference(tmp_path):
    spec = configs.sod(m=(32, 4, 4), stepN=3)
    a, b = _pair(tmp_path, spec)
    _run(REFBIN, "serial", a)
    _run(DROPIN, "serial", b)
    sa, fa = _last_fields(a)
    sb, fb = _last_fields(b)
    for f in FIELDS:
        assert np.array_equal(fa[f], fb[f])
