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


def test_shock_cylinder_body_fixture_belongs_to_the_named_case(tmp_path):
    """tests/golden/bodies_shock_cylinder.npz (the cylinder as the reference
    preprocesses it, read by bench.py) holds the partition and model of
    configs.shock_cylinder() at its full size; where the reference harness is
    built, its preprocessing of the same case gives the same surface."""
    from artracfd_b200.case import load_polyhedra
    z = np.load(os.path.join(ROOT, "tests", "golden", "bodies_shock_cylinder.npz"))
    part, model = configs.shock_cylinder().descriptors()
    assert bytes(part) == bytes(z["part"])
    assert bytes(model) == bytes(z["model"])
    geo, keep = load_polyhedra(z)
    assert len(geo) == 1 and geo[0].faceN > 0 and geo[0].state == 1
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        return
    ref = Reference()
    path = str(tmp_path / "sc")
    configs.shock_cylinder(m=(64, 32, 4)).write(path)  # same body file, small mesh
    ref.load(path)
    P = ref.geometry()[0]
    for key, rows in (("v", P.vertN), ("Nv", P.vertN), ("Nf", P.faceN), ("Ne", P.edgeN)):
        got = np.ctypeslib.as_array(getattr(P, key), (rows * 3,))
        assert np.array_equal(got, keep[0][key]), key


def test_sensor_threshold_leaves_uniform_stencils_to_the_linear_scheme():
    """A uniform stencil (all ten features zero) has WENO5 weights equal to the
    linear weights: the shipped threshold lies above the network's output
    there (by the stated logit margin), so uniform regions -- the quiescent
    gas ahead of a shock -- are not flagged."""
    import math
    from artracfd_b200 import sensor
    params, thr, meta = sensor.load(sensor.WEIGHTS)
    p0 = float(sensor.forward_cpu(params, np.zeros(sensor.N_IN))[0])
    assert thr > p0
    margin = math.log(thr / (1 - thr)) - math.log(p0 / (1 - p0))
    assert margin >= meta.get("uniform_margin", 0.25) - 1e-6, margin


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


def test_sensor_weights_file_holds_the_trained_sensor(tmp_path):
    """sensor_weights.bin (read by acfd_sensor_load_file and the drop-in
    program's hybrid mode) holds the parameters and threshold of
    sensor_weights.npz in the stated layout; save_bin writes that layout."""
    from artracfd_b200 import sensor
    params, thr, _ = sensor.load(sensor.WEIGHTS)

    def parse(path):
        raw = open(path, "rb").read()
        assert raw[:8] == b"ACFDSNS1"
        count = int(np.frombuffer(raw[8:12], dtype="<i4")[0])
        t = float(np.frombuffer(raw[12:16], dtype="<f4")[0])
        p = np.frombuffer(raw[16:], dtype="<f4")
        assert p.size == count
        return p, t

    p, t = parse(sensor.WEIGHTS_BIN)
    assert p.size == load_library().acfd_mlp_param_count()
    assert np.array_equal(p, params) and t == np.float32(thr)
    out = str(tmp_path / "w.bin")
    sensor.save_bin(out, params[::-1], 0.25)
    p2, t2 = parse(out)
    assert np.array_equal(p2, params[::-1]) and t2 == 0.25


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).reference_available(),
                    reason="reference harness oracle/_ref not built")
def test_case_files_carry_restart_and_output_count(tmp_path):
    """CaseSpec writes the restart tag and the space-data output count where
    the reference's loader reads them (case_loader.c:68-72): the reference
    loaded from the file starts its data count at the restart tag."""
    from oracle.oracle import Reference
    spec = configs.sod(m=(32, 4, 4))
    spec.restart, spec.dataW = 0, 3
    path = str(tmp_path / "sod")
    spec.write(path)
    text = open(os.path.join(path, "artracfd.case")).read().split("time begin")[1].split("time end")[0].split()
    assert text[0] == "0" and text[4] == "3"
    ref = Reference()
    ref.load(path)
    assert ref.time()["stepC"] == 0


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).reference_available(),
                    reason="reference harness oracle/_ref not built")
def test_contact_case_has_touching_spheres(tmp_path):
    """The rigid-body tests' contact case is what it claims: the reference's
    own contact search finds every sphere touching the other two."""
    from oracle.oracle import Reference
    spec = cases.contact_spheres(viscous=False)
    path = str(tmp_path / "contact")
    spec.write(path)
    ref = Reference()
    ref.load(path)
    lists = ref.collision_scan()
    assert [sorted(g for g, _ in c) for c in lists] == [[2, 3], [1, 3], [1, 2]]


def _bench():
    import importlib.util
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("acfd_bench", os.path.join(root, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _FakeNvml:
    """The NVML calls the clock sampler makes, answering like a GPU held at
    1965 MHz under its power cap."""
    NVML_CLOCK_SM = 1

    def __init__(self, fail_init=False):
        self.fail_init = fail_init
        self.calls = 0
        self.shut = False

    def nvmlInit(self):
        if self.fail_init:
            raise RuntimeError("no NVML")

    def nvmlShutdown(self):
        self.shut = True

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("gpu", i)

    def nvmlDeviceGetMaxClockInfo(self, h, clock):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, clock):
        self.calls += 1
        return 1965 if self.calls % 4 else 1950

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return 0x4 | 0x1  # power cap (and the idle bit, which is not reported)


def test_clock_sampler_polls_nvml_during_a_short_region(monkeypatch):
    import sys
    import time
    bench = _bench()
    fake = _FakeNvml()
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    with bench.ClockSampler(0) as clk:
        time.sleep(0.1)
    got = clk.summary()
    assert got["source"] == "nvml" and fake.shut
    assert got["samples"] >= 5
    assert got["sm_mhz"] == 1965.0 and got["sm_max_mhz"] == 1965.0
    assert got["reasons"] == ["sw_power_cap"]


def test_clock_sampler_without_nvml_falls_back_quietly(monkeypatch):
    import sys
    bench = _bench()
    monkeypatch.setitem(sys.modules, "pynvml", _FakeNvml(fail_init=True))
    monkeypatch.setenv("PATH", "/nonexistent")
    with bench.ClockSampler(0) as clk:
        pass
    got = clk.summary()
    assert got["source"] == "nvidia-smi" and got["samples"] == 0 and got["sm_mhz"] is None


_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_DROPIN = os.path.join(_ROOT, "artracfd_b200", "shim", "_build", "artracfd_gpu")
_REFBIN = os.path.join(_ROOT, "oracle", "_ref", "artracfd")


def _ensight(path):
    raw = open(path, "rb").read()
    return np.frombuffer(raw[80 + 80 + 4 + 80:], dtype=np.float32)


@pytest.mark.skipif(not (os.path.exists(_DROPIN) and os.path.exists(_REFBIN)), reason="programs not built")
def test_dropin_serial_mode_writes_the_reference_files(tmp_path):
    """The drop-in program in `-m serial` mode is the reference program: the
    renamed Solve / EvolveFluidDynamics / TreatBoundary route to the
    reference's own functions (no device is touched)."""
    import subprocess
    spec = configs.sod(m=(32, 4, 4), stepN=4)
    outs = []
    for name, binary in (("ref", _REFBIN), ("dropin", _DROPIN)):
        d = str(tmp_path / name)
        spec.write(d)
        r = subprocess.run([binary, "-m", "serial"], cwd=d, capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(d)
    names = sorted(f for f in os.listdir(outs[0]) if f.startswith("field0") and not f.endswith(".case"))
    assert names
    for f in names:
        assert np.array_equal(_ensight(os.path.join(outs[0], f)), _ensight(os.path.join(outs[1], f))), f


@pytest.mark.skipif(not os.path.exists(_DROPIN), reason="drop-in program not built")
def test_dropin_gpu_mode_fails_loudly_without_a_device(tmp_path):
    """No CPU fallback: `-m gpu` on a machine without a usable GPU stops with
    the library's error instead of computing on the host."""
    import subprocess
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    d = str(tmp_path / "case")
    configs.sod(m=(32, 4, 4), stepN=2).write(d)
    r = subprocess.run([_DROPIN, "-m", "gpu"], cwd=d, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "acfd_init failed" in r.stderr
    assert not any(f.startswith("field00001") for f in os.listdir(d))


def _header_prototypes():
    """name -> parameter count of every function declared in include/acfd.h."""
    header = open(os.path.join(ROOT, "include", "acfd.h")).read()
    header = re.sub(r"/\*.*?\*/", "", header, flags=re.S)
    out = {}
    for m in re.finditer(r"^(?:int|void|double|const char\s*\*)\s*\**\s*(acfd_\w+)\s*\(([^)]*)\)\s*;", header,
                         re.M | re.S):
        params = " ".join(m.group(2).split())
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_ctypes_binding_matches_every_prototype():
    """The ctypes binding declares every function of the header with the
    header's number of parameters (a drifted binding would pass wrong
    arguments without any error)."""
    protos = _header_prototypes()
    assert len(protos) >= 40
    lib = load_library()
    for name, count in protos.items():
        fn = getattr(lib, name)
        assert fn.argtypes is not None, name
        assert len(fn.argtypes) == count, (name, len(fn.argtypes), count)


@pytest.mark.skipif(not os.path.exists(_DROPIN), reason="drop-in program not built")
def test_dropin_bad_case_file_stops_before_the_device(tmp_path):
    """A bad case file (zero cells along x) stops the drop-in program in the
    reference's own case check (CheckCaseSettingData, case_loader.c:509-544)
    with its message, before any device work."""
    import subprocess
    d = str(tmp_path / "case")
    configs.sod(m=(32, 4, 4), stepN=2).write(d)
    path = os.path.join(d, "artracfd.case")
    text = open(path).read()
    assert "\n32, 4, 4\n" in text
    open(path, "w").write(text.replace("\n32, 4, 4\n", "\n0, 4, 4\n", 1))
    r = subprocess.run([_DROPIN, "-m", "gpu"], cwd=d, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "mesh number should be positive" in r.stderr
    assert "Solving" not in r.stdout


_TASKS_HARNESS = r"""
#include <cstdio>
#include <vector>
struct int2 { int x, y; };
struct int4 { int x, y, z, w; };
#include "ghost_tasks.h"
int main(int argc, char **argv)
{
    FILE *f = std::fopen(argv[1], "rb");
    std::vector<int2> pairs;
    int2 p;
    while (std::fread(&p, sizeof p, 1, f) == 1) pairs.push_back(p);
    std::fclose(f);
    std::vector<int4> tasks;
    std::vector<int2> single;
    ghost_copy_tasks_of<int2, int4>(pairs, tasks, single);
    FILE *o = std::fopen(argv[2], "wb");
    long long in_tasks = 0;
    for (const int4 &t : tasks) {
        if (t.z < 1 || t.z > kGhostLong) return 3;
        for (int q = 0; q < t.z; ++q) {
            const int2 e = {t.x + q, t.x + q + t.y};
            std::fwrite(&e, sizeof e, 1, o);
        }
        in_tasks += t.z;
    }
    for (const int2 &e : single) std::fwrite(&e, sizeof e, 1, o);
    std::fclose(o);
    std::printf("%zu %lld %zu\n", tasks.size(), in_tasks, single.size());
    return 0;
}
"""


def _periodic_fill_pairs(n, ng, pitch=None):
    """(destination, source) node pairs of the one-launch fill of a grid whose
    faces are all periodic: every ghost node takes the value of the computed
    node one period away along each axis where it lies outside (rows of
    `pitch` nodes, by default nx)."""
    nx, ny, nz = n
    px = nx if pitch is None else pitch
    lo = [ng, ng, ng]
    L = [nx - 2 * ng, ny - 2 * ng, nz - 2 * ng]
    out = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                c = [i, j, k]
                src = list(c)
                for a in range(3):
                    if c[a] < lo[a]:
                        src[a] += L[a]
                    elif c[a] >= lo[a] + L[a]:
                        src[a] -= L[a]
                if src != c:
                    out.append(((k * ny + j) * px + i, (src[2] * ny + src[1]) * px + src[0]))
    return np.array(out, dtype=np.int32)


def test_ghost_copy_tasks_cover_exactly_the_copies(tmp_path):
    """The copy tasks of the one-launch ghost fill (csrc/ghost_tasks.h,
    compiled here for the host): the tasks expanded, with the single copies,
    give back exactly the fill's (destination, source) copies -- periodic
    grids whose x faces are three nodes wide, a plane far longer than one
    task, the same copies in a random order, and an outflow-like list of
    short runs."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "tasks.cpp"
    src.write_text(_TASKS_HARNESS)
    exe = tmp_path / "tasks"
    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "artracfd_b200", "csrc")
    subprocess.run([gxx, "-O2", "-std=c++17", "-I" + csrc, str(src), "-o", str(exe)], check=True)
    rng = np.random.default_rng(7)
    cases_ = {
        "periodic 19^3": _periodic_fill_pairs((19, 19, 19), 3),
        "periodic thin z": _periodic_fill_pairs((70, 40, 11), 3),
        "plane longer than a task": np.stack([np.arange(5000, 12000), np.arange(20000, 27000)], 1).astype(np.int32),
    }
    shuffled = cases_["periodic 19^3"].copy()
    rng.shuffle(shuffled)
    cases_["shuffled"] = shuffled
    rows = [(r * 40 + c, r * 40 + c + 3) for r in range(60) for c in range(3)]
    cases_["outflow-like"] = np.array(rows, dtype=np.int32)
    for name, pairs in cases_.items():
        pin, pout = tmp_path / "pairs.bin", tmp_path / "out.bin"
        pairs.astype(np.int32).tofile(pin)
        r = subprocess.run([str(exe), str(pin), str(pout)], capture_output=True, text=True, check=True)
        got = np.fromfile(pout, dtype=np.int32).reshape(-1, 2)
        want = pairs.reshape(-1, 2)
        assert len(got) == len(want), name
        assert np.array_equal(got[np.lexsort(got.T[::-1])], want[np.lexsort(want.T[::-1])]), name
        ntask, in_tasks, nsingle = (int(x) for x in r.stdout.split())
        if name == "plane longer than a task":
            assert (ntask, in_tasks, nsingle) == (4, 7000, 0)  # three pieces of 2048 and the rest
        if name == "outflow-like":
            assert (ntask, nsingle) == (0, len(want))  # runs of three: single copies


_DIV_HARNESS = r"""
#include <cstdio>
#include <cstdint>
#include <initializer_list>
#include "fast_div.h"
// every divisor 1..4096 against numerators at and around its multiples and
// at random across the range the kernels use (n < 2^31), then random divisors
static uint64_t state = 88172645463325252ull;
static uint32_t rnd() { state ^= state << 13; state ^= state >> 7; state ^= state << 17; return (uint32_t)state; }
static int check(uint32_t d, uint32_t n)
{
    if (n >= (1u << 31)) return 0;
    return fast_div(n, make_fast_div(d)) != n / d;
}
int main()
{
    long long bad = 0, tried = 0;
    for (uint32_t d = 1; d <= 4096; ++d) {
        for (uint32_t q = 0; q < 2000; ++q) {
            for (int e = -1; e <= 1; ++e) {
                const long long n = (long long)q * d + e;
                if (n < 0) continue;
                bad += check(d, (uint32_t)n);
                ++tried;
            }
        }
        for (int r = 0; r < 2000; ++r) {
            bad += check(d, rnd() >> 1);
            ++tried;
        }
    }
    for (int r = 0; r < 200000; ++r) {
        const uint32_t d = (rnd() >> 1) | 1u, n = rnd() >> 1;
        bad += check(d, n) + check(d, n - n % d) + check(d, n - n % d - 1u * (n >= d));
        tried += 3;
    }
    const uint32_t edge[] = {0u, 1u, 2147483647u, 2147483646u, 1073741824u, 1073741823u};
    for (uint32_t d : {1u, 2u, 3u, 7u, 129u, 1023u, 65537u, 2147483647u})
        for (uint32_t n : edge) { bad += check(d, n); ++tried; }
    std::printf("%lld %lld\n", tried, bad);
    return bad != 0;
}
"""


def test_fast_division_matches_integer_division(tmp_path):
    """The multiply-high division of csrc/fast_div.h (the node index of the
    sensor and CFL kernels), compiled here for the host: equal to n / d for
    every divisor up to 4096 at and around its multiples and at random
    numerators below 2^31, and for random divisors up to 2^31."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "div.cpp"
    src.write_text(_DIV_HARNESS)
    exe = tmp_path / "div"
    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "artracfd_b200", "csrc")
    subprocess.run([gxx, "-O2", "-std=c++17", "-I" + csrc, str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    tried, bad = (int(x) for x in r.stdout.split())
    assert tried > 20_000_000 and bad == 0 and r.returncode == 0, (tried, bad)


_TRANSPOSE_HARNESS = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
struct int2 { int x, y; };
struct int4 { int x, y, z, w; };
#include "ghost_tasks.h"
int main(int argc, char **argv)
{
    FILE *f = std::fopen(argv[1], "rb");
    std::vector<int2> pairs;
    int2 p;
    while (std::fread(&p, sizeof p, 1, f) == 1) pairs.push_back(p);
    std::fclose(f);
    const std::vector<int2> xc = transposed_copies_of(pairs, std::atoi(argv[3]), std::atoi(argv[4]),
                                                      std::atoi(argv[5]), std::atoi(argv[6]));
    for (size_t q = 1; q < xc.size(); ++q)
        if (xc[q].x < xc[q - 1].x) return 3;  // destination order
    FILE *o = std::fopen(argv[2], "wb");
    std::fwrite(xc.data(), sizeof(int2), xc.size(), o);
    std::fclose(o);
    return 0;
}
"""


def test_transposed_fill_is_the_fill_of_the_transposed_grid(tmp_path):
    """The copies of a periodic fill remapped to the grid with axes 0 and 1
    exchanged (csrc/ghost_tasks.h, the fill of the transposed state that the
    FP32 forms' X half steps run on), compiled here for the host: exactly the
    periodic fill of the transposed grid, with padded rows on both sides."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "tr.cpp"
    src.write_text(_TRANSPOSE_HARNESS)
    exe = tmp_path / "tr"
    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "artracfd_b200", "csrc")
    subprocess.run([gxx, "-O2", "-std=c++17", "-I" + csrc, str(src), "-o", str(exe)], check=True)
    for (n0, n1, n2) in ((19, 13, 11), (25, 9, 10), (16, 16, 9)):
        pitch, xpitch = (n0 + 7) // 8 * 8, (n1 + 7) // 8 * 8
        pairs = _periodic_fill_pairs((n0, n1, n2), 3, pitch)
        pin, pout = tmp_path / "pairs.bin", tmp_path / "out.bin"
        pairs.astype(np.int32).tofile(pin)
        subprocess.run([str(exe), str(pin), str(pout), str(pitch), str(n0), str(n1), str(xpitch)], check=True)
        got = np.fromfile(pout, dtype=np.int32).reshape(-1, 2)
        want = _periodic_fill_pairs((n1, n0, n2), 3, xpitch)
        want = want[np.argsort(want[:, 0], kind="stable")]
        assert np.array_equal(got, want), (n0, n1, n2)
