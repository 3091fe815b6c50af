"""Benchmark of the fluid time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--mode fp64|fp64_exact|fp32] [--n 128]

Workload: the viscous Taylor-Green vortex at 128^3 cells (129^3 = 2,146,689
computed nodes), WENO5 + central viscous flux, Roe average, LLF splitting,
RK3, CFL 0.5 -- synthetic initial data of the named shape (no data set).
A step is one full time step: the CFL reduction (read back to the host),
the host dt, and EvolveFluidDynamics (6 directional half-step sweeps x 3 RK
stages, each followed by the ghost fill), replayed as one CUDA graph.

Metric: Mcell-steps/s = computed nodes x completed steps / seconds, device
timed with CUDA events on the solver's stream, max over ranks.  The state
(3 levels x 5 variables x 2.5 M nodes, 295 MB of FP64) is larger than L2, so
no flush is needed between steps.  With --gpus N each rank advances its own
replica (the path has no exchange step), so value = N x per-rank rate.

One JSON line is printed by rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s: learned-sensor FP32 vs plain FP64 WENO5 on B200 at L1 err<=1e-3"
UNIT = "Mcell-steps/s"
WORKLOAD = "viscous Taylor-Green vortex 128^3 cells (129^3 nodes), WENO5/LLF/Roe, RK3, CFL 0.5, Re 1600, Ma 0.1"

# algorithmic figures per computed node (3D split WENO5/RK3: 6 sweeps x 3 stages)
BYTES_PER_NODE_STEP = 1920.0          # FP64 state: stage 1 reads 40 B writes 40 B; stages 2,3 read 80 B write 40 B
FLOP_PER_NODE_STAGE_VISCOUS = 1535.0  # ComputeFhat 1380 + ComputeFvhat 115 + LU/SolveOperator 40 (reference C source)
STAGE_BYTES = (80.0, 120.0, 120.0)


def profiled_traffic(mode: str, tiles, axes=(0, 1, 2), transposed=()):
    """DRAM bytes per RK-stage-2 launch of this form's stage kernels, mean over
    the given sweep axes, from the committed ncu record profiles/dram_traffic.json
    (dram__bytes_read.sum + dram__bytes_write.sum of one capture per axis, the
    stage-kernel variant of each axis recorded beside it, and whether the X
    half step ran on the X sweep or as the Y sweep of the transposed state).
    Returns (bytes, source) or (None, reason) when the record does not hold
    this form with these variants."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if not os.path.exists(p):
        return None, "no profiles/dram_traffic.json"
    with open(p) as fh:
        rec = json.load(fh).get(mode)
    if not rec:
        return None, f"no capture of the {mode} form"
    vals = []
    for a in axes:
        caps = rec["axes"].get(str(a), [])
        caps = caps if isinstance(caps, list) else [caps]
        tr = a in transposed
        hit = [c for c in caps if int(tiles[a]) in [int(v) for v in c["variants"]]
               and bool(c.get("transposed", False)) == tr]
        if not hit:
            return None, f"no capture of variant {tiles[a]} on axis {a}" + (" (transposed)" if tr else "")
        vals.append(float(hit[0]["dram_bytes"]))
    return sum(vals) / len(vals), rec["source"]


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled from a thread every 5 ms when it answers (a timed
    region of ~0.1 s still gets tens of samples), else nvidia-smi every
    100 ms.  Read-only: no GPU setting is touched."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                   "hw_thermal_slowdown": 0x40}
    PERIOD_S = 0.005

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []  # NVML: (sm MHz, max sm MHz, reason bits)
        self.stop = threading.Event()
        self.thread = None

    def _start_nvml(self) -> bool:
        try:
            import pynvml
            pynvml.nvmlInit()
        except Exception:
            return False
        try:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            first = (float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)), smax, int(reasons(h)))
        except Exception:
            try:
                pynvml.nvmlShutdown()
            except Exception:
                pass
            return False
        self.nvml = (pynvml, h, reasons, smax)
        self.samples.append(first)
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()
        return True

    def _poll(self):
        pynvml, h, reasons, smax = self.nvml
        while not self.stop.wait(self.PERIOD_S):
            try:
                self.samples.append((float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)), smax,
                                     int(reasons(h))))
            except Exception:
                return

    def __enter__(self):
        if self._start_nvml():
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nvml:
            self.stop.set()
            self.thread.join(timeout=2)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        if self.nvml:
            for mhz, mx, bits in list(self.samples):
                sm.append(mhz)
                smax = mx
                reasons.update(nm for nm, b in self.REASON_BITS.items() if bits & b)
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def fp64_peak_tflops(torch, dtype=None):
    """Measured FP64 (or FP32) reference: cuBLAS DGEMM (SGEMM without TF32)
    8192^3, best of 5."""
    dtype = dtype or torch.float64
    tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, dtype=dtype, device="cuda")
    b = torch.randn(8192, 8192, dtype=dtype, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.backends.cuda.matmul.allow_tf32 = tf32
    return 2.0 * 8192 ** 3 / best / 1e12


def cpu_baseline_reference(n: int, steps: int = 1, procs: int = 1):
    """The unmodified reference (oracle/_ref, compiled from its own sources)
    on the host cores: ``procs`` independent processes, each one TGV case of
    the bench's shape timed for ``steps`` time steps (ComputeTimeStep +
    EvolveFluidDynamics).  Returns (Mcell-steps/s aggregate, details)."""
    from artracfd_b200 import configs
    spec = configs.tgv(n=n)
    work = tempfile.mkdtemp(prefix="acfd_cpu_")
    case = os.path.join(work, "tgv")
    spec.write(case)
    code = (
        "import sys,time,os; sys.path.insert(0,%r)\n"
        "from oracle.oracle import Reference\n"
        "import contextlib, io\n"
        "r=Reference(); d=sys.argv[1]\n"
        "devnull=os.open(os.devnull, os.O_WRONLY); os.dup2(devnull,1)\n"
        "r.load(d)\n"
        "t=[]\n"
        "for k in range(%d):\n"
        "    t0=time.perf_counter(); dt=r.time_step(); r.evolve_fluid(dt); t.append(time.perf_counter()-t0)\n"
        "sys.stderr.write('STEPTIMES '+' '.join('%%.6f'%%x for x in t)+'\\n')\n" % (ROOT, steps))
    ps = []
    for q in range(procs):
        d = os.path.join(work, f"p{q}")
        subprocess.run(["cp", "-r", case, d], check=True)
        ps.append(subprocess.Popen([sys.executable, "-c", code, d], stderr=subprocess.PIPE, stdout=subprocess.DEVNULL,
                                   text=True))
    times = []
    for p in ps:
        _, err = p.communicate()
        for line in err.splitlines():
            if line.startswith("STEPTIMES"):
                times.append([float(x) for x in line.split()[1:]])
    if not times:
        return None, {}
    nodes = (n + 1) ** 3
    per_step = max(sum(t) / len(t) for t in times)
    rate = len(times) * nodes / per_step / 1e6
    subprocess.run(["rm", "-rf", work])
    return rate, {"seconds_per_step": per_step, "procs": len(times), "steps": steps}


FORMS = {"fp64": "FP64", "fp64_exact": "FP64_EXACT", "fp32": "FP32_BULK", "hybrid": "FP64"}
# arithmetic-form codes of the C ABI (ACFD_FP64_EXACT .. ACFD_FP32_HYBRID) -> bench names
FORM_NAMES = {0: "fp64_exact", 1: "fp64", 2: "fp32", 3: "hybrid"}
DTYPES = {"fp64": "f64", "fp64_exact": "f64", "fp32": "f32/f64", "hybrid": "f32/f64"}


def max_over_ranks(torch, dist, x: float, device="cuda") -> float:
    """The largest of the ranks' values of x (x itself on one rank): every
    multi-rank time in the JSON line is the slowest rank's."""
    if not dist:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, nodes_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job Mcell-steps/s of N independent replicas (weak scaling: every
    rank advances its own copy of the workload) timed by the slowest rank."""
    return world * nodes_per_rank * steps / seconds / 1e6


def _tune(s, spec, steps=3):
    """The stage-kernel variants timed on the state after a few steps (the
    sensor flags of the initial field are not those of the timed steps)."""
    for _ in range(steps):
        s.evolve(s.time_step(spec.cfl))
    return s.autotune()


def _solver(part, model, form, stream):
    from artracfd_b200 import abi
    from artracfd_b200.solver import Solver
    s = Solver(part, model, getattr(abi, FORMS[form]))
    s.set_stream(stream.cuda_stream)
    if form == "hybrid":
        from artracfd_b200 import sensor as sensor_mod
        sensor_mod.attach(s)
    return s


def _timed_steps(torch, s, spec, steps, warmup, dist, stream, clock_index, label=None):
    """W untimed steps, then K steps between CUDA events on the solver's
    stream (barrier + synchronize on both sides); seconds (max over ranks),
    kernel launches and the clocks sampled meanwhile."""
    def step():
        s.evolve(s.time_step(spec.cfl), graph=True)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = s.launches()
    # NVTX range of the timed steps (an ncu launch list can be limited to it
    # with --nvtx --nvtx-include "timed_<form>/")
    torch.cuda.nvtx.range_push(label or ("timed_" + FORM_NAMES.get(s.mode, "form")))
    with ClockSampler(clock_index) as clk:
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        e1.synchronize()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    if dist:
        sec = max_over_ranks(torch, dist, sec)
        dist.barrier()
    return sec, s.launches() - launches0, clk.summary()


def _stage_profile(torch, s, spec, nodes_pin, stream, per_axis=None, other=None):
    """One eager step through acfd_profile_step, with CUDA events around each
    piece of the step on the solver's stream: mean stage-kernel and
    ghost-fill times (ms), and the algorithmic bytes per stage launch.
    per_axis (a dict, optional) receives the stage times and algorithmic
    bytes of each sweep axis (the X half steps' stages whether they run on
    the X sweep or transposed on the Y sweep), other (optional) the times of
    the remaining pieces (the sensor's flags, transposes)."""
    from artracfd_b200 import abi
    names = {abi.PIECE_TRANSPOSE: "transpose", abi.PIECE_SENSOR: "sensor_flags"}
    stage_ms, bc_ms, stage_bytes = [], [], []
    for kind, ax, q, ms in s.profile_step(s.time_step(spec.cfl)):
        if kind in (abi.PIECE_STAGE, abi.PIECE_STAGE_XT):
            stage_ms.append(ms)
            stage_bytes.append(STAGE_BYTES[q] * nodes_pin)
            if per_axis is not None:
                d = per_axis.setdefault(ax, {"ms": [], "bytes": [], "transposed": False})
                d["ms"].append(ms)
                d["bytes"].append(stage_bytes[-1])
                d["transposed"] = kind == abi.PIECE_STAGE_XT
        elif kind == abi.PIECE_FILL:
            bc_ms.append(ms)
        elif other is not None:
            other.setdefault(names.get(kind, str(kind)), []).append(ms)
    return sum(stage_ms) / len(stage_ms), sum(bc_ms) / len(bc_ms), sum(stage_bytes) / len(stage_bytes)


def _pin_mask(part):
    import numpy as np
    n = [int(x) for x in part.n]
    ns = np.array(part.ns)[0]
    m = np.zeros((n[2], n[1], n[0]), dtype=bool)
    m[ns[2, 0]:ns[2, 1], ns[1, 0]:ns[1, 1], ns[0, 0]:ns[0, 1]] = True
    return m.ravel()


def _start(part, model, node, form, stream, geo=None):
    """A solver of the given form on the case's initial state: the node
    array uploaded, the bodies (if any) uploaded and mapped onto the nodes
    (ComputeGeometricField), then TreatBoundary on U[TO] -- the steps of
    InitializeComputeDomain (initialization.c:38-55)."""
    from artracfd_b200 import abi
    s = _solver(part, model, form, stream)
    s.upload(node)
    if geo:
        s.geo_upload(geo)
        s.compute_geometric_field()
    s.treat_boundary(abi.TO)
    return s


def _accuracy(part, model, node, spec, form, steps, stream, geo=None):
    """The form against the plain FP64 path on the same initial state and
    the same dt sequence: relative L1 and Linf errors of density, pressure
    and momentum over the computed fluid nodes after `steps` steps."""
    import numpy as np
    ref = _start(part, model, node, "fp64", stream, geo)
    dts = []
    for _ in range(steps):
        dt = ref.time_step(spec.cfl)
        ref.evolve(dt, graph=True)
        dts.append(dt)
    got = ref.download()
    a = got["U"][:, 0, :].copy()
    fluid = got["did"] == 0
    ref.close()
    s = _start(part, model, node, form, stream, geo)
    for dt in dts:
        s.evolve(dt, graph=True)
    b = s.download()["U"][:, 0, :].copy()
    s.close()
    pin = _pin_mask(part) & fluid
    a, b = a[pin], b[pin]
    gm1 = model.gamma - 1.0

    def pres(u):
        return gm1 * (u[:, 4] - 0.5 * (u[:, 1] ** 2 + u[:, 2] ** 2 + u[:, 3] ** 2) / u[:, 0])

    out = {"steps": steps, "against": "plain FP64 path (fast form), same initial state and dt sequence"}
    for name, fa, fb in (("rho", a[:, 0], b[:, 0]), ("p", pres(a), pres(b)), ("mom", a[:, 1:4], b[:, 1:4])):
        d = np.abs(fb - fa)
        out["l1_" + name] = float(d.sum() / np.abs(fa).sum()) if np.isfinite(d).all() else float("inf")
        out["linf_" + name] = float(d.max() / np.abs(fa).max()) if np.isfinite(d).all() else float("inf")
    return out


def _form_block(torch, part, model, node, spec, form, nodes_pin, args, dist, stream, local_rank, geo=None,
                hbm_peak=None, profile=True, label=None):
    """One arithmetic form on one case: autotuned variants, W warm-up and K
    device-timed steps (CFL read back + host dt + graph replay each step),
    and optionally one profiled eager step (mean stage and ghost-fill
    times)."""
    s = _start(part, model, node, form, stream, geo)
    tiles = _tune(s, spec)
    sec, launches, clk = _timed_steps(torch, s, spec, args.steps, args.warmup, dist, stream, local_rank, label)
    out = {"value": job_rate(int(os.environ.get("WORLD_SIZE", "1")), nodes_pin, args.steps, sec),
           "ms_per_step": sec / args.steps * 1e3, "tiles": tiles, "clocks": clk, "gpu_launches": launches}
    if form == "hybrid":
        out["flagged_fraction"] = s.sensor_update() / (3.0 * nodes_pin)
    if profile:
        per_axis, other = {}, {}
        st, bc, by = _stage_profile(torch, s, spec, nodes_pin, stream, per_axis, other)
        out["stage_ms"] = {"sweep_mean": st, "ghost_fill_mean": bc,
                           "per_axis": {str(ax): sum(d["ms"]) / len(d["ms"]) for ax, d in sorted(per_axis.items())},
                           "x_transposed": any(d["transposed"] for d in per_axis.values()),
                           "other_per_step": {k: sum(v) for k, v in sorted(other.items())}}
        if hbm_peak:
            out["hbm_frac"] = by / (st / 1e3) / 1e9 / hbm_peak
        out["_stage_mean_ms"] = st
    s.close()
    return out


def shock_cylinder_block(torch, args, dist, stream, local_rank):
    """The learned sensor's own configuration: a Ma 2.81 planar shock over an
    extruded cylinder, [0,16]x[0,8]x[0,0.0625] at 1024x512x4 cells (1023 x
    511 x 5 = 2,613,765 computed nodes), inviscid, WENO5/LLF/Roe, RK3, CFL
    0.5.  The cylinder is the reference's own preprocessed surface
    (tests/golden/bodies_shock_cylinder.npz, made by make_bodies.py); the
    initial field follows the case file.  Hybrid and plain FP64 rates, and
    the hybrid's L1/Linf errors against the plain FP64 path after 100 steps
    on the same dt sequence."""
    import numpy as np
    from artracfd_b200 import configs
    from artracfd_b200.case import load_polyhedra

    path = os.path.join(ROOT, "tests", "golden", "bodies_shock_cylinder.npz")
    if not os.path.exists(path):
        return {"unavailable": "tests/golden/bodies_shock_cylinder.npz missing"}
    spec = configs.shock_cylinder()
    part, model = spec.descriptors()
    z = np.load(path)
    geo, keep = load_polyhedra(z)
    node = spec.initial_nodes(part, model)
    pin = int(np.prod(np.array(part.ns)[0, :, 1] - np.array(part.ns)[0, :, 0]))
    f64 = _form_block(torch, part, model, node, spec, "fp64", pin, args, dist, stream, local_rank, geo,
                      label="timed_sc_fp64")
    hyb = _form_block(torch, part, model, node, spec, "hybrid", pin, args, dist, stream, local_rank, geo,
                      label="timed_sc_hybrid")
    for blk in (f64, hyb):
        blk.pop("_stage_mean_ms", None)
    acc = None
    if args.sc_accuracy_steps > 0:
        acc = _accuracy(part, model, node, spec, "hybrid", args.sc_accuracy_steps, stream, geo)
    del keep
    return {"workload": "Ma 2.81 shock over an extruded cylinder (256 facets), 1024x512x4 cells "
                        "(2,613,765 computed nodes), inviscid WENO5/LLF/Roe, RK3, CFL 0.5",
            "nodes": pin, "hybrid": hyb, "plain_fp64": f64,
            "speedup_vs_plain_fp64": hyb["value"] / f64["value"], "accuracy": acc}


def run_ours(args, rank, world, local_rank):
    import torch

    from artracfd_b200 import abi, configs

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    spec = configs.tgv(n=args.n)
    part, model = spec.descriptors()
    nodes_pin = (args.n + 1) ** 3
    node = spec.initial_nodes(part, model)
    stream = torch.cuda.Stream()
    hbm_peak, peak_kind = load_peaks()

    # the plain FP64 path, timed first (the comparison of the headline)
    plain = None
    if args.mode != "fp64":
        plain = _form_block(torch, part, model, node, spec, "fp64", nodes_pin, args, dist, stream, local_rank,
                            hbm_peak=hbm_peak)
    # the FP32-bulk form without the sensor: what the sensor itself adds
    fp32 = None
    if args.mode == "hybrid":
        fp32 = _form_block(torch, part, model, node, spec, "fp32", nodes_pin, args, dist, stream, local_rank,
                           hbm_peak=hbm_peak)

    # the form named by --mode (default: the learned-sensor hybrid)
    s = _solver(part, model, args.mode, stream)
    s.upload(node)
    s.treat_boundary(abi.TO)
    tiles = _tune(s, spec)
    sensor_info = None
    if args.mode == "hybrid":
        flagged = s.sensor_update()
        sensor_info = {"flagged_fraction_at_start": flagged / (3.0 * nodes_pin)}
    sec, gpu_launches, clocks = _timed_steps(torch, s, spec, args.steps, args.warmup, dist, stream, local_rank)
    value = job_rate(world, nodes_pin, args.steps, sec)
    if args.mode == "hybrid":
        sensor_info["flagged_fraction_after_timed_steps"] = s.sensor_update() / (3.0 * nodes_pin)
    per_axis, other = {}, {}
    stage_mean, bc_mean, bytes_per_stage = _stage_profile(torch, s, spec, nodes_pin, stream, per_axis, other)
    # the dominant kernel: the stage-kernel family (tile variant class) with
    # the largest share of the stage time; its algorithmic bytes over its
    # mean launch duration
    fam_of = lambda v: "brick" if v < abi.BRICK_VARIANTS else ("plane" if v >= abi.PLANE_VARIANT else "line-march")
    fams = {}
    for ax, d in per_axis.items():
        f = fams.setdefault(fam_of(tiles[ax]), {"ms": [], "bytes": [], "axes": []})
        f["ms"] += d["ms"]
        f["bytes"] += d["bytes"]
        f["axes"].append(ax)
    dom_name, dom = max(fams.items(), key=lambda kv: sum(kv[1]["ms"]))
    dom_ms = sum(dom["ms"]) / len(dom["ms"])
    dom_bytes = sum(dom["bytes"]) / len(dom["bytes"])
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    dom_share = sum(dom["ms"]) / sum(sum(d["ms"]) for d in fams.values())
    # ncu traffic of RK stage 2 (120 B algorithmic per node), scaled to the
    # mean RK-stage mix of one step (106.7 B per node)
    tr2, tr_src = profiled_traffic(args.mode, tiles, tuple(sorted(dom["axes"])),
                                   tuple(ax for ax, d in per_axis.items() if d["transposed"]))
    traffic = tr2 * (dom_bytes / (STAGE_BYTES[1] * nodes_pin)) if tr2 else None
    flop_rate = FLOP_PER_NODE_STAGE_VISCOUS * nodes_pin / (stage_mean / 1e3) / 1e12
    fp64_peak = fp64_peak_tflops(torch) if rank == 0 else None
    fp32_peak = fp64_peak_tflops(torch, torch.float32) if rank == 0 and args.mode in ("fp32", "hybrid") else None
    # the FP64 pipe fraction belongs to the plain FP64 path's own stage time
    st64 = plain["_stage_mean_ms"] if plain else stage_mean
    flop_rate64 = FLOP_PER_NODE_STAGE_VISCOUS * nodes_pin / (st64 / 1e3) / 1e12
    # e2e through the C ABI with host buffers: upload of the host node array,
    # K steps (CFL read back each step), download of the result
    host = node.copy()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.upload(host)
    s.treat_boundary(abi.TO)
    for _ in range(args.steps):
        s.evolve(s.time_step(spec.cfl), graph=True)
    s.download(host)
    e2e_sec = time.perf_counter() - t0
    e2e_sec = max_over_ranks(torch, dist, e2e_sec)
    node_bytes = host.nbytes
    # the strictest drop-in use: the whole node array crosses PCIe both ways
    # every step (a host that touches its nodes between steps)
    rt_steps = max(1, min(args.steps, 5))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(rt_steps):
        s.upload(host)
        s.evolve(s.time_step(spec.cfl), graph=True)
        s.download(host)
    rt_sec = max_over_ranks(torch, dist, time.perf_counter() - t0)
    s.close()
    accuracy = None
    if args.mode in ("fp32", "hybrid") and args.accuracy_steps > 0:
        accuracy = _accuracy(part, model, node, spec, args.mode, args.accuracy_steps, stream)
    # the blocks of the other configurations are single-GPU figures: at N > 1
    # every rank times the headline replica only
    extra = args.mode == "hybrid" and world == 1
    shock_cyl = None
    if extra and not args.no_shock_cylinder:
        try:
            shock_cyl = shock_cylinder_block(torch, args, dist, stream, local_rank)
        except Exception as exc:  # the headline line is printed regardless
            shock_cyl = {"error": f"{type(exc).__name__}: {exc}"}
    ib = None
    if extra and args.ib_steps > 0:
        try:
            ib = ib_dropin_block(args)
        except Exception as exc:
            ib = {"error": f"{type(exc).__name__}: {exc}"}
    batch = None
    if extra and args.batch_steps > 0:
        try:
            batch = batch_block(args, args.batch_steps, local_rank)
        except Exception as exc:
            batch = {"error": f"{type(exc).__name__}: {exc}"}
    for blk in (plain, fp32):
        if blk:
            blk.pop("_stage_mean_ms", None)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        rate, det = cpu_baseline_reference(args.n, steps=1, procs=1)
        if rate is not None:
            cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"1 time step of the same TGV {args.n}^3 case by the unmodified reference "
                             f"(oracle/_ref, gcc -O2 -std=c99), 1 process on 1 core: "
                             f"{det['seconds_per_step']:.2f} s/step"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPES[args.mode],
        "data": "synthetic (analytic TGV initial field)",
        "config": {"workload": WORKLOAD, "form": args.mode, "nodes_per_gpu": nodes_pin,
                   "l2": "state 295 MB > 126 MB L2, no flush", "parallelism": f"replicas x{world}"},
        "plain_fp64": plain,
        "speedup_vs_plain_fp64": (value / plain["value"]) if plain else None,
        "fp32_bulk": fp32,
        "speedup_vs_fp32_bulk": (value / fp32["value"]) if fp32 else None,
        "accuracy": accuracy,
        "shock_cylinder": shock_cyl,
        "batch": batch,
        "ib_spheres_dropin": ib,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic,
                     "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum of an RK-stage-2 launch "
                                     f"of this kernel ({tr_src}), scaled to the mean "
                                     f"RK-stage mix; algorithmic bytes per launch = {dom_bytes:.4g}",
                     "kernel": f"{dom_name} stage kernel of sweep axes {sorted(dom['axes'])} "
                               f"({dom_share * 100:.0f}% of the stage time), mean over its launches in one step",
                     "all_stage_kernels": {"achieved": bytes_per_stage / (stage_mean / 1e3) / 1e9,
                                           "frac": bytes_per_stage / (stage_mean / 1e3) / 1e9 / hbm_peak},
                     "per_axis_ms": {str(ax): sum(d["ms"]) / len(d["ms"]) for ax, d in sorted(per_axis.items())},
                     "peak_kind": peak_kind,
                     "fp64": {"achieved_tflops": flop_rate64, "peak_tflops": fp64_peak,
                              "frac": (flop_rate64 / fp64_peak) if fp64_peak else None,
                              "peak_kind": "measured cuBLAS DGEMM 8192^3 in this run",
                              "flop_per_node_stage": FLOP_PER_NODE_STAGE_VISCOUS,
                              "stage_ms": st64,
                              "note": "the plain FP64 path's mean stage time against the reference's FP64 flop "
                                      "count of a stage (1,535 flop per node)"},
                     "fp32": ({"achieved_tflops": flop_rate, "peak_tflops": fp32_peak,
                               "frac": (flop_rate / fp32_peak) if fp32_peak else None,
                               "peak_kind": "measured cuBLAS SGEMM 8192^3 (no TF32) in this run",
                               "note": "the reference's flop count of the same stages over the FP32 form's stage time "
                                       "(reference-equivalent work: the hybrid computes fewer flops on smooth "
                                       "interfaces)"} if fp32_peak else None)},
        "stage_ms": {"sweep_mean": stage_mean, "ghost_fill_mean": bc_mean,
                     "x_transposed": any(d["transposed"] for d in per_axis.values()),
                     "other_per_step": {k: sum(v) for k, v in sorted(other.items())}},
        "clocks": clocks,
        "e2e": {"value": job_rate(world, nodes_pin, args.steps, e2e_sec), "unit": UNIT,
                "h2d_bytes_per_step": (node_bytes + 8 * args.steps) / args.steps,
                "d2h_bytes_per_step": (node_bytes + 24 * args.steps) / args.steps,
                "what": "C-ABI loop with host node arrays: acfd_sync_to_device, K x (acfd_cfl + host dt + "
                        "acfd_evolve_fluid_graph), acfd_sync_to_host; wall clock",
                "node_array_every_step": {"value": job_rate(world, nodes_pin, rt_steps, rt_sec), "steps": rt_steps,
                                          "h2d_bytes_per_step": node_bytes, "d2h_bytes_per_step": node_bytes,
                                          "what": "each step uploads and downloads the whole node array "
                                                  "(acfd_sync_to_device, acfd_cfl, acfd_evolve_fluid_graph, "
                                                  "acfd_sync_to_host); wall clock"}},
        "gpu_launches": gpu_launches,
        "tiles": tiles,
        "sensor": sensor_info,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def ib_dropin_block(args):
    """The immersed-boundary configuration through the drop-in program (the
    reference's own host code -- case loading, rigid-body kinematics --
    linked with libacfd_gpu): crossflow over eight moving 1280-facet spheres
    in [0,4]^3 at 192^3 cells (191 x 193 x 193 = 7,114,559 computed nodes),
    plain FP64 path, the rigid-body step's node scans, collisions and surface
    motion on the device.  Rate from the program's own per-step timer
    (host wall clock of a whole step, solid half steps included; the first
    step, which captures the step graph, is left out)."""
    import re
    import shutil
    from artracfd_b200 import configs
    exe = os.path.join(ROOT, "artracfd_b200", "shim", "_build", "artracfd_gpu")
    if not os.path.exists(exe):
        return {"unavailable": "drop-in program not built (it needs the reference sources)"}
    steps = max(2, args.ib_steps)
    spec = configs.ib_spheres(n=192)
    spec.stepN = steps
    work = tempfile.mkdtemp(prefix="acfd_ib_")
    case = os.path.join(work, "ib192")
    spec.write(case)
    env = dict(os.environ, ACFD_MODE="fp64")
    t0 = time.perf_counter()
    r = subprocess.run([exe, "-m", "gpu"], cwd=case, env=env, capture_output=True, text=True, timeout=900)
    wall = time.perf_counter() - t0
    shutil.rmtree(work, ignore_errors=True)
    if r.returncode != 0:
        return {"error": f"drop-in program exited {r.returncode}: {r.stdout[-300:]} {r.stderr[-300:]}"}
    el = [float(x) for x in re.findall(r"elapsed: ([0-9.eE+-]+)s", r.stdout)]
    if len(el) < 2:
        return {"error": "no step timer lines in the drop-in program's output"}
    per_step = sum(el[1:]) / len(el[1:])
    pin = 191 * 193 * 193
    return {"workload": "8 moving 1280-facet spheres in a Ma 0.3, Re 200 crossflow, 192^3 cells (7,114,559 "
                        "computed nodes), WENO5/RK3, drop-in program, plain FP64 path, solid step on the device",
            "value": pin / per_step / 1e6, "unit": UNIT, "ms_per_step": per_step * 1e3, "steps_timed": len(el) - 1,
            "wall_s": wall, "timer": "the program's own per-step host timer (solve.c:89 restated), first step "
                                     "(graph capture) left out"}


def batch_block(args, steps, local_rank):
    """The batched sweep: 48 independent viscous TGV and 3D Riemann cases
    (configs.batch_cases, seed 42) advanced together by the batch API in the
    learned-sensor FP32 form -- every RK stage of a step of every case in one
    persistent launch (ACFD_BATCH_PERSISTENT), and for comparison one
    plane-march launch per RK stage (ACFD_BATCH_PLANE) -- against the same
    cases run one at a time by the single-case API on the plain FP64 path.
    All are device-timed with CUDA events (the one-at-a-time runs include
    their per-step host dt, as a user running cases one by one does); the
    batch's dt stays on the device.  `steps` timed steps of each."""
    import numpy as np
    import torch
    from concurrent.futures import ThreadPoolExecutor

    from artracfd_b200 import abi, configs, sensor
    from artracfd_b200.batch import Batch
    from artracfd_b200.solver import Solver

    torch.cuda.set_device(local_rank)
    specs = configs.batch_cases(count=args.batch_cases, seed=42)
    descs = [s.descriptors() for s in specs]
    pin = [int(np.prod(np.array(p.ns)[0, :, 1] - np.array(p.ns)[0, :, 0])) for p, _ in descs]
    stream = torch.cuda.Stream()
    b = Batch(descs)
    b.set_stream(stream.cuda_stream)
    rho64 = []
    sec64 = 0.0
    pool = ThreadPoolExecutor(1)
    fut = pool.submit(specs[0].initial_nodes, *descs[0])
    for c, spec in enumerate(specs):
        node = fut.result()
        if c + 1 < len(specs):
            fut = pool.submit(specs[c + 1].initial_nodes, *descs[c + 1])
        b.upload(c, node)
        b.treat_boundary(c)
        with Solver(*descs[c], abi.FP64) as s:
            s.set_stream(stream.cuda_stream)
            s.upload(node)
            s.treat_boundary(abi.TO)
            s.evolve(s.time_step(spec.cfl), graph=True)  # graph capture outside the timed steps
            s.upload(node)
            s.treat_boundary(abi.TO)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                s.evolve(s.time_step(spec.cfl), graph=True)
            e1.record(stream)
            e1.synchronize()
            sec64 += e0.elapsed_time(e1) / 1e3
            rho64.append(s.download()["U"][:, 0, 0].copy())
        del node
    pool.shutdown()
    params, thr, _ = sensor.load(sensor.WEIGHTS)
    b.sensor_load(params, thr)
    b.set_precision(abi.FP32_HYBRID)
    cfl = [s.cfl for s in specs]
    total = sum(pin)
    # the default (one plane-march launch per RK stage) first: its rate is
    # the block's value; then the persistent step
    kernels = {"per_stage_plane": abi.BATCH_PLANE}
    try:
        b.set_kernel(abi.BATCH_PERSISTENT)
        kernels["persistent"] = abi.BATCH_PERSISTENT
    except abi.AcfdError:
        pass
    timed = {}
    errs = None
    for name, kern in kernels.items():
        b.set_kernel(kern)
        # the first advance captures the step graph (after the first kernel's
        # timed steps the cases continue from where they are: the rate of a
        # step does not depend on the state's time)
        b.advance(cfl, 1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = b.launches()
        nt = max(1, steps - 1)
        e0.record(stream)
        b.advance(cfl, nt)
        e1.record(stream)
        e1.synchronize()
        secb = e0.elapsed_time(e1) / 1e3
        timed[name] = {"value": total * nt / secb / 1e6, "ms_per_step": secb / nt * 1e3, "timed_steps": nt,
                       "gpu_launches_per_step": (b.launches() - l0) / nt}
        if errs is None:
            # first kernel: 1 + nt = steps steps from the start, as the FP64 runs
            errs = []
            for c in range(len(specs)):
                r = b.download(c)["U"][:, 0, 0]
                m = np.array(descs[c][0].ns)[0]
                n = list(descs[c][0].n)
                mask = np.zeros((n[2], n[1], n[0]), dtype=bool)
                mask[m[2, 0]:m[2, 1], m[1, 0]:m[1, 1], m[0, 0]:m[0, 1]] = True
                mask = mask.ravel()
                errs.append(float(np.abs(r[mask] - rho64[c][mask]).sum() / np.abs(rho64[c][mask]).sum()))
    b.close()
    head = next(iter(timed))
    v64 = total * steps / sec64 / 1e6
    return {
        "workload": f"{len(specs)} independent viscous TGV / 3D Riemann cases, n^3 with n in "
                    "{64..160 step 16}, Ma U[0.1,0.5], Re U[400,3200], seed 42; WENO5/RK3",
        "cases": len(specs), "pin_nodes": total,
        "kinds": {k: sum(1 for s in specs if s.kind == k) for k in ("tgv", "riemann")},
        "form": "hybrid (learned sensor, FP32 bulk)", "kernel": head,
        "value": timed[head]["value"], "ms_per_step": timed[head]["ms_per_step"], "steps": steps,
        "kernels": timed,
        "one_at_a_time_fp64": {"value": v64, "ms_per_step_all_cases": sec64 / steps * 1e3,
                               "what": "each case alone through the single-case API, plain FP64 path, host dt "
                                       "per step, CUDA graph per step"},
        "speedup_vs_one_at_a_time_fp64": timed[head]["value"] / v64,
        "accuracy": {"l1_rho_max_over_cases": max(errs), "l1_rho_mean": sum(errs) / len(errs),
                     "against": "each case on the plain FP64 path after the same number of steps (its own dt "
                                "sequence)"},
    }


def run_batch(args, rank, world, local_rank):
    """--workload batch: the batched sweep as its own JSON line."""
    blk = batch_block(args, args.steps, local_rank)
    line = {
        "metric": METRIC, "workload": "batch", "value": blk["value"], "unit": UNIT,
        "n_gpus": 1, "steps": args.steps, "higher_is_better": True, "dtype": "f32/f64",
        "data": "synthetic (seeded TGV and 3D Riemann initial fields)",
        "config": {k: blk[k] for k in ("workload", "cases", "pin_nodes", "kinds", "form", "kernel")},
        "ms_per_step": blk["ms_per_step"],
        "kernels": blk["kernels"],
        "one_at_a_time_fp64": blk["one_at_a_time_fp64"],
        "speedup_vs_one_at_a_time_fp64": blk["speedup_vs_one_at_a_time_fp64"],
        "accuracy": blk["accuracy"],
    }
    print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    # every host thread this process may use (one reference process each; the
    # reference is serial), at most one process per GB of available memory
    # (a TGV 128^3 reference process holds ~0.5 GB); --ref-procs caps it
    procs = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        import psutil
        procs = min(procs, max(1, int(psutil.virtual_memory().available // (1 << 30))))
    except Exception:
        pass
    if args.ref_procs > 0:
        procs = min(procs, args.ref_procs)
    procs = max(1, procs)
    t0 = time.perf_counter()
    rates = []
    # a bounded sample: two reference time steps per process whatever --steps
    # (one step of TGV 128^3 takes ~15 s on one core)
    rate, det = cpu_baseline_reference(args.n, steps=max(1, min(args.steps, 2)), procs=procs)
    if rate is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference harness oracle/_ref not built"}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
        # the steps each process ran (a bounded sample; --steps/--warmup asked for more)
        "steps": det["steps"], "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": det["seconds_per_step"] * 1e3,
        "ms_per_step_note": "seconds per time step of one process while all processes run (slowest process)",
        "per_core_value": rate / det["procs"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic TGV initial field)",
        "config": {"workload": WORKLOAD, "form": "reference CPU (serial C99)", "procs": det["procs"]},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": det["procs"], "kind": "reference",
                         "sample": f"{det['procs']} independent processes of the unmodified reference, "
                                   f"{det['steps']} time step(s) each of TGV {args.n}^3"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.perf_counter() - t0,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="hybrid", choices=["fp64", "fp64_exact", "fp32", "hybrid"])
    ap.add_argument("--accuracy-steps", type=int, default=200)
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-shock-cylinder", action="store_true", help="leave out the shock-cylinder block")
    ap.add_argument("--sc-accuracy-steps", type=int, default=100,
                    help="steps of the shock-cylinder accuracy comparison (0: none)")
    ap.add_argument("--ref-procs", type=int, default=0, help="reference processes (0: every usable host thread)")
    ap.add_argument("--workload", default="tgv", choices=["tgv", "batch"],
                    help="tgv: the headline line (TGV 128^3); batch: the 48-case batched sweep")
    ap.add_argument("--batch-cases", type=int, default=48)
    ap.add_argument("--ib-steps", type=int, default=6,
                    help="steps of the 192^3 moving-spheres drop-in block (0: leave it out)")
    ap.add_argument("--batch-steps", type=int, default=10,
                    help="timed steps of the batch block of the default line (0: leave it out)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "batch":
        run_batch(args, rank, world, local_rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
