"""Learned smoothness sensor: data, training and the weights file.

The network (10 -> 32 -> 32 -> 1, ReLU, ReLU, sigmoid) is trained on the GPU by
this library's own kernels (acfd_mlp_grad: forward and backward of the batch;
acfd_mlp_adam: the update).  PyTorch only holds device arrays.

Data: seeded 1D and 3D Riemann problems (rho in [0.1, 10], p in [0.1, 100],
|u| < 2) and Taylor-Green vortex states, advanced by the plain FP64 path; at
recorded steps acfd_sensor_features returns, for every node and sweep axis,
the 10 stencil features and how much the departure of the WENO5 nonlinear
weights from the linear weights changes the reconstruction at the node's two
interfaces (|sum_k (omega_k - C_k) q_k| relative to the stencil values).  A
node is labelled non-smooth when that change exceeds ``tau``.

    python -m artracfd_b200.sensor train [--tau 1e-3] [--out artracfd_b200/sensor_weights.npz]
    python -m artracfd_b200.sensor calibrate [--uniform-margin 0.25]   # threshold floor only
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np

from . import abi, configs
from .case import Boundary, CaseSpec, Region
from .solver import Solver

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "sensor_weights.npz")
N_IN, N_H = 10, 32


def param_count(lib=None) -> int:
    lib = lib or abi.load_library()
    return lib.acfd_mlp_param_count()


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised parameters in the library's layout."""
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0, math.sqrt(2.0 / N_IN), size=(N_H, N_IN))
    b1 = np.zeros(N_H)
    W2 = rng.normal(0, math.sqrt(2.0 / N_H), size=(N_H, N_H))
    b2 = np.zeros(N_H)
    w3 = rng.normal(0, math.sqrt(1.0 / N_H), size=N_H)
    b3 = np.zeros(1)
    return np.concatenate([W1.ravel(), b1, W2.ravel(), b2, w3, b3]).astype(np.float32)


# ----------------------------------------------------------------------
# seeded states
# ----------------------------------------------------------------------
def _prim_exprs(rho, u, p, v=0.0, w=0.0):
    return tuple("%.17g" % x for x in (rho, u, v, w, p))


def riemann_1d(seed: int, n: int = 48) -> CaseSpec:
    """Two random states separated by a plane of random orientation."""
    rng = np.random.default_rng(seed)
    s = [dict(rho=rng.uniform(0.1, 10), p=rng.uniform(0.1, 100), u=rng.uniform(-2, 2) / math.sqrt(3),
              v=rng.uniform(-2, 2) / math.sqrt(3), w=rng.uniform(-2, 2) / math.sqrt(3)) for _ in range(2)]
    nrm = rng.normal(size=3)
    nrm /= np.linalg.norm(nrm)
    O = Boundary(abi.OUTFLOW)
    return CaseSpec(domain_lo=(0, 0, 0), domain_hi=(1, 1, 1), m=(n, n, n), cfl=0.5, refMu=0.0,
                    init=_prim_exprs(s[0]["rho"], s[0]["u"], s[0]["p"], s[0]["v"], s[0]["w"]),
                    boundaries=[O] * 6,
                    regions=[Region("plane", p1=(0.5, 0.5, 0.5), p2=tuple(nrm),
                                    exprs=_prim_exprs(s[1]["rho"], s[1]["u"], s[1]["p"], s[1]["v"], s[1]["w"]))])


def riemann_3d(seed: int, n: int = 48) -> CaseSpec:
    """Eight random states in the octants of the unit cube."""
    rng = np.random.default_rng(1000 + seed)
    O = Boundary(abi.OUTFLOW)
    regions = []
    first = None
    for a in range(2):
        for b in range(2):
            for c in range(2):
                st = _prim_exprs(rng.uniform(0.1, 10), rng.uniform(-2, 2) / math.sqrt(3), rng.uniform(0.1, 100),
                                 rng.uniform(-2, 2) / math.sqrt(3), rng.uniform(-2, 2) / math.sqrt(3))
                if first is None:
                    first = st
                    continue
                regions.append(Region("box", p1=(0.5 * a, 0.5 * b, 0.5 * c),
                                      p2=(0.5 * a + 0.5, 0.5 * b + 0.5, 0.5 * c + 0.5), exprs=st))
    return CaseSpec(domain_lo=(0, 0, 0), domain_hi=(1, 1, 1), m=(n, n, n), cfl=0.5, refMu=0.0, init=first,
                    boundaries=[O] * 6, regions=regions)


def _pin_count(part) -> int:
    ns = np.array(part.ns)
    return int(np.prod(ns[0, :, 1] - ns[0, :, 0]))


def collect(specs, steps=24, every=8, mode=abi.FP64, verbose=False):
    """Run each case with the plain path and record (features, departure)
    for every fluid node and sweep axis at steps 0, every, 2*every, ..."""
    import torch

    feats, deps = [], []
    for spec in specs:
        part, model = spec.descriptors()
        node = spec.initial_nodes(part, model)
        n = _pin_count(part)
        with Solver(part, model, mode) as s:
            s.upload(node)
            s.treat_boundary(abi.TO)
            for k in range(steps + 1):
                if k % every == 0:
                    for d in range(3):
                        f = torch.empty((n, N_IN), dtype=torch.float32, device="cuda")
                        p = torch.empty(n, dtype=torch.float32, device="cuda")
                        abi.check(s.lib.acfd_sensor_features(s.h, d, ctypes.c_void_p(f.data_ptr()),
                                                             ctypes.c_void_p(p.data_ptr())), s.lib)
                        # fluid nodes with finite data only (a strong random
                        # Riemann problem can drive the unlimited scheme to a
                        # negative pressure; such states are not training data)
                        keep = (p >= 0) & torch.isfinite(p) & torch.isfinite(f).all(dim=1)
                        feats.append(f[keep])
                        deps.append(p[keep])
                if k < steps:
                    s.evolve(s.time_step(spec.cfl))
        if verbose:
            print(f"  collected {spec.m} case", flush=True)
    return torch.cat(feats), torch.cat(deps)


def default_specs(seeds=range(12), n=48):
    specs = []
    for q in seeds:
        specs.append(riemann_1d(q, n))
        specs.append(riemann_3d(q, n))
    # vortex states: the Taylor-Green flow over the Re and Ma range of the
    # batched workload, at two resolutions
    for Re, Ma in ((1600.0, 0.1), (400.0, 0.3), (3200.0, 0.5), (800.0, 0.2)):
        specs.append(configs.tgv(n=n, Re=Re, Ma=Ma))
        specs.append(configs.tgv(n=2 * n, Re=Re, Ma=Ma))
    return specs


# ----------------------------------------------------------------------
# training with the library's kernels
# ----------------------------------------------------------------------
def train(X, y, epochs=6, batch=16384, lr=3e-3, pos_weight=None, seed=0, verbose=False):
    """Adam on the weighted binary cross-entropy; returns (params, history)."""
    import torch

    lib = abi.load_library()
    npar = lib.acfd_mlp_param_count()
    g = torch.Generator(device="cuda").manual_seed(seed)
    params = torch.tensor(init_params(seed), device="cuda")
    grad = torch.zeros(npar, dtype=torch.float32, device="cuda")
    m = torch.zeros_like(grad)
    v = torch.zeros_like(grad)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    n = X.shape[0]
    if pos_weight is None:
        pos = float(y.sum().item())
        pos_weight = max(1.0, (n - pos) / max(pos, 1.0))
    step = 0
    hist = []
    vp = ctypes.c_void_p
    stream = torch.cuda.current_stream().cuda_stream
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        rate = lr * (0.5 * (1 + math.cos(math.pi * ep / epochs)) * 0.9 + 0.1)
        loss.zero_()
        for b0 in range(0, n, batch):
            idx = perm[b0:b0 + batch]
            xb = X[idx].contiguous()
            yb = y[idx].contiguous()
            grad.zero_()
            nb = xb.shape[0]
            abi.check(lib.acfd_mlp_grad(vp(params.data_ptr()), vp(xb.data_ptr()), vp(yb.data_ptr()), nb,
                                        float(pos_weight), vp(grad.data_ptr()), vp(loss.data_ptr()), vp(stream)),
                      lib)
            step += 1
            abi.check(lib.acfd_mlp_adam(vp(params.data_ptr()), vp(grad.data_ptr()), vp(m.data_ptr()),
                                        vp(v.data_ptr()), step, float(rate), float(1.0 / nb), vp(stream)), lib)
        hist.append(float(loss.item()) / n)
        if verbose:
            print(f"  epoch {ep}: loss {hist[-1]:.5f}", flush=True)
    return params.cpu().numpy(), hist, float(pos_weight)


def predict(params, X):
    import torch

    lib = abi.load_library()
    p = torch.tensor(params, device="cuda")
    out = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
    vp = ctypes.c_void_p
    abi.check(lib.acfd_mlp_forward(vp(p.data_ptr()), vp(X.contiguous().data_ptr()), X.shape[0],
                                   vp(out.data_ptr()), None), lib)
    return out


WEIGHTS_BIN = os.path.join(HERE, "sensor_weights.bin")


def save(path, params, threshold, meta):
    np.savez(path, params=np.asarray(params, dtype=np.float32), threshold=np.float32(threshold),
             meta=json.dumps(meta))
    save_bin(os.path.splitext(path)[0] + ".bin", params, threshold)


def save_bin(path, params, threshold):
    """The weights in the file format of acfd_sensor_load_file: "ACFDSNS1",
    int32 parameter count, float32 threshold, float32 parameters."""
    p = np.asarray(params, dtype="<f4")
    with open(path, "wb") as fh:
        fh.write(b"ACFDSNS1")
        fh.write(np.int32(p.size).astype("<i4").tobytes())
        fh.write(np.float32(threshold).astype("<f4").tobytes())
        fh.write(p.tobytes())


def load(path=WEIGHTS):
    z = np.load(path)
    return z["params"].astype(np.float32), float(z["threshold"]), json.loads(str(z["meta"]))


def attach(solver: Solver, path=WEIGHTS, threshold=None):
    """Load the sensor into a solver and switch it to the hybrid form."""
    params, thr, _ = load(path)
    solver.sensor_load(params, threshold if threshold is not None else thr)
    solver.set_precision(abi.FP32_HYBRID)


def forward_cpu(params, X):
    """The network on the CPU in float64 (for calibration; the GPU kernels
    evaluate it in FP32 / FP16 tensor-core arithmetic)."""
    p = np.asarray(params, dtype=np.float64)
    o = 0
    W1 = p[o:o + N_H * N_IN].reshape(N_H, N_IN); o += N_H * N_IN
    b1 = p[o:o + N_H]; o += N_H
    W2 = p[o:o + N_H * N_H].reshape(N_H, N_H); o += N_H * N_H
    b2 = p[o:o + N_H]; o += N_H
    w3 = p[o:o + N_H]; o += N_H
    b3 = p[o]
    h = np.maximum(0.0, np.atleast_2d(X) @ W1.T + b1)
    h = np.maximum(0.0, h @ W2.T + b2)
    return 1.0 / (1.0 + np.exp(-(h @ w3 + b3)))


def uniform_floor(params, margin):
    """The threshold floor of a trained network: its output on a uniform
    stencil (all features zero), raised by `margin` in logit."""
    p0 = float(forward_cpu(params, np.zeros(N_IN))[0])
    return p0, 1.0 / (1.0 + math.exp(-(math.log(p0 / (1.0 - p0)) + margin)))


def calibrate(path=WEIGHTS, margin=0.25):
    """Raise the threshold of a weights file to the uniform-stencil floor
    (parameters unchanged); rewrites the .npz and the .bin beside it."""
    params, thr, meta = load(path)
    p0, floor = uniform_floor(params, margin)
    new = min(max(thr, floor), 0.5)
    meta.update(threshold=new, threshold_before_calibration=thr, uniform_output=p0, uniform_margin=margin)
    save(path, params, new, meta)
    return thr, new, p0


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "calibrate"])
    ap.add_argument("--tau", type=float, default=1e-3)
    ap.add_argument("--recall", type=float, default=0.999)
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--seeds", type=int, default=12)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--uniform-margin", type=float, default=0.25,
                    help="logit margin of the threshold above the output at zero features")
    ap.add_argument("--out", default=WEIGHTS)
    args = ap.parse_args()
    if args.cmd == "calibrate":
        old, new, p0 = calibrate(args.out, args.uniform_margin)
        print(json.dumps(dict(threshold_before=old, threshold=new, uniform_output=p0)))
        return
    t0 = time.time()
    X, dep = collect(default_specs(range(args.seeds), args.n), verbose=True)
    y = (dep > args.tau).float()
    n = X.shape[0]
    # hold out 10% for the threshold choice and the reported scores
    g = torch.Generator(device="cuda").manual_seed(1)
    perm = torch.randperm(n, device="cuda", generator=g)
    nv = n // 10
    va, tr = perm[:nv], perm[nv:]
    params, hist, pw = train(X[tr], y[tr], epochs=args.epochs, verbose=True)
    prob = predict(params, X[va])
    pos = y[va] > 0.5
    # smallest threshold keeping the required recall on held-out positives
    ps = torch.sort(prob[pos]).values
    k = int(math.floor((1.0 - args.recall) * ps.numel()))
    thr = float(ps[k].item()) if ps.numel() else 0.5
    # a uniform stencil (all ten features zero) is smooth by construction: its
    # WENO5 weights equal the linear weights exactly.  Positives whose own
    # five-point features are flat (a jump just outside the stencil, which
    # the neighbouring nodes' flags cover in the hybrid sweep) pull the
    # recall threshold down onto the network's output at zero features; the
    # threshold is kept a logit margin above it, so that uniform regions
    # (the quiescent gas ahead of a shock) take the linear scheme
    p0, floor = uniform_floor(params, args.uniform_margin)
    thr = min(max(thr, floor, 1e-4), 0.5)
    flag = prob > thr
    recall = float((flag & pos).sum().item() / max(pos.sum().item(), 1))
    flagged = float(flag.float().mean().item())
    meta = dict(tau=args.tau, samples=int(n), positives=float(y.sum().item()), pos_weight=pw, epochs=args.epochs,
                loss=hist, threshold=thr, uniform_output=p0, uniform_margin=args.uniform_margin,
                heldout_recall=recall, heldout_flagged_fraction=flagged,
                heldout_positive_fraction=float(pos.float().mean().item()), seconds=time.time() - t0,
                data=f"{args.seeds} seeds x (1D + 3D Riemann) at {args.n}^3 + 4 TGV (Re, Ma) at {args.n}^3 and "
                     f"{2 * args.n}^3, 25 steps, every 8th recorded")
    save(args.out, params, thr, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
