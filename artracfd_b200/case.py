"""Case description in the reference's own terms.

``CaseSpec`` holds what an ArtraCFD case directory holds (artracfd.case and
artracfd.geo, case_loader.c:55-226, initialization.c:163-209).  It can

* write that case directory, so that the reference program or its harness
  runs the very same case (``write``);
* derive the ``acfd_partition_t``/``acfd_model_t`` descriptors that the GPU
  library consumes, restating ComputeParameters (cfd_parameters.c:28-186) and
  PartitionDomain (domain_partition.c:19-150) (``descriptors``);
* evaluate the initial field on the host with numpy (``initial_nodes``),
  following InitializeFieldData (initialization.c:68-162).
"""
from __future__ import annotations

import math
import os
import struct
from dataclasses import dataclass, field

import numpy as np

from . import abi

BC_NAMES = {abi.INFLOW: "inflow", abi.OUTFLOW: "outflow", abi.SLIPWALL: "slip wall",
            abi.NOSLIPWALL: "noslip wall", abi.PERIODIC: "periodic"}
FACE_NAMES = ["west", "east", "south", "north", "front", "back"]
GAS_R = 287.058  # cfd_parameters.c:169
GAMMA = 1.4      # cfd_parameters.c:168
INT_MAX = 2**31 - 1


@dataclass
class Boundary:
    kind: int
    values: tuple = ()   # inflow: rho,u,v,w,p; walls: (T,)


@dataclass
class Region:
    """Regional initializer: kind in {'plane','sphere','box','cylinder'}."""
    kind: str
    p1: tuple = (0.0, 0.0, 0.0)
    p2: tuple = (0.0, 0.0, 0.0)
    r: float = 0.0
    exprs: tuple = ("1", "0", "0", "0", "1")


@dataclass
class Body:
    """One immersed body (data_stream.c:154-188 field order)."""
    O: tuple
    r: float
    V: tuple = (0.0, 0.0, 0.0)
    W: tuple = (0.0, 0.0, 0.0)
    rho: float = 1.0e40
    T: float = -1.0
    cf: float = 0.0
    stl: str | None = None          # None: analytical sphere
    triangles: np.ndarray | None = None  # (faceN, 3, 3) float32 vertices for the STL file


@dataclass
class CaseSpec:
    domain_lo: tuple
    domain_hi: tuple
    m: tuple
    end: float = 1.0
    cfl: float = 0.6
    stepN: int = 0
    restart: int = 0   # data output to restart from (0: none)
    dataW: int = 1     # space data outputs over the run
    tScheme: int = 1
    sScheme: int = 1
    multidim: int = 0
    jacobMean: int = 1
    fluxSplit: int = 0
    psi: int = 0
    ibmLayer: int = 1
    refMu: float = 0.0
    gState: int = 0
    g: tuple = (0.0, 0.0, 0.0)
    refL: float = 1.0
    refRho: float = 1.0
    refV: float = 1.0
    refT: float = 1.0
    init: tuple = ("1", "0", "0", "0", "1")
    boundaries: list = field(default_factory=lambda: [Boundary(abi.PERIODIC)] * 6)
    regions: list = field(default_factory=list)
    bodies: list = field(default_factory=list)

    # ------------------------------------------------------------------
    # reference case directory
    # ------------------------------------------------------------------
    def write(self, path: str) -> None:
        os.makedirs(path, exist_ok=True)
        L = []
        L += ["space begin", "%.17g, %.17g, %.17g" % tuple(self.domain_lo),
              "%.17g, %.17g, %.17g" % tuple(self.domain_hi), "%d, %d, %d" % tuple(self.m), "space end"]
        L += ["time begin", "%d" % self.restart, "%.17g" % self.end, "%.17g" % self.cfl, "%d" % self.stepN,
              "%d" % self.dataW, "1", "time end"]
        L += ["numerical begin"] + ["%d" % v for v in (self.tScheme, self.sScheme, self.multidim,
                                                       self.jacobMean, self.fluxSplit, self.psi,
                                                       self.ibmLayer)] + ["numerical end"]
        L += ["material begin", "0", "%.17g" % self.refMu, "%d" % self.gState,
              "%.17g, %.17g, %.17g" % tuple(self.g), "material end"]
        L += ["reference begin"] + ["%.17g" % v for v in (self.refL, self.refRho, self.refV, self.refT)] + [
            "reference end"]
        L += ["initialization begin"] + list(self.init) + ["initialization end"]
        for f, b in zip(FACE_NAMES, self.boundaries):
            L += [f"{f} boundary begin", BC_NAMES[b.kind]]
            if b.kind == abi.INFLOW:
                L += ["%.17g" % v for v in b.values[:5]]
            elif b.kind in (abi.SLIPWALL, abi.NOSLIPWALL):
                L += ["%.17g" % (b.values[0] if b.values else -1.0)]
            L += [f"{f} boundary end"]
        for rg in self.regions:
            L += [f"{rg.kind} initialization begin"]
            L += ["%.17g, %.17g, %.17g" % tuple(rg.p1)]
            if rg.kind in ("plane", "box", "cylinder"):
                L += ["%.17g, %.17g, %.17g" % tuple(rg.p2)]
            if rg.kind in ("sphere", "cylinder"):
                L += ["%.17g" % rg.r]
            L += list(rg.exprs) + [f"{rg.kind} initialization end"]
        with open(os.path.join(path, "artracfd.case"), "w") as fh:
            fh.write("\n".join(L) + "\n")
        self._write_geo(path)

    def _write_geo(self, path: str) -> None:
        sph = [b for b in self.bodies if b.stl is None]
        stl = [b for b in self.bodies if b.stl is not None]
        if [b.stl is None for b in self.bodies] != [True] * len(sph) + [False] * len(stl):
            raise ValueError("analytical spheres must precede triangulated bodies")
        L = ["count begin", str(len(sph)), str(len(stl)), "count end"]

        def state(b):
            a = "%.17g, %.17g, %.17g, %.17g, " % (*b.O, b.r)
            a += "%.17g, %.17g, %.17g, %.17g, %.17g, %.17g, " % (*b.V, *b.W)
            a += "%.17g, %.17g, %.17g, 0, 0, 0" % (b.rho, b.T, b.cf)
            return [a, "0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0"]

        if sph:
            L += ["sphere state begin"]
            for b in sph:
                L += state(b)
            L += ["sphere state end"]
        if stl:
            L += ["polyhedron geometry begin"] + [b.stl for b in stl] + ["polyhedron geometry end"]
            L += ["polyhedron state begin"]
            for b in stl:
                L += state(b)
            L += ["polyhedron state end"]
            L += ["polyhedron transform begin"] + ["1, 1, 1, 0, 0, 0, 0, 0, 0"] * len(stl) + [
                "polyhedron transform end"]
            for b in stl:
                write_stl(os.path.join(path, b.stl), b.triangles)
        with open(os.path.join(path, "artracfd.geo"), "w") as fh:
            fh.write("\n".join(L) + "\n")

    # ------------------------------------------------------------------
    # descriptors for the GPU library
    # ------------------------------------------------------------------
    def descriptors(self):
        """Return (Partition, Model) exactly as the reference computes them."""
        part = abi.Partition()
        model = abi.Model()
        model.tScheme, model.sScheme, model.multidim = self.tScheme, self.sScheme, self.multidim
        model.jacobMean, model.fluxSplit, model.psi = self.jacobMean, self.fluxSplit, self.psi
        model.ibmLayer = self.ibmLayer
        model.gState = self.gState
        m = [int(v) for v in self.m]
        for q, b in enumerate(self.boundaries):
            part.typeBC[q + 1] = b.kind
            if b.kind == abi.INFLOW:
                for v in range(5):
                    part.varBC[q + 1][v] = b.values[v]
            elif b.kind in (abi.SLIPWALL, abi.NOSLIPWALL):
                part.varBC[q + 1][5] = b.values[0] if b.values else -1.0
        # SetNodeNumber (cfd_parameters.c:46-124)
        collapse = 0
        if m[2] - 1 == 0:
            collapse = 3
        if m[1] - 1 == 0:
            collapse = 2 * collapse + 2
        if m[0] - 1 == 0:
            collapse = 2 * collapse + 1
        part.collapse = collapse
        if self.sScheme == 0:
            model.sL, model.sR, part.gl = -1, 2, 2
        else:
            model.sL, model.sR, part.gl = -2, 3, 3
        ng = [part.gl - 1] * 3
        if self.multidim == 0:
            if collapse in (1, 5, 7):
                ng[0] = 0
            if collapse in (2, 5, 8):
                ng[1] = 0
            if collapse in (3, 7, 8):
                ng[2] = 0
        for s in range(3):
            if self.boundaries[2 * s].kind == abi.PERIODIC:
                ng[s] = part.gl
        for s in range(3):
            m[s] = max(m[s], 2)
            part.m[s] = m[s]
            part.ng[s] = ng[s]
            part.n[s] = m[s] + 1 + 2 * ng[s]
        # InitializeParameters (cfd_parameters.c:129-186)
        for s in range(3):
            hi = self.domain_hi[s] / self.refL
            lo = self.domain_lo[s] / self.refL
            part.domain[s][0] = lo
            part.domain[s][1] = hi
            part.d[s] = (hi - lo) / float(m[s])
            part.dd[s] = 1.0 / part.d[s]
        tiny = 1.0e-6 * min(part.d[0], min(part.d[1], part.d[2]))
        part.tinyL = tiny * tiny
        model.ibmLayer = INT_MAX if self.ibmLayer <= 0 else self.ibmLayer
        model.gamma = GAMMA
        gasR = GAS_R
        for s in range(3):
            model.g[s] = self.g[s] * self.refL / (self.refV * self.refV)
        model.sState = self.gState
        model.refMa = self.refV / math.sqrt(model.gamma * gasR * self.refT)
        model.refMu = self.refMu / (self.refRho * self.refV * self.refL)
        model.gasR = 1.0 / (model.gamma * model.refMa * model.refMa)
        model.cv = model.gasR / (model.gamma - 1.0)
        model.refL, model.refRho, model.refV, model.refT = self.refL, self.refRho, self.refV, self.refT
        partition_domain(part)
        return part, model

    @property
    def end_time(self) -> float:
        return self.end * self.refV / self.refL

    # ------------------------------------------------------------------
    # initial field
    # ------------------------------------------------------------------
    def initial_nodes(self, part: abi.Partition | None = None, model: abi.Model | None = None) -> np.ndarray:
        """Initial node array (reference layout), following InitializeFieldData
        (initialization.c:68-162): every node starts as junk with flags -1,
        PIN nodes get flags 0 and the initializers in order.  Expressions are
        evaluated with numpy, so values may differ from the reference's
        calculator in the last bits."""
        if part is None or model is None:
            part, model = self.descriptors()
        n = list(part.n)
        node = np.zeros(n[0] * n[1] * n[2], dtype=abi.NODE_DTYPE)
        node["U"] = np.frombuffer(b"\x01" * 8, dtype="<f8")[0]
        for f in ("did", "fid", "lid", "gst"):
            node[f] = -1
        ns = np.array(part.ns)
        lo = ns[0, :, 0]
        hi = ns[0, :, 1]
        k, j, i = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]),
                              indexing="ij")
        idx = ((k * n[1] + j) * n[0] + i).ravel()
        for f in ("did", "fid", "lid", "gst"):
            node[f][idx] = 0
        x = part.domain[0][0] + (i.ravel() - part.ng[0]) * part.d[0]
        y = part.domain[1][0] + (j.ravel() - part.ng[1]) * part.d[1]
        z = part.domain[2][0] + (k.ravel() - part.ng[2]) * part.d[2]
        U = np.empty((idx.size, 5))
        inits = [Region("global", exprs=self.init)] + list(self.regions)
        first = True
        for rg in inits:
            prim = [np.broadcast_to(np.asarray(_eval_expr(e, x, y, z), dtype=np.float64), x.shape)
                    for e in rg.exprs]
            mask = _region_mask(rg, x, y, z)
            cons = _to_conservative(model.gamma, prim)
            if first:
                U[:] = cons
                first = False
            else:
                U[mask] = cons[mask]
        node["U"][idx, 0, :] = U
        return node


def partition_domain(part: abi.Partition) -> None:
    """PartitionDomain (domain_partition.c:19-150)."""
    normals = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    for q in range(7):
        for s in range(3):
            part.N[q][s] = normals[q][s]
    for s in range(3):
        lo, hi = part.ng[s], part.n[s] - part.ng[s]
        if part.typeBC[1 + 2 * s] == abi.PERIODIC:
            part.ns[0][s][0], part.ns[0][s][1] = lo, hi
        else:
            part.ns[0][s][0], part.ns[0][s][1] = lo + 1, hi - 1
        for p in range(1, 7):
            part.ns[p][s][0], part.ns[p][s][1] = lo, hi
        for p in range(7, 13):
            part.ns[p][s][0], part.ns[p][s][1] = 0, part.n[s]
        part.ns[13][s][0], part.ns[13][s][1] = lo, hi
        part.ns[14][s][0], part.ns[14][s][1] = 0, part.n[s]
    for s in range(3):
        part.ns[1 + 2 * s][s][1] = part.ns[1 + 2 * s][s][0] + 1
        part.ns[2 + 2 * s][s][0] = part.ns[2 + 2 * s][s][1] - 1
        part.ns[7 + 2 * s][s][1] = part.ng[s]
        part.ns[8 + 2 * s][s][0] = part.n[s] - part.ng[s]
    pri = [(0, 1, 2), (1, 0, 2), (2, 0, 1)]
    for q in range(3):
        for s in range(3):
            part.np[q][s][0] = part.ns[0][pri[q][s]][0]
            part.np[q][s][1] = part.ns[0][pri[q][s]][1]
    path = []
    for s in range(3):
        for sg in (-1, 1):
            v = [0, 0, 0]
            v[s] = sg
            path.append(v)
    for a0, a1 in ((0, 1), (0, 2), (1, 2)):
        for b in (-1, 1):
            for a in (-1, 1):
                v = [0, 0, 0]
                v[a0], v[a1] = a, b
                path.append(v)
    for dist in (2, 3):
        for s in range(3):
            for sg in (-1, 1):
                v = [0, 0, 0]
                v[s] = sg * dist
                path.append(v)
    for q, v in enumerate(path):
        for s in range(3):
            part.path[q][s] = v[s]
    part.pathSep[1] = 6
    part.pathSep[2] = 24
    part.pathSep[3] = 30
    part.pathSep[0] = part.pathSep[part.gl]


_EXPR_NS = {"sin": np.sin, "cos": np.cos, "tan": np.tan, "exp": np.exp, "ln": np.log,
            "lg": np.log10, "abs": np.abs, "pi": math.pi}


def _eval_expr(expr: str, x, y, z):
    src = expr.replace("^", "**")
    return eval(src, {"__builtins__": {}}, dict(_EXPR_NS, x=x, y=y, z=z, t=0.0))  # noqa: S307


def _region_mask(rg: Region, x, y, z):
    """Region tests of ApplyInitializer (initialization.c:103-162)."""
    pc = np.stack([x, y, z], axis=-1)
    p1 = np.asarray(rg.p1, dtype=np.float64)
    p2 = np.asarray(rg.p2, dtype=np.float64)
    d = pc - p1
    if rg.kind == "global":
        return np.ones(x.shape, dtype=bool)
    if rg.kind == "plane":
        return (d[:, 0] * p2[0] + d[:, 1] * p2[1] + d[:, 2] * p2[2]) >= 0.0
    if rg.kind == "sphere":
        return rg.r * rg.r >= (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    if rg.kind == "box":
        e = d * (pc - p2)
        return (e[:, 0] <= 0) & (e[:, 1] <= 0) & (e[:, 2] <= 0)
    if rg.kind == "cylinder":
        ax = p2 - p1
        l2 = ax @ ax
        proj = d @ ax
        perp = (d * d).sum(axis=1) - proj * proj / l2
        return (proj >= 0) & (proj <= l2) & (rg.r * rg.r >= perp)
    raise ValueError(rg.kind)


def _to_conservative(gamma, prim):
    rho, u, v, w, p = prim
    U = np.empty(rho.shape + (5,))
    U[:, 0] = rho
    U[:, 1] = rho * u
    U[:, 2] = rho * v
    U[:, 3] = rho * w
    U[:, 4] = 0.5 * rho * (u * u + v * v + w * w) + p / (gamma - 1.0)
    return U


# ----------------------------------------------------------------------
# geometry files
# ----------------------------------------------------------------------
def write_stl(path: str, tris: np.ndarray) -> None:
    """Binary STL (stl.c:97-121 layout): 80-byte header, uint32 count,
    per facet normal + 3 vertices as float32 and a uint16 attribute."""
    tris = np.asarray(tris, dtype=np.float32)
    with open(path, "wb") as fh:
        fh.write(b"binary stl".ljust(80, b"\0"))
        fh.write(struct.pack("<I", tris.shape[0]))
        for t in tris:
            nrm = np.cross(t[1] - t[0], t[2] - t[0]).astype(np.float64)
            nn = np.linalg.norm(nrm)
            nrm = (nrm / nn if nn > 0 else nrm).astype(np.float32)
            fh.write(nrm.tobytes() + t.tobytes() + b"\0\0")


def icosphere(center, radius, level=3) -> np.ndarray:
    """Triangulated sphere by recursive subdivision of an icosahedron,
    outward-oriented; level 3 gives 1280 facets."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
             (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                v = verts[a] + verts[b]
                verts.append(v / np.linalg.norm(v))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius + np.asarray(center, dtype=np.float64)
    tris = V[np.array(faces)]
    # outward orientation
    for q in range(tris.shape[0]):
        nrm = np.cross(tris[q, 1] - tris[q, 0], tris[q, 2] - tris[q, 0])
        if nrm @ (tris[q].mean(axis=0) - np.asarray(center)) < 0:
            tris[q] = tris[q, ::-1]
    return tris.astype(np.float32)


def extruded_cylinder(center_xy, radius, z0, z1, segments=64) -> np.ndarray:
    """Closed prism approximating a cylinder along z (outward-oriented)."""
    ang = np.linspace(0.0, 2.0 * math.pi, segments, endpoint=False)
    cx, cy = center_xy
    ring = np.stack([cx + radius * np.cos(ang), cy + radius * np.sin(ang)], axis=1)
    tris = []
    for q in range(segments):
        a, b = ring[q], ring[(q + 1) % segments]
        A0, B0 = (a[0], a[1], z0), (b[0], b[1], z0)
        A1, B1 = (a[0], a[1], z1), (b[0], b[1], z1)
        tris.append((A0, B0, B1))
        tris.append((A0, B1, A1))
        tris.append(((cx, cy, z0), B0, A0))
        tris.append(((cx, cy, z1), A1, B1))
    return np.array(tris, dtype=np.float32)


# ----------------------------------------------------------------------
# preprocessed bodies
# ----------------------------------------------------------------------

def load_polyhedra(z, prefix: str = "geo_"):
    """Body descriptors (abi.Polyhedron) from arrays saved with the given key
    prefix: ``<prefix>count`` bodies, each with ``scal`` (faceN, edgeN, vertN,
    state), ``real`` (r, O, V, W, T, cf, box) and, for triangulated bodies,
    the surface arrays f, Nf, e, Ne, v, Nv of the reference's Polyhedron
    (commons.h:203-243) after its load-time preprocessing.  Returns
    (bodies, keep): ``keep`` holds the arrays the descriptors point into and
    must outlive them."""
    import ctypes
    keep = []
    geo = []
    if prefix + "count" not in z:
        return geo, keep
    for q in range(int(z[prefix + "count"])):
        p = f"{prefix}{q}_"
        P = abi.Polyhedron()
        P.faceN, P.edgeN, P.vertN, P.state = (int(v) for v in z[p + "scal"])
        real = z[p + "real"]
        P.r = real[0]
        for s in range(3):
            P.O[s] = real[1 + s]
            P.V[s] = real[4 + s]
            P.W[s] = real[7 + s]
        P.T = real[10]
        P.cf = real[11]
        for s in range(3):
            for m in range(2):
                P.box[s][m] = real[12 + 2 * s + m]
        if P.faceN > 0:
            arrs = {}
            for key, ct in (("f", ctypes.c_int), ("Nf", ctypes.c_double), ("e", ctypes.c_int),
                            ("Ne", ctypes.c_double), ("v", ctypes.c_double), ("Nv", ctypes.c_double)):
                a = np.ascontiguousarray(z[p + key], dtype=np.int32 if ct is ctypes.c_int else np.float64)
                arrs[key] = a
                setattr(P, key, a.ctypes.data_as(ctypes.POINTER(ct)))
            keep.append(arrs)
        geo.append(P)
    return geo, keep
