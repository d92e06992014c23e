"""Seeded synthetic transport workloads (no datasets are involved).

Builds the cell-average initial state and the face-normal velocity data of the
MantlePar coupled transport workloads:

* uniform ``nx x ny`` quads on ``[0, 0.5] x [0, 1]`` (src/core/mesh.cpp:27-55,
  uniform family: x_i = x0 + i*L/nx with the far endpoint snapped);
* cell averages ``H = (1 - y_c) + a_H * U_H``, ``C = 0.3 + 0.02 * U_C`` with
  ``U`` from the reference's stateless SplitMix64 finaliser
  (src/core/mesh.cpp:12-25) keyed ``seed + 2*cell + field``;
* solid velocity ``v_s = (d psi/dy, -d psi/dx)`` of the streamfunction
  ``psi = A sin(2 pi x) sin(pi y)`` and Darcy velocity ``u_d = (0, 0.01)``,
  sampled at the 5 Gauss points of every edge.  Normal components are taken
  against each edge's canonical right normal ``(dy, -dx)/len``
  (src/core/integral.cpp:62-89) in the reference's edge-id order
  (src/core/mesh_info.h:84: AlongI ids ``j*nx + i`` first, then AlongJ ids
  ``nx*(ny+1) + j*(nx+1) + i``).  ``psi = 0`` on the walls, so the solid
  normal velocity is set to exactly zero on boundary edges.

The material set ("S") keeps the reference defaults except Te0=250 K,
Tm0=1250 K, L=6e5, cp=1200, Xe=0.5, alpha0=0: with these the literal H, C
formulas populate the two-solid, eutectic and solid+liquid regions (with the
defaults C=0.3 exceeds Xe=0.25 and the reference rejects the state).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

GAUSS5_POINTS, GAUSS5_WEIGHTS = np.polynomial.legendre.leggauss(5)

_M1 = np.uint64(0x9E3779B97F4A7C15)
_M2 = np.uint64(0xBF58476D1CE4E5B9)
_M3 = np.uint64(0x94D049BB133111EB)


def mix64(v: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on uint64 arrays (src/core/mesh.cpp:12-18)."""
    with np.errstate(over="ignore"):
        v = v.astype(np.uint64) + _M1
        v = (v ^ (v >> np.uint64(30))) * _M2
        v = (v ^ (v >> np.uint64(27))) * _M3
        return v ^ (v >> np.uint64(31))


def unit_noise(seed: int, field: int, cells: np.ndarray) -> np.ndarray:
    """Uniform [0,1) per cell: top 53 bits of SplitMix64(seed + 2*cell + field)."""
    with np.errstate(over="ignore"):
        key = np.uint64(seed) + np.uint64(2) * cells.astype(np.uint64) + np.uint64(field)
    return (mix64(key) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


@dataclasses.dataclass
class Material:
    """Dimensional material inputs (src/phase/eutectic_rescaled.h:10-26)."""
    Tm0: float = 2000.0
    Te0: float = 1480.0
    nu: float = 6.5e6
    L: float = 5.0e5
    cp: float = 1200.0
    Xe: float = 0.25
    rho: float = 3000.0
    rhor: float = 500.0
    mus: float = 1.0e19
    mul: float = 1.0
    k0: float = 1.0e-8
    g: float = 10.0
    alpha0: float = 3.0e-5

    def astuple(self):
        return dataclasses.astuple(self)


def material_s() -> Material:
    """Material set S used by every transport workload."""
    return Material(Tm0=1250.0, Te0=250.0, L=6.0e5, cp=1200.0, Xe=0.5, alpha0=0.0)


@dataclasses.dataclass
class Workload:
    nx: int
    ny: int
    x0: float = 0.0
    x1: float = 0.5
    y0: float = 0.0
    y1: float = 1.0
    noise_H: float = 0.05
    noise_C: float = 0.02
    psi_amplitude: float = 0.1
    darcy: float = 0.01
    seed: int = 1
    cfl: float = 0.4
    steps: int = 200
    integrator: int = 3

    @property
    def cells(self) -> int:
        return self.nx * self.ny

    @property
    def edges(self) -> int:
        return self.nx * (self.ny + 1) + (self.nx + 1) * self.ny


def vertex_coords(n: int, lo: float, hi: float) -> np.ndarray:
    """Vertex coordinates of one axis as src/core/mesh.cpp VertexAt (uniform)."""
    h = (hi - lo) / float(n)
    v = lo + np.arange(n + 1, dtype=np.float64) * h
    v[0] = lo
    v[-1] = lo + (hi - lo)
    return v


def initial_state(w: Workload) -> tuple[np.ndarray, np.ndarray]:
    """Seeded cell averages H, C (x fastest, id = j*nx + i)."""
    ys = vertex_coords(w.ny, w.y0, w.y1)
    yc = 0.5 * (ys[:-1] + ys[1:])
    cells = np.arange(w.cells, dtype=np.uint64)
    H = (1.0 - np.repeat(yc, w.nx)) + w.noise_H * unit_noise(w.seed, 0, cells)
    C = 0.3 + w.noise_C * unit_noise(w.seed, 1, cells)
    return np.ascontiguousarray(H), np.ascontiguousarray(C)


def face_velocity(w: Workload) -> tuple[np.ndarray, np.ndarray]:
    """Normal solid / Darcy velocity at edge Gauss points, shape (edges, 5).

    Row e holds canonical edge id e; column q the q-th Gauss point along the
    canonical direction (increasing x for AlongI edges, increasing y for
    AlongJ edges).  Normals are the canonical right normals: (0,-1) for AlongI
    edges and (1,0) for AlongJ edges.
    """
    xs = vertex_coords(w.nx, w.x0, w.x1)
    ys = vertex_coords(w.ny, w.y0, w.y1)
    A = w.psi_amplitude
    t = 0.5 * (1.0 + GAUSS5_POINTS)
    two_pi = 2.0 * math.pi
    # AlongI edges: (i, j) for j in 0..ny, i in 0..nx-1; normal (0,-1).
    xi = xs[:-1, None] + t[None, :] * (xs[1:] - xs[:-1])[:, None]          # (nx, 5)
    yj = ys                                                               # (ny+1)
    vy = -two_pi * A * np.cos(two_pi * xi)[None, :, :] * np.sin(math.pi * yj)[:, None, None]
    vs_i = -vy                                                            # v_s . (0,-1)
    vs_i[0] = 0.0
    vs_i[-1] = 0.0
    ud_i = np.full_like(vs_i, -w.darcy)                                   # u_d . (0,-1)
    # AlongJ edges: (i, j) for j in 0..ny-1, i in 0..nx; normal (1,0).
    yq = ys[:-1, None] + t[None, :] * (ys[1:] - ys[:-1])[:, None]          # (ny, 5)
    vx = math.pi * A * np.sin(two_pi * xs)[None, :, None] * np.cos(math.pi * yq)[:, None, :]
    vs_j = vx
    vs_j[:, 0, :] = 0.0
    vs_j[:, -1, :] = 0.0
    ud_j = np.zeros_like(vs_j)
    vs = np.concatenate([vs_i.reshape(-1, 5), vs_j.reshape(-1, 5)])
    ud = np.concatenate([ud_i.reshape(-1, 5), ud_j.reshape(-1, 5)])
    return np.ascontiguousarray(vs), np.ascontiguousarray(ud)


def cell_velocity(w: Workload) -> tuple[np.ndarray, np.ndarray]:
    """Vertical solid / Darcy velocity at the 5x5 Gauss points of every cell,
    [cell*25 + b*5 + a] for the point (g_a, g_b), from the same streamfunction
    (v_s,y = -dpsi/dx) and u_d = (0, darcy)."""
    xs = vertex_coords(w.nx, w.x0, w.x1)
    ys = vertex_coords(w.ny, w.y0, w.y1)
    t = 0.5 * (1.0 + GAUSS5_POINTS)
    xq = xs[:-1, None] + t[None, :] * (xs[1:] - xs[:-1])[:, None]          # (nx, 5)
    yq = ys[:-1, None] + t[None, :] * (ys[1:] - ys[:-1])[:, None]          # (ny, 5)
    two_pi = 2.0 * math.pi
    A = w.psi_amplitude
    # (j, i, b, a)
    vy = -two_pi * A * np.cos(two_pi * xq)[None, :, None, :] * np.sin(math.pi * yq)[:, None, :, None]
    vs_y = np.ascontiguousarray(vy.reshape(-1))
    return vs_y, np.full_like(vs_y, w.darcy)


# ---------------------------------------------------------------- quad meshes

MESH_RECTANGULAR, MESH_PERTURBED, MESH_SINE_STRETCHED = 0, 1, 2


def quad_vertices(w: Workload, family: int = MESH_PERTURBED, perturbation: float = 0.2, seed: int = 11) -> np.ndarray:
    """Vertices of the reference's mesh families (src/core/mesh.cpp:27-55,
    VertexAt): (nx+1)*(ny+1) (x, y) pairs, x fastest. Perturbed: interior
    vertices moved by perturbation * spacing * (2U - 1), U the SplitMix64
    noise keyed seed + 2*index (+1 for y); sine-stretched:
    x = x0 + L sin(pi/2 * i/nx)."""
    M, N = w.nx + 1, w.ny + 1
    L, Hh = w.x1 - w.x0, w.y1 - w.y0
    hx, hy = L / float(M - 1), Hh / float(N - 1)
    i = np.arange(M, dtype=np.float64)[None, :].repeat(N, 0)
    j = np.arange(N, dtype=np.float64)[:, None].repeat(M, 1)
    x = w.x0 + i * hx
    y = w.y0 + j * hy
    if family == MESH_SINE_STRETCHED:
        x = w.x0 + L * np.sin(0.5 * math.pi * (i / (M - 1)))
        y = w.y0 + Hh * np.sin(0.5 * math.pi * (j / (N - 1)))
    elif family == MESH_PERTURBED:
        idx = (np.arange(N, dtype=np.uint64)[:, None] * np.uint64(M) + np.arange(M, dtype=np.uint64)[None, :])
        nxn = 2.0 * unit_noise(seed, 0, idx) - 1.0
        nyn = 2.0 * unit_noise(seed, 1, idx) - 1.0
        inner = np.zeros((N, M), bool)
        inner[1:-1, 1:-1] = True
        x = np.where(inner, x + perturbation * hx * nxn, x)
        y = np.where(inner, y + perturbation * hy * nyn, y)
    x[:, 0], x[:, -1] = w.x0, w.x0 + L
    y[0, :], y[-1, :] = w.y0, w.y0 + Hh
    return np.ascontiguousarray(np.stack([x, y], -1).reshape(-1))


def _flow(x, y, A):
    """Solid velocity of psi = A sin(2 pi x) sin(pi y): (dpsi/dy, -dpsi/dx)."""
    vx = math.pi * A * np.sin(2 * math.pi * x) * np.cos(math.pi * y)
    vy = -2 * math.pi * A * np.cos(2 * math.pi * x) * np.sin(math.pi * y)
    return vx, vy


def face_velocity_quads(w: Workload, xy: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """face_velocity on a general quad mesh: normal components of the same
    streamfunction flow and u_d = (0, darcy) at the 5 Gauss points of every
    edge against its canonical right normal (dy, -dx)/len; solid normal
    velocity exactly zero on wall edges."""
    V = xy.reshape(w.ny + 1, w.nx + 1, 2)
    t = 0.5 * (1.0 + GAUSS5_POINTS)
    out_vs, out_ud = [], []
    for a, b, wall in (
        (V[:, :-1], V[:, 1:], np.r_[True, np.zeros(w.ny - 1, bool), True][:, None].repeat(w.nx, 1)),      # AlongI
        (V[:-1, :], V[1:, :], np.zeros((w.ny, w.nx + 1), bool) | np.r_[True, np.zeros(w.nx - 1, bool), True][None, :]),
    ):
        d = b - a
        length = np.hypot(d[..., 0], d[..., 1])
        n = np.stack([d[..., 1], -d[..., 0]], -1) / length[..., None]
        p = a[..., None, :] + t[None, None, :, None] * d[..., None, :]          # (rows, cols, 5, 2)
        vx, vy = _flow(p[..., 0], p[..., 1], w.psi_amplitude)
        vs = vx * n[..., None, 0] + vy * n[..., None, 1]
        vs[wall] = 0.0
        ud = np.broadcast_to(w.darcy * n[..., None, 1], vs.shape)
        out_vs.append(vs.reshape(-1, 5))
        out_ud.append(np.ascontiguousarray(ud).reshape(-1, 5))
    return np.ascontiguousarray(np.concatenate(out_vs)), np.ascontiguousarray(np.concatenate(out_ud))


def uniform_face_velocity(w: Workload, xy: np.ndarray, U: float, V: float) -> np.ndarray:
    """Normal components of the uniform velocity (U, V) at the 5 Gauss points
    of every edge against its canonical right normal (dy, -dx)/len, [edge*5 + q];
    xy: the mesh vertices (quad_vertices, any family)."""
    P = xy.reshape(w.ny + 1, w.nx + 1, 2)
    out = []
    for a, b in ((P[:, :-1], P[:, 1:]), (P[:-1, :], P[1:, :])):   # AlongI, then AlongJ
        d = b - a
        length = np.hypot(d[..., 0], d[..., 1])
        vn = (U * d[..., 1] - V * d[..., 0]) / length
        out.append(np.repeat(vn.reshape(-1, 1), 5, axis=1))
    return np.ascontiguousarray(np.concatenate(out).reshape(-1))


def cell_centroids(w: Workload, xy: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Area centroids of the cells of a quad mesh, [j*nx + i] (the shoelace
    formula in coordinates relative to each cell's first corner, so that the
    products do not cancel on small cells)."""
    P = xy.reshape(w.ny + 1, w.nx + 1, 2)
    o = P[:-1, :-1]
    v = [P[:-1, :-1] - o, P[:-1, 1:] - o, P[1:, 1:] - o, P[1:, :-1] - o]   # counter-clockwise
    A2 = 0.0
    sx = 0.0
    sy_ = 0.0
    for k in range(4):
        a, b = v[k], v[(k + 1) % 4]
        cr = a[..., 0] * b[..., 1] - b[..., 0] * a[..., 1]
        A2 = A2 + cr
        sx = sx + (a[..., 0] + b[..., 0]) * cr
        sy_ = sy_ + (a[..., 1] + b[..., 1]) * cr
    return (o[..., 0] + sx / (3 * A2)).reshape(-1), (o[..., 1] + sy_ / (3 * A2)).reshape(-1)


def cell_velocity_quads(w: Workload, xy: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """cell_velocity on a general quad mesh: the vertical components at the
    bilinear images of the 5x5 Gauss points, [cell*25 + b*5 + a]."""
    V = xy.reshape(w.ny + 1, w.nx + 1, 2)
    c0, c1, c2, c3 = V[:-1, :-1], V[:-1, 1:], V[1:, 1:], V[1:, :-1]
    g = GAUSS5_POINTS
    s = 0.5 * (1 - g)[None, :, None]
    r = 0.5 * (1 + g)[None, :, None]
    out = np.zeros((w.ny, w.nx, 5, 5))
    for b in range(5):
        sb, tb = 0.5 * (1 - g[b]), 0.5 * (1 + g[b])
        for a in range(5):
            sa, ta = 0.5 * (1 - g[a]), 0.5 * (1 + g[a])
            lo = sa * c0 + ta * c1
            hi = sa * c3 + ta * c2
            p = sb * lo + tb * hi
            out[:, :, b, a] = _flow(p[..., 0], p[..., 1], w.psi_amplitude)[1]
    del s, r
    vs_y = np.ascontiguousarray(out.reshape(-1))
    return vs_y, np.full_like(vs_y, w.darcy)


# The BASELINE workloads, named by what they are.
def plain_small() -> Workload:
    """20x20 plain FP64 instance, 200 steps (the run.sh --grid 20 size)."""
    return Workload(nx=20, ny=20, steps=200)


def plain_large() -> Workload:
    """1280x2560 plain FP64 single instance, 100 steps."""
    return Workload(nx=1280, ny=2560, steps=100)


def mixed_large() -> Workload:
    """4096x4096 mixed-precision instance, H noise 0.1, 50 steps."""
    return Workload(nx=4096, ny=4096, noise_H=0.1, steps=50)


def batched_instances(count: int = 256, seed: int = 3) -> list[Workload]:
    """Uneven meshes: nx, ny log-uniform on [40,640] and [40,960], step 20."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nx = int(20 * round(math.exp(rng.uniform(math.log(40), math.log(640))) / 20))
        ny = int(20 * round(math.exp(rng.uniform(math.log(40), math.log(960))) / 20))
        amp = float(rng.uniform(0.05, 0.2))
        out.append(Workload(nx=max(nx, 40), ny=max(ny, 40), psi_amplitude=amp, seed=1000 + i, steps=100))
    return out
