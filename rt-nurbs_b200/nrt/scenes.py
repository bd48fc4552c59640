"""Seeded synthetic scenes for the NURBS intersection path.

Every scene is a list of NURBS surfaces in the reference's layout
(ParametricSurf::nurbsSurf, src/math/nurbs.h:17-22): control points are
weighted-homogeneous (w*x, w*y, w*z, w), row-major with index i*(m+1)+j and i
along u; knot vectors hold n+p+2 and m+q+2 values.  Cameras follow the
reference's pinhole camera (src/core/camera.h:63-174): eye, look-at point, up
vector, field of view on the short image axis, and resolution.

The workloads (sizes, degrees, distributions) are the ones this engine is
benchmarked on; where a distribution leaves a choice open, the choice is
written next to the generator.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Surface:
    cp: np.ndarray        # ((n+1)*(m+1), 4) float32, weighted-homogeneous
    U: np.ndarray         # (n+p+2,) float32
    V: np.ndarray         # (m+q+2,) float32
    n: int
    m: int
    p: int
    q: int


@dataclass
class Camera:
    eye: tuple
    look: tuple
    up: tuple
    fov_deg: float
    width: int
    height: int
    spp: int = 1
    seed: int = 0

    @property
    def n_rays(self) -> int:
        return self.width * self.height * self.spp

    @property
    def cam_k(self) -> float:
        # 0.5*H/tan(fov/2): pixels per unit distance at depth 1 (intersect.cu:212)
        return 0.5 * self.height / np.tan(np.radians(self.fov_deg) / 2.0)


@dataclass
class Scene:
    name: str
    surfaces: list
    camera: Camera
    notes: dict = field(default_factory=dict)


def _homogeneous(xyz: np.ndarray, w: np.ndarray) -> np.ndarray:
    out = np.empty((xyz.shape[0], 4), np.float32)
    out[:, :3] = (xyz * w[:, None]).astype(np.float32)
    out[:, 3] = w.astype(np.float32)
    return out


def clamped_uniform_knots(n: int, p: int) -> np.ndarray:
    inner = [(k + 1) / (n - p + 1) for k in range(n - p)]
    return np.array([0.0] * (p + 1) + inner + [1.0] * (p + 1), np.float32)


# --------------------------------------------------------------------------
# Small height-field scene: one bicubic surface, 8x8 net, 25 patches.
def heightfield_scene(seed: int = 0, width: int = 256, height: int = 256, spp: int = 1) -> Scene:
    """One bicubic NURBS surface with an 8x8 net on [-1,1]^2 and clamped uniform
    knots (25 Bezier patches).  z = 0.3 sin(3x) cos(2y) + N(0, 0.02), weights
    U[0.5, 2].  Pinhole camera at (0,-3,2) looking at the origin, up (0,0,1),
    45 degree field of view, 256x256 pixel-centre rays."""
    rng = np.random.default_rng(seed)
    n = m = 7
    p = q = 3
    g = np.linspace(-1.0, 1.0, n + 1)
    X, Y = np.meshgrid(g, g, indexing="ij")          # i along u (x), j along v (y)
    Z = 0.3 * np.sin(3 * X) * np.cos(2 * Y) + rng.normal(0.0, 0.02, X.shape)
    W = rng.uniform(0.5, 2.0, X.shape)
    xyz = np.stack([X, Y, Z], -1).reshape(-1, 3)
    surf = Surface(_homogeneous(xyz, W.reshape(-1)), clamped_uniform_knots(n, p), clamped_uniform_knots(m, q),
                   n, m, p, q)
    cam = Camera((0.0, -3.0, 2.0), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 45.0, width, height, spp, seed)
    return Scene("heightfield", [surf], cam)


# --------------------------------------------------------------------------
# Exact rational torus and sphere (src/core/benchmark.cpp:52-79 and
# src/core/main.cpp:70-98): 9-point rational circles with weights sqrt(2)/2,
# quarter-arc knots.  Ray hits are known in closed form.
_S = 0.70710678
_CX = [1, 1, 0, -1, -1, -1, 0, 1, 1]
_CY = [0, 1, 1, 1, 0, -1, -1, -1, 0]
_CW = [1, _S, 1, _S, 1, _S, 1, _S, 1]
_QUARTER = np.array([0, 0, 0, .25, .25, .5, .5, .75, .75, 1, 1, 1], np.float32)


def torus_surface(R: float = 1.0, r: float = 0.4, cz: float = 6.0) -> Surface:
    cp = np.empty((81, 4), np.float32)
    for i in range(9):
        for j in range(9):
            radial = R + r * _CX[j]
            w = _CW[i] * _CW[j]
            cp[i * 9 + j] = (w * radial * _CX[i], w * radial * _CY[i], w * (r * _CY[j] + cz), w)
    return Surface(cp, _QUARTER.copy(), _QUARTER.copy(), 8, 8, 2, 2)


def sphere_surface(Rs: float = 1.0, cz: float = 6.0) -> Surface:
    svr = [0, Rs, Rs, Rs, 0]
    svz = [Rs, Rs, 0, -Rs, -Rs]
    svw = [1, _S, 1, _S, 1]
    cp = np.empty((45, 4), np.float32)
    for i in range(9):
        for j in range(5):
            w = _CW[i] * svw[j]
            cp[i * 5 + j] = (w * svr[j] * _CX[i], w * svr[j] * _CY[i], w * (svz[j] + cz), w)
    V = np.array([0, 0, 0, .5, .5, 1, 1, 1], np.float32)
    return Surface(cp, _QUARTER.copy(), V, 8, 4, 2, 2)


def analytic_scene(kind: str = "torus", width: int = 192, height: int = 108) -> Scene:
    """Torus or sphere centred on (0,0,6), camera at (3,3,0) looking at
    (0,0,6) with up (0,1,0) and a 60 degree field of view, as the reference's
    benchmark sets it up (src/core/benchmark.cpp:123-131)."""
    surf = torus_surface() if kind == "torus" else sphere_surface()
    cam = Camera((3.0, 3.0, 0.0), (0.0, 0.0, 6.0), (0.0, 1.0, 0.0), 60.0, width, height)
    return Scene(kind, [surf], cam)


# --------------------------------------------------------------------------
# Many-surface scenes of mixed degree.
def _random_knots(rng, n: int, p: int) -> np.ndarray:
    """Clamped knot vector whose n-p interior slots hold U(0,1) values, each
    repeated 1 or 2 times (never more than p)."""
    slots = n - p
    vals = []
    while len(vals) < slots:
        v = float(rng.uniform(0.0, 1.0))
        mult = int(rng.integers(1, 3))
        mult = min(mult, p, slots - len(vals))
        vals.extend([v] * mult)
    vals.sort()
    return np.array([0.0] * (p + 1) + vals + [1.0] * (p + 1), np.float32)


def _random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def random_surface(rng, centre, deg_range=(2, 5), net_range=(16, 32), relief: float = 1.0) -> Surface:
    """One random NURBS surface.  Control points lie in a unit box: a regular
    (n+1)x(m+1) grid over the box's x/y extent with heights U(0, relief); the
    box is then rotated by a uniformly random rotation about its centre and
    moved to `centre`.  Weights are lognormal(0, 0.5)."""
    p = int(rng.integers(deg_range[0], deg_range[1] + 1))
    q = int(rng.integers(deg_range[0], deg_range[1] + 1))
    n = int(rng.integers(net_range[0], net_range[1] + 1)) - 1
    m = int(rng.integers(net_range[0], net_range[1] + 1)) - 1
    gx = np.linspace(0.0, 1.0, n + 1)
    gy = np.linspace(0.0, 1.0, m + 1)
    X, Y = np.meshgrid(gx, gy, indexing="ij")
    Z = rng.uniform(0.0, relief, X.shape)
    local = np.stack([X - 0.5, Y - 0.5, Z - 0.5 * relief], -1).reshape(-1, 3)
    Rm = _random_rotation(rng)
    xyz = local @ Rm.T + np.asarray(centre)[None, :]
    w = rng.lognormal(0.0, 0.5, (n + 1) * (m + 1))
    return Surface(_homogeneous(xyz, w), _random_knots(rng, n, p), _random_knots(rng, m, q), n, m, p, q)


def surfaces_grid_scene(n_surfaces: int, seed: int, width: int, height: int, spp: int, relief: float = 1.0,
                        deg_range=(2, 5), net_range=(16, 32), spacing: float = 1.0, layers: int = 4,
                        name: str = "surfaces") -> Scene:
    """n_surfaces random surfaces (see random_surface) whose boxes sit on a
    lattice of `layers` levels with the given spacing (64 -> 4x4x4,
    256 -> 8x8x4), so that most camera rays cross several surfaces.  The camera
    looks at the lattice centre from the direction (1, -1.3, 0.8), close
    enough (0.55x the distance at which the lattice's bounding sphere would
    just fit the short image axis) that the lattice fills the frame."""
    rng = np.random.default_rng(seed)
    layers = max(1, min(layers, n_surfaces))
    per_layer = int(np.ceil(n_surfaces / layers))
    side = int(np.ceil(np.sqrt(per_layer)))
    dims = np.array([side, int(np.ceil(per_layer / side)), layers], np.float64)
    half = 0.5 * spacing * (dims - 1)
    surfs = []
    for k in range(n_surfaces):
        ix, iy, iz = k % side, (k // side) % int(dims[1]), k // per_layer
        centre = (-half[0] + spacing * ix, -half[1] + spacing * iy, -half[2] + spacing * iz)
        surfs.append(random_surface(rng, centre, deg_range, net_range, relief))
    radius = float(np.linalg.norm(half + 0.5 * spacing))
    fov = 60.0
    dist = 0.55 * radius / np.sin(np.radians(fov / 2.0))
    view = np.array([1.0, -1.3, 0.8])
    view /= np.linalg.norm(view)
    eye = tuple(float(x) for x in dist * view)
    cam = Camera(eye, (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), fov, width, height, spp, seed)
    return Scene(name, surfs, cam, {"lattice": dims.astype(int).tolist(), "spacing": spacing, "relief": relief})


def mixed_degree_scene(seed: int = 1, width: int = 1920, height: int = 1080, spp: int = 4) -> Scene:
    """64 surfaces of degree 2-5, nets 16x16 to 32x32, about 10k Bezier
    patches; 1920x1080 with 4 jittered samples per pixel (8,294,400 rays)."""
    return surfaces_grid_scene(64, seed, width, height, spp, name="mixed64")


def wavefront_scene(seed: int = 3, width: int = 2048, height: int = 2048, spp: int = 4) -> Scene:
    """256 surfaces from the same generator (about 40k-100k Bezier patches);
    2048x2048 with 4 jittered samples (2^24 primary rays per batch)."""
    return surfaces_grid_scene(256, seed, width, height, spp, name="wave256")


# --------------------------------------------------------------------------
# Precision stress: degree 7x7 rational patches, extreme weights, collapsed
# edges, grazing rays.
def _bernstein(n: int, t: np.ndarray):
    """Bernstein values and derivatives of degree n at t (float64), shape (len(t), n+1)."""
    from math import comb

    k = np.arange(n + 1)
    c = np.array([comb(n, i) for i in k], np.float64)
    t = t[:, None]
    B = c * t ** k * (1.0 - t) ** (n - k)
    km = np.arange(n)
    cm = np.array([comb(n - 1, i) for i in km], np.float64)
    Bm = cm * t ** km * (1.0 - t) ** (n - 1 - km)
    dB = np.zeros_like(B)
    dB[:, :-1] -= n * Bm
    dB[:, 1:] += n * Bm
    return B, dB


def patch_points(cp: np.ndarray, p: int, q: int, u: np.ndarray, v: np.ndarray):
    """S, dS/du, dS/dv (float64) of rational Bezier patches cp[k] ((p+1)(q+1) x 4,
    weighted-homogeneous, index i*(q+1)+j) at (u[k], v[k])."""
    P = cp.reshape(-1, p + 1, q + 1, 4).astype(np.float64)
    Bu, dBu = _bernstein(p, u)
    Bv, dBv = _bernstein(q, v)
    H = np.einsum("ki,kj,kijc->kc", Bu, Bv, P)
    Hu = np.einsum("ki,kj,kijc->kc", dBu, Bv, P)
    Hv = np.einsum("ki,kj,kijc->kc", Bu, dBv, P)
    w = H[:, 3:4]
    S = H[:, :3] / w
    return S, (Hu[:, :3] - S * Hu[:, 3:4]) / w, (Hv[:, :3] - S * Hv[:, 3:4]) / w


def precision_patches(seed: int = 5, n_patches: int = 32, collapsed: int = 8):
    """n_patches rational Bezier patches of degree 7x7 on an 8-wide wall of unit
    squares (spacing 1.1) facing -y, gentle random relief, weights log-uniform
    in [1e-2, 1e2]; the first `collapsed` patches have their u = 0 edge
    collapsed to one point (a degenerate, triangle-like net).  Returns
    (cp (n*64, 4) float32 weighted-homogeneous, offsets, degrees)."""
    rng = np.random.default_rng(seed)
    p = q = 7
    cps, off, deg = [], [], []
    cols = 8
    for k in range(n_patches):
        ix, iz = k % cols, k // cols
        g = np.linspace(0.0, 1.0, p + 1)
        X, Z = np.meshgrid(g, g, indexing="ij")
        Y = 0.15 * rng.normal(size=X.shape)
        xyz = np.stack([X + 1.1 * ix - 0.55 * cols, Y, Z + 1.1 * iz - 0.55 * (n_patches // cols)], -1)
        if k < collapsed:
            xyz[0, :, :] = xyz[0, (q + 1) // 2, :]  # the whole u = 0 row at one point
        w = 10.0 ** rng.uniform(-2.0, 2.0, (p + 1) * (q + 1))
        cps.append(_homogeneous(xyz.reshape(-1, 3), w))
        off.append(k * (p + 1) * (q + 1))
        deg.append((p, q))
    return np.concatenate(cps), np.array(off, np.int32), np.array(deg, np.int32)


def precision_camera(width: int = 3840, height: int = 2160, seed: int = 5) -> Camera:
    """A pinhole camera in front of the precision wall (pixel-centre rays)."""
    return Camera((0.3, -7.0, 0.4), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 40.0, width, height, 1, seed)


def grazing_rays(cp: np.ndarray, off: np.ndarray, deg: np.ndarray, m: int, seed: int = 5, max_deg: float = 2.0):
    """m rays within max_deg degrees of a patch's tangent plane: a surface point
    S is drawn (random patch, (u, v) in [0.05, 0.95]^2, FP64), a direction d
    at U(0, max_deg) degrees from a random tangent direction towards the
    patch's front (-y) side, and the origin backed off along it by U(1, 3):
    O = S - L d.  Returns float32 arrays (ox, oy, oz, dx, dy, dz)."""
    rng = np.random.default_rng(seed + 1000)
    k = rng.integers(0, len(off), m)
    p, q = int(deg[0, 0]), int(deg[0, 1])
    n_pts = (p + 1) * (q + 1)
    blocks = np.stack([cp[off[i]:off[i] + n_pts] for i in range(len(off))])[k]
    u = rng.uniform(0.05, 0.95, m)
    v = rng.uniform(0.05, 0.95, m)
    S, Su, Sv = patch_points(blocks.reshape(m, -1), p, q, u, v)
    nrm = np.cross(Su, Sv)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True) + 1e-300
    nrm *= np.where(nrm[:, 1:2] > 0, -1.0, 1.0)  # towards the front (-y)
    t1 = Su / (np.linalg.norm(Su, axis=1, keepdims=True) + 1e-300)
    t2 = np.cross(nrm, t1)
    phi = rng.uniform(0.0, 2.0 * np.pi, m)[:, None]
    tang = np.cos(phi) * t1 + np.sin(phi) * t2
    a = np.radians(rng.uniform(0.0, max_deg, m))[:, None]
    d = np.cos(a) * tang - np.sin(a) * nrm  # enters the surface from the front
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    L = rng.uniform(1.0, 3.0, m)[:, None]
    o = S - L * d
    return tuple(np.ascontiguousarray(x, np.float32) for x in (o[:, 0], o[:, 1], o[:, 2], d[:, 0], d[:, 1], d[:, 2]))


def precision_workload(width: int = 3840, height: int = 2160, seed: int = 5, grazing: float = 0.25):
    """The precision-stress workload: the patches of precision_patches, camera
    rays of precision_camera with every round(1/grazing)-th ray replaced by a
    grazing ray.  Returns (patches (cp, off, deg), rays as 6 float32 CUDA
    tensors, indices of the grazing rays)."""
    import torch

    from . import lib_module as L

    cp, off, deg = precision_patches(seed)
    rays = L.camera_rays(precision_camera(width, height, seed))
    n = rays[0].numel()
    step = max(1, int(round(1.0 / grazing)))
    idx = np.arange(0, n, step)
    g = grazing_rays(cp, off, deg, idx.size, seed)
    ti = torch.from_numpy(idx).to(rays[0].device)
    for a, b in zip(rays, g):
        a[ti] = torch.from_numpy(b).to(a.device)
    return (cp, off, deg), rays, idx
