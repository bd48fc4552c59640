"""Python binding of the test oracle (TEST INFRASTRUCTURE ONLY).

Two CPU implementations of the reference's intersection path sit behind this
module:

* ``liboracle.so`` (oracle/oracle.cpp): this project's restatement of the
  reference path, in float (reference order of operations) and in double (the
  FP64 oracle).  It builds anywhere (``make -C oracle``).
* ``_ref/libnrt_ref_it{7,8}.so`` (oracle/ref_driver.cpp): the reference's own
  host-compilable functions compiled from its sources, used to pin the
  restatement.  It exists only where the reference sources were present at
  build time (``make -C oracle ref``).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this
module, and only to check (or to time the CPU baseline); the product library
never calls it.
"""
from __future__ import annotations

import ctypes as C
import ctypes as C_
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


class OrcOpts(C.Structure):
    _fields_ = [("init_mode", C.c_int), ("max_iter", C.c_int), ("eps", C.c_float), ("det_eps", C.c_float),
                ("flat_threshold", C.c_float), ("cam_k", C.c_float)]


def reference_dir() -> str:
    """The reference checkout whose sources `make ref` compiles: $NRT_REFERENCE,
    else the build container's mount point (absent on the GPU hosts, where the
    prebuilt _ref libraries are used)."""
    return os.environ.get("NRT_REFERENCE", "/root/reference")


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and, if ref and the reference sources exist, the _ref libraries)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and os.path.isdir(os.path.join(reference_dir(), "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"NRT_REFERENCE={reference_dir()}"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_patch_grid.argtypes = [f32p, f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]
        L.orc_decompose.argtypes = [f32p, f32p, f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
        L.orc_patch_boxes.argtypes = [f32p, i32p, i32p, C.c_int, f32p]
        L.orc_build_bvh.argtypes = [f32p, C.c_int, f32p, u32p, u32p, i32p]
        L.orc_build_bvh.restype = C.c_int
        L.orc_build_bvh_binned.argtypes = [f32p, C.c_int, C.c_int, f32p, u32p, u32p, i32p]
        L.orc_build_bvh_binned.restype = C.c_int
        L.orc_roots_f64.argtypes = [f64p, i32p, i32p, f32p, C.c_int] + [f32p] * 6 + [
            C.c_long, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, i32p, f64p, f64p, f64p,
            C.c_void_p]
        common = [i32p, i32p, C.c_void_p, f32p, u32p, u32p, i32p, f32p, f32p, f32p, f32p, f32p, f32p, C.c_long,
                  C.POINTER(OrcOpts), i32p]
        L.orc_intersect_f32.argtypes = [f32p] + common + [f32p, f32p, f32p, i32p, i32p, C.c_void_p,
                                                          C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
        L.orc_intersect_f64.argtypes = [f64p] + common + [f64p, f64p, f64p, i32p, i32p, C.c_void_p,
                                                          C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
        L.orc_newton_f32.argtypes = [f32p, C.c_int, C.c_int, f32p, f32p, C.c_float, C.c_float, C.c_float, C.c_float,
                                     C.c_uint32, C.c_int, f32p]
        L.orc_patch_eval_f64.argtypes = [f64p, C.c_int, C.c_int, C.c_double, C.c_double, f64p]
        L.orc_ray_planes_f32.argtypes = [f32p, f32p, f32p]
        L.orc_surface_point_f64.argtypes = [f32p, f32p, f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                            C.c_double, f64p]
        L.orc_camera_rays.argtypes = [f32p, f32p, f32p, C.c_float, C.c_int, C.c_int, C.c_int, C.c_uint32] + [f32p] * 6
        L.orc_patch_delta.argtypes = [f32p, i32p, i32p, C.c_int, f32p]
        _LIB = L
    return _LIB


def ref_available(iters: int = 7) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libnrt_ref_it{iters}.so"))


def ref_lib(iters: int = 7):
    if iters not in _REF:
        L = C.CDLL(os.path.join(HERE, "_ref", f"libnrt_ref_it{iters}.so"))
        L.ref_decompose.argtypes = [f32p, f32p, f32p, C.c_int, C.c_int, C.c_int, C.c_int, f32p, f32p]
        L.ref_decompose.restype = C.c_int
        L.ref_build_bvh.argtypes = [f32p, i32p, i32p, C.c_int, f32p, u32p, u32p, i32p]
        L.ref_camera_rays.argtypes = [f32p, f32p, f32p, C.c_float, C.c_int, C.c_int] + [f32p] * 6
        L.ref_intersect.argtypes = [f32p, i32p, i32p, C.c_void_p, C.c_int, f32p, u32p, u32p] + [f32p] * 6 + [
            C.c_long, C.c_float, C.c_float, C.c_int, C.c_float, i32p, f32p, f32p, f32p, C.c_void_p,
            C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
        L.ref_iterations.restype = C.c_int
        _REF[iters] = L
    return _REF[iters]


# ---------------------------------------------------------------------------
@dataclass
class Patches:
    """A flat set of Bezier patches: cp (P,4) points, off[k] = first point of
    patch k, deg[k] = (p, q), ranges[k] = (u0,u1,v0,v1), surf[k] = surface index.
    cp64 holds the same patches decomposed in double (FP64 oracle)."""
    cp: np.ndarray
    off: np.ndarray
    deg: np.ndarray
    ranges: np.ndarray
    surf: np.ndarray
    cp64: np.ndarray | None = None

    @property
    def n(self) -> int:
        return int(self.off.shape[0])

    def subset(self, order: np.ndarray) -> "Patches":
        """Patches re-ordered (e.g. into BVH order), points copied contiguously."""
        sizes = (self.deg[:, 0] + 1) * (self.deg[:, 1] + 1)
        new_off = np.zeros(len(order), np.int32)
        new_off[1:] = np.cumsum(sizes[order])[:-1]
        idx = np.concatenate([np.arange(self.off[k], self.off[k] + sizes[k]) for k in order]) if len(order) else []
        return Patches(np.ascontiguousarray(self.cp[idx]), new_off, np.ascontiguousarray(self.deg[order]),
                       np.ascontiguousarray(self.ranges[order]), np.ascontiguousarray(self.surf[order]),
                       None if self.cp64 is None else np.ascontiguousarray(self.cp64[idx]))


def decompose(surf, f64: bool = True):
    """(cp float32, cp float64 or None, ranges) of one surface, patch (i,j) at i*nbV+j."""
    L = lib()
    nbU, nbV = C.c_int(), C.c_int()
    L.orc_patch_grid(surf.U, surf.V, surf.n, surf.m, surf.p, surf.q, C.byref(nbU), C.byref(nbV))
    N = nbU.value * nbV.value
    piece = (surf.p + 1) * (surf.q + 1)
    cp = np.zeros((N * piece, 4), np.float32)
    cp64 = np.zeros((N * piece, 4), np.float64) if f64 else None
    ranges = np.zeros((N, 4), np.float32)
    L.orc_decompose(np.ascontiguousarray(surf.cp, np.float32), surf.U, surf.V, surf.n, surf.m, surf.p, surf.q,
                    cp.ctypes.data, None if cp64 is None else cp64.ctypes.data, ranges.ctypes.data)
    return cp, cp64, ranges, (nbU.value, nbV.value)


def decompose_scene(surfaces, f64: bool = True) -> Patches:
    cps, cp64s, rngs, degs, surf_ids, offs = [], [], [], [], [], []
    base = 0
    for s_idx, s in enumerate(surfaces):
        cp, cp64, ranges, (nu, nv) = decompose(s, f64)
        N = nu * nv
        piece = (s.p + 1) * (s.q + 1)
        cps.append(cp)
        if f64:
            cp64s.append(cp64)
        rngs.append(ranges)
        degs.append(np.tile(np.array([[s.p, s.q]], np.int32), (N, 1)))
        surf_ids.append(np.full(N, s_idx, np.int32))
        offs.append(base + piece * np.arange(N, dtype=np.int32))
        base += N * piece
    return Patches(np.ascontiguousarray(np.concatenate(cps)), np.concatenate(offs).astype(np.int32),
                   np.ascontiguousarray(np.concatenate(degs)), np.concatenate(rngs), np.concatenate(surf_ids),
                   np.ascontiguousarray(np.concatenate(cp64s)) if f64 else None)


def patch_boxes(P: Patches) -> np.ndarray:
    out = np.zeros((P.n, 6), np.float32)
    lib().orc_patch_boxes(P.cp, P.off, P.deg, P.n, out)
    return out


def patch_delta(P: Patches) -> np.ndarray:
    out = np.zeros(P.n, np.float32)
    lib().orc_patch_delta(P.cp, P.off, P.deg, P.n, out)
    return out


@dataclass
class BinaryBVH:
    box: np.ndarray     # (M, 6) float32
    lf: np.ndarray      # (M,) uint32
    cnt: np.ndarray     # (M,) uint32
    order: np.ndarray   # (N,) int32: BVH slot -> input patch index
    used: int


def build_bvh(boxes: np.ndarray) -> BinaryBVH:
    N = boxes.shape[0]
    M = max(2 * N - 1, 1)
    nb = np.zeros((M, 6), np.float32)
    lf = np.zeros(M, np.uint32)
    cnt = np.zeros(M, np.uint32)
    order = np.zeros(N, np.int32)
    used = lib().orc_build_bvh(np.ascontiguousarray(boxes, np.float32), N, nb, lf, cnt, order)
    return BinaryBVH(nb, lf, cnt, order, used)


def build_bvh_binned(boxes: np.ndarray, max_leaf: int = 1) -> BinaryBVH:
    """32-bin SAH binary BVH (the tree this project builds for scenes), from
    the oracle's own C restatement."""
    N = boxes.shape[0]
    M = max(2 * N - 1, 1)
    nb = np.zeros((M, 6), np.float32)
    lf = np.zeros(M, np.uint32)
    cnt = np.zeros(M, np.uint32)
    order = np.zeros(N, np.int32)
    used = lib().orc_build_bvh_binned(np.ascontiguousarray(boxes, np.float32), N, max_leaf, nb, lf, cnt, order)
    return BinaryBVH(nb, lf, cnt, order, used)


@dataclass
class Rays:
    ox: np.ndarray
    oy: np.ndarray
    oz: np.ndarray
    dx: np.ndarray
    dy: np.ndarray
    dz: np.ndarray

    @property
    def n(self) -> int:
        return int(self.ox.shape[0])

    def take(self, idx) -> "Rays":
        return Rays(*[np.ascontiguousarray(a[idx]) for a in (self.ox, self.oy, self.oz, self.dx, self.dy, self.dz)])

    def arrays(self):
        return (self.ox, self.oy, self.oz, self.dx, self.dy, self.dz)


def camera_rays(cam) -> Rays:
    R = cam.width * cam.height * cam.spp
    arr = [np.zeros(R, np.float32) for _ in range(6)]
    lib().orc_camera_rays(np.array(cam.eye, np.float32), np.array(cam.look, np.float32), np.array(cam.up, np.float32),
                          cam.fov_deg, cam.width, cam.height, cam.spp, cam.seed, *arr)
    return Rays(*arr)


@dataclass
class Hits:
    patch: np.ndarray   # input patch index, -1 = miss
    t: np.ndarray
    u: np.ndarray
    v: np.ndarray
    evals: np.ndarray   # Newton evaluations of the winning solve
    tests: np.ndarray   # (ray, patch) tests performed
    geo: np.ndarray | None
    newton_total: int
    skip_total: int


def intersect(P: Patches, bvh: BinaryBVH, rays: Rays, init_mode: int = 0, max_iter: int = 8, eps: float = 1e-6,
              det_eps: float = 1e-5, f64: bool = False, delta=None, flat_threshold: float = 0.0, cam_k: float = 0.0,
              geo: bool = False) -> Hits:
    """Closest hit by the reference traversal.  init_mode 0 = patch midpoint,
    1 = the reference's bilinear guess.  f64 runs the FP64 oracle."""
    L = lib()
    R = rays.n
    dt = np.float64 if f64 else np.float32
    hit = np.zeros(R, np.int32)
    t = np.zeros(R, dt)
    u = np.zeros(R, dt)
    v = np.zeros(R, dt)
    ev = np.zeros(R, np.int32)
    te = np.zeros(R, np.int32)
    g = np.zeros((R, 9), dt) if geo else None
    nc, sc = C.c_ulonglong(), C.c_ulonglong()
    opts = OrcOpts(init_mode, max_iter, eps, det_eps, flat_threshold, cam_k)
    delta_arr = None if delta is None else np.ascontiguousarray(delta, np.float32)
    if f64:
        if P.cp64 is None:
            raise ValueError("FP64 oracle needs patches decomposed with f64=True")
        fn, cp = L.orc_intersect_f64, P.cp64
    else:
        fn, cp = L.orc_intersect_f32, P.cp
    fn(cp, P.off, P.deg, None if delta_arr is None else delta_arr.ctypes.data, bvh.box, bvh.lf, bvh.cnt, bvh.order,
       *rays.arrays(), R, C.byref(opts), hit, t, u, v, ev, te, None if g is None else g.ctypes.data, C.byref(nc),
       C.byref(sc))
    return Hits(hit, t, u, v, ev, te, g, nc.value, sc.value)


@dataclass
class Roots:
    patch: np.ndarray   # nearest root's patch (input order), -1 = none
    t: np.ndarray
    u: np.ndarray
    v: np.ndarray
    n_roots: np.ndarray | None


def true_closest_hits(P: Patches, rays: Rays, grid: int = 4, max_iter: int = 40, eps: float = 1e-11) -> Roots:
    """Multi-start FP64 diagnostic: for every ray the nearest root over all
    patches whose box it crosses, from a grid x grid lattice of Newton starts
    plus the midpoint on each (double, eps on |r1|+|r2|), with the number of
    distinct roots found.  Needs P.cp64."""
    R = rays.n
    patch = np.zeros(R, np.int32)
    t, u, v = (np.zeros(R, np.float64) for _ in range(3))
    nr = np.zeros(R, np.int32)
    lib().orc_roots_f64(P.cp64, P.off, P.deg, patch_boxes(P), P.n, *rays.arrays(), R, grid, max_iter, eps, None,
                        None, None, patch, t, u, v, nr.ctypes.data)
    return Roots(patch, t, u, v, nr)


def polish_hits(P: Patches, rays: Rays, patch: np.ndarray, u0: np.ndarray, v0: np.ndarray, max_iter: int = 40,
                eps: float = 1e-11) -> Roots:
    """FP64 Newton on patch[i] from (u0[i], v0[i]) (patch < 0: skipped): the
    exact root next to a reported hit, or patch -1 where none is reached."""
    R = rays.n
    only = np.ascontiguousarray(patch, np.int32)
    a0 = np.ascontiguousarray(u0, np.float64)
    b0 = np.ascontiguousarray(v0, np.float64)
    out = np.zeros(R, np.int32)
    t, u, v = (np.zeros(R, np.float64) for _ in range(3))
    lib().orc_roots_f64(P.cp64, P.off, P.deg, patch_boxes(P), P.n, *rays.arrays(), R, 0, max_iter, eps,
                        only.ctypes.data, a0.ctypes.data, b0.ctypes.data, out, t, u, v, None)
    return Roots(out, t, u, v, None)


def newton_f32(cp: np.ndarray, p: int, q: int, o, d, u0=0.5, v0=0.5, det_eps=1e-5, eps=1e-6, seed=0, max_iter=8):
    out = np.zeros(11, np.float32)
    r = lib().orc_newton_f32(np.ascontiguousarray(cp, np.float32), p, q, np.asarray(o, np.float32),
                             np.asarray(d, np.float32), u0, v0, det_eps, eps, seed, max_iter, out)
    return r, out


def surface_point(surf, u: float, v: float) -> np.ndarray:
    out = np.zeros(3, np.float64)
    lib().orc_surface_point_f64(np.ascontiguousarray(surf.cp, np.float32), surf.U, surf.V, surf.n, surf.m, surf.p,
                                surf.q, u, v, out)
    return out


def patch_eval_f64(cp64: np.ndarray, p: int, q: int, u: float, v: float) -> np.ndarray:
    out = np.zeros(12, np.float64)
    lib().orc_patch_eval_f64(np.ascontiguousarray(cp64, np.float64), p, q, u, v, out)
    return out.reshape(3, 4)


# ---------------------------------------------------------------------------
# The reference's own code (oracle/_ref), for pinning the restatement.
def ref_refine(surf, C: float, iters: int = 7):
    """The reference's curvatureRefinementU then V (src/math/nurbs.h:289-486) on a copy
    of surf: (cp (P,4), U, V, n, m)."""
    L = ref_lib(iters)
    L.ref_refine.argtypes = [f32p, f32p, f32p, C_int := C_.c_int, C_int, C_int, C_int, C_.c_float, f32p, f32p, f32p,
                             C_.c_long, C_int, C_int, C_.POINTER(C_int), C_.POINTER(C_int)]
    cap_pts, cap_k = 1 << 21, 1 << 16
    cp = np.zeros((cap_pts, 4), np.float32)
    U = np.zeros(cap_k, np.float32)
    V = np.zeros(cap_k, np.float32)
    n, m = C_.c_int(), C_.c_int()
    rc = L.ref_refine(np.ascontiguousarray(surf.cp, np.float32), np.ascontiguousarray(surf.U, np.float32),
                      np.ascontiguousarray(surf.V, np.float32), surf.n, surf.m, surf.p, surf.q, float(C), cp, U, V,
                      cap_pts, cap_k, cap_k, C_.byref(n), C_.byref(m))
    if rc != 0:
        raise RuntimeError(f"ref_refine failed ({rc})")
    n, m = n.value, m.value
    return cp[:(n + 1) * (m + 1)].copy(), U[:n + surf.p + 2].copy(), V[:m + surf.q + 2].copy(), n, m


def ref_decompose(surf, iters: int = 7):
    L = ref_lib(iters)
    nbU, nbV = C.c_int(), C.c_int()
    lib().orc_patch_grid(surf.U, surf.V, surf.n, surf.m, surf.p, surf.q, C.byref(nbU), C.byref(nbV))
    N = nbU.value * nbV.value
    piece = (surf.p + 1) * (surf.q + 1)
    cp = np.zeros((N * piece, 4), np.float32)
    ranges = np.zeros((N, 4), np.float32)
    got = L.ref_decompose(np.ascontiguousarray(surf.cp, np.float32), surf.U, surf.V, surf.n, surf.m, surf.p, surf.q,
                          cp, ranges)
    assert got == N
    return cp, ranges


def ref_build_bvh(P: Patches, iters: int = 7) -> BinaryBVH:
    N = P.n
    M = 2 * N - 1
    nb = np.zeros((M, 6), np.float32)
    lf = np.zeros(M, np.uint32)
    cnt = np.zeros(M, np.uint32)
    order = np.zeros(N, np.int32)
    ref_lib(iters).ref_build_bvh(P.cp, P.off, P.deg, N, nb, lf, cnt, order)
    used = int(np.max(np.nonzero(np.any(nb != 0, axis=1) | (cnt != 0) | (lf != 0))[0]) + 1) if N > 1 else 1
    return BinaryBVH(nb, lf, cnt, order, used)


def ref_camera_rays(cam, iters: int = 7) -> Rays:
    R = cam.width * cam.height
    arr = [np.zeros(R, np.float32) for _ in range(6)]
    ref_lib(iters).ref_camera_rays(np.array(cam.eye, np.float32), np.array(cam.look, np.float32),
                                   np.array(cam.up, np.float32), cam.fov_deg, cam.width, cam.height, *arr)
    return Rays(*arr)


def ref_intersect(P_bvh: Patches, bvh: BinaryBVH, rays: Rays, bilinear_init: bool = True, eps: float = 1e-4,
                  iters: int = 7, delta=None, flat_threshold: float = 0.0, cam_k: float = 0.0, geo: bool = False):
    """The reference traversal over patches already in BVH order (P_bvh = P.subset(bvh.order)).
    Returns (hit slot, t, u, v, geo, newton_total, skip_total)."""
    L = ref_lib(iters)
    R = rays.n
    hit = np.zeros(R, np.int32)
    t = np.zeros(R, np.float32)
    u = np.zeros(R, np.float32)
    v = np.zeros(R, np.float32)
    g = np.zeros((R, 9), np.float32) if geo else None
    nc, sc = C.c_ulonglong(), C.c_ulonglong()
    delta_arr = None if delta is None else np.ascontiguousarray(delta, np.float32)
    L.ref_intersect(P_bvh.cp, P_bvh.off, P_bvh.deg, None if delta_arr is None else delta_arr.ctypes.data, P_bvh.n,
                    bvh.box, bvh.lf, bvh.cnt, *rays.arrays(), R, flat_threshold, cam_k, int(bilinear_init), eps, hit,
                    t, u, v, None if g is None else g.ctypes.data, C.byref(nc), C.byref(sc))
    return hit, t, u, v, g, nc.value, sc.value
