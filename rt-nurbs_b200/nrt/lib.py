"""ctypes declarations of include/nrt.h and thin Python wrappers."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))  # rt-nurbs_b200/
_LIB = None

INIT_MIDPOINT, INIT_BILINEAR, INIT_LEARNED = 0, 1, 2
SCHED_PIXEL, SCHED_WAVEFRONT = 0, 1
BVH_BINNED_SAH, BVH_EXACT_SAH, BVH_BINNED_SAH_DEVICE = 0, 1, 2


class NrtError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"nrt error {status}: {msg}")
        self.status = status


class NurbsSurface(C.Structure):
    _fields_ = [("control_points", C.c_void_p), ("u_knots", C.c_void_p), ("v_knots", C.c_void_p),
                ("n", C.c_int), ("m", C.c_int), ("p", C.c_int), ("q", C.c_int)]


class BuildOpts(C.Structure):
    _fields_ = [("builder", C.c_int), ("max_leaf", C.c_int), ("device", C.c_int), ("wavefront_chunk", C.c_int64)]


class SceneInfo(C.Structure):
    _fields_ = [("n_patches", C.c_int), ("n_surfaces", C.c_int), ("n_nodes", C.c_int), ("bvh_depth", C.c_int),
                ("device_bytes", C.c_size_t), ("degree_hist", C.c_int * 64)]


class RaysC(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("ox", "oy", "oz", "dx", "dy", "dz")]


class HitsC(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("patch", "t", "u", "v", "iters", "tests", "geom")]


class IntersectOpts(C.Structure):
    _fields_ = [("init_mode", C.c_int), ("max_iter", C.c_int), ("eps", C.c_float), ("det_eps", C.c_float),
                ("cond_fp64", C.c_float), ("fp64_final", C.c_int), ("hull_cull", C.c_int), ("schedule", C.c_int),
                ("seed_offset", C.c_int), ("flat_threshold", C.c_float), ("cam_k", C.c_float),
                ("learned_iters", C.c_int)]

    def replace(self, **kw) -> "IntersectOpts":
        o = IntersectOpts()
        C.pointer(o)[0] = self
        for k, v in kw.items():
            setattr(o, k, v)
        return o

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_COUNTER_NAMES = ("rays", "box_tests", "patch_candidates", "patch_culled", "newton_solves", "newton_evals",
                  "fp64_solves", "fp64_final_steps", "hits", "errors", "learned_solves", "learned_fallbacks")


class Counters(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in _COUNTER_NAMES] + [("evals_by_degree", C.c_uint64 * 64),
                                                            ("hull_tests_by_degree", C.c_uint64 * 64),
                                                            ("kernel_launches", C.c_uint64), ("rounds", C.c_uint64),
                                                            ("newton_kernel_ms", C.c_double),
                                                            ("newton_kernel_launches", C.c_uint64),
                                                            ("flat_skips", C.c_uint64),
                                                            ("learned_converged", C.c_uint64),
                                                            ("learned_fallback_converged", C.c_uint64)]

    def as_dict(self) -> dict:
        d = {k: int(getattr(self, k)) for k in _COUNTER_NAMES}
        d["evals_by_degree"] = {(k // 8, k % 8): int(v) for k, v in enumerate(self.evals_by_degree) if v}
        d["hull_tests_by_degree"] = {(k // 8, k % 8): int(v) for k, v in enumerate(self.hull_tests_by_degree) if v}
        d["kernel_launches"] = int(self.kernel_launches)
        d["rounds"] = int(self.rounds)
        d["newton_kernel_ms"] = float(self.newton_kernel_ms)
        d["newton_kernel_launches"] = int(self.newton_kernel_launches)
        d["flat_skips"] = int(self.flat_skips)
        d["learned_converged"] = int(self.learned_converged)
        d["learned_fallback_converged"] = int(self.learned_fallback_converged)
        return d


class Tuning(C.Structure):
    _fields_ = [("step_blocks", C.c_int64), ("scatter_blocks", C.c_int64), ("class_blocks", C.c_int32),
                ("graph", C.c_int32), ("chunk", C.c_int64), ("quota0", C.c_int32), ("quota_max", C.c_int32),
                ("stage_nodes", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TrainOpts(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("seed", C.c_uint32)]


class CameraC(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("look", C.c_float * 3), ("up", C.c_float * 3), ("fov_deg", C.c_float),
                ("width", C.c_int), ("height", C.c_int), ("spp", C.c_int), ("seed", C.c_uint32)]


def lib_path() -> str:
    return os.path.join(PKG, "lib", "libnrt.so")


def lib():
    """Load libnrt.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise NrtError(-1, f"{path} is missing: build it with `make -C rt-nurbs_b200` (or __graft_entry__.build())")
        L = C.CDLL(path)
        vp = C.c_void_p
        L.nrt_last_error.restype = C.c_char_p
        L.nrt_version.restype = C.c_char_p
        L.nrt_decompose_count.argtypes = [C.POINTER(NurbsSurface), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.nrt_decompose.argtypes = [C.POINTER(NurbsSurface), vp, vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.nrt_patch_bounds.argtypes = [vp, vp, vp, C.c_int, vp]
        L.nrt_build_bvh_binary.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp, C.POINTER(C.c_int)]
        L.nrt_scene_create.argtypes = [C.POINTER(NurbsSurface), C.c_int, C.POINTER(BuildOpts), C.POINTER(vp)]
        L.nrt_scene_create_from_patches.argtypes = [vp, vp, vp, C.c_int, C.POINTER(BuildOpts), C.POINTER(vp)]
        L.nrt_scene_destroy.argtypes = [vp]
        L.nrt_scene_get_info.argtypes = [vp, C.POINTER(SceneInfo)]
        L.nrt_scene_patch_table.argtypes = [vp, vp, vp]
        L.nrt_scene_copy_arena.argtypes = [vp, vp, C.c_size_t]
        L.nrt_default_opts.argtypes = [C.POINTER(IntersectOpts)]
        L.nrt_default_opts.restype = None
        L.nrt_reference_opts.argtypes = [C.POINTER(IntersectOpts)]
        L.nrt_reference_opts.restype = None
        L.nrt_intersect.argtypes = [vp, C.POINTER(RaysC), C.c_int64, C.POINTER(IntersectOpts), C.POINTER(HitsC), vp]
        L.nrt_enable_counters.argtypes = [vp, C.c_int]
        L.nrt_enable_kernel_timing.argtypes = [vp, C.c_int]
        L.nrt_scene_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.nrt_scene_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.nrt_autotune.argtypes = [vp, C.POINTER(RaysC), C.c_int64, C.POINTER(IntersectOpts), C.POINTER(HitsC), C.c_int,
                                   C.POINTER(Tuning), C.POINTER(C.c_float), vp]
        L.nrt_get_counters.argtypes = [vp, C.POINTER(Counters), vp]
        L.nrt_generate_camera_rays.argtypes = [C.POINTER(CameraC), C.POINTER(RaysC), vp]
        L.nrt_shade.argtypes = [C.POINTER(HitsC), C.c_int64, C.c_int, vp, vp, vp, vp]
        L.nrt_compare_hits.argtypes = [C.POINTER(RaysC), C.POINTER(HitsC), C.POINTER(HitsC), C.c_int64, C.c_float, vp,
                                       vp, vp, vp]
        L.nrt_write_ppm.argtypes = [C.c_char_p, C.c_int, C.c_int, vp, vp, vp]
        L.nrt_refine_count.argtypes = [C.POINTER(NurbsSurface), C.c_float, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.nrt_refine_surface.argtypes = [C.POINTER(NurbsSurface), C.c_float, vp, vp, vp, C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]
        L.nrt_refine_surface_device.argtypes = [C.POINTER(NurbsSurface), C.c_float, C.c_int, vp, C.c_int64, vp, C.c_int,
                                                vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.nrt_bounce_scratch_bytes.argtypes = [C.c_int64]
        L.nrt_bounce_scratch_bytes.restype = C.c_size_t
        L.nrt_generate_bounce_rays.argtypes = [C.POINTER(RaysC), C.POINTER(HitsC), C.c_int64, C.c_uint32, C.c_float,
                                               C.POINTER(RaysC), vp, C.POINTER(C.c_int64), vp, vp]
        L.nrt_mlp_param_count.restype = C.c_size_t
        L.nrt_mlp_create.argtypes = [C.c_int, C.c_uint32, C.POINTER(vp)]
        L.nrt_mlp_destroy.argtypes = [vp]
        L.nrt_mlp_get_params.argtypes = [vp, vp]
        L.nrt_mlp_set_params.argtypes = [vp, vp]
        L.nrt_mlp_forward.argtypes = [vp, vp, C.c_int64, vp, vp]
        L.nrt_mlp_gradients.argtypes = [vp, vp, vp, C.c_int64, vp, C.POINTER(C.c_float), vp]
        L.nrt_mlp_train.argtypes = [vp, vp, vp, C.c_int64, C.POINTER(TrainOpts), vp, vp]
        L.nrt_mlp_save.argtypes = [vp, C.c_char_p]
        L.nrt_mlp_load.argtypes = [C.c_char_p, C.c_int, C.POINTER(vp)]
        L.nrt_scene_set_mlp.argtypes = [vp, vp]
        L.nrt_collect_training_data.argtypes = [vp, C.POINTER(RaysC), C.c_int64, C.POINTER(IntersectOpts), vp, vp,
                                                C.c_int64, C.POINTER(C.c_int64), vp]
        L.nrt_intersect_noalloc.argtypes = [vp, C.POINTER(RaysC), C.c_int64, C.POINTER(IntersectOpts),
                                            C.POINTER(HitsC), vp]
        _LIB = L
    return _LIB


def _check(status: int):
    if status != 0:
        raise NrtError(status, lib().nrt_last_error().decode())


def default_opts(**kw) -> IntersectOpts:
    o = IntersectOpts()
    lib().nrt_default_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def reference_opts(**kw) -> IntersectOpts:
    o = IntersectOpts()
    lib().nrt_reference_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _surface_struct(s):
    cp = np.ascontiguousarray(s.cp, np.float32)
    U = np.ascontiguousarray(s.U, np.float32)
    V = np.ascontiguousarray(s.V, np.float32)
    st = NurbsSurface(cp.ctypes.data, U.ctypes.data, V.ctypes.data, s.n, s.m, s.p, s.q)
    return st, (cp, U, V)


def refine(s, c: float):
    """nrt_refine_surface: the surface after curvature-driven knot insertion with
    constant c (a scenes.Surface)."""
    from .scenes import Surface

    L = lib()
    st, keep = _surface_struct(s)
    n, m = C.c_int(), C.c_int()
    _check(L.nrt_refine_count(C.byref(st), float(c), C.byref(n), C.byref(m)))
    cp = np.zeros(((n.value + 1) * (m.value + 1), 4), np.float32)
    U = np.zeros(n.value + s.p + 2, np.float32)
    V = np.zeros(m.value + s.q + 2, np.float32)
    _check(L.nrt_refine_surface(C.byref(st), float(c), cp.ctypes.data, U.ctypes.data, V.ctypes.data, C.byref(n),
                                C.byref(m)))
    return Surface(cp, U, V, n.value, m.value, s.p, s.q)


def refine_device(s, c: float, device: int = 0):
    """nrt_refine_surface_device: the same refinement computed on the GPU."""
    from .scenes import Surface

    L = lib()
    st, keep = _surface_struct(s)
    n, m = C.c_int(), C.c_int()
    rc = L.nrt_refine_surface_device(C.byref(st), float(c), int(device), None, 0, None, 0, None, 0, C.byref(n),
                                     C.byref(m))
    if rc not in (0, 1) or n.value < 0:
        _check(rc)
    cp = np.zeros(((n.value + 1) * (m.value + 1), 4), np.float32)
    U = np.zeros(n.value + s.p + 2, np.float32)
    V = np.zeros(m.value + s.q + 2, np.float32)
    _check(L.nrt_refine_surface_device(C.byref(st), float(c), int(device), cp.ctypes.data, cp.shape[0],
                                       U.ctypes.data, U.size, V.ctypes.data, V.size, C.byref(n), C.byref(m)))
    return Surface(cp, U, V, n.value, m.value, s.p, s.q)


def decompose(s):
    """Host decomposition of one surface: (cp (P,4) float32, ranges (N,4), (nbU, nbV))."""
    L = lib()
    st, keep = _surface_struct(s)
    nu, nv = C.c_int(), C.c_int()
    _check(L.nrt_decompose_count(C.byref(st), C.byref(nu), C.byref(nv)))
    N = nu.value * nv.value
    cp = np.zeros((N * (s.p + 1) * (s.q + 1), 4), np.float32)
    ranges = np.zeros((N, 4), np.float32)
    _check(L.nrt_decompose(C.byref(st), cp.ctypes.data, ranges.ctypes.data, C.byref(nu), C.byref(nv)))
    return cp, ranges, (nu.value, nv.value)


def patch_bounds(cp, off, deg) -> np.ndarray:
    cp = np.ascontiguousarray(cp, np.float32)
    off = np.ascontiguousarray(off, np.int32)
    deg = np.ascontiguousarray(deg, np.int32)
    out = np.zeros((off.shape[0], 6), np.float32)
    _check(lib().nrt_patch_bounds(cp.ctypes.data, off.ctypes.data, deg.ctypes.data, off.shape[0], out.ctypes.data))
    return out


def build_bvh_binary(boxes, builder=BVH_EXACT_SAH):
    boxes = np.ascontiguousarray(boxes, np.float32)
    N = boxes.shape[0]
    M = 2 * N - 1
    nb = np.zeros((M, 6), np.float32)
    lf = np.zeros(M, np.uint32)
    cnt = np.zeros(M, np.uint32)
    order = np.zeros(N, np.int32)
    used = C.c_int()
    _check(lib().nrt_build_bvh_binary(boxes.ctypes.data, N, builder, nb.ctypes.data, lf.ctypes.data,
                                      cnt.ctypes.data, order.ctypes.data, C.byref(used)))
    return nb, lf, cnt, order, used.value


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        import torch

        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Scene:
    """A device scene (decomposition + BVH + upload), nrt_scene_create."""

    def __init__(self, surfaces=None, patches=None, builder=BVH_BINNED_SAH, max_leaf=1, device=0, wavefront_chunk=0):
        L = lib()
        self._h = C.c_void_p()
        opts = BuildOpts(builder, max_leaf, device, wavefront_chunk)
        if surfaces is not None:
            arr = (NurbsSurface * len(surfaces))()
            keep = []
            for i, s in enumerate(surfaces):
                st, k = _surface_struct(s)
                arr[i] = st
                keep.append(k)
            _check(L.nrt_scene_create(arr, len(surfaces), C.byref(opts), C.byref(self._h)))
        else:
            cp, off, deg = (np.ascontiguousarray(patches[0], np.float32), np.ascontiguousarray(patches[1], np.int32),
                            np.ascontiguousarray(patches[2], np.int32))
            _check(L.nrt_scene_create_from_patches(cp.ctypes.data, off.ctypes.data, deg.ctypes.data, off.shape[0],
                                                   C.byref(opts), C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().nrt_scene_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        inf = SceneInfo()
        _check(lib().nrt_scene_get_info(self._h, C.byref(inf)))
        hist = {(k // 8, k % 8): int(v) for k, v in enumerate(inf.degree_hist) if v}
        return {"n_patches": inf.n_patches, "n_surfaces": inf.n_surfaces, "n_nodes": inf.n_nodes,
                "bvh_depth": inf.bvh_depth, "device_bytes": int(inf.device_bytes), "degree_hist": hist}

    def arena(self) -> np.ndarray:
        """The scene's device arena as host bytes (nrt_scene_copy_arena)."""
        out = np.zeros(self.info()["device_bytes"], np.uint8)
        _check(lib().nrt_scene_copy_arena(self._h, out.ctypes.data, out.nbytes))
        return out

    def patch_table(self):
        n = self.info()["n_patches"]
        surf = np.zeros(n, np.int32)
        ranges = np.zeros((n, 4), np.float32)
        _check(lib().nrt_scene_patch_table(self._h, surf.ctypes.data, ranges.ctypes.data))
        return surf, ranges

    def enable_counters(self, on=True):
        _check(lib().nrt_enable_counters(self._h, int(on)))

    def counters(self, stream=None) -> dict:
        c = Counters()
        _check(lib().nrt_get_counters(self._h, C.byref(c), _stream_ptr(stream)))
        return c.as_dict()

    def enable_kernel_timing(self, on=True):
        _check(lib().nrt_enable_kernel_timing(self._h, int(on)))

    def tuning(self) -> dict:
        t = Tuning()
        _check(lib().nrt_scene_get_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        """Wavefront launch shapes (nrt_scene_set_tuning); unspecified fields are kept."""
        t = Tuning(**{k: int(v) for k, v in kw.items()})
        _check(lib().nrt_scene_set_tuning(self._h, C.byref(t)))

    def autotune(self, rays, opts: IntersectOpts | None = None, out=None, reps=3, stream=None):
        """nrt_autotune on these rays: keeps the fastest wavefront launch shapes on
        the scene; returns (tuning dict, ms per call)."""
        import torch

        opts = opts or default_opts(schedule=SCHED_WAVEFRONT)
        n = rays[0].numel()
        if out is None:
            out = {k: torch.empty(n, dtype=torch.int32 if k == "patch" else torch.float32, device=rays[0].device)
                   for k in ("patch", "t", "u", "v")}
        r = RaysC(*[C.c_void_p(a.data_ptr()) for a in rays])
        h = HitsC(_ptr(out["patch"]), _ptr(out["t"]), _ptr(out["u"]), _ptr(out["v"]), _ptr(out.get("iters")),
                  _ptr(out.get("tests")), _ptr(out.get("geom")))
        t, ms = Tuning(), C.c_float()
        _check(lib().nrt_autotune(self._h, C.byref(r), n, C.byref(opts), C.byref(h), int(reps), C.byref(t),
                                  C.byref(ms), _stream_ptr(stream)))
        return t.as_dict(), float(ms.value)

    def set_mlp(self, mlp: "Mlp"):
        _check(lib().nrt_scene_set_mlp(self._h, mlp.handle))

    def collect_training_data(self, rays, opts: IntersectOpts | None = None, capacity=None, stream=None):
        """(features (m,12), targets (m,2)) CUDA tensors of converged plain-Newton solves."""
        import torch

        if opts is None:
            opts = default_opts(schedule=SCHED_WAVEFRONT)
        n = rays[0].numel()
        cap = int(capacity if capacity is not None else 16 * n)
        feat = torch.empty((cap, 12), dtype=torch.float32, device=rays[0].device)
        targ = torch.empty((cap, 2), dtype=torch.float32, device=rays[0].device)
        cnt = C.c_int64()
        r = RaysC(*[C.c_void_p(a.data_ptr()) for a in rays])
        _check(lib().nrt_collect_training_data(self._h, C.byref(r), n, C.byref(opts), C.c_void_p(feat.data_ptr()),
                                               C.c_void_p(targ.data_ptr()), cap, C.byref(cnt), _stream_ptr(stream)))
        m = min(cnt.value, cap)
        return feat[:m], targ[:m], cnt.value

    def intersect(self, rays, opts: IntersectOpts | None = None, out=None, stream=None, geom=False, extra=True):
        """rays: 6 float32 CUDA tensors (ox, oy, oz, dx, dy, dz).  Returns a dict of CUDA tensors."""
        import torch

        if opts is None:
            opts = default_opts()
        n = rays[0].numel()
        dev = rays[0].device
        if out is None:
            out = {"patch": torch.empty(n, dtype=torch.int32, device=dev),
                   "t": torch.empty(n, dtype=torch.float32, device=dev),
                   "u": torch.empty(n, dtype=torch.float32, device=dev),
                   "v": torch.empty(n, dtype=torch.float32, device=dev)}
            if extra:
                out["iters"] = torch.empty(n, dtype=torch.int32, device=dev)
                out["tests"] = torch.empty(n, dtype=torch.int32, device=dev)
            if geom:
                out["geom"] = torch.empty((n, 9), dtype=torch.float32, device=dev)
        r = RaysC(*[C.c_void_p(a.data_ptr()) for a in rays])
        h = HitsC(_ptr(out["patch"]), _ptr(out["t"]), _ptr(out["u"]), _ptr(out["v"]), _ptr(out.get("iters")),
                  _ptr(out.get("tests")), _ptr(out.get("geom")))
        _check(lib().nrt_intersect(self._h, C.byref(r), n, C.byref(opts), C.byref(h), _stream_ptr(stream)))
        return out


def bounce_rays(rays, hits, seed=0, offset=1e-4, out=None, stream=None):
    """nrt_generate_bounce_rays: (6 ray tensors of length m, source-index tensor, m) for the
    rays that hit; hits must carry "geom" (intersect(..., geom=True))."""
    import torch

    n = rays[0].numel()
    dev = rays[0].device
    if out is None:
        out = [torch.empty(n, dtype=torch.float32, device=dev) for _ in range(6)]
        src = torch.empty(n, dtype=torch.int32, device=dev)
    else:
        out, src = out
    scratch = torch.empty(max(1, int(lib().nrt_bounce_scratch_bytes(n))), dtype=torch.uint8, device=dev)
    r = RaysC(*[C.c_void_p(a.data_ptr()) for a in rays])
    h = HitsC(_ptr(hits["patch"]), _ptr(hits["t"]), _ptr(hits["u"]), _ptr(hits["v"]), None, None, _ptr(hits["geom"]))
    o = RaysC(*[C.c_void_p(a.data_ptr()) for a in out])
    m = C.c_int64()
    _check(lib().nrt_generate_bounce_rays(C.byref(r), C.byref(h), n, int(seed) & 0xFFFFFFFF, float(offset), C.byref(o),
                                          _ptr(src), C.byref(m), _ptr(scratch), _stream_ptr(stream)))
    k = int(m.value)
    return [a[:k] for a in out], src[:k], k


def _hits_struct(h):
    return HitsC(_ptr(h["patch"]), _ptr(h["t"]), _ptr(h["u"]), _ptr(h["v"]), _ptr(h.get("iters")),
                 _ptr(h.get("tests")), _ptr(h.get("geom")))


def shade(hits, mode=1, stream=None):
    """nrt_shade: (r, g, b) float32 CUDA tensors; mode 0 hit mask, 1 normal map."""
    import torch

    n = hits["patch"].numel()
    rgb = [torch.empty(n, dtype=torch.float32, device=hits["patch"].device) for _ in range(3)]
    h = _hits_struct(hits)
    _check(lib().nrt_shade(C.byref(h), n, int(mode), *[_ptr(a) for a in rgb], _stream_ptr(stream)))
    return rgb


def compare_hits(rays, ref, test, cam_k, stream=None):
    """nrt_compare_hits: (pixel error, normal angle in degrees, mismatch) CUDA tensors per ray."""
    import torch

    n = ref["patch"].numel()
    dev = ref["patch"].device
    px, deg = torch.empty(n, device=dev), torch.empty(n, device=dev)
    mm = torch.empty(n, dtype=torch.int32, device=dev)
    r = RaysC(*[C.c_void_p(a.data_ptr()) for a in rays])
    a, b = _hits_struct(ref), _hits_struct(test)
    _check(lib().nrt_compare_hits(C.byref(r), C.byref(a), C.byref(b), n, float(cam_k), _ptr(px), _ptr(deg), _ptr(mm),
                                  _stream_ptr(stream)))
    return px, deg, mm


def write_ppm(path, width, height, r, g, b):
    """nrt_write_ppm from host float arrays (numpy) in [0, 1]."""
    arrs = [np.ascontiguousarray(x, np.float32) for x in (r, g, b)]
    _check(lib().nrt_write_ppm(str(path).encode(), int(width), int(height), *[a.ctypes.data for a in arrs]))


class Camera(CameraC):
    pass


def camera_rays(cam, device="cuda", stream=None):
    """Primary rays for a scenes.Camera as 6 CUDA tensors."""
    import torch

    c = CameraC((C.c_float * 3)(*cam.eye), (C.c_float * 3)(*cam.look), (C.c_float * 3)(*cam.up), cam.fov_deg,
                cam.width, cam.height, cam.spp, cam.seed)
    n = cam.width * cam.height * cam.spp
    arrs = [torch.empty(n, dtype=torch.float32, device=device) for _ in range(6)]
    r = RaysC(*[C.c_void_p(a.data_ptr()) for a in arrs])
    _check(lib().nrt_generate_camera_rays(C.byref(c), C.byref(r), _stream_ptr(stream)))
    return arrs


class Mlp:
    """The learned-initial-guess network (nrt_mlp_*)."""

    N_PARAMS = 5122

    def __init__(self, seed=0, device=0, handle=None):
        self._h = C.c_void_p()
        if handle is not None:
            self._h = handle
        else:
            _check(lib().nrt_mlp_create(device, seed, C.byref(self._h)))

    @classmethod
    def load(cls, path, device=0):
        h = C.c_void_p()
        _check(lib().nrt_mlp_load(str(path).encode(), device, C.byref(h)))
        return cls(handle=h)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().nrt_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.zeros(self.N_PARAMS, np.float32)
        _check(lib().nrt_mlp_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, theta):
        theta = np.ascontiguousarray(theta, np.float32)
        assert theta.size == self.N_PARAMS
        _check(lib().nrt_mlp_set_params(self._h, theta.ctypes.data))

    def forward(self, features, stream=None):
        import torch

        n = features.shape[0]
        out = torch.empty((n, 2), dtype=torch.float32, device=features.device)
        _check(lib().nrt_mlp_forward(self._h, C.c_void_p(features.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                     _stream_ptr(stream)))
        return out

    def gradients(self, features, targets, stream=None):
        g = np.zeros(self.N_PARAMS, np.float32)
        loss = C.c_float()
        _check(lib().nrt_mlp_gradients(self._h, C.c_void_p(features.data_ptr()), C.c_void_p(targets.data_ptr()),
                                       features.shape[0], g.ctypes.data, C.byref(loss), _stream_ptr(stream)))
        return float(loss.value), g

    def train(self, features, targets, epochs=20, batch=4096, lr=1e-3, seed=0, stream=None):
        losses = np.zeros(epochs, np.float32)
        o = TrainOpts(epochs, batch, lr, 0.0, 0.0, 0.0, seed)
        _check(lib().nrt_mlp_train(self._h, C.c_void_p(features.data_ptr()), C.c_void_p(targets.data_ptr()),
                                   features.shape[0], C.byref(o), losses.ctypes.data, _stream_ptr(stream)))
        return losses

    def save(self, path):
        _check(lib().nrt_mlp_save(self._h, str(path).encode()))
