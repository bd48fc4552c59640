"""Python binding of libnrt.so (the engine's C ABI, include/nrt.h).

This module is plumbing for tests, benchmarks and Python users: device
buffers are torch CUDA tensors whose pointers are handed to the C ABI, and
every compute call goes to the CUDA kernels in libnrt.so.  There is no CPU
fallback: if the library or a GPU is missing, calls raise.
"""
from . import lib as lib_module  # noqa: F401
from .lib import (  # noqa: F401
    BuildOpts,
    Camera,
    Counters,
    IntersectOpts,
    Mlp,
    NrtError,
    Scene,
    bounce_rays,
    build_bvh_binary,
    camera_rays,
    compare_hits,
    decompose,
    default_opts,
    lib,
    lib_path,
    patch_bounds,
    reference_opts,
    shade,
    write_ppm,
    refine,
    refine_device,
    INIT_BILINEAR,
    INIT_LEARNED,
    INIT_MIDPOINT,
    SCHED_PIXEL,
    SCHED_WAVEFRONT,
    BVH_BINNED_SAH,
    BVH_EXACT_SAH,
    BVH_BINNED_SAH_DEVICE,
)
