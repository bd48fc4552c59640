"""Autotuner front end: the launch shapes nrt_autotune picks, cached per
(GPU, scene statistics, ray count, options) in a JSON file.

    from nrt import autotune
    tuning, ms = autotune.tune(scene, rays, opts)   # sets the scene's tuning

The search itself runs in the library (nrt_autotune: CUDA-event timing of
candidate traversal/scatter grids, class-launch blocks and rays per pass, one
knob at a time; the rounds stay in the CUDA graph unless the caller chose
host-driven rounds).  The cache file is
NRT_TUNING_CACHE, else .tuning_cache.json beside this package.
"""
from __future__ import annotations

import hashlib
import json
import os

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def cache_path() -> str:
    return os.environ.get("NRT_TUNING_CACHE", os.path.join(PKG, ".tuning_cache.json"))


def key(scene, n_rays: int, opts) -> str:
    """GPU name, patch count, degree histogram, ray count and options."""
    import torch

    info = scene.info()
    degs = sorted((f"{p}x{q}", v) for (p, q), v in info.get("degree_hist", {}).items())
    hist = hashlib.sha1(json.dumps(degs).encode()).hexdigest()[:12]
    o = {k: (round(v, 9) if isinstance(v, float) else v) for k, v in opts.as_dict().items()}
    return json.dumps({"gpu": torch.cuda.get_device_name(), "patches": info["n_patches"], "degrees": hist,
                       "rays": int(n_rays), "opts": o}, sort_keys=True)


def load(path: str | None = None) -> dict:
    try:
        with open(path or cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def tune(scene, rays, opts, out=None, reps: int = 3, path: str | None = None, refresh: bool = False):
    """Sets the scene's wavefront tuning from the cache, or runs the autotuner
    and records its choice.  Returns (tuning dict, ms per call or None when
    the tuning came from the cache)."""
    path = path or cache_path()
    k = key(scene, rays[0].numel(), opts)
    cache = load(path)
    if not refresh and k in cache:
        scene.set_tuning(**cache[k])
        return cache[k], None
    tuning, ms = scene.autotune(rays, opts, out=out, reps=reps)
    cache[k] = tuning
    try:
        with open(path, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
    except OSError:
        pass  # a read-only location only loses the cache
    return tuning, ms
