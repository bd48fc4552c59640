"""Helpers shared by the GPU parity tests: run the CUDA path through the C ABI
and compare its hits with the oracle's."""
import numpy as np


def to_numpy(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


def gpu_rays(rays_np):
    import torch

    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in rays_np.arrays()]


def compare(gpu, patch_ref, t_ref, u_ref=None, v_ref=None):
    """Agreement statistics of GPU hits against a reference hit set.
    Returns hit/miss agreement, same-patch fraction among rays both hit, and
    relative t / absolute (u,v) errors over rays that hit the same patch."""
    gp = gpu["patch"]
    hit_g, hit_r = gp >= 0, patch_ref >= 0
    both = hit_g & hit_r
    same = both & (gp == patch_ref)
    st = {"n": int(gp.size), "hit_rate": float(hit_g.mean()), "agree": float((hit_g == hit_r).mean()),
          "disagree": int((hit_g != hit_r).sum()), "both": int(both.sum()),
          "same_patch": float(same.sum() / max(both.sum(), 1))}
    if same.any():
        rel = np.abs(gpu["t"][same].astype(np.float64) - t_ref[same]) / np.abs(t_ref[same])
        st["t_rel_max"] = float(rel.max())
        st["t_rel_p999"] = float(np.quantile(rel, 0.999))
        st["t_rel_gt_1e-4"] = float((rel > 1e-4).mean())
        if u_ref is not None:
            duv = np.maximum(np.abs(gpu["u"][same] - u_ref[same]), np.abs(gpu["v"][same] - v_ref[same]))
            st["uv_abs_max"] = float(duv.max())
            st["uv_abs_p999"] = float(np.quantile(duv, 0.999))
    # over rays that both hit (any patch): nearest-surface distance agreement
    if both.any():
        relb = np.abs(gpu["t"][both].astype(np.float64) - t_ref[both]) / np.abs(t_ref[both])
        st["t_rel_gt_1e-4_any"] = float((relb > 1e-4).mean())
    return st
