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


def crossing_cos(rays_np, geom):
    """|cos| of the angle between each ray and the surface normal dS/du x dS/dv
    of its hit (from the hit's 9-float geometry): t's condition number is about
    1 / |cos|, so near-tangent crossings (|cos| -> 0) are ill-conditioned."""
    d = np.stack(rays_np[3:], 1).astype(np.float64)
    g = geom.astype(np.float64)
    n = np.cross(g[:, 3:6], g[:, 6:9])
    return np.abs(np.sum(n * d, 1)) / np.maximum(np.linalg.norm(n, axis=1) * np.linalg.norm(d, axis=1), 1e-300)


def root_stats(oracle_mod, P, rays_np, got, ref, cosang=None):
    """Hits of the engine and of the FP64 oracle on the same rays, each refined
    to the exact root next to it (FP64 Newton to |r1|+|r2| < 1e-11 from the
    reported (u, v) on the reported patch; the oracle itself stops at the
    method's eps, so its t is only good to about eps / sin(angle)).  Returns:
    genuine (fraction of engine hits that refine to a root), t_err / uv_err
    (engine hit against its exact root, t relative to t or to 1e4 FP32 ulps of
    the ray origin's largest coordinate, whichever is larger; max and
    quantiles; with cosang, the
    |cos| of each hit's crossing angle, t_err_max is taken over the hits with
    |cos| >= 1e-2 and t_err_tangent counts the others above 1e-4), same_root
    (fraction of rays both hit where the two exact roots coincide) and the
    counts of rays both hit on different roots, by which one is nearer."""
    rays = oracle_mod.Rays(*rays_np)
    he, ho = got["patch"] >= 0, ref.patch >= 0
    pe = oracle_mod.polish_hits(P, rays, np.where(he, got["patch"], -1), got["u"], got["v"])
    po = oracle_mod.polish_hits(P, rays, ref.patch, ref.u, ref.v)
    ok = he & (pe.patch >= 0)
    st = {"genuine": float(ok.sum() / max(he.sum(), 1))}
    if ok.any():
        # An absolute error below one FP32 ulp of the origin's largest
        # coordinate is not counted against t: the hit point o + t d cannot be
        # stored more finely than that (it matters only for rays that end very
        # near their origin, such as bounce rays reaching the next patch of a
        # crease at t ~ 1e-6).
        o_ulp = np.spacing(np.max(np.abs(np.stack(rays_np[:3], 1)), axis=1).astype(np.float32)).astype(np.float64)
        rel = np.abs(got["t"][ok].astype(np.float64) - pe.t[ok]) / np.maximum(np.abs(pe.t[ok]), 1e4 * o_ulp[ok])
        duv = np.maximum(np.abs(got["u"][ok] - pe.u[ok]), np.abs(got["v"][ok] - pe.v[ok]))
        wc = np.ones(rel.size, bool) if cosang is None else cosang[ok] >= 1e-2
        st.update({"t_err_max": float(rel[wc].max()) if wc.any() else 0.0,
                   "t_err_max_all": float(rel.max()), "t_err_p9999": float(np.quantile(rel, 0.9999)),
                   "t_err_gt_1e-4": int((rel > 1e-4).sum()), "t_err_tangent": int(((rel > 1e-4) & ~wc).sum()),
                   "uv_err_max": float(duv.max()), "uv_err_p999": float(np.quantile(duv, 0.999))})
    both = he & ho & (pe.patch >= 0) & (po.patch >= 0)
    same = both & (got["patch"] == ref.patch) & (np.abs(pe.t - po.t) <= 1e-6 * np.abs(po.t))
    st["same_root"] = float(same.sum() / max(both.sum(), 1))
    other = both & ~same
    st["other_root_engine_nearer"] = int((other & (pe.t < po.t)).sum())
    st["other_root_engine_farther"] = int((other & (pe.t >= po.t)).sum())
    return st
