// wf_solve.cu -- the per-degree-class kernels of the wavefront schedule:
// k_wf_newton<P,Q,MODE> (hull tests, compaction and Newton over one class's
// work items) and k_wf_resolve<P,Q,LEARNED> (recompute the winners and write
// the hit records).  wavefront.cu holds the rest of the schedule.
//
// This file is compiled once per u-degree (-DNRT_WF_P=1..7) so that the
// 7x7 degree classes build in parallel.  The mode is a template argument so
// that the plain solve does not carry the registers of the network's
// inference (MODE: plain, plain + training-pair collection, learned guess).
#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "wavefront.h"

#ifndef NRT_WF_P
#error "wf_solve.cu is compiled with -DNRT_WF_P=<u degree 1..7>"
#endif

namespace nrt {
namespace dev {

namespace {

__device__ __forceinline__ void item_ray(const WfItem& it, RayFrame& r) {
    r.ox = it.ox; r.oy = it.oy; r.oz = it.oz;
    r.dx = it.dx; r.dy = it.dy; r.dz = it.dz;
    ray_planes(r);
}


// One (ray, patch) solve with the options' initial guess.  With the learned
// guess (init_mode 2) Newton first runs from the network's (u, v) for
// learned_iters evaluations; if that does not converge it falls back to plain
// Newton from (0.5, 0.5) with the full budget, which stays the judge of hits.
// When the network's raw guess lies outside [-0.25, 1.25]^2 (it predicts no
// root in the patch) the learned attempt is skipped and plain Newton runs
// directly.  evals counts both attempts.  With flat_threshold > 0 (midpoint or
// bilinear guess) the flat-skip test runs first, as in the per-pixel kernel;
// an accepted guess comes back with flat = 1 and evals 0.
template <int P, int Q, bool LEARNED>
__device__ __forceinline__ NewtonOut solve_item(const Scene& sc, int slot, const RayFrame& r, const PatchRay& pr,
                                                const float* __restrict__ blk, float lu, float lv, uint32_t seed,
                                                const Opts& op, const NewtonOpts& nw_in, int& fell_back) {
    fell_back = 0;
    NewtonOpts nw = nw_in;  // the FP64 decisions apply to patches with widely spread weights
    nw.fp64_band = nw_in.fp64_band && ((__ldg(&sc.hdr[slot].y) >> 8) & kFlagWideWeights);
    if constexpr (LEARNED) {
        // the attempts, through one call site (the solve is compiled once): from the network's
        // guess for learned_iters evaluations, then from the midpoint with the full budget
        const bool inside = lu >= -0.25f && lu <= 1.25f && lv >= -0.25f && lv <= 1.25f;
        fell_back = inside ? 0 : 2;  // 2: gated off, plain Newton only
        int first_evals = 0, first_f64 = 0, first_done = 0;
        NewtonOut o;
        for (int attempt = inside ? 0 : 1; attempt < 2; ++attempt) {
            NewtonOpts na = nw;
            float u0 = 0.5f, v0 = 0.5f;
            if (attempt == 0) {
                if (op.learned_iters > 0 && op.learned_iters < nw.max_iter) na.max_iter = op.learned_iters;
                u0 = fminf(fmaxf(lu, 0.f), 1.f);
                v0 = fminf(fmaxf(lv, 0.f), 1.f);
            }
            o = newton<P, Q>(blk, r, pr, u0, v0, seed, na);
            if (attempt == 0) {
                if (o.evals > 0) return o;
                fell_back = 1;
                first_evals = o.evals;
                first_f64 = o.fp64_solves;
                first_done = o.done;
            }
        }
        if (fell_back == 1) {
            o.evals = o.evals > 0 ? o.evals - first_evals : o.evals + first_evals;
            o.fp64_solves += first_f64;
            o.done += first_done;
        }
        return o;
    } else {
        float gu = 0.5f, gv = 0.5f;
        if (op.init_mode == 1) bilinear_guess(sc.corners + 4 * slot, r, gu, gv);
        if (op.flat_threshold > 0.f) {
            // the ray's entry into the slot's leaf box, computed as the traversal does
            const float4 lo = __ldg(sc.leafbox + 2 * slot), hi = __ldg(sc.leafbox + 2 * slot + 1);
            const float te =
                slab(lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, r, __frcp_rn(r.dx), __frcp_rn(r.dy), __frcp_rn(r.dz));
            NewtonOut o;
            if (flat_accept<P, Q>(blk, r, pr, __ldg(sc.delta + slot), te, op, gu, gv, o) && 0.f < o.t) return o;
        }
        return newton<P, Q>(blk, r, pr, gu, gv, seed, nw);
    }
}

// Lower the ray's nearest-hit record to {key, uv} if key is smaller: a 128-bit
// compare-and-swap loop.  Every failed swap means another lane lowered the
// key, so the loop ends after at most as many tries as there are competing
// hits; the bound only guards against a fault, and reports false.
__device__ __forceinline__ bool record_hit(ulonglong2* rec, unsigned long long key, unsigned long long uv) {
    unsigned __int128* p = reinterpret_cast<unsigned __int128*>(rec);
    const unsigned __int128 want = ((unsigned __int128)uv << 64) | key;
    unsigned __int128 cur = *p;  // a torn read only costs one failed swap
    for (int tries = 0; tries < (1 << 16); ++tries) {
        if (key >= (unsigned long long)cur) return true;
        const unsigned __int128 old = atomicCAS(p, cur, want);
        if (old == cur) return true;
        cur = old;
    }
    return false;
}

// Features of the lane's item for the network (zeros for an idle lane).
__device__ __forceinline__ void item_features(const Scene& sc, bool valid, int slot, const int4& h, const double4& C,
                                              const RayFrame& r, const PatchRay& pr, float (&x)[kMlpIn]) {
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) x[k] = 0.f;
    if (valid) features(sc.frames[slot], h.y & 15, (h.y >> 4) & 15, r, pr, C.x, C.y, C.z, x);
}

// The network's raw (u, v) guess for every work item in [offsets[rank_lo],
// offsets[rank_hi]) into wb.guess (learned mode).  Inference is
// warp-synchronous (mma.sync on the warp's 32 items); it runs here, in a
// kernel whose warps never diverge, and not inside the Newton kernels, whose
// lanes leave their solves at different times: there the tensor-core
// instructions were not always reached by the whole warp at once, and the
// learned kernels stalled.
template <int P, int Q>
__global__ void __launch_bounds__(256) k_wf_guess(Scene sc, WfBuffers wb, int rank_lo, int rank_hi, Opts op) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    MlpSmem* ms = reinterpret_cast<MlpSmem*>(dyn_smem);
    mlp_load(*ms, op.mlp);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int begin = wb.offsets[rank_lo], end = wb.offsets[rank_hi];
    for (long long base = begin + ((long long)blockIdx.x * 8 + warp) * 32; base < end;
         base += (long long)gridDim.x * 256) {
        const long long k = base + lane;
        const bool valid = k < end;
        RayFrame r;
        int4 h = make_int4(0, 0, 0, 0);
        double4 C = make_double4(0.0, 0.0, 0.0, 0.0);
        PatchRay pr{};
        int slot = 0;
        if (valid) {
            const WfItem it = wb.items[k];
            item_ray(it, r);
            slot = it.slot;
            h = sc.hdr[slot];
            C = sc.centre[slot];
            pr = patch_ray(r, C.x, C.y, C.z);
        }
        float x[kMlpIn];
        item_features(sc, valid, slot, h, C, r, pr, x);
        float lu, lv;
        mlp_infer_warp(*ms, warp, lane, x, lu, lv);
        if (valid) wb.guess[k] = make_float2(lu, lv);
    }
}

// Newton over the items of one degree class.  Each warp takes 32 items at a
// time (chunks in a fixed stride), runs the hull tests on them (one lane per item;
// the items of a warp mostly share a patch, so control point loads broadcast),
// and queues the survivors in shared memory; Newton then runs on full warps of
// survivors, so culled items do not leave lanes idle.
template <int P, int Q, int MODE>
__global__ void __launch_bounds__(256, MODE == kWfPlain ? 2 : 1) k_wf_newton(Scene sc, Rays rays, WfBuffers wb, int cls, int rank_lo,
                                                   int rank_hi, Opts op, int32_t* tests, unsigned long long* ctr) {
    constexpr unsigned kFull = 0xffffffffu;
    constexpr bool kUseNet = MODE == kWfLearned;
    __shared__ int queue[8][64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* qu = queue[warp];
    const int begin = wb.offsets[rank_lo], end = wb.offsets[rank_hi];
    unsigned long long solves = 0, evals = 0, f64 = 0, culled = 0, hull_tests = 0, learned = 0, fallbacks = 0,
                       flats = 0, cas_err = 0, learned_conv = 0, fallback_conv = 0;
    NewtonOpts nw = op.nw;
    nw.fp64_final = 0;  // applied to the winner only, in k_wf_resolve
    const float cull_eps = op.nw.eps;
    int qn = 0;
    bool more = true;
    // warps take 32-item chunks in a fixed stride (no shared cursor to contend on)
    const int n_warps = gridDim.x * (blockDim.x >> 5);
    int chunk = blockIdx.x * (blockDim.x >> 5) + warp;
    while (true) {
        while (more && qn < 32) {
            const int base = begin + 32 * chunk;
            chunk += n_warps;
            if (base >= end) {
                more = false;
                break;
            }
            const int k = base + lane;
            bool keep = false;
            if (k < end) {
                keep = true;
                // level 3 is the traversal's oriented-box test alone: after it the per-pair
                // hull tests cost more than the solves they remove (16.4 against 18.3 ms per
                // step on the 64-surface workload, with the same hits)
                if (op.hull_cull && op.hull_cull != 3) {
                    const WfItem it = wb.items[k];
                    const int4 h = sc.hdr[it.slot];
                    if ((h.y >> 8) & kFlagPositiveWeights) {
                        RayFrame r;
                        item_ray(it, r);
                        const double4 C = sc.centre[it.slot];
                        const PatchRay pr = patch_ray(r, C.x, C.y, C.z);
                        const float lim = cull_eps + 8e-6f * (float)C.w;
                        ++hull_tests;
                        const bool miss = op.hull_cull >= 4
                                              ? clip_misses<P, Q>(sc.cp + h.x, r, pr, lim)
                                              : hull_misses<P, Q>(sc.cp + h.x, r, pr, lim) ||
                                                    (op.hull_cull == 2 && subdiv_misses<P, Q>(sc.cp + h.x, r, pr, lim));
                        if (miss) {
                            keep = false;
                            ++culled;
                        }
                    }
                }
            }
            const unsigned m = __ballot_sync(kFull, keep);
            if (keep) qu[qn + __popc(m & ((1u << lane) - 1))] = k;
            qn += __popc(m);
            __syncwarp();
        }
        if (qn == 0) break;
        const int take = qn < 32 ? qn : 32;
        const int k = lane < take ? qu[qn - take + lane] : -1;
        qn -= take;
        __syncwarp();
        WfItem it;
        RayFrame r;
        int4 h = make_int4(0, 0, 0, 0);
        double4 C = make_double4(0.0, 0.0, 0.0, 0.0);
        PatchRay pr{};
        if (k >= 0) {
            it = wb.items[k];
            item_ray(it, r);
            h = sc.hdr[it.slot];
            C = sc.centre[it.slot];
            pr = patch_ray(r, C.x, C.y, C.z);
        }
        float x[kMlpIn];
        float lu = 0.5f, lv = 0.5f;
        if constexpr (MODE == kWfCollect) item_features(sc, k >= 0, k >= 0 ? it.slot : 0, h, C, r, pr, x);
        if constexpr (kUseNet) {
            if (k >= 0) {  // the network's guess, from k_wf_guess
                const float2 g = wb.guess[k];
                lu = g.x;
                lv = g.y;
            }
        }
        if (k >= 0) {
            int fell = 0;
            const NewtonOut o = solve_item<P, Q, kUseNet>(sc, it.slot, r, pr, sc.cp + h.x, lu, lv,
                                                           (uint32_t)it.ray + op.seed_offset, op, nw, fell);
            ++solves;
            learned += (kUseNet && fell != 2) ? 1 : 0;
            fallbacks += fell == 1 ? 1ull : 0ull;
            learned_conv += (kUseNet && fell == 0) ? 1ull : 0ull;      // the guess's own solve converged
            fallback_conv += (fell == 1 && o.evals > 0) ? 1ull : 0ull;  // it did not, plain Newton did
            evals += (unsigned long long)o.done;
            f64 += (unsigned long long)o.fp64_solves;
            if (tests) atomicAdd(tests + it.ray, 1);
            flats += (unsigned long long)o.flat;
            if ((o.evals > 0 || o.flat) && o.t > 0.f) {
                const unsigned long long key = ((unsigned long long)__float_as_uint(o.t) << 32) |
                                               ((unsigned)it.slot << 1) | (unsigned)o.flat;
                const unsigned long long uv =
                    ((unsigned long long)__float_as_uint(o.u) << 32) | __float_as_uint(o.v);
                if (!record_hit(wb.best + it.ray, key, uv)) ++cas_err;
            }
            if constexpr (MODE == kWfCollect) {  // a training pair: features -> converged (u, v), or (-1, -1)
                const unsigned long long at = atomicAdd(op.col_count, 1ull);
                if ((long long)at < op.col_cap) {
#pragma unroll
                    for (int q2 = 0; q2 < kMlpIn; ++q2) op.col_feat[at * kMlpIn + q2] = x[q2];
                    op.col_targ[2 * at] = o.evals > 0 ? o.u : -1.f;
                    op.col_targ[2 * at + 1] = o.evals > 0 ? o.v : -1.f;
                }
            }
        }
        __syncwarp();
    }
    if (ctr && op.counters) {
        count_add(ctr, kSolves, solves);
        count_add(ctr, kEvals, evals);
        count_add(ctr, kFp64Solves, f64);
        count_add(ctr, kCulled, culled);
        count_add(ctr, kLearned, learned);
        count_add(ctr, kFallbacks, fallbacks);
        count_add(ctr, kLearnedConverged, learned_conv);
        count_add(ctr, kFallbackConverged, fallback_conv);
        count_add(ctr, kFlatSkips, flats);
        if (evals) atomicAdd(ctr + kEvalsByDegree + P * 8 + Q, evals);
        if (hull_tests) atomicAdd(ctr + kHullByDegree + P * 8 + Q, hull_tests);
    }
    if (ctr && cas_err) atomicAdd(ctr + kErrors, cas_err);
}

// Resolve, step 1: rays without a hit get their miss record; rays with one

// Resolve, step 2 (one launch per degree class): rebuild the winning solve's
// point from the (u, v) recorded with its key (one evaluation, the same one
// the solve converged on), apply the FP64 final step, and write the hit
// record; when per-ray evaluation counts are requested the solve itself is
// run again instead (same code and inputs, so the same iterate).
template <int P, int Q, bool LEARNED>
__global__ void __launch_bounds__(256) k_wf_resolve(Scene sc, WfBuffers wb, int rank_lo, int rank_hi, Opts op,
                                                    Hits out, unsigned long long* ctr) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int begin = wb.offsets[rank_lo], end = wb.offsets[rank_hi];
    unsigned long long f64f = 0, hits = 0, err = 0;
    for (long long base = begin + ((long long)blockIdx.x * 8 + warp) * 32; base < end;
         base += (long long)gridDim.x * 256) {
        const long long k = base + lane;
        const bool valid = k < end;
        WfItem it;
        RayFrame r;
        int4 h = make_int4(0, 0, 0, 0);
        double4 C = make_double4(0.0, 0.0, 0.0, 0.0);
        PatchRay pr{};
        if (valid) {
            it = wb.items[k];
            item_ray(it, r);
            h = sc.hdr[it.slot];
            C = sc.centre[it.slot];
            pr = patch_ray(r, C.x, C.y, C.z);
        }
        if (valid) {
        const long long i = it.ray;
        NewtonOut o;
        if (out.iters) {  // the evaluation count is wanted: solve again
            float lu = 0.5f, lv = 0.5f;
            if constexpr (LEARNED) {  // the network's guess, from k_wf_guess over these items
                const float2 g = wb.guess[k];
                lu = g.x;
                lv = g.y;
            }
            int fell = 0;
            o = solve_item<P, Q, LEARNED>(sc, it.slot, r, pr, sc.cp + h.x, lu, lv, (uint32_t)it.ray + op.seed_offset,
                                          op, op.nw, fell);
        } else {  // rebuild the winner at its recorded (u, v): the solve's last evaluation
            const ulonglong2 rec = wb.best[i];
            const float u = __uint_as_float((unsigned)(rec.y >> 32)), v = __uint_as_float((unsigned)rec.y);
            const float* __restrict__ blk = sc.cp + h.x;
            float H[4], Hu[4], Hv[4];
            eval_patch<P, Q>(blk, u, v, H, Hu, Hv);
            const float iw = __frcp_rn(H[3]);
            const float sx = H[0] * iw, sy = H[1] * iw, sz = H[2] * iw;
            o.fp64_solves = 0;
            o.fp64_final = 0;
            o.flat = (int)(rec.x & 1ull);
            o.evals = o.flat ? 0 : 1;  // converged (the count itself is not recorded)
            o.done = 0;
            o.u = u; o.v = v;
            o.sx = sx; o.sy = sy; o.sz = sz;
            o.ux = (Hu[0] - sx * Hu[3]) * iw; o.uy = (Hu[1] - sy * Hu[3]) * iw; o.uz = (Hu[2] - sz * Hu[3]) * iw;
            o.vx = (Hv[0] - sx * Hv[3]) * iw; o.vy = (Hv[1] - sy * Hv[3]) * iw; o.vz = (Hv[2] - sz * Hv[3]) * iw;
            o.t = fmaf(sx, r.dx, fmaf(sy, r.dy, fmaf(sz, r.dz, pr.tc)));
            if (!o.flat && op.nw.fp64_final) final_step_fp64<P, Q>(blk, r, pr, o);
        }
        if ((o.evals > 0 || o.flat) && o.t > 0.f) {
            ++hits;
            f64f += (unsigned long long)o.fp64_final;
            out.patch[i] = h.z;
            out.t[i] = o.t;
            out.u[i] = o.u;
            out.v[i] = o.v;
            if (out.iters) out.iters[i] = o.evals;
            if (out.geom) {
                float* g = out.geom + 9 * i;
                g[0] = (float)(C.x + (double)o.sx); g[1] = (float)(C.y + (double)o.sy); g[2] = (float)(C.z + (double)o.sz);
                g[3] = o.ux; g[4] = o.uy; g[5] = o.uz;
                g[6] = o.vx; g[7] = o.vy; g[8] = o.vz;
            }
        } else {
            if (o.evals <= 0 && !o.flat) ++err;  // the recomputed winner must converge again
            out.patch[i] = -1;
            out.t[i] = -1.f;
            out.u[i] = 0.f;
            out.v[i] = 0.f;
            if (out.iters) out.iters[i] = 0;
            if (out.geom)
                for (int a = 0; a < 9; ++a) out.geom[9 * i + a] = 0.f;
        }
        }
        __syncwarp();
    }
    if (ctr) {
        if (op.counters) {
            count_add(ctr, kFp64Final, f64f);
            count_add(ctr, kHits, hits);
        }
        if (err) atomicAdd(ctr + kErrors, err);
    }
}

// Dynamic shared memory for the network: the attribute is set once per kernel
// (per process; every kernel of this file runs on devices of one architecture).
template <class K>
void allow_mlp_smem(K kernel, bool& done) {
    if (!done) {
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
        done = true;
    }
}

template <int Q>
void newton_class(const WfClassLaunch& L) {
    constexpr int P = NRT_WF_P;
    switch (L.mode) {
        case kWfLearned: {
            static bool done = false;
            allow_mlp_smem(k_wf_guess<P, Q>, done);
            k_wf_guess<P, Q><<<L.grid, 256, sizeof(MlpSmem), L.stream>>>(*L.sc, *L.wb, L.rank_lo, L.rank_hi, *L.op);
            k_wf_newton<P, Q, kWfLearned><<<L.grid, 256, 0, L.stream>>>(*L.sc, *L.rays, *L.wb, L.cls, L.rank_lo,
                                                                        L.rank_hi, *L.op, L.tests, L.ctr);
            break;
        }
        case kWfCollect:
            k_wf_newton<P, Q, kWfCollect><<<L.grid, 256, 0, L.stream>>>(*L.sc, *L.rays, *L.wb, L.cls, L.rank_lo,
                                                                        L.rank_hi, *L.op, L.tests, L.ctr);
            break;
        default:
            k_wf_newton<P, Q, kWfPlain><<<L.grid, 256, 0, L.stream>>>(*L.sc, *L.rays, *L.wb, L.cls, L.rank_lo,
                                                                      L.rank_hi, *L.op, L.tests, L.ctr);
    }
}

template <int Q>
void resolve_class(const WfClassLaunch& L) {
    constexpr int P = NRT_WF_P;
    if (L.mode == kWfLearned) {
        if (L.out->iters) {  // the winners are solved again: their guesses first
            static bool done = false;
            allow_mlp_smem(k_wf_guess<P, Q>, done);
            k_wf_guess<P, Q><<<L.grid, 256, sizeof(MlpSmem), L.stream>>>(*L.sc, *L.wb, L.rank_lo, L.rank_hi, *L.op);
        }
        k_wf_resolve<P, Q, true><<<L.grid, 256, 0, L.stream>>>(*L.sc, *L.wb, L.rank_lo, L.rank_hi, *L.op, *L.out,
                                                               L.ctr);
    } else {
        k_wf_resolve<P, Q, false><<<L.grid, 256, 0, L.stream>>>(*L.sc, *L.wb, L.rank_lo, L.rank_hi, *L.op, *L.out,
                                                                L.ctr);
    }
}

}  // namespace

#define NRT_WF_CAT2(a, b) a##b
#define NRT_WF_CAT(a, b) NRT_WF_CAT2(a, b)

void NRT_WF_CAT(wf_newton_p, NRT_WF_P)(int q, const WfClassLaunch& L) {
    switch (q) {
        case 1: newton_class<1>(L); break;
        case 2: newton_class<2>(L); break;
        case 3: newton_class<3>(L); break;
        case 4: newton_class<4>(L); break;
        case 5: newton_class<5>(L); break;
        case 6: newton_class<6>(L); break;
        case 7: newton_class<7>(L); break;
        default: break;
    }
}

void NRT_WF_CAT(wf_resolve_p, NRT_WF_P)(int q, const WfClassLaunch& L) {
    switch (q) {
        case 1: resolve_class<1>(L); break;
        case 2: resolve_class<2>(L); break;
        case 3: resolve_class<3>(L); break;
        case 4: resolve_class<4>(L); break;
        case 5: resolve_class<5>(L); break;
        case 6: resolve_class<6>(L); break;
        case 7: resolve_class<7>(L); break;
        default: break;
    }
}

}  // namespace dev
}  // namespace nrt
