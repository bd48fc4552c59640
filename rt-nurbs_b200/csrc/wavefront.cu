// wavefront.cu -- the batched intersection schedule.
//
// The per-pixel kernel (intersect_pixel.cu) lets every lane of a warp walk its
// own ray through the BVH and run Newton on whatever patch it reaches, so a
// warp executes many (p,q) instantiations side by side.  Here the work is
// regrouped, in rounds r = 0, 1, 2, ... until no ray is left traversing:
//
//   k_wf_step        one thread per active ray: resumes the ray's saved BVH
//                    stack, pruning every entry whose box entry is not nearer
//                    than the ray's best hit so far (the reference's rule,
//                    src/gpu/intersect.cu:169-183), and emits the leaf patches
//                    it reaches, up to round_quota(r) of them; counts them per
//                    patch rank; saves the stack; rays with a non-empty stack
//                    stay active.
//   k_wf_scan        exclusive scan of the per-rank counts.
//   k_wf_scatter     work items (ray origin and direction, ray index, slot) in
//                    rank order, ranks sorted by (p, q, slot).
//   k_wf_newton<P,Q> one launch per degree class present in the scene: each
//                    warp takes 32 consecutive items (mostly one patch, so
//                    control point loads broadcast), runs the exact hull tests
//                    on them, compacts the survivors by ballot into a shared
//                    queue and runs Newton on full warps of survivors; a
//                    converged hit with t > 0 lowers the ray's 64-bit key
//                    (t bits << 32 | slot) with atomicMin.
//
// The resolve pass sorts the rays that hit by their winner's (p, q, slot) and
// k_wf_resolve<P,Q> recomputes each winning solve (same code and inputs) with
// the FP64 final step and writes the hit record.  The closest hit is the
// minimum over all candidates nearer than the best hit, so the order in which
// candidates are solved does not change it.
#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "kernels.h"
#include "wavefront.h"

namespace nrt {
namespace dev {

namespace {

__device__ __forceinline__ float key_t(unsigned long long key) {
    return key == kNoHit ? INFINITY : __uint_as_float((unsigned)(key >> 32));
}

__device__ __forceinline__ void load_ray(const Rays& rays, long long i, RayFrame& r) {
    r.ox = __ldg(rays.ox + i); r.oy = __ldg(rays.oy + i); r.oz = __ldg(rays.oz + i);
    r.dx = __ldg(rays.dx + i); r.dy = __ldg(rays.dy + i); r.dz = __ldg(rays.dz + i);
    ray_planes(r);
}

// Warp-aggregated increment of hist[key]: lanes with equal keys add once.
__device__ __forceinline__ int aggregated_add(int* hist, int key) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == leader) base = atomicAdd(hist + key, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane) - 1));
}

}  // namespace

__global__ void __launch_bounds__(128) k_wf_step(Scene sc, Rays rays, long long n, int round, int n_active,
                                                 int quota, Opts op, WfBuffers wb, int cur, int32_t* tests,
                                                 unsigned long long* ctr, const int32_t* rank_of) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_active) return;
    const long long i = round == 0 ? (long long)j : (long long)wb.active[cur][j];
    RayFrame r;
    load_ray(rays, i, r);
    const float rdx = __frcp_rn(r.dx), rdy = __frcp_rn(r.dy), rdz = __frcp_rn(r.dz);
    int st[kStack];
    float stt[kStack];
    int sp;
    float best;
    if (round == 0) {
        sp = 1;
        st[0] = 0;
        stt[0] = 0.f;
        best = INFINITY;
        wb.best_key[i] = kNoHit;
        if (tests) tests[i] = 0;
    } else {
        sp = wb.stack_sp[i];
        for (int k = 0; k < sp; ++k) {
            st[k] = wb.stack_ref[(long long)k * n + i];
            stt[k] = wb.stack_t[(long long)k * n + i];
        }
        best = key_t(wb.best_key[i]);
    }
    int32_t* emit = wb.emit_slot + (long long)j * kEmitMax;
    int emitted = 0;
    unsigned long long boxes = 0, cands = 0, culled = 0, err = 0;
    while (sp > 0 && emitted < quota) {
        --sp;
        const int ref = st[sp];
        const float te = stt[sp];
        if (te >= best) continue;
        if (ref >= 0) {
            const float4* nd = reinterpret_cast<const float4*>(sc.nodes + ref);
            const float4 lx = __ldg(nd + 0), hx = __ldg(nd + 1), ly = __ldg(nd + 2), hy = __ldg(nd + 3);
            const float4 lz = __ldg(nd + 4), hz = __ldg(nd + 5);
            const int4 ch = __ldg(reinterpret_cast<const int4*>(nd + 6));
            const int4 cn = __ldg(reinterpret_cast<const int4*>(nd + 7));
            const float LX[4] = {lx.x, lx.y, lx.z, lx.w}, HX[4] = {hx.x, hx.y, hx.z, hx.w};
            const float LY[4] = {ly.x, ly.y, ly.z, ly.w}, HY[4] = {hy.x, hy.y, hy.z, hy.w};
            const float LZ[4] = {lz.x, lz.y, lz.z, lz.w}, HZ[4] = {hz.x, hz.y, hz.z, hz.w};
            const int CH[4] = {ch.x, ch.y, ch.z, ch.w}, CN[4] = {cn.x, cn.y, cn.z, cn.w};
            float tt[4];
            int rr[4], k = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (CH[q] < 0 && CN[q] == 0) continue;
                ++boxes;
                const float t = slab(LX[q], LY[q], LZ[q], HX[q], HY[q], HZ[q], r, rdx, rdy, rdz);
                if (t < best) {
                    tt[k] = t;
                    rr[k] = CH[q] >= 0 ? CH[q] : leaf_ref(~CH[q], CN[q]);
                    ++k;
                }
            }
            for (int a = 1; a < k; ++a)  // farthest pushed first: nearest popped next
                for (int b = a; b > 0 && tt[b] > tt[b - 1]; --b) {
                    const float tf = tt[b]; tt[b] = tt[b - 1]; tt[b - 1] = tf;
                    const int rf = rr[b]; rr[b] = rr[b - 1]; rr[b - 1] = rf;
                }
            for (int a = 0; a < k; ++a) {
                if (sp < kStack) {
                    st[sp] = rr[a];
                    stt[sp] = tt[a];
                    ++sp;
                } else {
                    ++err;  // stack overflow: the subtree is dropped and the error counted
                }
            }
        } else {
            const int first = leaf_first(ref), lc = leaf_count(ref);
            for (int s = first; s < first + lc; ++s) {
                ++cands;
                emit[emitted++] = s;  // quota <= 8 and a leaf holds <= 8: stays below kEmitMax
                aggregated_add(wb.hist, rank_of[s]);
            }
        }
    }
    for (int k = 0; k < sp; ++k) {
        wb.stack_ref[(long long)k * n + i] = st[k];
        wb.stack_t[(long long)k * n + i] = stt[k];
    }
    wb.stack_sp[i] = sp;
    wb.emit_cnt[j] = emitted;
    if (sp > 0) {
        const int at = aggregated_add(wb.counts + (1 - cur), 0);
        wb.active[1 - cur][at] = (int)i;
    }
    if (ctr) {
        if (op.counters) {
            if (round == 0) count_add(ctr, kRays, 1);
            count_add(ctr, kBoxTests, boxes);
            count_add(ctr, kCandidates, cands);
            count_add(ctr, kCulled, culled);
        }
        if (err) atomicAdd(ctr + kErrors, err);
    }
}

__global__ void __launch_bounds__(256) k_wf_scatter(Rays rays, int round, int n_active, WfBuffers wb, int cur,
                                                    const int32_t* rank_of) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_active) return;
    const int i = round == 0 ? j : wb.active[cur][j];
    const int m = wb.emit_cnt[j];
    if (m == 0) return;
    WfItem it;
    it.ox = __ldg(rays.ox + i); it.oy = __ldg(rays.oy + i); it.oz = __ldg(rays.oz + i);
    it.dx = __ldg(rays.dx + i); it.dy = __ldg(rays.dy + i); it.dz = __ldg(rays.dz + i);
    it.ray = i;
    for (int e = 0; e < m; ++e) {
        const int s = wb.emit_slot[(long long)j * kEmitMax + e];
        const int rk = rank_of[s];
        const int pos = wb.offsets[rk] + aggregated_add(wb.cursor, rk);
        it.slot = s;
        wb.items[pos] = it;
    }
}

__device__ __forceinline__ void item_ray(const WfItem& it, RayFrame& r) {
    r.ox = it.ox; r.oy = it.oy; r.oz = it.oz;
    r.dx = it.dx; r.dy = it.dy; r.dz = it.dz;
    ray_planes(r);
}

// Exclusive scan of hist[0..m) into offsets[0..m] (offsets[m] = total), and
// cursor[] cleared; one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_wf_scan(int m, WfBuffers wb) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int per = (m + 1023) / 1024;
    const int a = min(m, t * per), b = min(m, a + per);
    int s = 0;
    for (int k = a; k < b; ++k) s += wb.hist[k];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // Hillis-Steele inclusive scan
        const int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - s;
    for (int k = a; k < b; ++k) {
        wb.offsets[k] = run;
        run += wb.hist[k];
        wb.cursor[k] = 0;
    }
    if (t == 1023) wb.offsets[m] = part[1023];
}

// One (ray, patch) solve with the options' initial guess.  With the learned
// guess (init_mode 2) Newton first runs from the network's (u, v) for
// learned_iters evaluations; if that does not converge it falls back to plain
// Newton from (0.5, 0.5) with the full budget, which stays the judge of hits.
// When the network's raw guess lies outside [-0.25, 1.25]^2 (it predicts no
// root in the patch) the learned attempt is skipped and plain Newton runs
// directly.  evals counts both attempts.
template <int P, int Q>
__device__ __forceinline__ NewtonOut solve_item(const Scene& sc, int slot, const RayFrame& r, const PatchRay& pr,
                                                const float* __restrict__ blk, float lu, float lv, uint32_t seed,
                                                const Opts& op, const NewtonOpts& nw, int& fell_back) {
    fell_back = 0;
    const bool inside = lu >= -0.25f && lu <= 1.25f && lv >= -0.25f && lv <= 1.25f;
    if (op.init_mode == 2 && inside) {
        NewtonOpts nl = nw;
        if (op.learned_iters > 0 && op.learned_iters < nw.max_iter) nl.max_iter = op.learned_iters;
        const NewtonOut o = newton<P, Q>(blk, r, pr, fminf(fmaxf(lu, 0.f), 1.f), fminf(fmaxf(lv, 0.f), 1.f), seed, nl);
        if (o.evals > 0) return o;
        fell_back = 1;
        NewtonOut f = newton<P, Q>(blk, r, pr, 0.5f, 0.5f, seed, nw);
        f.evals = f.evals > 0 ? f.evals - o.evals : f.evals + o.evals;
        f.fp64_solves += o.fp64_solves;
        return f;
    }
    if (op.init_mode == 2) fell_back = 2;  // gated off: plain Newton only
    float gu = 0.5f, gv = 0.5f;
    if (op.init_mode == 1) bilinear_guess(sc.corners + 4 * slot, r, gu, gv);
    return newton<P, Q>(blk, r, pr, gu, gv, seed, nw);
}

// Features of the lane's item for the network (zeros for an idle lane).
__device__ __forceinline__ void item_features(const Scene& sc, bool valid, int slot, const int4& h, const double4& C,
                                              const RayFrame& r, const PatchRay& pr, float (&x)[kMlpIn]) {
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) x[k] = 0.f;
    if (valid) features(sc.frames[slot], h.y & 15, (h.y >> 4) & 15, r, pr, C.x, C.y, C.z, x);
}

// Newton over the items of one degree class.  Each warp takes 32 items at a
// time (chunks in a fixed stride), runs the hull tests on them (one lane per item;
// the items of a warp mostly share a patch, so control point loads broadcast),
// and queues the survivors in shared memory; Newton then runs on full warps of
// survivors, so culled items do not leave lanes idle.
template <int P, int Q>
__global__ void __launch_bounds__(256) k_wf_newton(Scene sc, Rays rays, WfBuffers wb, int cls, int rank_lo,
                                                   int rank_hi, Opts op, int32_t* tests, unsigned long long* ctr) {
    constexpr unsigned kFull = 0xffffffffu;
    __shared__ int queue[8][64];
    extern __shared__ __align__(16) unsigned char dyn_smem[];  // the network, when init_mode == 2
    MlpSmem* ms = reinterpret_cast<MlpSmem*>(dyn_smem);
    if (op.init_mode == 2) {
        mlp_load(*ms, op.mlp);
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int* qu = queue[warp];
    const int begin = wb.offsets[rank_lo], end = wb.offsets[rank_hi];
    unsigned long long solves = 0, evals = 0, f64 = 0, culled = 0, hull_tests = 0, learned = 0, fallbacks = 0;
    NewtonOpts nw = op.nw;
    nw.fp64_final = 0;  // applied to the winner only, in k_wf_resolve
    const bool need_features = op.init_mode == 2 || op.col_feat != nullptr;
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
                if (op.hull_cull) {
                    const WfItem it = wb.items[k];
                    const int4 h = sc.hdr[it.slot];
                    if ((h.y >> 8) & kFlagPositiveWeights) {
                        RayFrame r;
                        item_ray(it, r);
                        const double4 C = sc.centre[it.slot];
                        const PatchRay pr = patch_ray(r, C.x, C.y, C.z);
                        const float lim = cull_eps + 8e-6f * (float)C.w;
                        ++hull_tests;
                        if (hull_misses<P, Q>(sc.cp + h.x, r, pr, lim) ||
                            (op.hull_cull >= 2 && subdiv_misses<P, Q>(sc.cp + h.x, r, pr, lim))) {
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
        if (need_features) item_features(sc, k >= 0, k >= 0 ? it.slot : 0, h, C, r, pr, x);
        if (op.init_mode == 2) mlp_infer_warp(*ms, warp, lane, x, lu, lv);  // warp-synchronous
        if (k >= 0) {
            int fell = 0;
            const NewtonOut o = solve_item<P, Q>(sc, it.slot, r, pr, sc.cp + h.x, lu, lv,
                                                 (uint32_t)it.ray + op.seed_offset, op, nw, fell);
            ++solves;
            learned += (op.init_mode == 2 && fell != 2) ? 1 : 0;
            fallbacks += fell == 1 ? 1ull : 0ull;
            evals += (unsigned long long)(o.evals > 0 ? o.evals : -o.evals);
            f64 += (unsigned long long)o.fp64_solves;
            if (tests) atomicAdd(tests + it.ray, 1);
            if (o.evals > 0 && o.t > 0.f) {
                const unsigned long long key = ((unsigned long long)__float_as_uint(o.t) << 32) | (unsigned)it.slot;
                atomicMin(wb.best_key + it.ray, key);
            }
            if (op.col_feat) {  // a training pair: features -> converged (u, v), or (-1, -1) if none
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
        if (evals) atomicAdd(ctr + kEvalsByDegree + P * 8 + Q, evals);
        if (hull_tests) atomicAdd(ctr + kHullByDegree + P * 8 + Q, hull_tests);
    }
}

// Resolve, step 1: rays without a hit get their miss record; rays with one
// emit their winning slot (counted per rank, as a round's candidates are).
__global__ void __launch_bounds__(256) k_wf_resolve_emit(long long n, Opts op, WfBuffers wb, Hits out,
                                                         const int32_t* rank_of, unsigned long long* ctr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long key = wb.best_key[i];
    if (key == kNoHit) {
        wb.emit_cnt[i] = 0;
        out.patch[i] = -1;
        out.t[i] = -1.f;
        out.u[i] = 0.f;
        out.v[i] = 0.f;
        if (out.iters) out.iters[i] = 0;
        if (out.geom)
            for (int a = 0; a < 9; ++a) out.geom[9 * (long long)i + a] = 0.f;
        return;
    }
    const int s = (int)(key & 0xffffffffu);
    wb.emit_cnt[i] = 1;
    wb.emit_slot[(long long)i * kEmitMax] = s;
    aggregated_add(wb.hist, rank_of[s]);
}

// Resolve, step 2 (one launch per degree class): recompute the winning solve
// (same code and inputs, so the same iterate) with the FP64 final step, and
// write the hit record.
template <int P, int Q>
__global__ void __launch_bounds__(256) k_wf_resolve(Scene sc, WfBuffers wb, int rank_lo, int rank_hi, Opts op,
                                                    Hits out, unsigned long long* ctr) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    MlpSmem* ms = reinterpret_cast<MlpSmem*>(dyn_smem);
    if (op.init_mode == 2) {
        mlp_load(*ms, op.mlp);
        __syncthreads();
    }
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
        float lu = 0.5f, lv = 0.5f;
        if (op.init_mode == 2) {
            float x[kMlpIn];
            item_features(sc, valid, valid ? it.slot : 0, h, C, r, pr, x);
            mlp_infer_warp(*ms, warp, lane, x, lu, lv);
        }
        if (valid) {  // idle lanes wait at the __syncwarp below, so the next mma runs converged
        int fell = 0;
        const NewtonOut o = solve_item<P, Q>(sc, it.slot, r, pr, sc.cp + h.x, lu, lv, (uint32_t)it.ray + op.seed_offset,
                                             op, op.nw, fell);
        const long long i = it.ray;
        if (o.evals > 0 && o.t > 0.f) {
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
            if (o.evals <= 0) ++err;  // the recomputed winner must converge again
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
template <int P, int Q>
void allow_mlp_smem_newton() {
    static bool done = false;
    if (!done) {
        cudaFuncSetAttribute(k_wf_newton<P, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
        done = true;
    }
}
template <int P, int Q>
void allow_mlp_smem_resolve() {
    static bool done = false;
    if (!done) {
        cudaFuncSetAttribute(k_wf_resolve<P, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
        done = true;
    }
}

// ---------------------------------------------------------------------------
size_t wavefront_scratch_bytes(long long n, int n_slots) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t N = (size_t)n, S = (size_t)n_slots + 1;
    return 2 * al(N * kStack * 4) + al(N * 4) + al(N * 8) + 2 * al(N * 4) + al(16) + al(N * kEmitMax * 4) +
           al(N * 4) + al(N * kEmitMax * sizeof(WfItem)) + 3 * al(S * 4) + al(64 * 4);
}

WfBuffers wavefront_carve(void* base, long long n, int n_slots) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t N = (size_t)n, S = (size_t)n_slots + 1;
    char* p = static_cast<char*>(base);
    WfBuffers b;
    b.stack_ref = reinterpret_cast<int32_t*>(p); p += al(N * kStack * 4);
    b.stack_t = reinterpret_cast<float*>(p); p += al(N * kStack * 4);
    b.stack_sp = reinterpret_cast<int32_t*>(p); p += al(N * 4);
    b.best_key = reinterpret_cast<unsigned long long*>(p); p += al(N * 8);
    b.active[0] = reinterpret_cast<int32_t*>(p); p += al(N * 4);
    b.active[1] = reinterpret_cast<int32_t*>(p); p += al(N * 4);
    b.counts = reinterpret_cast<int32_t*>(p); p += al(16);
    b.emit_slot = reinterpret_cast<int32_t*>(p); p += al(N * kEmitMax * 4);
    b.emit_cnt = reinterpret_cast<int32_t*>(p); p += al(N * 4);
    b.items = reinterpret_cast<WfItem*>(p); p += al(N * kEmitMax * sizeof(WfItem));
    b.hist = reinterpret_cast<int32_t*>(p); p += al(S * 4);
    b.cursor = reinterpret_cast<int32_t*>(p); p += al(S * 4);
    b.offsets = reinterpret_cast<int32_t*>(p); p += al(S * 4);
    b.class_cursor = reinterpret_cast<int32_t*>(p);
    return b;
}

cudaError_t launch_wavefront(const Scene& sc, const WfPlan& plan, const Rays& rays, long long n, const Opts& op,
                             const Hits& out, const WfBuffers& wb, int32_t* host_count, unsigned long long* ctr,
                             cudaStream_t stream, long long* launches, long long* rounds) {
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    int n_active = (int)n, cur = 0;
    const size_t smem = op.init_mode == 2 ? sizeof(MlpSmem) : 0;
    for (int round = 0; n_active > 0; ++round) {
        if (round > 4096) return cudaErrorUnknown;  // unreachable: every round pops at least one entry per ray
        e = cudaMemsetAsync(wb.hist, 0, sizeof(int) * plan.n_slots, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(wb.counts + (1 - cur), 0, sizeof(int), stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(wb.class_cursor, 0, sizeof(int) * 64, stream);
        if (e != cudaSuccess) return e;
        k_wf_step<<<(unsigned)((n_active + 127) / 128), 128, 0, stream>>>(sc, rays, n, round, n_active,
                                                                         round_quota(round), op, wb, cur, out.tests,
                                                                         ctr, plan.rank_of);
        k_wf_scan<<<1, 1024, 0, stream>>>(plan.n_slots, wb);
        k_wf_scatter<<<(unsigned)((n_active + 255) / 256), 256, 0, stream>>>(rays, round, n_active, wb, cur,
                                                                             plan.rank_of);
        *launches += 3 + plan.n_classes;
        *rounds += 1;
        for (int c = 0; c < plan.n_classes; ++c) {
            const int pq = plan.class_pq[c], rl = plan.class_rank[c], rh = plan.class_rank[c + 1];
            const unsigned grid = plan.class_grid[c];
            switch (pq) {
#define NRT_CASE(P, Q) \
    case (P) | ((Q) << 4):                                                                              \
        if (smem) allow_mlp_smem_newton<P, Q>();                                                        \
        k_wf_newton<P, Q><<<grid, 256, smem, stream>>>(sc, rays, wb, c, rl, rh, op, out.tests, ctr);     \
        break;
                NRT_FOR_EACH_DEGREE(NRT_CASE)
#undef NRT_CASE
                default: break;
            }
        }
        e = cudaMemcpyAsync(host_count, wb.counts + (1 - cur), sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        n_active = *host_count;
        cur = 1 - cur;
    }
    // resolve: hit rays sorted by their winner's (p, q, slot), one kernel per class
    e = cudaMemsetAsync(wb.hist, 0, sizeof(int) * plan.n_slots, stream);
    if (e != cudaSuccess) return e;
    k_wf_resolve_emit<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(n, op, wb, out, plan.rank_of, ctr);
    k_wf_scan<<<1, 1024, 0, stream>>>(plan.n_slots, wb);
    k_wf_scatter<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(rays, 0, (int)n, wb, cur, plan.rank_of);
    for (int c = 0; c < plan.n_classes; ++c) {
        const int pq = plan.class_pq[c], rl = plan.class_rank[c], rh = plan.class_rank[c + 1];
        const unsigned grid = plan.class_grid[c];
        switch (pq) {
#define NRT_CASE(P, Q) \
    case (P) | ((Q) << 4):                                                                              \
        if (smem) allow_mlp_smem_resolve<P, Q>();                                                       \
        k_wf_resolve<P, Q><<<grid, 256, smem, stream>>>(sc, wb, rl, rh, op, out, ctr);                   \
        break;
            NRT_FOR_EACH_DEGREE(NRT_CASE)
#undef NRT_CASE
            default: break;
        }
    }
    *launches += 3 + plan.n_classes;
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace nrt
