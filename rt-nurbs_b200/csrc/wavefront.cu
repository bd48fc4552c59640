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
//                    src/gpu/intersect.cu:169-183), runs the ray-space hull test
//                    on each leaf patch, and emits up to round_quota(r)
//                    surviving candidates; counts them per patch rank; saves
//                    the stack; rays with a non-empty stack stay active.
//   k_wf_scan        exclusive scan of the per-rank counts.
//   k_wf_scatter     (ray, slot) work items in rank order, ranks sorted by
//                    (p, q, slot).
//   k_wf_newton<P,Q> one launch per degree class present in the scene:
//                    consecutive lanes take consecutive items, so a warp
//                    shares one patch (broadcast loads) and one code path; a
//                    converged hit with t > 0 lowers the ray's 64-bit key
//                    (t bits << 32 | slot) with atomicMin.
//
// k_wf_resolve then recomputes each ray's winning solve (with the FP64 final
// step) and writes the hit record.  The closest hit is the minimum over all
// candidates nearer than the best hit, so the order in which candidates are
// solved does not change it.
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

// Hull test with a runtime degree (one code path for all patches).
__device__ __forceinline__ bool hull_misses_any(const float* __restrict__ blk, int n, int np, const RayFrame& r,
                                                const PatchRay& pr, float lim) {
    bool pos1 = true, neg1 = true, pos2 = true, neg2 = true;
    const float4* X = reinterpret_cast<const float4*>(blk);
    const float4* Y = reinterpret_cast<const float4*>(blk + np);
    const float4* Z = reinterpret_cast<const float4*>(blk + 2 * np);
    const float4* W = reinterpret_cast<const float4*>(blk + 3 * np);
    for (int k = 0; k < np / 4; ++k) {
        const float4 x = __ldg(X + k), y = __ldg(Y + k), z = __ldg(Z + k), w = __ldg(W + k);
        const float xs[4] = {x.x, x.y, x.z, x.w}, ys[4] = {y.x, y.y, y.z, y.w};
        const float zs[4] = {z.x, z.y, z.z, z.w}, ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            if (4 * k + l < n) {
                const float a = fmaf(r.n1x, xs[l], fmaf(r.n1y, ys[l], fmaf(r.n1z, zs[l], pr.e1 * ws[l])));
                const float b = fmaf(r.n2x, xs[l], fmaf(r.n2y, ys[l], fmaf(r.n2z, zs[l], pr.e2 * ws[l])));
                const float m = lim * ws[l];
                pos1 &= a > m;
                neg1 &= a < -m;
                pos2 &= b > m;
                neg2 &= b < -m;
            }
        }
    }
    return pos1 | neg1 | pos2 | neg2;
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
                const int4 h = sc.hdr[s];
                const double4 C = sc.centre[s];
                const int p = h.y & 15, q = (h.y >> 4) & 15;
                ++cands;
                if (op.hull_cull && ((h.y >> 8) & kFlagPositiveWeights)) {
                    const PatchRay pr = patch_ray(r, C.x, C.y, C.z);
                    if (ctr && op.counters) atomicAdd(ctr + kHullByDegree + p * 8 + q, 1ull);
                    if (hull_misses_any(sc.cp + h.x, (p + 1) * (q + 1), padded_points(p, q), r, pr,
                                        op.nw.eps + 8e-6f * (float)C.w)) {
                        ++culled;
                        continue;
                    }
                }
                emit[emitted++] = s;  // quota <= 24 and a leaf holds <= 8: stays below kEmitMax
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

__global__ void __launch_bounds__(256) k_wf_scatter(int round, int n_active, WfBuffers wb, int cur,
                                                    const int32_t* rank_of) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_active) return;
    const int i = round == 0 ? j : wb.active[cur][j];
    const int m = wb.emit_cnt[j];
    for (int e = 0; e < m; ++e) {
        const int s = wb.emit_slot[(long long)j * kEmitMax + e];
        const int rk = rank_of[s];
        const int pos = wb.offsets[rk] + aggregated_add(wb.cursor, rk);
        wb.items[pos] = make_int2(i, s);
    }
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

template <int P, int Q>
__global__ void __launch_bounds__(256) k_wf_newton(Scene sc, Rays rays, WfBuffers wb, int rank_lo, int rank_hi,
                                                   Opts op, int32_t* tests, unsigned long long* ctr) {
    const int begin = wb.offsets[rank_lo], end = wb.offsets[rank_hi];
    unsigned long long solves = 0, evals = 0, f64 = 0;
    NewtonOpts nw = op.nw;
    nw.fp64_final = 0;  // applied to the winner only, in k_wf_resolve
    for (int k = begin + blockIdx.x * blockDim.x + threadIdx.x; k < end; k += gridDim.x * blockDim.x) {
        const int2 it = wb.items[k];
        RayFrame r;
        load_ray(rays, it.x, r);
        const int4 h = sc.hdr[it.y];
        const double4 C = sc.centre[it.y];
        const PatchRay pr = patch_ray(r, C.x, C.y, C.z);
        float gu = 0.5f, gv = 0.5f;
        if (op.init_mode == 1) bilinear_guess(sc.corners + 4 * it.y, r, gu, gv);
        const NewtonOut o = newton<P, Q>(sc.cp + h.x, r, pr, gu, gv, (uint32_t)it.x + op.seed_offset, nw);
        ++solves;
        evals += (unsigned long long)(o.evals > 0 ? o.evals : -o.evals);
        f64 += (unsigned long long)o.fp64_solves;
        if (tests) atomicAdd(tests + it.x, 1);
        if (o.evals > 0 && o.t > 0.f) {
            const unsigned long long key = ((unsigned long long)__float_as_uint(o.t) << 32) | (unsigned)it.y;
            atomicMin(wb.best_key + it.x, key);
        }
    }
    if (ctr && op.counters) {
        count_add(ctr, kSolves, solves);
        count_add(ctr, kEvals, evals);
        count_add(ctr, kFp64Solves, f64);
        if (evals) atomicAdd(ctr + kEvalsByDegree + P * 8 + Q, evals);
    }
}

template <int P, int Q>
__device__ __forceinline__ NewtonOut resolve_one(const Scene& sc, int slot, const RayFrame& r, const Opts& op,
                                                 uint32_t seed) {
    const int4 h = sc.hdr[slot];
    const double4 C = sc.centre[slot];
    const PatchRay pr = patch_ray(r, C.x, C.y, C.z);
    float gu = 0.5f, gv = 0.5f;
    if (op.init_mode == 1) bilinear_guess(sc.corners + 4 * slot, r, gu, gv);
    return newton<P, Q>(sc.cp + h.x, r, pr, gu, gv, seed, op.nw);
}

__device__ __noinline__ NewtonOut resolve_any(const Scene& sc, int slot, const RayFrame& r, const Opts& op,
                                              uint32_t seed) {
    switch (sc.hdr[slot].y & 0xff) {
#define NRT_CASE(P, Q) \
    case (P) | ((Q) << 4): return resolve_one<P, Q>(sc, slot, r, op, seed);
        NRT_FOR_EACH_DEGREE(NRT_CASE)
#undef NRT_CASE
        default: break;
    }
    NewtonOut o;
    o.evals = 0;
    return o;
}

__global__ void __launch_bounds__(128) k_wf_resolve(Scene sc, Rays rays, long long n, Opts op, WfBuffers wb,
                                                    Hits out, unsigned long long* ctr) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long key = wb.best_key[i];
    bool hit = false;
    if (key != kNoHit) {
        const int slot = (int)(key & 0xffffffffu);
        RayFrame r;
        load_ray(rays, i, r);
        const NewtonOut o = resolve_any(sc, slot, r, op, (uint32_t)i + op.seed_offset);
        if (o.evals > 0 && o.t > 0.f) {
            hit = true;
            out.patch[i] = sc.hdr[slot].z;
            out.t[i] = o.t;
            out.u[i] = o.u;
            out.v[i] = o.v;
            if (out.iters) out.iters[i] = o.evals;
            if (out.geom) {
                const double4 C = sc.centre[slot];
                float* g = out.geom + 9 * i;
                g[0] = (float)(C.x + (double)o.sx); g[1] = (float)(C.y + (double)o.sy); g[2] = (float)(C.z + (double)o.sz);
                g[3] = o.ux; g[4] = o.uy; g[5] = o.uz;
                g[6] = o.vx; g[7] = o.vy; g[8] = o.vz;
            }
            if (ctr && op.counters) count_add(ctr, kFp64Final, (unsigned long long)o.fp64_final);
        } else if (ctr && o.evals <= 0) {
            atomicAdd(ctr + kErrors, 1ull);  // the recomputed winner must converge again
        }
    }
    if (!hit) {
        out.patch[i] = -1;
        out.t[i] = -1.f;
        out.u[i] = 0.f;
        out.v[i] = 0.f;
        if (out.iters) out.iters[i] = 0;
        if (out.geom)
            for (int a = 0; a < 9; ++a) out.geom[9 * i + a] = 0.f;
    }
    if (ctr && op.counters) count_add(ctr, kHits, hit ? 1 : 0);
}

// ---------------------------------------------------------------------------
size_t wavefront_scratch_bytes(long long n, int n_slots) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t N = (size_t)n, S = (size_t)n_slots + 1;
    return 2 * al(N * kStack * 4) + al(N * 4) + al(N * 8) + 2 * al(N * 4) + al(16) + al(N * kEmitMax * 4) +
           al(N * 4) + al(N * kEmitMax * 8) + 3 * al(S * 4);
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
    b.items = reinterpret_cast<int2*>(p); p += al(N * kEmitMax * 8);
    b.hist = reinterpret_cast<int32_t*>(p); p += al(S * 4);
    b.cursor = reinterpret_cast<int32_t*>(p); p += al(S * 4);
    b.offsets = reinterpret_cast<int32_t*>(p);
    return b;
}

cudaError_t launch_wavefront(const Scene& sc, const WfPlan& plan, const Rays& rays, long long n, const Opts& op,
                             const Hits& out, const WfBuffers& wb, int32_t* host_count, unsigned long long* ctr,
                             cudaStream_t stream, long long* launches, long long* rounds) {
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    int n_active = (int)n, cur = 0;
    for (int round = 0; n_active > 0; ++round) {
        if (round > 4096) return cudaErrorUnknown;  // unreachable: every round pops at least one entry per ray
        e = cudaMemsetAsync(wb.hist, 0, sizeof(int) * plan.n_slots, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(wb.counts + (1 - cur), 0, sizeof(int), stream);
        if (e != cudaSuccess) return e;
        k_wf_step<<<(unsigned)((n_active + 127) / 128), 128, 0, stream>>>(sc, rays, n, round, n_active,
                                                                         round_quota(round), op, wb, cur, out.tests,
                                                                         ctr, plan.rank_of);
        k_wf_scan<<<1, 1024, 0, stream>>>(plan.n_slots, wb);
        k_wf_scatter<<<(unsigned)((n_active + 255) / 256), 256, 0, stream>>>(round, n_active, wb, cur, plan.rank_of);
        *launches += 3 + plan.n_classes;
        *rounds += 1;
        for (int c = 0; c < plan.n_classes; ++c) {
            const int pq = plan.class_pq[c], rl = plan.class_rank[c], rh = plan.class_rank[c + 1];
            const unsigned grid = plan.class_grid[c];
            switch (pq) {
#define NRT_CASE(P, Q) \
    case (P) | ((Q) << 4): k_wf_newton<P, Q><<<grid, 256, 0, stream>>>(sc, rays, wb, rl, rh, op, out.tests, ctr); break;
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
    k_wf_resolve<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(sc, rays, n, op, wb, out, ctr);
    *launches += 1;
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace nrt
