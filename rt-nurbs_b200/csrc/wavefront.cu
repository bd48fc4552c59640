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
//                    it reaches, up to the round's quota of them; counts them per
//                    patch rank; saves the stack; rays with a non-empty stack
//                    stay active.
//   k_wf_scan        exclusive scan of the per-rank counts.
//   k_wf_scatter     work items (ray origin and direction, ray index, slot) in
//                    rank order, ranks sorted by (p, q, slot).
//   k_wf_newton<P,Q,MODE> one launch per degree class present in the scene: each
//                    warp takes 32 consecutive items (mostly one patch, so
//                    control point loads broadcast), runs the exact hull tests
//                    on them, compacts the survivors by ballot into a shared
//                    queue and runs Newton on full warps of survivors; a
//                    converged hit with t > 0 lowers the ray's 64-bit key
//                    (t bits << 32 | slot << 1 | flat) with a 128-bit
//                    compare-and-swap that stores the hit's (u, v) beside it.
//
// The resolve pass sorts the rays that hit by their winner's (p, q, slot) and
// k_wf_resolve<P,Q,LEARNED> recomputes each winning solve (same code and inputs) with
// the FP64 final step and writes the hit record.  The closest hit is the
// minimum over all candidates nearer than the best hit, so the order in which
// candidates are solved does not change it.
#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "kernels.h"
#include "wavefront.h"

#include <algorithm>

namespace nrt {
namespace dev {

namespace {

__device__ __forceinline__ float key_t(unsigned long long key) {
    return key == kNoHit ? INFINITY : __uint_as_float((unsigned)(key >> 32));
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

struct StepTally {
    unsigned long long boxes, cands, culled, err;
};

// One active ray j (ray index i) for one round: resume its saved stack, emit
// up to `quota` leaf patches, save the stack, and queue the ray for the next
// round if its stack is not empty.
// A stack entry (node, entry distance bits) is one 8-byte word, in local
// memory and in the saved stacks: one load or store per entry (4.5 % less
// step time than separate node and distance arrays).  Visiting the nearest
// child directly, without its push and pop, was slower (register pressure).
__device__ __forceinline__ void step_ray(const Scene& sc, const float4* top, int n_top, const Rays& rays, long long n,
                                         int round, int j, long long i, int quota, const Opts& op, const WfBuffers& wb,
                                         int cur, int32_t* tests, const int32_t* rank_of, StepTally& c) {
    RayFrame r;
    r.ox = __ldg(rays.ox + i); r.oy = __ldg(rays.oy + i); r.oz = __ldg(rays.oz + i);
    r.dx = __ldg(rays.dx + i); r.dy = __ldg(rays.dy + i); r.dz = __ldg(rays.dz + i);
    const float rdx = __frcp_rn(r.dx), rdy = __frcp_rn(r.dy), rdz = __frcp_rn(r.dz);
    int2 st[kStack];
    int sp;
    float best;
    if (round == 0) {
        sp = 1;
        st[0] = make_int2(0, 0);
        best = INFINITY;
        wb.best[i] = make_ulonglong2(kNoHit, 0ull);
        if (tests) tests[i] = 0;
    } else {
        sp = wb.stack_sp[i];
        for (int k = 0; k < sp; ++k) st[k] = wb.stack[(long long)k * n + i];
        best = key_t(wb.best[i].x);
    }
    int32_t* emit = wb.emit_slot + (long long)j * kEmitMax;
    int emitted = 0;
    while (sp > 0 && emitted < quota) {
        --sp;
        const int ref = st[sp].x;
        if (__int_as_float(st[sp].y) >= best) continue;
        if (ref >= 0) {
            // a node of the staged top of the tree from shared memory, any other through L1
            float4 lx, hx, ly, hy, lz, hz;
            int4 ch, cn;
            if (ref < n_top) {
                const float4* nd = top + 8 * ref;
                lx = nd[0]; hx = nd[1]; ly = nd[2]; hy = nd[3]; lz = nd[4]; hz = nd[5];
                ch = reinterpret_cast<const int4*>(nd)[6];
                cn = reinterpret_cast<const int4*>(nd)[7];
            } else {
                const float4* nd = reinterpret_cast<const float4*>(sc.nodes + ref);
                lx = __ldg(nd + 0); hx = __ldg(nd + 1); ly = __ldg(nd + 2); hy = __ldg(nd + 3);
                lz = __ldg(nd + 4); hz = __ldg(nd + 5);
                ch = __ldg(reinterpret_cast<const int4*>(nd + 6));
                cn = __ldg(reinterpret_cast<const int4*>(nd + 7));
            }
            const float LX[4] = {lx.x, lx.y, lx.z, lx.w}, HX[4] = {hx.x, hx.y, hx.z, hx.w};
            const float LY[4] = {ly.x, ly.y, ly.z, ly.w}, HY[4] = {hy.x, hy.y, hy.z, hy.w};
            const float LZ[4] = {lz.x, lz.y, lz.z, lz.w}, HZ[4] = {hz.x, hz.y, hz.z, hz.w};
            const int CH[4] = {ch.x, ch.y, ch.z, ch.w}, CN[4] = {cn.x, cn.y, cn.z, cn.w};
            float tt[4];
            int rr[4], k = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (CH[q] < 0 && CN[q] == 0) continue;
                ++c.boxes;
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
                    st[sp] = make_int2(rr[a], __float_as_int(tt[a]));
                    ++sp;
                } else {
                    ++c.err;  // stack overflow: the subtree is dropped and the error counted
                }
            }
        } else {
            const int first = leaf_first(ref), lc = leaf_count(ref);
            for (int s = first; s < first + lc; ++s) {
                ++c.cands;
                if (op.hull_cull >= 3 && obb_misses(sc.obb + 4 * s, r, op.nw.eps)) {
                    ++c.culled;
                    continue;
                }
                emit[emitted++] = s;  // quota <= 8 and a leaf holds <= 8: stays below kEmitMax
                aggregated_add(wb.hist, rank_of[s]);
            }
        }
    }
    for (int k = 0; k < sp; ++k) wb.stack[(long long)k * n + i] = st[k];
    wb.stack_sp[i] = sp;
    wb.emit_cnt[j] = emitted;
    if (sp > 0) {
        const int at = aggregated_add(wb.counts + (1 - cur), 0);
        wb.active[1 - cur][at] = (int)i;
    }
}

__device__ __forceinline__ void step_count(unsigned long long* ctr, const Opts& op, unsigned long long rays,
                                           const StepTally& c) {
    if (!ctr) return;
    if (op.counters) {
        count_add(ctr, kRays, rays);
        count_add(ctr, kBoxTests, c.boxes);
        count_add(ctr, kCandidates, c.cands);
        count_add(ctr, kCulled, c.culled);
    }
    if (c.err) atomicAdd(ctr + kErrors, c.err);
}

// The top of the 4-wide tree in shared memory: the tree is numbered breadth
// first, so its first `stage` nodes are its top levels (1, 5, 21, 85, 341
// nodes are whole levels), which every ray entering the tree visits.  The
// whole block copies them once (eight 16-byte words per node) before any of
// its threads traverses; returns how many nodes were staged.
__device__ __forceinline__ int stage_top(const Scene& sc, float4* top, int stage) {
    const int k = sc.n_nodes < stage ? sc.n_nodes : stage;
    const float4* src = reinterpret_cast<const float4*>(sc.nodes);
    for (int w = threadIdx.x; w < 8 * k; w += blockDim.x) top[w] = __ldg(src + w);
    __syncthreads();
    return k;
}

// Host-driven round: the host passes the round, its active count and list.
__global__ void __launch_bounds__(128) k_wf_step(Scene sc, Rays rays, long long n, int round, int n_active,
                                                 int quota, Opts op, WfBuffers wb, int cur, int32_t* tests,
                                                 unsigned long long* ctr, const int32_t* rank_of, int stage) {
    extern __shared__ float4 top[];
    const int n_top = stage_top(sc, top, stage);
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    StepTally c{};
    const long long i = j < n_active ? (round == 0 ? (long long)j : (long long)wb.active[cur][j]) : 0;
    if (j < n_active) step_ray(sc, top, n_top, rays, n, round, j, i, quota, op, wb, cur, tests, rank_of, c);
    step_count(ctr, op, (round == 0 && j < n_active) ? 1ull : 0ull, c);
}

// Device-driven round (inside the CUDA graph's loop): the round number is
// counts[2], the active list and count follow from it.  Persistent warps
// take 32 rays at a time from the round's work counter (counts[4]), each warp
// on its own (a block-wide grab made every warp wait for its block's slowest
// ray: 430 -> 461 Mrays/s without it), so the grid can be sized to the GPU
// and a round with few active rays costs no empty blocks.
__global__ void __launch_bounds__(128) k_wf_step_dev(Scene sc, Rays rays, long long n, Opts op, WfBuffers wb,
                                                     int32_t* tests, unsigned long long* ctr, const int32_t* rank_of,
                                                     int quota0, int quota_max, int stage) {
    extern __shared__ float4 top[];
    const int n_top = stage_top(sc, top, stage);  // once per block: the block stays for the whole round
    const int round = wb.counts[2], cur = round & 1;
    const int n_active = round == 0 ? (int)n : wb.counts[cur];
    const int quota = round_quota(round, quota0, quota_max);
    const int lane = threadIdx.x & 31;
    StepTally c{};
    unsigned long long seen = 0;
    for (;;) {  // each warp takes 32 rays at a time, without waiting for the rest of its block
        int base = 0;
        if (lane == 0) base = atomicAdd(wb.counts + 4, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n_active) break;
        const int j = base + lane;
        const long long i = j < n_active ? (round == 0 ? (long long)j : (long long)wb.active[cur][j]) : 0;
        if (j < n_active) step_ray(sc, top, n_top, rays, n, round, j, i, quota, op, wb, cur, tests, rank_of, c);
        if (j < n_active) ++seen;
    }
    step_count(ctr, op, round == 0 ? seen : 0ull, c);
}

// Work items of active ray j (ray index i), placed in rank order.
__device__ __forceinline__ void scatter_ray(const Rays& rays, int j, int i, const WfBuffers& wb,
                                            const int32_t* rank_of) {
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

__global__ void __launch_bounds__(256) k_wf_scatter(Rays rays, int round, int n_active, WfBuffers wb, int cur,
                                                    const int32_t* rank_of) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_active) return;
    scatter_ray(rays, j, round == 0 ? j : wb.active[cur][j], wb, rank_of);
}

// Persistent as k_wf_step_dev, on its own work counter (counts[5]).
__global__ void __launch_bounds__(256) k_wf_scatter_dev(Rays rays, long long n, WfBuffers wb,
                                                        const int32_t* rank_of) {
    const int round = wb.counts[2], cur = round & 1;
    const int n_active = round == 0 ? (int)n : wb.counts[cur];
    const int lane = threadIdx.x & 31;
    for (;;) {  // each warp takes 32 rays at a time
        int base = 0;
        if (lane == 0) base = atomicAdd(wb.counts + 5, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n_active) break;
        const int j = base + lane;
        if (j < n_active) scatter_ray(rays, j, round == 0 ? j : wb.active[cur][j], wb, rank_of);
    }
}

// Graph loop bookkeeping.  init: round 0, empty lists and work counters, and
// a clear histogram.  round_end: clear what the next round counts into (its
// active list's count and the work counters; k_wf_scan already cleared the
// histogram), advance the round and continue the loop while rays are left.
__global__ void __launch_bounds__(256) k_wf_init(WfBuffers wb, int n_slots) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_slots; k += gridDim.x * blockDim.x) wb.hist[k] = 0;
    if (blockIdx.x == 0 && threadIdx.x < 8) wb.counts[threadIdx.x] = 0;
}

constexpr int kMaxRounds = 4096;  // every round pops at least one stack entry per active ray

__global__ void k_wf_round_end(WfBuffers wb, cudaGraphConditionalHandle loop, unsigned long long* ctr) {
    if (threadIdx.x != 0) return;
    const int round = wb.counts[2], cur = round & 1;
    const int next = wb.counts[1 - cur];
    const bool more = next > 0 && round + 1 < kMaxRounds;
    if (ctr) {
        atomicAdd(ctr + kRoundsDone, 1ull);
        if (next > 0 && !more) atomicAdd(ctr + kErrors, 1ull);
    }
    wb.counts[cur] = 0;  // the next round queues its survivors into this list
    wb.counts[4] = 0;
    wb.counts[5] = 0;
    wb.counts[2] = round + 1;
    cudaGraphSetConditional(loop, more ? 1u : 0u);
}

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
        const int hk = wb.hist[k];
        wb.offsets[k] = run;
        run += hk;
        wb.cursor[k] = 0;
        wb.hist[k] = 0;  // cleared for the next round
    }
    if (t == 1023) wb.offsets[m] = part[1023];
}

// emit their winning slot (counted per rank, as a round's candidates are).
__global__ void __launch_bounds__(256) k_wf_resolve_emit(long long n, Opts op, WfBuffers wb, Hits out,
                                                         const int32_t* rank_of, unsigned long long* ctr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long key = wb.best[i].x;
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
    const int s = (int)((key & 0xffffffffu) >> 1);
    wb.emit_cnt[i] = 1;
    wb.emit_slot[(long long)i * kEmitMax] = s;
    aggregated_add(wb.hist, rank_of[s]);
}

// ---------------------------------------------------------------------------
size_t wavefront_scratch_bytes(long long n, int n_slots) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t N = (size_t)n, S = (size_t)n_slots + 1;
    return al(N * kStack * 8) + al(N * 4) + al(N * 16) + 2 * al(N * 4) + al(32) + al(N * kEmitMax * 4) +
           al(N * 4) + al(N * kEmitMax * sizeof(WfItem)) + al(N * kEmitMax * 8) + 3 * al(S * 4) + al(64 * 4);
}

WfBuffers wavefront_carve(void* base, long long n, int n_slots) {
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t N = (size_t)n, S = (size_t)n_slots + 1;
    char* p = static_cast<char*>(base);
    WfBuffers b;
    b.stack = reinterpret_cast<int2*>(p); p += al(N * kStack * 8);
    b.stack_sp = reinterpret_cast<int32_t*>(p); p += al(N * 4);
    b.best = reinterpret_cast<ulonglong2*>(p); p += al(N * 16);
    b.active[0] = reinterpret_cast<int32_t*>(p); p += al(N * 4);
    b.active[1] = reinterpret_cast<int32_t*>(p); p += al(N * 4);
    b.counts = reinterpret_cast<int32_t*>(p); p += al(32);
    b.emit_slot = reinterpret_cast<int32_t*>(p); p += al(N * kEmitMax * 4);
    b.emit_cnt = reinterpret_cast<int32_t*>(p); p += al(N * 4);
    b.items = reinterpret_cast<WfItem*>(p); p += al(N * kEmitMax * sizeof(WfItem));
    b.guess = reinterpret_cast<float2*>(p); p += al(N * kEmitMax * 8);
    b.hist = reinterpret_cast<int32_t*>(p); p += al(S * 4);
    b.cursor = reinterpret_cast<int32_t*>(p); p += al(S * 4);
    b.offsets = reinterpret_cast<int32_t*>(p); p += al(S * 4);
    b.class_cursor = reinterpret_cast<int32_t*>(p);
    return b;
}

// The per-class kernels live in wf_solve.cu, one object per u-degree.
static void wf_newton_class(int p, int q, const WfClassLaunch& L) {
    switch (p) {
        case 1: wf_newton_p1(q, L); break;
        case 2: wf_newton_p2(q, L); break;
        case 3: wf_newton_p3(q, L); break;
        case 4: wf_newton_p4(q, L); break;
        case 5: wf_newton_p5(q, L); break;
        case 6: wf_newton_p6(q, L); break;
        case 7: wf_newton_p7(q, L); break;
        default: break;
    }
}

static void wf_resolve_class(int p, int q, const WfClassLaunch& L) {
    switch (p) {
        case 1: wf_resolve_p1(q, L); break;
        case 2: wf_resolve_p2(q, L); break;
        case 3: wf_resolve_p3(q, L); break;
        case 4: wf_resolve_p4(q, L); break;
        case 5: wf_resolve_p5(q, L); break;
        case 6: wf_resolve_p6(q, L); break;
        case 7: wf_resolve_p7(q, L); break;
        default: break;
    }
}

cudaError_t launch_wavefront(const Scene& sc, const WfPlan& plan, const Rays& rays, long long n, const Opts& op,
                             const Hits& out, const WfBuffers& wb, int32_t* host_count, unsigned long long* ctr,
                             cudaStream_t stream, long long* launches, long long* rounds, cudaEvent_t* ev,
                             double* newton_ms, long long* newton_launches, int quota0, int quota_max,
                             int stage_nodes) {
    if (n <= 0) return cudaSuccess;
    const int stage = stage_nodes < 1 ? 1 : (stage_nodes > kMaxStagedNodes ? kMaxStagedNodes : stage_nodes);
    cudaError_t e = cudaSuccess;
    int n_active = (int)n, cur = 0;
    WfClassLaunch L{};
    L.sc = &sc; L.rays = &rays; L.wb = &wb; L.op = &op; L.out = &out;
    L.tests = out.tests; L.ctr = ctr; L.stream = stream;
    L.mode = op.init_mode == 2 ? kWfLearned : (op.col_feat ? kWfCollect : kWfPlain);
    for (int round = 0; n_active > 0; ++round) {
        if (round > 4096) return cudaErrorUnknown;  // unreachable: every round pops at least one entry per ray
        e = cudaMemsetAsync(wb.hist, 0, sizeof(int) * plan.n_slots, stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(wb.counts + (1 - cur), 0, sizeof(int), stream);
        if (e != cudaSuccess) return e;
        k_wf_step<<<(unsigned)((n_active + 127) / 128), 128, staged_bytes(stage), stream>>>(
            sc, rays, n, round, n_active, round_quota(round, quota0, quota_max), op, wb, cur, out.tests, ctr,
            plan.rank_of, stage);
        k_wf_scan<<<1, 1024, 0, stream>>>(plan.n_slots, wb);
        k_wf_scatter<<<(unsigned)((n_active + 255) / 256), 256, 0, stream>>>(rays, round, n_active, wb, cur,
                                                                             plan.rank_of);
        *launches += 3 + plan.n_classes * (L.mode == kWfLearned ? 2 : 1);  // learned: the guess kernels too
        *rounds += 1;
        const bool timed = ev && newton_ms;
        if (timed) cudaEventRecord(ev[0], stream);
        for (int c = 0; c < plan.n_classes; ++c) {
            L.cls = c;
            L.rank_lo = plan.class_rank[c];
            L.rank_hi = plan.class_rank[c + 1];
            L.grid = plan.class_grid[c];
            wf_newton_class(plan.class_pq[c] & 15, plan.class_pq[c] >> 4, L);
        }
        if (timed) cudaEventRecord(ev[1], stream);
        e = cudaMemcpyAsync(host_count, wb.counts + (1 - cur), sizeof(int), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return e;
        if (timed) {
            float ms = 0.f;
            e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
            if (e != cudaSuccess) return e;
            *newton_ms += ms;
            if (newton_launches) *newton_launches += plan.n_classes;
        }
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
        L.cls = c;
        L.rank_lo = plan.class_rank[c];
        L.rank_hi = plan.class_rank[c + 1];
        L.grid = plan.class_grid[c];
        wf_resolve_class(plan.class_pq[c] & 15, plan.class_pq[c] >> 4, L);
    }
    *launches += 3 + plan.n_classes * ((L.mode == kWfLearned && out.iters) ? 2 : 1);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace nrt

namespace nrt {
namespace dev {

namespace {

// Records the launches of `fill` on stream cs into a new graph.
template <class F>
cudaError_t capture(cudaStream_t cs, cudaGraph_t* g, F&& fill) {
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return e;
    fill();
    const cudaError_t le = cudaGetLastError();
    e = cudaStreamEndCapture(cs, g);
    return le != cudaSuccess ? le : e;
}

// The degree classes' kernels of one step as parallel branches of the graph
// being captured on cs: they touch disjoint work items and meet only in
// atomics (the nearest-hit records, the counters), so the GPU may run one
// class's blocks in another's tail.  launch(c) issues class c on L.stream.
constexpr int kClassBranches = 4;

template <class F>
void fork_classes(cudaStream_t cs, cudaStream_t* side, cudaEvent_t* ev, int n_classes, WfClassLaunch& L,
                  F&& launch) {
    cudaEventRecord(ev[0], cs);
    const int nb = std::min(n_classes, kClassBranches);
    for (int b = 0; b < nb; ++b) cudaStreamWaitEvent(side[b], ev[0], 0);
    for (int c = 0; c < n_classes; ++c) {
        L.stream = side[c % kClassBranches];
        launch(c);
    }
    for (int b = 0; b < nb; ++b) {
        cudaEventRecord(ev[1 + b], side[b]);
        cudaStreamWaitEvent(cs, ev[1 + b], 0);
    }
    L.stream = cs;
}

}  // namespace

cudaError_t build_wavefront_graph(const Scene& sc, const WfPlan& plan, const Rays& rays, long long n,
                                  long long chunk, const Opts& op, const Hits& out, const WfBuffers& wb,
                                  unsigned long long* ctr, const WfTuning& tu, cudaGraphExec_t* exec,
                                  long long* passes) {
    *exec = nullptr;
    *passes = 0;
    if (n <= 0 || chunk <= 0) return cudaErrorInvalidValue;
    cudaGraph_t g = nullptr;
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    cudaStream_t side[kClassBranches] = {};
    cudaEvent_t ev[1 + kClassBranches] = {};
    for (int b = 0; b < kClassBranches && e == cudaSuccess; ++b) e = cudaStreamCreateWithFlags(&side[b], cudaStreamNonBlocking);
    for (int b = 0; b < 1 + kClassBranches && e == cudaSuccess; ++b) e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
    cudaGraphNode_t prev = nullptr;
    const int mode = op.init_mode == 2 ? kWfLearned : (op.col_feat ? kWfCollect : kWfPlain);
    for (long long at = 0; at < n && e == cudaSuccess; at += chunk) {
        const long long m = std::min(chunk, n - at);
        const Rays rc{rays.ox + at, rays.oy + at, rays.oz + at, rays.dx + at, rays.dy + at, rays.dz + at};
        const Hits hc{out.patch + at, out.t + at, out.u + at, out.v + at, out.iters ? out.iters + at : nullptr,
                      out.tests ? out.tests + at : nullptr, out.geom ? out.geom + 9 * at : nullptr};
        Opts oc = op;
        oc.seed_offset = op.seed_offset + (uint32_t)at;  // seeds follow the global ray index
        WfClassLaunch L{};
        L.sc = &sc; L.rays = &rc; L.wb = &wb; L.op = &oc; L.out = &hc;
        L.tests = hc.tests; L.ctr = ctr; L.stream = cs; L.mode = mode;
        // the pass's set-up
        cudaGraph_t pre = nullptr;
        e = capture(cs, &pre, [&] {
            k_wf_init<<<std::max(1u, std::min(148u * 2, (unsigned)((plan.n_slots + 255) / 256))), 256, 0, cs>>>(
                wb, plan.n_slots);
        });
        cudaGraphNode_t n_pre = nullptr;
        if (e == cudaSuccess) e = cudaGraphAddChildGraphNode(&n_pre, g, prev ? &prev : nullptr, prev ? 1 : 0, pre);
        if (pre) cudaGraphDestroy(pre);
        // the rounds: a while node whose body is one round
        cudaGraphConditionalHandle loop = 0;
        if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault);
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = loop;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t n_loop = nullptr;
        if (e == cudaSuccess) e = cudaGraphAddNode(&n_loop, g, &n_pre, 1, &cp);
        if (e == cudaSuccess) {
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
            if (e == cudaSuccess) {
                const unsigned step_grid = (unsigned)std::max(1LL, std::min<long long>((m + 127) / 128, tu.step_blocks));
                const unsigned scat_grid = (unsigned)std::max(1LL, std::min<long long>((m + 255) / 256, tu.scatter_blocks));
                const int stage = tu.stage_nodes < 1 ? 1 : (tu.stage_nodes > kMaxStagedNodes ? kMaxStagedNodes
                                                                                               : tu.stage_nodes);
                k_wf_step_dev<<<step_grid, 128, staged_bytes(stage), cs>>>(sc, rc, m, oc, wb, hc.tests, ctr,
                                                                           plan.rank_of, tu.quota0, tu.quota_max,
                                                                           stage);
                k_wf_scan<<<1, 1024, 0, cs>>>(plan.n_slots, wb);
                k_wf_scatter_dev<<<scat_grid, 256, 0, cs>>>(rc, m, wb, plan.rank_of);
                fork_classes(cs, side, ev, plan.n_classes, L, [&](int c) {
                    L.cls = c;
                    L.rank_lo = plan.class_rank[c];
                    L.rank_hi = plan.class_rank[c + 1];
                    L.grid = tu.class_blocks > 0 ? (unsigned)tu.class_blocks : plan.class_grid[c];
                    wf_newton_class(plan.class_pq[c] & 15, plan.class_pq[c] >> 4, L);
                });
                k_wf_round_end<<<1, 32, 0, cs>>>(wb, loop, ctr);
                const cudaError_t le = cudaGetLastError();
                cudaGraph_t got = nullptr;
                e = cudaStreamEndCapture(cs, &got);
                if (e == cudaSuccess) e = le;
            }
        }
        // resolve: hit rays sorted by their winner's (p, q, slot), one kernel per class
        cudaGraph_t post = nullptr;
        if (e == cudaSuccess)
            e = capture(cs, &post, [&] {
                cudaMemsetAsync(wb.hist, 0, sizeof(int) * plan.n_slots, cs);
                k_wf_resolve_emit<<<(unsigned)((m + 255) / 256), 256, 0, cs>>>(m, oc, wb, hc, plan.rank_of, ctr);
                k_wf_scan<<<1, 1024, 0, cs>>>(plan.n_slots, wb);
                k_wf_scatter<<<(unsigned)((m + 255) / 256), 256, 0, cs>>>(rc, 0, (int)m, wb, 0, plan.rank_of);
                fork_classes(cs, side, ev, plan.n_classes, L, [&](int c) {
                    L.cls = c;
                    L.rank_lo = plan.class_rank[c];
                    L.rank_hi = plan.class_rank[c + 1];
                    L.grid = plan.class_grid[c];
                    wf_resolve_class(plan.class_pq[c] & 15, plan.class_pq[c] >> 4, L);
                });
            });
        cudaGraphNode_t n_post = nullptr;
        if (e == cudaSuccess) e = cudaGraphAddChildGraphNode(&n_post, g, &n_loop, 1, post);
        if (post) cudaGraphDestroy(post);
        prev = n_post;
        ++*passes;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(exec, g, 0);
    if (e != cudaSuccess) *exec = nullptr;
    if (g) cudaGraphDestroy(g);
    if (cs) cudaStreamDestroy(cs);
    for (cudaStream_t st : side)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    return e;
}

}  // namespace dev
}  // namespace nrt
