// intersect_pixel.cu -- one thread per ray: 4-wide BVH traversal, per-patch
// hull test, initial guess, Newton.  The SIMT counterpart of the reference's
// calculateIntersect (src/gpu/intersect.cu:20-194), with the same closest-hit
// rule (accept 0 < t < t_max, strictly nearer than the current hit) and the
// same per-patch method; it is the plain baseline the wavefront path is
// measured against.
#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "kernels.h"
#include "wavefront.h"

namespace nrt {
namespace dev {

struct Best {
    float t_max;
    int slot;
    NewtonOut o;
};

struct Tally {
    unsigned long long box, cand, culled, solves, evals, f64s, f64f, err, flat;
};

template <int P, int Q, bool FINAL>
__device__ __forceinline__ void test_patch(const Scene& sc, int slot, const RayFrame& r, float te, const Opts& op,
                                           uint32_t seed, Best& b, Tally& c, unsigned long long* ctr) {
    const int4 h = sc.hdr[slot];
    const double4 C = sc.centre[slot];
    const float* __restrict__ blk = sc.cp + h.x;
    const PatchRay pr = patch_ray(r, C.x, C.y, C.z);
    ++c.cand;
    if (op.hull_cull && ((h.y >> 8) & kFlagPositiveWeights)) {
        const float lim = op.nw.eps + 8e-6f * (float)C.w;
        if (op.counters) atomicAdd(ctr + kHullByDegree + P * 8 + Q, 1ull);
        if (hull_misses<P, Q>(blk, r, pr, lim)) {
            ++c.culled;
            return;
        }
    }
    float gu = 0.5f, gv = 0.5f;
    if (op.init_mode == 1) bilinear_guess(sc.corners + 4 * slot, r, gu, gv);
    {
        NewtonOut o;
        if (flat_accept<P, Q>(blk, r, pr, sc.delta[slot], te, op, gu, gv, o) && 0.f < o.t && o.t < b.t_max) {
            ++c.flat;
            b.t_max = o.t; b.slot = slot; b.o = o;
            return;
        }
    }
    NewtonOpts nw = op.nw;  // the FP64 decisions apply to patches with widely spread weights
    nw.fp64_band = op.nw.fp64_band && ((h.y >> 8) & kFlagWideWeights);
    const NewtonOut o = newton<P, Q, FINAL>(blk, r, pr, gu, gv, seed, nw);
    ++c.solves;
    c.evals += (unsigned long long)o.done;
    c.f64s += (unsigned long long)o.fp64_solves;
    c.f64f += (unsigned long long)o.fp64_final;
    if (op.counters) atomicAdd(ctr + kEvalsByDegree + P * 8 + Q, (unsigned long long)o.done);
    if (o.evals > 0 && 0.f < o.t && o.t < b.t_max) {
        b.t_max = o.t;
        b.slot = slot;
        b.o = o;
    }
}

// Degree dispatch: one specialised, fully unrolled instantiation per (p, q).
template <bool FINAL>
__device__ __noinline__ void test_patch_any(const Scene& sc, int slot, const RayFrame& r, float te, const Opts& op,
                                            uint32_t seed, Best& b, Tally& c, unsigned long long* ctr) {
    const int pq = sc.hdr[slot].y & 0xff;
    switch (pq) {
#define NRT_CASE(P, Q) \
    case (P) | ((Q) << 4): test_patch<P, Q, FINAL>(sc, slot, r, te, op, seed, b, c, ctr); break;
        NRT_FOR_EACH_DEGREE(NRT_CASE)
#undef NRT_CASE
        default: ++c.err; break;
    }
}

template <bool FINAL>
__device__ __forceinline__ void trace_pixel(const Scene& sc, const Rays& rays, long long i, const Opts& op,
                                            const Hits& out, unsigned long long* ctr) {
    RayFrame r;
    r.ox = rays.ox[i]; r.oy = rays.oy[i]; r.oz = rays.oz[i];
    r.dx = rays.dx[i]; r.dy = rays.dy[i]; r.dz = rays.dz[i];
    ray_planes(r);
    const float rdx = __frcp_rn(r.dx), rdy = __frcp_rn(r.dy), rdz = __frcp_rn(r.dz);
    const uint32_t seed = (uint32_t)i + op.seed_offset;
    Best b;
    b.t_max = INFINITY;
    b.slot = -1;
    Tally c = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int st_ref[kStack];
    float st_t[kStack];
    int sp = 0;
    st_ref[sp] = 0;
    st_t[sp] = 0.f;
    ++sp;
    while (sp > 0) {
        --sp;
        const int ref = st_ref[sp];
        const float te = st_t[sp];
        if (te >= b.t_max) continue;
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
            int rr[4];
            int k = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (CH[q] < 0 && CN[q] == 0) continue;  // empty slot
                ++c.box;
                const float t = slab(LX[q], LY[q], LZ[q], HX[q], HY[q], HZ[q], r, rdx, rdy, rdz);
                if (t < b.t_max) {
                    tt[k] = t;
                    rr[k] = CH[q] >= 0 ? CH[q] : leaf_ref(~CH[q], CN[q]);
                    ++k;
                }
            }
            // push farthest first so the nearest child is popped next
            for (int a = 1; a < k; ++a)
                for (int j = a; j > 0 && tt[j] > tt[j - 1]; --j) {
                    const float tf = tt[j]; tt[j] = tt[j - 1]; tt[j - 1] = tf;
                    const int rf = rr[j]; rr[j] = rr[j - 1]; rr[j - 1] = rf;
                }
            for (int a = 0; a < k; ++a) {
                if (sp < kStack) {
                    st_ref[sp] = rr[a];
                    st_t[sp] = tt[a];
                    ++sp;
                } else {
                    ++c.err;  // stack overflow: the subtree is dropped and the error counted
                }
            }
        } else {
            const int first = leaf_first(ref), cnt = leaf_count(ref);
            for (int s = first; s < first + cnt; ++s) test_patch_any<FINAL>(sc, s, r, te, op, seed, b, c, ctr);
        }
    }
    if (b.slot >= 0) {
        const int4 h = sc.hdr[b.slot];
        out.patch[i] = h.z;
        out.t[i] = b.o.t;
        out.u[i] = b.o.u;
        out.v[i] = b.o.v;
        if (out.iters) out.iters[i] = b.o.evals;
        if (out.geom) {
            const double4 C = sc.centre[b.slot];
            float* g = out.geom + 9 * i;
            g[0] = (float)(C.x + (double)b.o.sx); g[1] = (float)(C.y + (double)b.o.sy); g[2] = (float)(C.z + (double)b.o.sz);
            g[3] = b.o.ux; g[4] = b.o.uy; g[5] = b.o.uz;
            g[6] = b.o.vx; g[7] = b.o.vy; g[8] = b.o.vz;
        }
    } else {
        out.patch[i] = -1;
        out.t[i] = -1.f;
        out.u[i] = 0.f;
        out.v[i] = 0.f;
        if (out.iters) out.iters[i] = 0;
        if (out.geom)
            for (int a = 0; a < 9; ++a) out.geom[9 * i + a] = 0.f;
    }
    if (out.tests) out.tests[i] = (int)c.solves;
    if (ctr && op.counters) {
        count_add(ctr, kRays, 1);
        count_add(ctr, kBoxTests, c.box);
        count_add(ctr, kCandidates, c.cand);
        count_add(ctr, kCulled, c.culled);
        count_add(ctr, kSolves, c.solves);
        count_add(ctr, kEvals, c.evals);
        count_add(ctr, kFp64Solves, c.f64s);
        count_add(ctr, kFp64Final, c.f64f);
        count_add(ctr, kHits, b.slot >= 0 ? 1 : 0);
        count_add(ctr, kErrors, c.err);
        count_add(ctr, kFlatSkips, c.flat);
    } else if (ctr && c.err) {
        atomicAdd(ctr + kErrors, c.err);
    }
}

// FINAL: instantiated with and without the FP64 final step (op.nw.fp64_final
// picks one at launch).
template <bool FINAL>
__global__ void __launch_bounds__(128) k_intersect_pixel(Scene sc, Rays rays, long long n, Opts op, Hits out,
                                                         unsigned long long* ctr) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) trace_pixel<FINAL>(sc, rays, i, op, out, ctr);
}

// Same, for the ray indices list[0 .. *count) (count known only on the device).
template <bool FINAL>
__global__ void __launch_bounds__(128) k_intersect_pixel_list(Scene sc, Rays rays, const int32_t* list,
                                                              const int32_t* count, Opts op, Hits out,
                                                              unsigned long long* ctr) {
    const int m = *count;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        trace_pixel<FINAL>(sc, rays, list[k], op, out, ctr);
}

cudaError_t launch_intersect_pixel(const Scene& sc, const Rays& rays, long long n, const Opts& op, const Hits& out,
                                   unsigned long long* ctr, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int threads = 128;
    const long long blocks = (n + threads - 1) / threads;
    if (op.nw.fp64_final) k_intersect_pixel<true><<<(unsigned)blocks, threads, 0, stream>>>(sc, rays, n, op, out, ctr);
    else k_intersect_pixel<false><<<(unsigned)blocks, threads, 0, stream>>>(sc, rays, n, op, out, ctr);
    return cudaGetLastError();
}

cudaError_t launch_intersect_pixel_list(const Scene& sc, const Rays& rays, const int32_t* list,
                                        const int32_t* list_count, long long max_n, const Opts& op, const Hits& out,
                                        unsigned long long* ctr, cudaStream_t stream) {
    if (max_n <= 0) return cudaSuccess;
    long long blocks = (max_n + 127) / 128;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (op.nw.fp64_final)
        k_intersect_pixel_list<true><<<(unsigned)blocks, 128, 0, stream>>>(sc, rays, list, list_count, op, out, ctr);
    else
        k_intersect_pixel_list<false><<<(unsigned)blocks, 128, 0, stream>>>(sc, rays, list, list_count, op, out, ctr);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace nrt
