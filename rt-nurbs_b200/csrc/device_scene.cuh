// device_scene.cuh -- device-side views of a scene, rays, hits and options.
#pragma once

#include <cstdint>

#include "mlp.cuh"
#include "patch_math.cuh"

namespace nrt {
namespace dev {

struct Node4 {  // same layout as nrt::Node4 (128 bytes)
    float lo_x[4], hi_x[4], lo_y[4], hi_y[4], lo_z[4], hi_z[4];
    int32_t child[4];
    int32_t count[4];
};

struct Scene {
    const Node4* nodes;      // 4-wide BVH, root at 0
    const int4* hdr;         // per slot: block offset, p|q<<4|flags<<8, global id, surface
    const double4* centre;   // per slot: patch centre (x, y, z) and radius of the local points
    const float* cp;         // SoA blocks in patch-local homogeneous coordinates
    const float4* corners;   // per slot: four dehomogenised world-space corners q00, q10, q11, q01
    const float* delta;      // per slot: flatness (patchDelta) for flat-skip
    const PatchFrame* frames;  // per slot: frame of the learned guess's features
    const float4* obb;       // per slot: oriented box of the control points, 4 float4 (see obb_misses)
    const float4* leafbox;   // per slot: the box of its BVH leaf (lo xyz, hi xyz in two float4), as the
                             // parent node stores it (the flat-skip's entry distance)
    int n_slots;
    int n_nodes;             // 4-wide nodes (breadth-first: the top levels come first)
};

struct Rays {
    const float *ox, *oy, *oz, *dx, *dy, *dz;
};

struct Hits {
    int32_t* patch;
    float *t, *u, *v;
    int32_t* iters;
    int32_t* tests;
    float* geom;
};

struct Opts {
    NewtonOpts nw;
    int init_mode;      // 0 midpoint, 1 reference bilinear, 2 learned
    int hull_cull;
    uint32_t seed_offset;
    float flat_threshold;
    float cam_k;
    int counters;       // 1: accumulate all counters; 0: only the error count
    int learned_iters;  // evaluations from the network's guess before the plain fallback
    MlpParams mlp;      // network (init_mode 2)
    float* col_feat;    // training-pair collection (null: off): capacity x 12
    float* col_targ;    // capacity x 2
    unsigned long long* col_count;
    long long col_cap;
};

// Flat-skip (src/gpu/intersect.cu:104-123): when the patch's projected
// flatness delta * cam_k / te (te: the ray's entry distance into the leaf box)
// is below the pixel threshold, the patch is evaluated at the initial guess
// and the guess is accepted when its projected plane residual is below the
// threshold too.  Returns true with o holding the point (evals 0, flat 1);
// the caller still requires 0 < t (and t below its best hit).
template <int P, int Q>
__device__ __forceinline__ bool flat_accept(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                            float delta, float te, const Opts& op, float gu, float gv, NewtonOut& o) {
    if (!(op.flat_threshold > 0.f && delta * op.cam_k / te < op.flat_threshold)) return false;
    float H[4], Hu[4], Hv[4];
    eval_patch<P, Q>(blk, gu, gv, H, Hu, Hv);
    const float iw = __frcp_rn(H[3]);
    const float sx = H[0] * iw, sy = H[1] * iw, sz = H[2] * iw;
    const float r1 = fmaf(r.n1x, sx, fmaf(r.n1y, sy, fmaf(r.n1z, sz, pr.e1)));
    const float r2 = fmaf(r.n2x, sx, fmaf(r.n2y, sy, fmaf(r.n2z, sz, pr.e2)));
    if (!((fabsf(r1) + fabsf(r2)) * op.cam_k / te < op.flat_threshold)) return false;
    o.evals = 0;
    o.u = gu; o.v = gv;
    o.t = fmaf(sx, r.dx, fmaf(sy, r.dy, fmaf(sz, r.dz, pr.tc)));
    o.sx = sx; o.sy = sy; o.sz = sz;
    o.ux = (Hu[0] - sx * Hu[3]) * iw; o.uy = (Hu[1] - sy * Hu[3]) * iw; o.uz = (Hu[2] - sz * Hu[3]) * iw;
    o.vx = (Hv[0] - sx * Hv[3]) * iw; o.vy = (Hv[1] - sy * Hv[3]) * iw; o.vz = (Hv[2] - sz * Hv[3]) * iw;
    o.fp64_solves = 0;
    o.fp64_final = 0;
    o.flat = 1;
    o.done = 1;  // the one evaluation at the guess
    return true;
}

// Indices into the device counter block (nrt_counters order).
enum Counter : int {
    kRays = 0, kBoxTests, kCandidates, kCulled, kSolves, kEvals, kFp64Solves, kFp64Final, kHits, kErrors, kLearned,
    kFallbacks, kRoundsDone, kFlatSkips, kLearnedConverged, kFallbackConverged, kNumCounters
};
// Followed by 64 per-degree evaluation counts and 64 per-degree hull-test counts.
constexpr int kEvalsByDegree = kNumCounters, kHullByDegree = kNumCounters + 64, kCounterWords = kNumCounters + 128;

constexpr int kStack = 48;

// Leaf reference on the traversal stack: ~(first << 3 | (count - 1)).
__device__ __forceinline__ int leaf_ref(int first, int count) { return ~((first << 3) | (count - 1)); }
__device__ __forceinline__ int leaf_first(int ref) { return (~ref) >> 3; }
__device__ __forceinline__ int leaf_count(int ref) { return ((~ref) & 7) + 1; }

// Warp-aggregated counter add (per-lane atomics when the warp is partial).
__device__ __forceinline__ void count_add(unsigned long long* ctr, int which, unsigned long long v) {
    if (!ctr) return;
    const unsigned mask = __activemask();
    if (mask == 0xffffffffu) {
        unsigned long long s = v;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && s) atomicAdd(ctr + which, s);
    } else if (v) {
        atomicAdd(ctr + which, v);
    }
}

}  // namespace dev
}  // namespace nrt
