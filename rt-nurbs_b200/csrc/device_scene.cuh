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
    int n_slots;
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

// Indices into the device counter block (nrt_counters order).
enum Counter : int {
    kRays = 0, kBoxTests, kCandidates, kCulled, kSolves, kEvals, kFp64Solves, kFp64Final, kHits, kErrors, kLearned,
    kFallbacks, kRoundsDone, kNumCounters
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
