// wavefront.h -- buffers and plan of the batched (wavefront) schedule.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device_scene.cuh"

namespace nrt {
namespace dev {

constexpr int kEmitMax = 16;   // candidates one ray may emit in one round (quota <= 8, plus one leaf)

// A (ray, patch) work item carries its ray so that the per-class kernels read
// items sequentially instead of gathering rays at random.
struct __align__(16) WfItem {
    float ox, oy, oz, dx, dy, dz;
    int32_t ray, slot;
};
constexpr unsigned long long kNoHit = ~0ull;

// Candidates per ray in round r: q0, 2 q0, 4 q0, ... up to qmax (the
// launch-shape default is 4, then 8, and nrt_intersect_noalloc runs with the
// scene's tuned values too; the training-pair collection uses 1, 2, 4, 8).  qmax <= 8 keeps a round's emissions (quota plus the rest
// of one leaf of <= 8 patches) within kEmitMax.
__host__ __device__ constexpr int round_quota(int r, int q0 = 1, int qmax = 8) {
    return r >= 4 ? qmax : ((q0 << r) < qmax ? (q0 << r) : qmax);
}

// Scratch of one wavefront launch over n rays (device pointers).
struct WfBuffers {
    int2* stack;                   // kStack * n (node, entry distance bits), entry k of ray i at [k * n + i]
    int32_t* stack_sp;             // n
    ulonglong2* best;              // n: the nearest hit so far, {key, (u bits << 32) | v bits}; the key
                                   // (t bits << 32) | slot << 1 | flat orders hits by t, then slot
    int32_t* active[2];            // n each: ray indices still traversing (ping-pong)
    int32_t* counts;               // 8 ints: active counts of the two lists, round (graph), -, work
                                   // counters of the persistent step and scatter kernels (graph)
    int32_t* emit_slot;            // n * kEmitMax: candidates emitted this round, by active position
    int32_t* emit_cnt;             // n
    WfItem* items;                 // n * kEmitMax: work items of a round, in rank order
    float2* guess;                 // n * kEmitMax: the network's raw (u, v) for each work item (learned guess)
    int32_t* hist;                 // n_slots + 1
    int32_t* cursor;               // n_slots + 1
    int32_t* offsets;              // n_slots + 1
    int32_t* class_cursor;         // 64: next unclaimed item of each degree class
};

// Per-scene schedule data: patch ranks in (p, q, slot) order and the degree
// classes present.
struct WfPlan {
    const int32_t* rank_of;   // device: slot -> rank
    int n_slots;
    int n_classes;
    int class_pq[64];         // p | q << 4
    int class_rank[65];       // first rank of each class; [n_classes] = n_slots
    unsigned class_grid[64];  // blocks of 256 threads for the class's Newton kernel
};

// Kernel variants of a degree class: plain solve, plain solve that records
// training pairs, solve from the network's guess.
enum WfMode : int { kWfPlain = 0, kWfCollect = 1, kWfLearned = 2 };

// Arguments of one per-class launch (k_wf_newton or k_wf_resolve).
struct WfClassLaunch {
    const Scene* sc;
    const Rays* rays;
    const WfBuffers* wb;
    const Opts* op;
    const Hits* out;
    int32_t* tests;
    unsigned long long* ctr;
    cudaStream_t stream;
    int mode;
    int cls, rank_lo, rank_hi;
    unsigned grid;
};

// Launchers of the per-class kernels for u-degree p (wf_solve.cu, one object
// per p); q selects the v-degree.
void wf_newton_p1(int q, const WfClassLaunch& L);
void wf_newton_p2(int q, const WfClassLaunch& L);
void wf_newton_p3(int q, const WfClassLaunch& L);
void wf_newton_p4(int q, const WfClassLaunch& L);
void wf_newton_p5(int q, const WfClassLaunch& L);
void wf_newton_p6(int q, const WfClassLaunch& L);
void wf_newton_p7(int q, const WfClassLaunch& L);
void wf_resolve_p1(int q, const WfClassLaunch& L);
void wf_resolve_p2(int q, const WfClassLaunch& L);
void wf_resolve_p3(int q, const WfClassLaunch& L);
void wf_resolve_p4(int q, const WfClassLaunch& L);
void wf_resolve_p5(int q, const WfClassLaunch& L);
void wf_resolve_p6(int q, const WfClassLaunch& L);
void wf_resolve_p7(int q, const WfClassLaunch& L);

// Bytes of scratch for n rays and a scene of n_slots patches.
size_t wavefront_scratch_bytes(long long n, int n_slots);
// Carve WfBuffers out of one block of at least wavefront_scratch_bytes(n, n_slots).
WfBuffers wavefront_carve(void* base, long long n, int n_slots);

// Launch shapes of the graph's per-round kernels (the autotuner's knobs).
struct WfTuning {
    long long step_blocks = 148 * 8;     // persistent k_wf_step_dev blocks of 128 (capped at one ray per thread)
    long long scatter_blocks = 148 * 8;  // persistent k_wf_scatter_dev blocks of 256 (same)
    int class_blocks = 0;               // k_wf_newton blocks of 256 per class launch; 0 = the plan's
    int quota0 = 4;                     // candidates per ray in the first round (doubling each round)
    int quota_max = 8;                  // ... up to this many (<= 8)
    int stage_nodes = 1;                // top nodes of the tree each traversal block stages in shared memory
};

// The staged top of the tree: at most the top five levels of the 4-wide tree
// (341 nodes of 128 bytes, 43.6 KB of shared memory per traversal block).
constexpr int kMaxStagedNodes = 341;
inline size_t staged_bytes(int stage) { return (size_t)stage * 128; }

// The whole intersection of n rays as one executable CUDA graph, in passes of
// `chunk` rays.  Per pass: a set-up kernel, a while-loop node whose body is
// one round (step, scan, scatter, one Newton kernel per degree class,
// round_end, which sets the loop condition from the device-side count of
// rays still traversing), then the resolve kernels.  No host
// synchronisation; the graph is launched on any stream.  *passes gets the
// number of passes.
cudaError_t build_wavefront_graph(const Scene& sc, const WfPlan& plan, const Rays& rays, long long n,
                                  long long chunk, const Opts& op, const Hits& out, const WfBuffers& wb,
                                  unsigned long long* ctr, const WfTuning& tu, cudaGraphExec_t* exec,
                                  long long* passes);

// Runs the rounds; synchronises `stream` once per round to read the number of
// rays still traversing into host_count (pinned host memory).
// With ev[2] (two events) and newton_ms, each round's per-class Newton
// launches are bracketed by the events and their time added to *newton_ms.
cudaError_t launch_wavefront(const Scene& sc, const WfPlan& plan, const Rays& rays, long long n, const Opts& op,
                             const Hits& out, const WfBuffers& wb, int32_t* host_count, unsigned long long* ctr,
                             cudaStream_t stream, long long* launches, long long* rounds,
                             cudaEvent_t* ev = nullptr, double* newton_ms = nullptr, long long* newton_launches = nullptr,
                             int quota0 = 1, int quota_max = 8, int stage_nodes = 1);

// Per-pixel kernel over a device list of ray indices (count read on the device).
cudaError_t launch_intersect_pixel_list(const Scene& sc, const Rays& rays, const int32_t* list,
                                        const int32_t* list_count, long long max_n, const Opts& op, const Hits& out,
                                        unsigned long long* ctr, cudaStream_t stream);

}  // namespace dev

struct NoallocViews {
    dev::Scene scene;
    dev::WfPlan plan;
    dev::Opts opts;
    unsigned long long* counters;
    int device;
    int quota0, quota_max, stage_nodes;
};

}  // namespace nrt
