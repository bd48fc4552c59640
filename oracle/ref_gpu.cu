// ref_gpu.cu -- runs the reference's own CUDA kernel on the GPU
// (TEST INFRASTRUCTURE ONLY).
//
// Compiled by oracle/Makefile (target ref) together with the reference's
// src/gpu/intersect.cu where it lies (-I <reference>/src, forced-include
// ref_constants.h for the degree capacity) into oracle/_ref/libref_gpu.so.
// The entry point builds the reference's data structures in device memory
// (bezierPatch records pointing into one control-point block, BVHNode array,
// SoAQueue::ray_queue over the caller's device rays, surfaceInteraction
// array, a zero flatness array) and calls the reference's unchanged
// calculateIntersectWrapper (src/gpu/intersect.cu:199-220), timing it with
// CUDA events.  Nothing of the reference is copied into this repository.
//
// The reference kernel keeps its traversal stack in a 32-entry local array
// with no overflow check (src/gpu/intersect.cu:59); a push happens only when
// descending from an inner node, so the stack never holds more entries than
// the current node has ancestors.  refgpu_intersect therefore refuses any
// tree deeper than 31 inner levels before launching anything.

#include "core/bvh.h"
#include "gpu/intersect.h"
#include "gpu/soa.h"
#include "gpu/interact.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

int depth_of(const std::vector<BVHNode>& nodes, int i, int d) {
    if (nodes[i].prim_count > 0) return d;
    const int l = depth_of(nodes, nodes[i].left_first, d + 1);
    const int r = depth_of(nodes, nodes[i].left_first + 1, d + 1);
    return l > r ? l : r;
}

}  // namespace

extern "C" {

// Inner levels above the deepest leaf (the bound on the reference kernel's stack).
int refgpu_tree_depth(const uint32_t* lf, const uint32_t* cnt, int n_nodes) {
    std::vector<BVHNode> nodes(n_nodes);
    for (int i = 0; i < n_nodes; ++i) {
        nodes[i].left_first = lf[i];
        nodes[i].prim_count = cnt[i];
    }
    return depth_of(nodes, 0, 0);
}

// cp/off/deg: host patches in BVH slot order (off in points); node_box/lf/cnt:
// host binary BVH in the reference's layout; rays: device SoA of W*H rays.
// Outputs (device, W*H each): hit ray index or -1, t, u, v.  reps timed calls
// after one untimed call; *ms gets the mean CUDA-event time of one call.
// Returns 0, or -1 when the tree is too deep for the kernel's stack, or the
// CUDA error code.
int refgpu_intersect(const float* cp, long n_points, const int* off, const int* deg, int n_patches,
                     const float* node_box, const uint32_t* lf, const uint32_t* cnt, int n_nodes, float* ox,
                     float* oy, float* oz, float* dx, float* dy, float* dz, int W, int H, int* idx_interact,
                     float* t_out, float* u_out, float* v_out, int reps, float* ms) {
    std::vector<BVHNode> nodes(n_nodes);
    for (int i = 0; i < n_nodes; ++i) {
        const float* b = node_box + 6 * i;
        nodes[i].node_bound = MathExtra::bounds3f{b[0], b[1], b[2], b[3], b[4], b[5]};
        nodes[i].left_first = lf[i];
        nodes[i].prim_count = cnt[i];
    }
    if (depth_of(nodes, 0, 0) > 31) return -1;
    const long R = (long)W * H;
    MathTypes::vector4f* d_cp = nullptr;
    bezierPatch* d_patches = nullptr;
    BVHNode* d_nodes = nullptr;
    float* d_delta = nullptr;
    surfaceInteraction* d_inter = nullptr;
    cudaError_t e = cudaMalloc(&d_cp, sizeof(MathTypes::vector4f) * n_points);
    if (e == cudaSuccess) e = cudaMalloc(&d_patches, sizeof(bezierPatch) * n_patches);
    if (e == cudaSuccess) e = cudaMalloc(&d_nodes, sizeof(BVHNode) * n_nodes);
    if (e == cudaSuccess) e = cudaMalloc(&d_delta, sizeof(float) * n_patches);
    if (e == cudaSuccess) e = cudaMalloc(&d_inter, sizeof(surfaceInteraction) * R);
    if (e == cudaSuccess) e = cudaMemcpy(d_cp, cp, sizeof(MathTypes::vector4f) * n_points, cudaMemcpyHostToDevice);
    std::vector<bezierPatch> patches(n_patches);
    for (int k = 0; k < n_patches; ++k) {
        patches[k].control_point = d_cp + off[k];
        patches[k].u0 = patches[k].v0 = 0.f;
        patches[k].u1 = patches[k].v1 = 1.f;
        patches[k].p = deg[2 * k];
        patches[k].q = deg[2 * k + 1];
        patches[k].heap_pointer = nullptr;
    }
    if (e == cudaSuccess) e = cudaMemcpy(d_patches, patches.data(), sizeof(bezierPatch) * n_patches, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_nodes, nodes.data(), sizeof(BVHNode) * n_nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_delta, 0, sizeof(float) * n_patches);
    SoAQueue::ray_queue q{ox, oy, oz, dx, dy, dz, idx_interact};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float total = 0.f;
    for (int k = 0; k <= reps && e == cudaSuccess; ++k) {
        e = cudaMemset(idx_interact, 0xff, sizeof(int) * R);  // the caller's pre-set (src/core/benchmark.cpp:191)
        if (e != cudaSuccess) break;
        if (k > 0) cudaEventRecord(e0);
        calculateIntersectWrapper(q, d_nodes, d_patches, d_inter, W, H, 0.f, 1.f, d_delta);
        e = cudaGetLastError();
        if (k > 0 && e == cudaSuccess) {
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            total += t;
        }
    }
    if (e == cudaSuccess && ms) *ms = reps > 0 ? total / reps : 0.f;
    // hit records: t, (u, v) of the interaction where idx_interact != -1
    if (e == cudaSuccess) {
        std::vector<surfaceInteraction> h(R);
        std::vector<int> idx(R);
        e = cudaMemcpy(h.data(), d_inter, sizeof(surfaceInteraction) * R, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(idx.data(), idx_interact, sizeof(int) * R, cudaMemcpyDeviceToHost);
        std::vector<float> t(R), u(R), v(R);
        for (long i = 0; i < R; ++i) {
            t[i] = idx[i] >= 0 ? h[i].t_hit : -1.f;
            u[i] = idx[i] >= 0 ? h[i].uv.v[0] : 0.f;
            v[i] = idx[i] >= 0 ? h[i].uv.v[1] : 0.f;
        }
        if (e == cudaSuccess) e = cudaMemcpy(t_out, t.data(), sizeof(float) * R, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(u_out, u.data(), sizeof(float) * R, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(v_out, v.data(), sizeof(float) * R, cudaMemcpyHostToDevice);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_cp);
    cudaFree(d_patches);
    cudaFree(d_nodes);
    cudaFree(d_delta);
    cudaFree(d_inter);
    return e == cudaSuccess ? 0 : (int)e;
}

}  // extern "C"
