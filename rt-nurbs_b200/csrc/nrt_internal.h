// nrt_internal.h -- host-side structures shared by the engine's C++ and CUDA
// translation units.  Not part of the public ABI (include/nrt.h is).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/nrt.h"

namespace nrt {

// Thread-local error text behind nrt_last_error().
void set_error(const char* fmt, ...);
int fail(int status, const char* fmt, ...);

// A flat set of Bezier patches on the host.
struct PatchSet {
    std::vector<float> cp;        // 4 floats per point, weighted-homogeneous
    std::vector<int32_t> off;     // first point of each patch
    std::vector<int32_t> deg;     // (p, q) per patch
    std::vector<float> ranges;    // (u0, u1, v0, v1) per patch
    std::vector<int32_t> surf;    // surface index per patch
    // Instead of ranges/surf (device builder): per surface its first patch,
    // span counts and the offsets of its u and v breakpoints in `breaks`.
    struct Spans {
        int patch0, nbU, nbV;
        size_t bu, bv;
    };
    std::vector<Spans> spans;
    std::vector<float> breaks;
    int count() const { return (int)off.size(); }
};

// Algorithm A5.7 on one surface (float, the reference's order of operations).
int decompose_surface(const nrt_nurbs_surface& s, std::vector<float>& cp, std::vector<float>& ranges, int& nbU,
                      int& nbV);
int check_surface(const nrt_nurbs_surface& s);

// Axis-aligned box.
struct Box3 {
    float lo[3], hi[3];
};

// Binary BVH in the reference's layout (used as the builders' common output).
struct BinaryBVH {
    std::vector<Box3> box;
    std::vector<uint32_t> left_first, prim_count;
    std::vector<int32_t> order;   // leaf slot -> primitive index
    int used = 0;
};
void patch_boxes(const PatchSet& ps, std::vector<Box3>& out);
void build_exact_sah(const std::vector<Box3>& prims, BinaryBVH& out);
void build_binned_sah(const std::vector<Box3>& prims, int max_leaf, BinaryBVH& out);

// 4-wide node as stored on the device: child boxes SoA, 128 bytes.
// child[c] >= 0: inner node index; child[c] < 0: leaf holding patch slots
// [~child[c], ~child[c] + count[c]); count 0 with an inverted box = empty.
struct alignas(16) Node4 {
    float lo_x[4], hi_x[4], lo_y[4], hi_y[4], lo_z[4], hi_z[4];
    int32_t child[4];
    int32_t count[4];
};
static_assert(sizeof(Node4) == 128, "Node4 must be 128 bytes");

// Collapse a binary BVH into 4-wide nodes; leaf slots keep the binary order.
void collapse_to_wide(const BinaryBVH& bin, std::vector<Node4>& out, int& depth);

// Scene views for nrt_intersect_noalloc (defined in engine.cu, used by noalloc.cu).
struct NoallocViews;
int noalloc_views(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                  const nrt_hits* hits, NoallocViews* v);
void noalloc_record(nrt_scene* scene, long long launches, long long rounds);

}  // namespace nrt
