// scene_build.h -- pieces of scene creation shared by the host builder
// (engine.cu) and the device builder (scene_build.cu).
#pragma once

#include <cuda_runtime.h>

#include "nrt_internal.h"
#include "wavefront.h"

namespace nrt {

int cuda_fail(cudaError_t e, const char* what);

// Byte offsets of the scene's arrays in its device arena.
struct ArenaLayout {
    size_t nodes, hdr, centre, cp, corners, delta, counters, rank, frames, obb, leafbox, total;
};
ArenaLayout arena_layout(size_t n_wide, int N, size_t n_floats);
void plan_classes(const int* degree_hist, int N, dev::WfPlan& plan);
int new_scene(const nrt_build_opts& o, const ArenaLayout& L, nrt_scene** out, char** arena);
void finish_scene(nrt_scene* sc, const ArenaLayout& L, int N, dev::WfPlan plan, nrt_scene_info info, PatchSet&& ps,
                  int n_surfaces);

// Host builder: patches already decomposed on the host.  given: use this
// binary tree (its order maps leaf slots to patches) instead of building one;
// delta_by_patch: flatness per patch (input order) for flat-skip instead of
// the computed one.
int build_scene(PatchSet&& ps, int n_surfaces, const nrt_build_opts* opts, nrt_scene** out,
                const BinaryBVH* given = nullptr, const float* delta_by_patch = nullptr);

// Device builder.  Surfaces (nets and knots in host memory) or patches are
// copied to the device once; decomposition, patch boxes, the binned SAH, the
// 4-wide collapse and the per-slot packing run there, producing the same
// arena as build_scene with NRT_BVH_BINNED_SAH.
int build_scene_device_surfaces(const nrt_nurbs_surface* surfaces, int n_surfaces, const nrt_build_opts& o,
                                nrt_scene** out);
int build_scene_device_patches(const float* cp, const int32_t* cp_offset, const int32_t* degrees, int n_patches,
                               const nrt_build_opts& o, nrt_scene** out);

}  // namespace nrt
