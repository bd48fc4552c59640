/* nrt_compat.h -- the reference's own C++ entry points, served by libnrt.so.
 *
 * A program written against Frostbite16/rt-nurbs (src/core/benchmark.cpp,
 * src/core/main.cpp) links against libnrt.so unchanged: libnrt.so exports
 * calculateIntersectWrapper and calculateRaysWrapper with the reference's
 * exact C++ signatures (same names, parameter types and mangled symbols), and
 * runs them on this engine.  Such a program includes the reference's headers
 * (src/gpu/intersect.h, src/gpu/generateRaysKernel.h); this header declares
 * the same entry points for programs that do not have them, with the
 * reference's types restated: same names, namespaces and member layout
 * (the symbol names and the memory the caller passes depend on both).
 * Do not include it together with the reference's headers.
 *
 * Semantics, as the reference's (src/gpu/intersect.cu:20-220,
 * src/gpu/generateRaysKernel.cu:15-69):
 *  - all buffers are the caller's device or managed memory;
 *  - both calls are synchronous (they end in cudaDeviceSynchronize) and run
 *    on the legacy default stream;
 *  - they return nothing; a failure is printed to stderr with
 *    nrt_last_error()'s text and leaves the outputs untouched.
 */
#ifndef NRT_COMPAT_H
#define NRT_COMPAT_H

#ifndef __cplusplus
#error "nrt_compat.h declares C++ entry points"
#endif

/* src/math/math_types.h:5-97 (column-major matrices, plain float arrays). */
namespace MathTypes {
struct matrix4x4f { float m[16]; };
struct vector4f { float v[4]; };
struct vector3f { float v[3]; };
struct point2f { float v[2]; };
}  // namespace MathTypes

namespace MathExtra {
struct bounds2f { float p_min_x, p_min_y; float p_max_x, p_max_y; };
struct bounds3f { float p_min_x, p_min_y, p_min_z; float p_max_x, p_max_y, p_max_z; };
}  // namespace MathExtra

/* src/gpu/soa.h:6-14: the ray queue.  idx_interact[i] becomes i for a ray that
 * hits; it is not written for a miss (callers preset it to -1). */
namespace SoAQueue {
struct ray_queue {
    float* origin_x;
    float* origin_y;
    float* origin_z;
    float* direction_x;
    float* direction_y;
    float* direction_z;
    int* idx_interact;
};
}  // namespace SoAQueue

/* src/math/bezier_patch.h:10-16: one Bezier patch, (p+1)*(q+1) weighted-
 * homogeneous control points, index i*(q+1)+j with i along u. */
struct bezierPatch {
    MathTypes::vector4f* control_point;
    float u0, u1, v0, v1;
    int p, q;
    MathTypes::vector4f* heap_pointer;
};

/* src/core/bvh.h:13-17: binary BVH node; prim_count 0 = inner node with
 * children left_first and left_first + 1, else a leaf over
 * patches[left_first, left_first + prim_count). */
struct BVHNode {
    MathExtra::bounds3f node_bound;
    unsigned int left_first;
    unsigned int prim_count;
};

/* src/gpu/interact.h:6-21: per-pixel hit record (72 bytes).  For a hit:
 * t_hit, uv (patch-local), dpdu, dpdv (world-space partials of the
 * dehomogenised surface) and wo = -direction; dndu, dndv are never written. */
struct surfaceInteraction {
    float t_hit;
    MathTypes::vector3f wo;
    MathTypes::point2f uv;
    MathTypes::vector3f dpdu;
    MathTypes::vector3f dpdv;
    MathTypes::vector3f dndu;
    MathTypes::vector3f dndv;
};

/* src/core/camera.h:12-42. */
struct camera_config {
    MathTypes::matrix4x4f world_from_camera;
    MathTypes::matrix4x4f screen_from_camera;
    MathTypes::matrix4x4f NDC_from_screen;
    MathTypes::matrix4x4f raster_from_NDC;
    MathTypes::matrix4x4f raster_from_screen;
    MathTypes::matrix4x4f screen_from_raster;
    MathTypes::matrix4x4f camera_from_raster;
    int screen_resolution_x;
    int screen_resolution_y;
    MathExtra::bounds2f screen_window;
};
enum projection { orthographic, perspective };

/* Closest hit of the screen_res_x * screen_res_y rays of ray_queue against the
 * caller's patches and binary BVH (patches in the BVH's leaf order, as
 * BvhOps::buildBVH leaves them).  Replaces calculateIntersectWrapper
 * (src/gpu/intersect.h:9-13, src/gpu/intersect.cu:199-220): the reference's
 * settings (bilinear initial guess, 7 Newton evaluations, stop at
 * |r1| + |r2| < 1e-4, pull below |det J| < 1e-5), flat-skip with
 * flat_threshold pixels and delta[] per patch (0 = off), cam_k =
 * 0.5 * screen_res_y / tan(v_fov / 2) with v_fov in radians (the definition
 * names this parameter v_fov, the declaration cam_k; it is the field of view).
 * The first call with a scene packs the caller's patches and tree into the
 * engine's layout, keeping the caller's tree; later calls reuse that scene
 * while the patches, control points, nodes and delta are unchanged (checked
 * by content every call).  newton_count / skip_count, when given, are
 * incremented by the Newton solves and flat-skip acceptances of the call
 * (counted on the engine's traversal, which visits the tree 4 children at a
 * time). */
void calculateIntersectWrapper(SoAQueue::ray_queue& ray_queue, BVHNode* nodes, bezierPatch* patches,
                               surfaceInteraction* interact, int screen_res_x, int screen_res_y, float flat_threshold,
                               float cam_k, float* delta, unsigned long long* newton_count = nullptr,
                               unsigned long long* skip_count = nullptr);

/* Pixel-centre rays of a perspective or orthographic camera_config into
 * ray_queue, idx_interact preset to -1.  Replaces calculateRaysWrapper
 * (src/gpu/generateRaysKernel.h:6, src/gpu/generateRaysKernel.cu:15-69,
 * CameraOps::calculateRay src/core/camera.h:142-174), in round-to-nearest
 * float arithmetic without contraction, the reference's host arithmetic. */
void calculateRaysWrapper(SoAQueue::ray_queue& ray_queue, projection proj, camera_config& camera);

#endif /* NRT_COMPAT_H */
