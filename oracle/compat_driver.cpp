// compat_driver.cpp -- a program written against the reference, linked
// against libnrt.so (TEST INFRASTRUCTURE ONLY).
//
// Compiled by oracle/Makefile with the reference's own headers where they lie
// (-I <reference>/src): it includes src/gpu/intersect.h and
// src/gpu/generateRaysKernel.h for the declarations of
// calculateIntersectWrapper / calculateRaysWrapper and links against
// rt-nurbs_b200/lib/libnrt.so, which defines them -- the drop-in a caller of
// the reference gets.  The flow mirrors the reference's benchmark
// (src/core/benchmark.cpp:122-204): getPatch per surface, buildBVH over the
// patches, managed copies of nodes, patches, rebased control points and the
// flatness array, calculateRaysWrapper(perspective), idx_interact preset to
// -1, then calculateIntersectWrapper with counters.  The call runs twice (the
// second on the cached scene) and must give the same bytes.
//
//   compat_driver <input file> <output file>
// input: int32 n_surfaces; per surface int32 n, m, p, q, float32 points
// ((n+1)(m+1)x4), u knots (n+p+2), v knots (m+q+2); float32 eye[3], look[3],
// up[3], fov_deg; int32 W, H; float32 flat_threshold; int32 count, float32
// delta[count] (per patch, in BVH order).
// output: int32 W*H idx_interact, W*H surfaceInteraction records (72 bytes),
// 6 x W*H float32 rays, uint64 newton, skip, int32 n_patches.
#include "gpu/intersect.h"
#include "gpu/generateRaysKernel.h"
#include "math/transform.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

template <class T>
static T* managed(size_t n) {
    T* p = nullptr;
    if (cudaMallocManaged(&p, n * sizeof(T)) != cudaSuccess) {
        std::fprintf(stderr, "cudaMallocManaged failed\n");
        std::exit(2);
    }
    return p;
}

template <class T>
static void take(FILE* f, T* dst, size_t n) {
    if (std::fread(dst, sizeof(T), n, f) != n) {
        std::fprintf(stderr, "short input\n");
        std::exit(2);
    }
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    int n_surf = 0;
    take(in, &n_surf, 1);
    std::vector<bezierPatch> all;
    std::vector<bezierPatch*> owned;
    for (int s = 0; s < n_surf; ++s) {
        int nmpq[4];
        take(in, nmpq, 4);
        const int n = nmpq[0], m = nmpq[1], p = nmpq[2], q = nmpq[3];
        ParametricSurf::nurbsSurf surf;
        surf.n = n; surf.m = m; surf.p = p; surf.q = q;
        surf.control_point = new MathTypes::vector4f[(size_t)(n + 1) * (m + 1)];
        surf.u_knots = new float[n + p + 2];
        surf.v_knots = new float[m + q + 2];
        take(in, reinterpret_cast<float*>(surf.control_point), 4 * (size_t)(n + 1) * (m + 1));
        take(in, surf.u_knots, n + p + 2);
        take(in, surf.v_knots, m + q + 2);
        int nbU = 0, nbV = 0;
        bezierPatch* patches = BezierPatchOps::getPatch(surf, nbU, nbV);
        for (int k = 0; k < nbU * nbV; ++k) all.push_back(patches[k]);
        owned.push_back(patches);
        delete[] surf.u_knots;
        delete[] surf.v_knots;
        delete[] surf.control_point;
    }
    float cam[10];
    take(in, cam, 10);
    int WH[2];
    take(in, WH, 2);
    float flat = 0.f;
    take(in, &flat, 1);
    int n_delta = 0;
    take(in, &n_delta, 1);
    std::vector<float> delta_in(n_delta);
    take(in, delta_in.data(), n_delta);
    std::fclose(in);
    const int W = WH[0], H = WH[1], max_pixels = W * H;
    const int nP = (int)all.size();
    if (n_delta != nP) {
        std::fprintf(stderr, "delta has %d values for %d patches\n", n_delta, nP);
        return 2;
    }

    // scene: BVH over the patches (reordered in place), managed copies with rebased points
    BVHNode* nodes = managed<BVHNode>(2 * (size_t)nP - 1);
    bezierPatch* arr = all.data();
    BvhOps::buildBVH(nodes, 0, arr, nP);
    size_t total = 0;
    for (const bezierPatch& b : all) total += (size_t)(b.p + 1) * (b.q + 1);
    MathTypes::vector4f* gpu_cp = managed<MathTypes::vector4f>(total);
    bezierPatch* gpu_patches = managed<bezierPatch>(nP);
    float* delta = managed<float>(nP);
    size_t at = 0;
    for (int i = 0; i < nP; ++i) {
        const size_t np = (size_t)(all[i].p + 1) * (all[i].q + 1);
        std::memcpy(gpu_cp + at, all[i].control_point, np * sizeof(MathTypes::vector4f));
        gpu_patches[i] = all[i];
        gpu_patches[i].control_point = gpu_cp + at;
        gpu_patches[i].heap_pointer = gpu_cp;
        delta[i] = delta_in[i];
        at += np;
    }
    for (bezierPatch* p : owned) BezierPatchOps::freePatches(p);

    // camera and rays through the reference's entry point
    MathTypes::matrix4x4f world_from_camera = Transform::lookAt(
        MathTypes::point3f{cam[0], cam[1], cam[2]}, MathTypes::point3f{cam[3], cam[4], cam[5]},
        MathTypes::vector3f{cam[6], cam[7], cam[8]});
    camera_config main_cam = CameraOps::init_camera(world_from_camera, W, H);
    main_cam = CameraOps::getPerspectiveCamera(main_cam, cam[9], 0.01f, 1000.0f);
    SoAQueue::ray_queue rq = {managed<float>(max_pixels), managed<float>(max_pixels), managed<float>(max_pixels),
                              managed<float>(max_pixels), managed<float>(max_pixels), managed<float>(max_pixels),
                              managed<int>(max_pixels)};
    calculateRaysWrapper(rq, perspective, main_cam);

    surfaceInteraction* interact = managed<surfaceInteraction>(max_pixels);
    std::memset(interact, 0, sizeof(surfaceInteraction) * max_pixels);
    unsigned long long* d_newton = managed<unsigned long long>(1);
    unsigned long long* d_skip = managed<unsigned long long>(1);
    const float v_fov = MathUtils::radians(cam[9]);
    std::vector<int> idx_first(max_pixels);
    std::vector<surfaceInteraction> si_first(max_pixels);
    for (int run = 0; run < 2; ++run) {
        cudaMemset(rq.idx_interact, 0xFF, max_pixels * sizeof(int));
        *d_newton = 0;
        *d_skip = 0;
        calculateIntersectWrapper(rq, nodes, gpu_patches, interact, W, H, flat, v_fov, delta, d_newton, d_skip);
        if (cudaGetLastError() != cudaSuccess) return 3;
        if (run == 0) {
            std::memcpy(idx_first.data(), rq.idx_interact, max_pixels * sizeof(int));
            std::memcpy(si_first.data(), interact, max_pixels * sizeof(surfaceInteraction));
        } else if (std::memcmp(idx_first.data(), rq.idx_interact, max_pixels * sizeof(int)) != 0 ||
                   std::memcmp(si_first.data(), interact, max_pixels * sizeof(surfaceInteraction)) != 0) {
            std::fprintf(stderr, "second call differs from the first\n");
            return 4;
        }
    }

    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    std::fwrite(rq.idx_interact, sizeof(int), max_pixels, out);
    std::fwrite(interact, sizeof(surfaceInteraction), max_pixels, out);
    for (float* a : {rq.origin_x, rq.origin_y, rq.origin_z, rq.direction_x, rq.direction_y, rq.direction_z})
        std::fwrite(a, sizeof(float), max_pixels, out);
    const unsigned long long counts[2] = {*d_newton, *d_skip};
    std::fwrite(counts, sizeof(counts), 1, out);
    std::fwrite(&nP, sizeof(int), 1, out);
    std::fclose(out);
    return 0;
}
