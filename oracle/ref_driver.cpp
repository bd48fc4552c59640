// ref_driver.cpp -- runs the reference's own host-compilable code
// (TEST INFRASTRUCTURE ONLY).
//
// Compiled by oracle/Makefile against the reference's headers where they lie
// (-I <reference>/src, plus the forced-include ref_constants.h) into
// oracle/_ref/libnrt_ref_it{7,8}.so.  The library exposes C entry points that
// call, unchanged:
//   BezierPatchOps::getPatch          src/math/bezier_patch.h:86-139
//   BvhOps::buildBVH                  src/core/bvh.h:148-179
//   Transform::lookAt, CameraOps::*   src/math/transform.h:46-60, src/core/camera.h:63-174
//   MathUtils::getRayPlanes, BoundsOps::intersectBound, corners,
//   BezierPatchOps::biliniearRay / newtonRhapson / evalPointNormal
// The one piece that cannot compile on the host is the traversal loop of the
// __global__ kernel calculateIntersect (src/gpu/intersect.cu:33-193); it is
// restated below as a host loop over rays (OpenMP) that calls the reference
// functions above.  No reference file is copied into this repository.

#include "math/bezier_patch.h"
#include "core/bvh.h"
#include "core/camera.h"
#include "math/math_utils.h"
#include "math/bounds_ops.h"

#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

using MathTypes::vector3f;
using MathTypes::vector4f;

extern "C" {

int ref_iterations(void) { return NEWTON_MAX_ITERATIONS; }

// curvatureRefinementU then curvatureRefinementV (src/math/nurbs.h:289-486) on
// a copy of the surface, as src/core/main.cpp:100-102.  Writes the refined
// points and knots when they fit the capacities (points, u knots, v knots);
// returns 0, -1 when the V pass would overrun the reference's own scratch
// (it sizes a curve by n+1 and fills m+1 points), -2 when the outputs do not fit.
int ref_refine(const float* cp, const float* U, const float* V, int n, int m, int p, int q, float C, float* cp_out,
               float* U_out, float* V_out, long cap_pts, int cap_u, int cap_v, int* n_out, int* m_out) {
    float* Uk = new float[n + p + 2];
    float* Vk = new float[m + q + 2];
    vector4f* P = new vector4f[(size_t)(n + 1) * (m + 1)];
    std::memcpy(Uk, U, sizeof(float) * (n + p + 2));
    std::memcpy(Vk, V, sizeof(float) * (m + q + 2));
    std::memcpy(P, cp, sizeof(vector4f) * (size_t)(n + 1) * (m + 1));
    NurbsOps::curvatureRefinementU(Uk, p, n, m, C, P);
    int rc = 0;
    if (m > n) rc = -1;
    else NurbsOps::curvatureRefinementV(Vk, q, m, n, C, P);
    if (rc == 0) {
        *n_out = n;
        *m_out = m;
        if ((long)(n + 1) * (m + 1) > cap_pts || n + p + 2 > cap_u || m + q + 2 > cap_v) rc = -2;
        else {
            std::memcpy(cp_out, P, sizeof(vector4f) * (size_t)(n + 1) * (m + 1));
            std::memcpy(U_out, Uk, sizeof(float) * (n + p + 2));
            std::memcpy(V_out, Vk, sizeof(float) * (m + q + 2));
        }
    }
    delete[] Uk;
    delete[] Vk;
    delete[] P;
    return rc;
}

// getPatch on one surface; cp_out gets nbU*nbV*(p+1)*(q+1) points, ranges 4 floats per patch.
int ref_decompose(const float* cp, const float* U, const float* V, int n, int m, int p, int q, float* cp_out,
                  float* ranges) {
    std::vector<float> Uk(U, U + n + p + 2), Vk(V, V + m + q + 2);
    std::vector<vector4f> P((size_t)(n + 1) * (m + 1));
    std::memcpy(P.data(), cp, sizeof(vector4f) * P.size());
    ParametricSurf::nurbsSurf s{Uk.data(), Vk.data(), P.data(), n, m, p, q};
    int nbU = 0, nbV = 0;
    bezierPatch* patches = BezierPatchOps::getPatch(s, nbU, nbV);
    const int piece = (p + 1) * (q + 1);
    for (int k = 0; k < nbU * nbV; ++k) {
        if (cp_out) std::memcpy(cp_out + 4 * (size_t)k * piece, patches[k].control_point, sizeof(vector4f) * piece);
        if (ranges) {
            ranges[4 * k + 0] = patches[k].u0; ranges[4 * k + 1] = patches[k].u1;
            ranges[4 * k + 2] = patches[k].v0; ranges[4 * k + 3] = patches[k].v1;
        }
    }
    BezierPatchOps::freePatches(patches);
    return nbU * nbV;
}

// buildBVH over patches given as (cp, offsets in points, degrees).  Writes the
// 2N-1 nodes (6 bounds floats + left_first + prim_count) and order[k] = input
// index of the patch in BVH slot k.
void ref_build_bvh(const float* cp, const int* cp_off, const int* deg, int N, float* node_box, uint32_t* lf,
                   uint32_t* cnt, int32_t* order) {
    std::vector<bezierPatch> patches(N);
    std::map<const vector4f*, int> slot_of;
    const vector4f* base = reinterpret_cast<const vector4f*>(cp);
    for (int k = 0; k < N; ++k) {
        patches[k].control_point = const_cast<vector4f*>(base + cp_off[k]);
        patches[k].p = deg[2 * k];
        patches[k].q = deg[2 * k + 1];
        patches[k].u0 = patches[k].v0 = 0;
        patches[k].u1 = patches[k].v1 = 1;
        patches[k].heap_pointer = nullptr;
        slot_of[patches[k].control_point] = k;
    }
    std::vector<BVHNode> nodes(2 * (size_t)N - 1);
    std::memset(nodes.data(), 0, sizeof(BVHNode) * nodes.size());
    bezierPatch* arr = patches.data();
    BvhOps::buildBVH(nodes.data(), 0, arr, N);
    for (size_t i = 0; i < nodes.size(); ++i) {
        const MathExtra::bounds3f& b = nodes[i].node_bound;
        float* o = node_box + 6 * i;
        o[0] = b.p_min_x; o[1] = b.p_min_y; o[2] = b.p_min_z;
        o[3] = b.p_max_x; o[4] = b.p_max_y; o[5] = b.p_max_z;
        lf[i] = nodes[i].left_first;
        cnt[i] = nodes[i].prim_count;
    }
    for (int k = 0; k < N; ++k) order[k] = slot_of[arr[k].control_point];
}

// Perspective pixel-centre rays from the reference camera code.
void ref_camera_rays(const float* eye, const float* look, const float* up, float fov_deg, int W, int H, float* ox,
                     float* oy, float* oz, float* dx, float* dy, float* dz) {
    MathTypes::matrix4x4f wfc = Transform::lookAt(MathTypes::point3f{eye[0], eye[1], eye[2]},
                                                  MathTypes::point3f{look[0], look[1], look[2]},
                                                  MathTypes::vector3f{up[0], up[1], up[2]});
    camera_config cam = CameraOps::init_camera(wfc, W, H);
    cam = CameraOps::getPerspectiveCamera(cam, fov_deg, 0.01f, 1000.0f);
    camera_gpu_payload pay = {cam.world_from_camera, cam.camera_from_raster};
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            MathExtra::ray r = CameraOps::calculateRay<perspective_projection>(pay, x, y);
            const long i = (long)y * W + x;
            ox[i] = r.origin.v[0]; oy[i] = r.origin.v[1]; oz[i] = r.origin.v[2];
            dx[i] = r.direction.v[0]; dy[i] = r.direction.v[1]; dz[i] = r.direction.v[2];
        }
}

// Per-ray closest hit (restated traversal of intersect.cu:33-193, calling the
// reference's functions).  Patches are given in BVH order (slot k = patch k).
// Outputs follow the reference's surfaceInteraction semantics: hit[i] = -1 on
// a miss, else the BVH slot of the closest patch; t, uv, dpdu, dpdv as written
// by the reference kernel.
void ref_intersect(const float* cp, const int* cp_off, const int* deg, const float* delta, int N,
                   const float* node_box, const uint32_t* lf, const uint32_t* cnt, const float* ox, const float* oy,
                   const float* oz, const float* dx, const float* dy, const float* dz, long R, float flat_threshold,
                   float cam_k, int bilinear_init, float eps, int32_t* hit, float* t_out, float* u_out, float* v_out,
                   float* geo_out, unsigned long long* newton_total, unsigned long long* skip_total) {
    std::vector<bezierPatch> patches(N);
    const vector4f* base = reinterpret_cast<const vector4f*>(cp);
    for (int k = 0; k < N; ++k) {
        patches[k].control_point = const_cast<vector4f*>(base + cp_off[k]);
        patches[k].p = deg[2 * k];
        patches[k].q = deg[2 * k + 1];
        patches[k].heap_pointer = nullptr;
    }
    std::vector<BVHNode> nodes(2 * (size_t)N - 1);
    for (size_t i = 0; i < nodes.size(); ++i) {
        const float* b = node_box + 6 * i;
        nodes[i].node_bound = MathExtra::bounds3f{b[0], b[1], b[2], b[3], b[4], b[5]};
        nodes[i].left_first = lf[i];
        nodes[i].prim_count = cnt[i];
    }
    unsigned long long nc_all = 0, sc_all = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nc_all, sc_all)
    for (long idx = 0; idx < R; ++idx) {
        MathExtra::ray ray{vector3f{ox[idx], oy[idx], oz[idx]}, vector3f{dx[idx], dy[idx], dz[idx]}};
        vector3f rd{1 / ray.direction.v[0], 1 / ray.direction.v[1], 1 / ray.direction.v[2]};
        MathExtra::ray_plane plane = MathUtils::getRayPlanes(ray);
        int stack[64];
        int sp = 0;
        float t_max = INFINITY;
        int best = -1;
        float bu = 0, bv = 0;
        vector3f bS{}, bSu{}, bSv{};
        unsigned long long nc = 0, sc = 0;
        auto box_t = [&](const BVHNode& nd) {
            const MathExtra::bounds3f& b = nd.node_bound;
            return BoundsOps::intersectBound(b.p_min_x, b.p_max_x, b.p_min_y, b.p_max_y, b.p_min_z, b.p_max_z,
                                             ray.origin.v[0], ray.origin.v[1], ray.origin.v[2], rd.v[0], rd.v[1],
                                             rd.v[2]);
        };
        BVHNode cur = nodes[0];
        float it = box_t(cur);
        bool live = it < t_max;
        while (live) {
            if (cur.prim_count > 0) {
                it = box_t(cur);
                for (uint32_t i = 0; i < cur.prim_count; ++i) {
                    const int slot = (int)(cur.left_first + i);
                    bezierPatch patch = patches[slot];
                    vector3f q00, q10, q11, q01;
                    MathTypes::vector2f g{0.5f, 0.5f};
                    if (bilinear_init) {
                        corners(patch, q00, q10, q11, q01);
                        g = BezierPatchOps::biliniearRay(q00, q10, q11, q01, ray.origin, ray.direction);
                    }
                    bool do_newton = true;
                    if (delta && delta[slot] * cam_k / it < flat_threshold) {
                        vector3f S, Su, Sv;
                        BezierPatchOps::evalPointNormal(patch, g.v[0], g.v[1], ray.direction, S, Su, Sv);
                        float res = fabsf(VectorOps::dotProduct(plane.n1, S) + plane.d1) +
                                    fabsf(VectorOps::dotProduct(plane.n2, S) + plane.d2);
                        if (res * cam_k / it < flat_threshold) {
                            ++sc;
                            float t = VectorOps::dotProduct(VectorOps::subtract(S, ray.origin), ray.direction);
                            if (0 < t && t < t_max) {
                                t_max = t; best = slot; bu = g.v[0]; bv = g.v[1]; bS = S; bSu = Su; bSv = Sv;
                                do_newton = false;
                            }
                        }
                    }
                    if (do_newton) {
                        ++nc;
                        newtonRhapsonPayload r =
                            BezierPatchOps::newtonRhapson(plane, patch, g.v[0], g.v[1], 1e-5f, eps, (uint)idx);
                        if (r.hit) {
                            float t = (r.s.v[0] - ray.origin.v[0]) * ray.direction.v[0] +
                                      (r.s.v[1] - ray.origin.v[1]) * ray.direction.v[1] +
                                      (r.s.v[2] - ray.origin.v[2]) * ray.direction.v[2];
                            if (0 < t && t < t_max) {
                                t_max = t; best = slot; bu = r.u; bv = r.v; bS = r.s; bSu = r.su; bSv = r.sv;
                            }
                        }
                    }
                }
                if (sp == 0) break;
                cur = nodes[stack[--sp]];
            } else {
                const float tl = box_t(nodes[cur.left_first]), tr = box_t(nodes[cur.left_first + 1]);
                it = fminf(tl, tr);
                if (it >= t_max) {
                    if (sp == 0) break;
                    cur = nodes[stack[--sp]];
                } else if (tl <= it) {
                    if (tr < t_max && sp < 64) stack[sp++] = (int)cur.left_first + 1;
                    cur = nodes[cur.left_first];
                } else {
                    if (tl < t_max && sp < 64) stack[sp++] = (int)cur.left_first;
                    cur = nodes[cur.left_first + 1];
                }
            }
        }
        nc_all += nc;
        sc_all += sc;
        hit[idx] = best;
        t_out[idx] = best >= 0 ? t_max : -1.0f;
        u_out[idx] = bu;
        v_out[idx] = bv;
        if (geo_out) {
            float* g = geo_out + 9 * idx;
            for (int k = 0; k < 3; ++k) { g[k] = bS.v[k]; g[3 + k] = bSu.v[k]; g[6 + k] = bSv.v[k]; }
        }
    }
    if (newton_total) *newton_total = nc_all;
    if (skip_total) *skip_total = sc_all;
}

}  // extern "C"
