// engine.cu -- the C ABI (include/nrt.h): host pipeline, device packing,
// launches and error reporting.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "kernels.h"
#include "nrt_internal.h"
#include "wavefront.h"

// ---------------------------------------------------------------------------
namespace nrt {

static thread_local std::string g_error;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

int fail(int status, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return status;
}

static int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? NRT_ERR_NOMEM : NRT_ERR_CUDA, "%s: %s (%s)", what,
                cudaGetErrorName(e), cudaGetErrorString(e));
}

#define NRT_CUDA(call, what)                               \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// Flatness of a patch: largest distance from a control point to the bilinear
// interpolation of the four corners at its (i/p, j/q) node; patchDelta,
// src/core/main.cpp:18-43.
static float patch_delta(const float* P, int p, int q) {
    const int row = q + 1;
    auto dh = [&](int i, float o[3]) {
        const float iw = 1.0f / P[4 * i + 3];
        o[0] = P[4 * i] * iw; o[1] = P[4 * i + 1] * iw; o[2] = P[4 * i + 2] * iw;
    };
    float c00[3], c10[3], c01[3], c11[3];
    dh(0, c00); dh(p * row, c10); dh(q, c01); dh(p * row + q, c11);
    float d = 0.f;
    for (int i = 0; i <= p; ++i)
        for (int j = 0; j <= q; ++j) {
            const float u = (float)i / p, v = (float)j / q;
            const float a = (1 - u) * (1 - v), b = u * (1 - v), c = (1 - u) * v, e = u * v;
            float Pij[3];
            dh(i * row + j, Pij);
            float s = 0.f;
            for (int k = 0; k < 3; ++k) {
                const float B = a * c00[k] + b * c10[k] + c * c01[k] + e * c11[k];
                s += (Pij[k] - B) * (Pij[k] - B);
            }
            d = fmaxf(d, sqrtf(s));
        }
    return d;
}

// Oriented bounding box of a patch's dehomogenised control points (their
// convex hull holds the patch when every weight is positive): axes from the
// principal directions of the points (cyclic Jacobi on the 3x3 covariance, in
// double), extents from the points' projections.  Four float4 per slot:
// (axis_k, half extent_k) for k = 0..2, then (centre, 0).  A patch with a
// non-positive weight gets infinite extents, so that it is never culled.
static void patch_obb(const float* P, int p, int q, float4 out[4]) {
    const int n = (p + 1) * (q + 1);
    std::vector<double> X(3 * (size_t)n);
    bool pos = true;
    double m[3] = {0, 0, 0};
    for (int i = 0; i < n; ++i) {
        const double w = P[4 * i + 3];
        pos = pos && w > 0.0;
        for (int k = 0; k < 3; ++k) {
            X[3 * i + k] = w != 0.0 ? P[4 * i + k] / w : 0.0;
            m[k] += X[3 * i + k] / n;
        }
    }
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) A[a][b] += (X[3 * i + a] - m[a]) * (X[3 * i + b] - m[b]);
    for (int sweep = 0; sweep < 32; ++sweep) {
        const double off = std::fabs(A[0][1]) + std::fabs(A[0][2]) + std::fabs(A[1][2]);
        if (off <= 1e-300 + 1e-15 * (std::fabs(A[0][0]) + std::fabs(A[1][1]) + std::fabs(A[2][2]))) break;
        for (int a = 0; a < 2; ++a)
            for (int b = a + 1; b < 3; ++b) {
                if (A[a][b] == 0.0) continue;
                const double th = 0.5 * std::atan2(2.0 * A[a][b], A[b][b] - A[a][a]);
                const double c = std::cos(th), s = std::sin(th);
                for (int k = 0; k < 3; ++k) {  // A <- A J
                    const double ka = A[k][a], kb = A[k][b];
                    A[k][a] = c * ka - s * kb;
                    A[k][b] = s * ka + c * kb;
                }
                for (int k = 0; k < 3; ++k) {  // A <- J^T A
                    const double ak = A[a][k], bk = A[b][k];
                    A[a][k] = c * ak - s * bk;
                    A[b][k] = s * ak + c * bk;
                }
                for (int k = 0; k < 3; ++k) {  // V <- V J
                    const double ka = V[k][a], kb = V[k][b];
                    V[k][a] = c * ka - s * kb;
                    V[k][b] = s * ka + c * kb;
                }
            }
    }
    double ctr[3] = {m[0], m[1], m[2]}, half[3];
    for (int a = 0; a < 3; ++a) {
        // round the axis to float first: the device projects with the stored axis
        float ax[3] = {(float)V[0][a], (float)V[1][a], (float)V[2][a]};
        double lo = 1e300, hi = -1e300;
        for (int i = 0; i < n; ++i) {
            const double t = ax[0] * (X[3 * i] - m[0]) + ax[1] * (X[3 * i + 1] - m[1]) + ax[2] * (X[3 * i + 2] - m[2]);
            lo = std::min(lo, t);
            hi = std::max(hi, t);
        }
        half[a] = 0.5 * (hi - lo);
        for (int k = 0; k < 3; ++k) ctr[k] += ax[k] * 0.5 * (lo + hi);
        out[a] = make_float4(ax[0], ax[1], ax[2], 0.f);
    }
    double cmax = 0.0;
    for (int k = 0; k < 3; ++k) cmax = std::max(cmax, std::fabs(ctr[k]));
    for (int a = 0; a < 3; ++a) {
        // extents cover the float-rounded centre and axes
        const double h = half[a] * (1.0 + 1e-6) + 4e-7 * cmax + 1e-30;
        out[a].w = pos ? (float)(h * (1.0 + 1e-6)) : INFINITY;
    }
    out[3] = make_float4((float)ctr[0], (float)ctr[1], (float)ctr[2], 0.f);
}

// Frame of the learned guess's features (see mlp.cuh): the tangent frame of
// the patch at (u, v) = (1/2, 1/2), in patch-local coordinates.  Axes A = dS/du,
// B = dS/dv and the normal of A x B scaled by sqrt|A x B|; origin
// S(1/2, 1/2) - A/2 - B/2, so that a point's frame coordinates (s, t) are its
// (u, v) to first order (the iterate of one Newton step from the midpoint).
// Rational evaluation in double from the weighted-homogeneous points.
// Degenerate nets (collapsed tangents) fall back to the box, normalised.
static dev::PatchFrame patch_frame(const float* P, int p, int q, double cx, double cy, double cz, const Box3& b,
                                   float delta) {
    auto pt = [&](int i, int j, double o[3]) {
        const float* c = P + 4 * (i * (q + 1) + j);
        o[0] = c[0] / (double)c[3] - cx; o[1] = c[1] / (double)c[3] - cy; o[2] = c[2] / (double)c[3] - cz;
    };
    // Bernstein values and derivatives at 1/2
    auto bern = [](int n, double* B, double* dB) {
        double c = 1.0;
        for (int i = 0; i <= n; ++i) {
            B[i] = c / std::ldexp(1.0, n);
            c = c * (n - i) / (i + 1);
        }
        double cm = 1.0, Bm[8];
        for (int i = 0; i < n; ++i) {
            Bm[i] = cm / std::ldexp(1.0, n - 1);
            cm = cm * (n - 1 - i) / (i + 1);
        }
        for (int i = 0; i <= n; ++i) dB[i] = n * ((i > 0 ? Bm[i - 1] : 0.0) - (i < n ? Bm[i] : 0.0));
    };
    double Bu[8], dBu[8], Bv[8], dBv[8];
    bern(p, Bu, dBu);
    bern(q, Bv, dBv);
    double H[4] = {0, 0, 0, 0}, Hu[4] = {0, 0, 0, 0}, Hv[4] = {0, 0, 0, 0};
    for (int i = 0; i <= p; ++i)
        for (int j = 0; j <= q; ++j) {
            const float* c = P + 4 * (i * (q + 1) + j);
            const double w = c[3];
            const double X[4] = {c[0] - w * cx, c[1] - w * cy, c[2] - w * cz, w};
            for (int k = 0; k < 4; ++k) {
                H[k] += Bu[i] * Bv[j] * X[k];
                Hu[k] += dBu[i] * Bv[j] * X[k];
                Hv[k] += Bu[i] * dBv[j] * X[k];
            }
        }
    double A[3], B[3], o[3];
    for (int k = 0; k < 3; ++k) {
        const double S = H[k] / H[3];
        A[k] = (Hu[k] - S * Hu[3]) / H[3];
        B[k] = (Hv[k] - S * Hv[3]) / H[3];
        o[k] = S - 0.5 * A[k] - 0.5 * B[k];
    }
    const double N[3] = {A[1] * B[2] - A[2] * B[1], A[2] * B[0] - A[0] * B[2], A[0] * B[1] - A[1] * B[0]};
    const double nn = std::sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    const double aa = A[0] * A[0] + A[1] * A[1] + A[2] * A[2], bb = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
    dev::PatchFrame f{};
    double M[3][3];  // columns A, B, N/sqrt|N|
    double scale;
    if (nn > 1e-9 * (aa + bb) && aa > 0 && bb > 0) {
        const double s = 1.0 / std::sqrt(nn);
        for (int k = 0; k < 3; ++k) { M[k][0] = A[k]; M[k][1] = B[k]; M[k][2] = N[k] * s; }
        scale = std::sqrt(std::max(aa, bb));
    } else {
        for (int k = 0; k < 3; ++k) {
            o[k] = (double)b.lo[k] - (k == 0 ? cx : k == 1 ? cy : cz);
            for (int l = 0; l < 3; ++l) M[k][l] = k == l ? std::max((double)b.hi[k] - b.lo[k], 1e-12) : 0.0;
        }
        scale = std::max({M[0][0], M[1][1], M[2][2]});
    }
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                       M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    const double id = 1.0 / det;
    const double inv[9] = {(M[1][1] * M[2][2] - M[1][2] * M[2][1]) * id, (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * id,
                           (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * id, (M[1][2] * M[2][0] - M[1][0] * M[2][2]) * id,
                           (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * id, (M[0][2] * M[1][0] - M[0][0] * M[1][2]) * id,
                           (M[1][0] * M[2][1] - M[1][1] * M[2][0]) * id, (M[0][1] * M[2][0] - M[0][0] * M[2][1]) * id,
                           (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * id};
    f.ox = (float)o[0]; f.oy = (float)o[1]; f.oz = (float)o[2];
    for (int k = 0; k < 9; ++k) f.m[k] = (float)inv[k];
    double hmax = 0.0;  // half-thickness of the control net along the frame's h axis
    for (int i = 0; i <= p; ++i)
        for (int j = 0; j <= q; ++j) {
            double X[3];
            pt(i, j, X);
            const double d3[3] = {X[0] - o[0], X[1] - o[1], X[2] - o[2]};
            hmax = std::max(hmax, std::fabs(inv[6] * d3[0] + inv[7] * d3[1] + inv[8] * d3[2]));
        }
    f.slab = (float)std::max(hmax, 1e-6);
    f.flat = (float)(hmax * std::sqrt(std::fabs(det)) / std::max(scale * scale, 1e-30));
    (void)delta;
    f.lo[0] = (float)(b.lo[0] - cx); f.lo[1] = (float)(b.lo[1] - cy); f.lo[2] = (float)(b.lo[2] - cz);
    f.hi_x = (float)(b.hi[0] - cx); f.hi_y = (float)(b.hi[1] - cy); f.hi_z = (float)(b.hi[2] - cz);
    return f;
}

dev::MlpParams blob_params(const void* blob);
size_t mlp_blob_bytes();
const void* mlp_device_blob(const nrt_mlp* m);
int mlp_device(const nrt_mlp* m);

}  // namespace nrt

using namespace nrt;

struct nrt_scene {
    int device = 0;
    PatchSet ps;
    int n_surfaces = 0;
    std::vector<int32_t> slot_patch;   // device slot -> global patch id
    void* arena = nullptr;
    size_t arena_bytes = 0;
    unsigned long long* counters = nullptr;
    int counters_on = 0;
    dev::Scene view{};
    nrt_scene_info info{};
    dev::WfPlan plan{};
    void* wf_ws = nullptr;       // wavefront scratch, grown on demand
    size_t wf_bytes = 0;
    long long wf_rays = 0;       // rays the scratch was carved for
    long long wf_chunk = 0;      // rays per wavefront pass
    int32_t* host_count = nullptr;  // pinned word for the per-round active count
    long long last_launches = 0, last_rounds = 0;  // of the last nrt_intersect
    void* mlp_blob = nullptr;    // the scene's copy of the learned guess's network
    // The wavefront as CUDA graphs: the last few built (most recent last), each
    // with the arguments it was built for (pointers, sizes, options, launch
    // shapes) and its pass count.
    struct WfGraph {
        std::vector<unsigned char> key;
        cudaGraphExec_t exec = nullptr;
        long long passes = 0;
    };
    std::vector<WfGraph> wf_graphs;
    long long wf_graph_passes = 0;  // passes of the graph the last call ran
    bool last_graph = false;     // the last nrt_intersect ran the graph (rounds counted on the device)
    dev::WfTuning tuning{};
    bool use_graph = true;       // false: host-driven rounds
    bool timing_on = false;      // events around the per-class Newton launches (host-driven rounds)
    cudaEvent_t tev[2] = {nullptr, nullptr};
    double newton_ms = 0.0;
    long long newton_launches = 0;
};



namespace {

int build_scene(PatchSet&& ps, int n_surfaces, const nrt_build_opts* opts, nrt_scene** out) {
    if (!out) return fail(NRT_ERR_INVALID, "out is null");
    *out = nullptr;
    const int N = ps.count();
    if (N <= 0) return fail(NRT_ERR_INVALID, "scene has no patches");
    nrt_build_opts o{NRT_BVH_BINNED_SAH, 1, 0, 0};
    if (opts) o = *opts;
    if (o.wavefront_chunk < 0) return fail(NRT_ERR_INVALID, "negative wavefront_chunk");
    if (o.max_leaf < 1 || o.max_leaf > 8) return fail(NRT_ERR_INVALID, "max_leaf must be in 1..8");
    if (N >= (1 << 27)) return fail(NRT_ERR_INVALID, "too many patches (%d)", N);
    for (int k = 0; k < N; ++k) {
        const int p = ps.deg[2 * k], q = ps.deg[2 * k + 1];
        if (p < 1 || q < 1 || p > NRT_MAX_DEGREE || q > NRT_MAX_DEGREE)
            return fail(NRT_ERR_INVALID, "patch %d has degree (%d,%d) outside 1..%d", k, p, q, NRT_MAX_DEGREE);
    }
    // BVH over patch boxes
    std::vector<Box3> boxes;
    patch_boxes(ps, boxes);
    BinaryBVH bin;
    if (o.builder == NRT_BVH_EXACT_SAH) build_exact_sah(boxes, bin);
    else build_binned_sah(boxes, o.max_leaf, bin);
    for (int i = 0; i < bin.used; ++i)
        if (bin.prim_count[i] > 8)  // coincident centroids can leave bigger leaves
            return fail(NRT_ERR_UNSUPPORTED, "BVH leaf with %u patches (limit 8)", bin.prim_count[i]);
    std::vector<Node4> wide;
    int depth = 0;
    collapse_to_wide(bin, wide, depth);

    // Pack patches in leaf order.
    std::vector<int4> hdr(N);
    std::vector<double4> centre(N);
    std::vector<float4> corners(4 * (size_t)N);
    std::vector<float> delta(N);
    std::vector<dev::PatchFrame> frames(N);
    std::vector<float4> obbs(4 * (size_t)N);
    // each slot's leaf box as its parent node stores it (the flat-skip's entry distance)
    std::vector<float4> leafbox(2 * (size_t)N, make_float4(0.f, 0.f, 0.f, 0.f));
    for (const Node4& nd : wide)
        for (int c = 0; c < 4; ++c)
            if (nd.child[c] < 0 && nd.count[c] > 0)
                for (int k = ~nd.child[c]; k < ~nd.child[c] + nd.count[c]; ++k) {
                    leafbox[2 * (size_t)k] = make_float4(nd.lo_x[c], nd.lo_y[c], nd.lo_z[c], 0.f);
                    leafbox[2 * (size_t)k + 1] = make_float4(nd.hi_x[c], nd.hi_y[c], nd.hi_z[c], 0.f);
                }
    std::vector<float> blocks;
    std::vector<int32_t> slot_patch(N);
    size_t total_floats = 0;
    for (int s = 0; s < N; ++s) {
        const int k = bin.order[s];
        total_floats += 4 * (size_t)dev::padded_points(ps.deg[2 * k], ps.deg[2 * k + 1]);
    }
    blocks.assign(total_floats, 0.f);
    size_t off = 0;
    nrt_scene_info info{};
    for (int s = 0; s < N; ++s) {
        const int k = bin.order[s];
        slot_patch[s] = k;
        const int p = ps.deg[2 * k], q = ps.deg[2 * k + 1], n = (p + 1) * (q + 1);
        const int np = dev::padded_points(p, q);
        const float* P = &ps.cp[4 * (size_t)ps.off[k]];
        const Box3& b = boxes[k];
        const double cx = 0.5 * ((double)b.lo[0] + b.hi[0]), cy = 0.5 * ((double)b.lo[1] + b.hi[1]),
                     cz = 0.5 * ((double)b.lo[2] + b.hi[2]);
        bool pos = true;
        double rad = 0.0;
        for (int i = 0; i < n; ++i) {
            const double w = P[4 * i + 3];
            pos = pos && (w > 0.0);
            blocks[off + i] = (float)((double)P[4 * i + 0] - w * cx);
            blocks[off + np + i] = (float)((double)P[4 * i + 1] - w * cy);
            blocks[off + 2 * np + i] = (float)((double)P[4 * i + 2] - w * cz);
            blocks[off + 3 * np + i] = (float)w;
            if (w != 0.0) {
                const double dx = P[4 * i] / w - cx, dy = P[4 * i + 1] / w - cy, dz = P[4 * i + 2] / w - cz;
                rad = std::max(rad, std::sqrt(dx * dx + dy * dy + dz * dz));
            }
        }
        for (int i = n; i < np; ++i) blocks[off + 3 * np + i] = 1.f;  // padding never read as a point
        hdr[s] = make_int4((int)off, p | (q << 4) | ((pos ? dev::kFlagPositiveWeights : 0) << 8), k, ps.surf[k]);
        centre[s] = make_double4(cx, cy, cz, rad);
        const int ci[4] = {0, p * (q + 1), p * (q + 1) + q, q};  // q00, q10, q11, q01 (bezier_patch.h:37-44)
        for (int c = 0; c < 4; ++c) {
            const float* X = P + 4 * ci[c];
            const float iw = 1.f / X[3];
            corners[4 * (size_t)s + c] = make_float4(X[0] * iw, X[1] * iw, X[2] * iw, 0.f);
        }
        delta[s] = patch_delta(P, p, q);
        frames[s] = patch_frame(P, p, q, cx, cy, cz, b, delta[s]);
        patch_obb(P, p, q, &obbs[4 * (size_t)s]);
        info.degree_hist[p * 8 + q] += 1;
        off += 4 * (size_t)np;
    }

    // One device arena, every array 256-byte aligned.
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t sz_nodes = align(wide.size() * sizeof(Node4)), sz_hdr = align(N * sizeof(int4)),
                 sz_cen = align(N * sizeof(double4)), sz_cp = align(blocks.size() * sizeof(float)),
                 sz_cor = align(corners.size() * sizeof(float4)), sz_del = align(N * sizeof(float)),
                 sz_ctr = align(dev::kCounterWords * sizeof(unsigned long long)),
                 sz_rank = align(N * sizeof(int32_t)), sz_frm = align(N * sizeof(dev::PatchFrame)),
                 sz_obb = align(obbs.size() * sizeof(float4)), sz_lbx = align(leafbox.size() * sizeof(float4));
    const size_t total =
        sz_nodes + sz_hdr + sz_cen + sz_cp + sz_cor + sz_del + sz_ctr + sz_rank + sz_frm + sz_obb + sz_lbx;
    // wavefront plan: patches ranked by (p, q, slot); one class per degree pair present
    std::vector<int32_t> by_rank(N), rank_of(N);
    for (int s2 = 0; s2 < N; ++s2) by_rank[s2] = s2;
    std::stable_sort(by_rank.begin(), by_rank.end(), [&](int a, int b) { return (hdr[a].y & 0xff) < (hdr[b].y & 0xff); });
    dev::WfPlan plan{};
    plan.n_slots = N;
    for (int rk = 0; rk < N; ++rk) {
        rank_of[by_rank[rk]] = rk;
        const int pq = hdr[by_rank[rk]].y & 0xff;
        if (plan.n_classes == 0 || plan.class_pq[plan.n_classes - 1] != pq) {
            plan.class_pq[plan.n_classes] = pq;
            plan.class_rank[plan.n_classes] = rk;
            plan.class_grid[plan.n_classes] = 148 * 4;
            ++plan.n_classes;
        }
    }
    plan.class_rank[plan.n_classes] = N;
    nrt_scene* sc = new (std::nothrow) nrt_scene();
    if (!sc) return fail(NRT_ERR_NOMEM, "host allocation failed");
    sc->device = o.device;
    sc->wf_chunk = o.wavefront_chunk > 0 ? o.wavefront_chunk : (1LL << 23);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(o.device);
    if (e != cudaSuccess) { delete sc; return cuda_fail(e, "cudaSetDevice"); }
    e = cudaMalloc(&sc->arena, total);
    if (e != cudaSuccess) { delete sc; cudaSetDevice(prev); return cuda_fail(e, "cudaMalloc(scene)"); }
    char* base = static_cast<char*>(sc->arena);
    size_t at = 0;
    auto put = [&](const void* src, size_t bytes, size_t slot) -> void* {
        void* dst = base + at;
        if (bytes) e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
        at += slot;
        return dst;
    };
    sc->view.nodes = static_cast<const dev::Node4*>(put(wide.data(), wide.size() * sizeof(Node4), sz_nodes));
    sc->view.hdr = static_cast<const int4*>(put(hdr.data(), N * sizeof(int4), sz_hdr));
    sc->view.centre = static_cast<const double4*>(put(centre.data(), N * sizeof(double4), sz_cen));
    sc->view.cp = static_cast<const float*>(put(blocks.data(), blocks.size() * sizeof(float), sz_cp));
    sc->view.corners = static_cast<const float4*>(put(corners.data(), corners.size() * sizeof(float4), sz_cor));
    sc->view.delta = static_cast<const float*>(put(delta.data(), N * sizeof(float), sz_del));
    sc->counters = reinterpret_cast<unsigned long long*>(base + at);
    if (e == cudaSuccess) e = cudaMemset(sc->counters, 0, sz_ctr);
    at += sz_ctr;
    plan.rank_of = static_cast<const int32_t*>(put(rank_of.data(), N * sizeof(int32_t), sz_rank));
    sc->view.frames = static_cast<const dev::PatchFrame*>(put(frames.data(), N * sizeof(dev::PatchFrame), sz_frm));
    sc->view.obb = static_cast<const float4*>(put(obbs.data(), obbs.size() * sizeof(float4), sz_obb));
    sc->view.leafbox = static_cast<const float4*>(put(leafbox.data(), leafbox.size() * sizeof(float4), sz_lbx));
    sc->plan = plan;
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaFree(sc->arena);
        delete sc;
        return cuda_fail(e, "scene upload");
    }
    sc->view.n_slots = N;
    sc->arena_bytes = total;
    info.n_patches = N;
    info.n_surfaces = n_surfaces;
    info.n_nodes = (int)wide.size();
    info.bvh_depth = depth;
    info.device_bytes = total;
    sc->info = info;
    sc->slot_patch = std::move(slot_patch);
    sc->ps = std::move(ps);
    sc->n_surfaces = n_surfaces;
    *out = sc;
    return NRT_OK;
}

void to_dev_opts(const nrt_intersect_opts& o, dev::Opts& d, int counters) {
    d.nw.max_iter = o.max_iter;
    d.nw.eps = o.eps;
    d.nw.det_eps = o.det_eps;
    d.nw.cond_fp64 = o.cond_fp64;
    d.nw.fp64_final = o.fp64_final;
    d.init_mode = o.init_mode;
    d.hull_cull = o.hull_cull;
    d.seed_offset = (uint32_t)o.seed_offset;
    d.flat_threshold = o.flat_threshold;
    d.cam_k = o.cam_k;
    d.counters = counters;
    d.learned_iters = o.learned_iters;
    d.mlp = dev::MlpParams{};
    d.col_feat = nullptr;
    d.col_targ = nullptr;
    d.col_count = nullptr;
    d.col_cap = 0;
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" {

const char* nrt_last_error(void) { return g_error.c_str(); }
const char* nrt_version(void) { return "nrt 0.1 (sm_100a)"; }

int nrt_decompose_count(const nrt_nurbs_surface* surf, int* nbU, int* nbV) {
    if (!surf || !nbU || !nbV) return fail(NRT_ERR_INVALID, "null argument");
    if (int st = check_surface(*surf)) return st;
    int nu = 1, nv = 1;
    for (int i = surf->p + 1; i <= surf->n; ++i) nu += surf->u_knots[i] != surf->u_knots[i - 1];
    for (int j = surf->q + 1; j <= surf->m; ++j) nv += surf->v_knots[j] != surf->v_knots[j - 1];
    *nbU = nu;
    *nbV = nv;
    return NRT_OK;
}

int nrt_decompose(const nrt_nurbs_surface* surf, float* cp_out, float* ranges_out, int* nbU, int* nbV) {
    if (!surf || !cp_out || !nbU || !nbV) return fail(NRT_ERR_INVALID, "null argument");
    std::vector<float> cp, ranges;
    int nu = 0, nv = 0;
    if (int st = decompose_surface(*surf, cp, ranges, nu, nv)) return st;
    std::memcpy(cp_out, cp.data(), cp.size() * sizeof(float));
    if (ranges_out) std::memcpy(ranges_out, ranges.data(), ranges.size() * sizeof(float));
    *nbU = nu;
    *nbV = nv;
    return NRT_OK;
}

int nrt_patch_bounds(const float* cp, const int32_t* cp_offset, const int32_t* degrees, int n_patches,
                     float* boxes) {
    if (n_patches < 0 || (n_patches > 0 && (!cp || !cp_offset || !degrees || !boxes)))
        return fail(NRT_ERR_INVALID, "null argument");
    PatchSet ps;
    int max_point = 0;
    for (int k = 0; k < n_patches; ++k)
        max_point = std::max(max_point, cp_offset[k] + (degrees[2 * k] + 1) * (degrees[2 * k + 1] + 1));
    ps.cp.assign(cp, cp + 4 * (size_t)max_point);
    ps.off.assign(cp_offset, cp_offset + n_patches);
    ps.deg.assign(degrees, degrees + 2 * (size_t)n_patches);
    std::vector<Box3> b;
    patch_boxes(ps, b);
    for (int k = 0; k < n_patches; ++k)
        for (int a = 0; a < 3; ++a) { boxes[6 * k + a] = b[k].lo[a]; boxes[6 * k + 3 + a] = b[k].hi[a]; }
    return NRT_OK;
}

int nrt_build_bvh_binary(const float* boxes, int n, int builder, float* node_bounds, uint32_t* left_first,
                         uint32_t* prim_count, int32_t* order, int* n_nodes) {
    if (n <= 0 || !boxes || !node_bounds || !left_first || !prim_count || !order)
        return fail(NRT_ERR_INVALID, "null argument or empty input");
    std::vector<Box3> prims(n);
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) { prims[i].lo[a] = boxes[6 * i + a]; prims[i].hi[a] = boxes[6 * i + 3 + a]; }
    BinaryBVH bin;
    if (builder == NRT_BVH_EXACT_SAH) build_exact_sah(prims, bin);
    else if (builder == NRT_BVH_BINNED_SAH) build_binned_sah(prims, 1, bin);
    else return fail(NRT_ERR_INVALID, "unknown BVH builder %d", builder);
    const size_t M = 2 * (size_t)n - 1;
    for (size_t i = 0; i < M; ++i) {
        for (int a = 0; a < 3; ++a) {
            node_bounds[6 * i + a] = bin.box[i].lo[a];
            node_bounds[6 * i + 3 + a] = bin.box[i].hi[a];
        }
        left_first[i] = bin.left_first[i];
        prim_count[i] = bin.prim_count[i];
    }
    std::memcpy(order, bin.order.data(), sizeof(int32_t) * n);
    if (n_nodes) *n_nodes = bin.used;
    return NRT_OK;
}

int nrt_scene_create(const nrt_nurbs_surface* surfaces, int n_surfaces, const nrt_build_opts* opts,
                     nrt_scene** out) {
    if (!surfaces || n_surfaces <= 0 || !out) return fail(NRT_ERR_INVALID, "null or empty surface list");
    PatchSet ps;
    for (int si = 0; si < n_surfaces; ++si) {
        std::vector<float> cp, ranges;
        int nu = 0, nv = 0;
        if (int st = decompose_surface(surfaces[si], cp, ranges, nu, nv)) {
            set_error("surface %d: %s", si, nrt_last_error());
            return st;
        }
        const int piece = (surfaces[si].p + 1) * (surfaces[si].q + 1);
        const int base = (int)(ps.cp.size() / 4);
        ps.cp.insert(ps.cp.end(), cp.begin(), cp.end());
        ps.ranges.insert(ps.ranges.end(), ranges.begin(), ranges.end());
        for (int k = 0; k < nu * nv; ++k) {
            ps.off.push_back(base + k * piece);
            ps.deg.push_back(surfaces[si].p);
            ps.deg.push_back(surfaces[si].q);
            ps.surf.push_back(si);
        }
    }
    return build_scene(std::move(ps), n_surfaces, opts, out);
}

int nrt_scene_create_from_patches(const float* cp, const int32_t* cp_offset, const int32_t* degrees, int n_patches,
                                  const nrt_build_opts* opts, nrt_scene** out) {
    if (!cp || !cp_offset || !degrees || n_patches <= 0 || !out) return fail(NRT_ERR_INVALID, "null or empty input");
    PatchSet ps;
    int max_point = 0;
    for (int k = 0; k < n_patches; ++k) {
        if (cp_offset[k] < 0) return fail(NRT_ERR_INVALID, "negative control point offset");
        max_point = std::max(max_point, cp_offset[k] + (degrees[2 * k] + 1) * (degrees[2 * k + 1] + 1));
    }
    ps.cp.assign(cp, cp + 4 * (size_t)max_point);
    ps.off.assign(cp_offset, cp_offset + n_patches);
    ps.deg.assign(degrees, degrees + 2 * (size_t)n_patches);
    ps.ranges.assign(4 * (size_t)n_patches, 0.f);
    for (int k = 0; k < n_patches; ++k) { ps.ranges[4 * k + 1] = 1.f; ps.ranges[4 * k + 3] = 1.f; }
    ps.surf.assign(n_patches, 0);
    return build_scene(std::move(ps), 1, opts, out);
}

int nrt_scene_destroy(nrt_scene* scene) {
    if (!scene) return NRT_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(scene->device);
    cudaError_t e = cudaFree(scene->arena);
    if (scene->wf_ws) {
        const cudaError_t e2 = cudaFree(scene->wf_ws);
        if (e == cudaSuccess) e = e2;
    }
    if (scene->host_count) cudaFreeHost(scene->host_count);
    if (scene->mlp_blob) cudaFree(scene->mlp_blob);
    for (auto& g : scene->wf_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (cudaEvent_t ev : scene->tev)
        if (ev) cudaEventDestroy(ev);
    cudaSetDevice(prev);
    delete scene;
    if (e != cudaSuccess) return cuda_fail(e, "cudaFree(scene)");
    return NRT_OK;
}

int nrt_scene_get_info(const nrt_scene* scene, nrt_scene_info* info) {
    if (!scene || !info) return fail(NRT_ERR_INVALID, "null argument");
    *info = scene->info;
    return NRT_OK;
}

int nrt_scene_patch_table(const nrt_scene* scene, int32_t* surface_of, float* ranges) {
    if (!scene) return fail(NRT_ERR_INVALID, "null scene");
    const int N = scene->ps.count();
    if (surface_of) std::memcpy(surface_of, scene->ps.surf.data(), sizeof(int32_t) * N);
    if (ranges) std::memcpy(ranges, scene->ps.ranges.data(), sizeof(float) * 4 * N);
    return NRT_OK;
}

void nrt_default_opts(nrt_intersect_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->init_mode = NRT_INIT_MIDPOINT;
    o->max_iter = 8;
    o->eps = 1e-6f;
    o->det_eps = 1e-5f;
    o->cond_fp64 = 0.f;
    o->fp64_final = 0;
    o->hull_cull = 0;
    o->schedule = NRT_SCHED_PIXEL;
}

void nrt_reference_opts(nrt_intersect_opts* o) {
    nrt_default_opts(o);
    if (!o) return;
    o->init_mode = NRT_INIT_BILINEAR;
    o->max_iter = 7;
    o->eps = 1e-4f;
}

int nrt_intersect(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                  const nrt_hits* hits, void* stream) {
    if (!scene || !rays || !opts || !hits) return fail(NRT_ERR_INVALID, "null argument");
    if (n < 0) return fail(NRT_ERR_INVALID, "negative ray count");
    if (n == 0) return NRT_OK;
    if (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz)
        return fail(NRT_ERR_INVALID, "null ray array");
    if (!hits->patch || !hits->t || !hits->u || !hits->v) return fail(NRT_ERR_INVALID, "null hit array");
    const nrt_intersect_opts& o = *opts;
    if (o.max_iter < 1 || o.max_iter > 256) return fail(NRT_ERR_INVALID, "max_iter %d outside 1..256", o.max_iter);
    if (!(o.eps > 0.f)) return fail(NRT_ERR_INVALID, "eps must be positive");
    if (o.init_mode != NRT_INIT_MIDPOINT && o.init_mode != NRT_INIT_BILINEAR) {
        if (o.init_mode != NRT_INIT_LEARNED) return fail(NRT_ERR_INVALID, "unknown init mode %d", o.init_mode);
        if (!scene->mlp_blob) return fail(NRT_ERR_INVALID, "learned init: no network set on this scene");
        if (o.schedule != NRT_SCHED_WAVEFRONT)
            return fail(NRT_ERR_UNSUPPORTED, "learned init runs on the wavefront schedule");
    }
    if (o.schedule != NRT_SCHED_PIXEL && o.schedule != NRT_SCHED_WAVEFRONT)
        return fail(NRT_ERR_INVALID, "unknown schedule %d", o.schedule);
    if (o.flat_threshold > 0.f && o.init_mode == NRT_INIT_LEARNED)
        return fail(NRT_ERR_UNSUPPORTED, "flat-skip tests the midpoint or bilinear guess, not the learned one");
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != scene->device) NRT_CUDA(cudaSetDevice(scene->device), "cudaSetDevice");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    dev::Opts d;
    std::memset(&d, 0, sizeof(d));  // padding too: the options are part of the graph's key
    to_dev_opts(o, d, scene->counters_on);
    if (scene->mlp_blob) d.mlp = blob_params(scene->mlp_blob);
    if (scene->counters_on)
        NRT_CUDA(cudaMemsetAsync(scene->counters, 0, dev::kCounterWords * sizeof(unsigned long long), st),
                 "counter reset");
    dev::Rays r{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz};
    dev::Hits h{hits->patch, hits->t, hits->u, hits->v, hits->iters, hits->tests, hits->geom};
    cudaError_t e = cudaSuccess;
    scene->last_launches = 0;
    scene->last_rounds = 0;
    scene->last_graph = false;
    if (o.schedule == NRT_SCHED_PIXEL) {
        e = dev::launch_intersect_pixel(scene->view, r, (long long)n, d, h, scene->counters, st);
        scene->last_launches = 1;
    } else {
        const long long chunk = std::min<long long>(n, scene->wf_chunk);
        if (scene->wf_rays < chunk) {
            // (re)allocate scratch for `chunk` rays; cudaFree synchronises the device
            if (scene->wf_ws) cudaFree(scene->wf_ws);
            scene->wf_ws = nullptr;
            scene->wf_rays = 0;
            const size_t bytes = dev::wavefront_scratch_bytes(chunk, scene->plan.n_slots);
            e = cudaMalloc(&scene->wf_ws, bytes);
            if (e != cudaSuccess) {
                scene->wf_ws = nullptr;
                if (prev != scene->device) cudaSetDevice(prev);
                return cuda_fail(e, "cudaMalloc(wavefront scratch)");
            }
            scene->wf_bytes = bytes;
            scene->wf_rays = chunk;
        }
        if (!scene->host_count) {
            e = cudaMallocHost(&scene->host_count, sizeof(int32_t));
            if (e != cudaSuccess) {
                scene->host_count = nullptr;
                if (prev != scene->device) cudaSetDevice(prev);
                return cuda_fail(e, "cudaMallocHost(count)");
            }
        }
        const dev::WfBuffers wb = dev::wavefront_carve(scene->wf_ws, scene->wf_rays, scene->plan.n_slots);
        // the graph is rebuilt when any of its arguments changed
        std::vector<unsigned char> key;
        auto add = [&](const void* p, size_t b) {
            const unsigned char* c = static_cast<const unsigned char*>(p);
            key.insert(key.end(), c, c + b);
        };
        const long long nn = n;
        add(&r, sizeof(r));
        add(&h, sizeof(h));
        add(&nn, sizeof(nn));
        add(&chunk, sizeof(chunk));
        add(&scene->wf_ws, sizeof(scene->wf_ws));
        add(&scene->wf_rays, sizeof(scene->wf_rays));  // the scratch layout follows from it
        add(&d, sizeof(d));
        add(&scene->tuning, sizeof(scene->tuning));
        scene->newton_ms = 0.0;
        scene->newton_launches = 0;
        if (scene->timing_on && !scene->tev[0]) {
            e = cudaEventCreate(&scene->tev[0]);
            if (e == cudaSuccess) e = cudaEventCreate(&scene->tev[1]);
            if (e != cudaSuccess) {
                if (prev != scene->device) cudaSetDevice(prev);
                return cuda_fail(e, "cudaEventCreate");
            }
        }
        if (!scene->use_graph || scene->timing_on) {
            for (long long at = 0; at < n && e == cudaSuccess; at += chunk) {
                const long long m = std::min(chunk, (long long)n - at);
                dev::Rays rc{r.ox + at, r.oy + at, r.oz + at, r.dx + at, r.dy + at, r.dz + at};
                dev::Hits hc{h.patch + at, h.t + at, h.u + at, h.v + at, h.iters ? h.iters + at : nullptr,
                             h.tests ? h.tests + at : nullptr, h.geom ? h.geom + 9 * at : nullptr};
                dev::Opts dc = d;
                dc.seed_offset = d.seed_offset + (uint32_t)at;  // seeds follow the global ray index
                e = dev::launch_wavefront(scene->view, scene->plan, rc, m, dc, hc, wb, scene->host_count,
                                          scene->counters, st, &scene->last_launches, &scene->last_rounds,
                                          scene->timing_on ? scene->tev : nullptr,
                                          scene->timing_on ? &scene->newton_ms : nullptr, &scene->newton_launches,
                                          scene->tuning.quota0, scene->tuning.quota_max);
            }
            if (prev != scene->device) cudaSetDevice(prev);
            if (e != cudaSuccess) return cuda_fail(e, "intersect launch");
            return NRT_OK;
        }
        constexpr size_t kGraphsKept = 4;
        auto& gs = scene->wf_graphs;
        size_t at = 0;
        while (at < gs.size() && gs[at].key != key) ++at;
        if (at == gs.size()) {
            nrt_scene::WfGraph g;
            e = dev::build_wavefront_graph(scene->view, scene->plan, r, (long long)n, chunk, d, h, wb,
                                           scene->counters, scene->tuning, &g.exec, &g.passes);
            if (e == cudaSuccess) {
                g.key = std::move(key);
                if (gs.size() == kGraphsKept) {  // drop the least recently used
                    cudaGraphExecDestroy(gs.front().exec);
                    gs.erase(gs.begin());
                }
                gs.push_back(std::move(g));
                at = gs.size() - 1;
            }
        } else if (at + 1 != gs.size()) {  // most recent last
            std::rotate(gs.begin() + at, gs.begin() + at + 1, gs.end());
            at = gs.size() - 1;
        }
        if (e == cudaSuccess) {
            e = cudaGraphLaunch(gs[at].exec, st);
            scene->wf_graph_passes = gs[at].passes;
        }
        scene->last_graph = true;
    }
    if (prev != scene->device) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "intersect launch");
    return NRT_OK;
}

int nrt_scene_get_tuning(const nrt_scene* scene, nrt_wavefront_tuning* out) {
    if (!scene || !out) return fail(NRT_ERR_INVALID, "null argument");
    out->step_blocks = scene->tuning.step_blocks;
    out->scatter_blocks = scene->tuning.scatter_blocks;
    out->class_blocks = scene->tuning.class_blocks > 0 ? scene->tuning.class_blocks : (int32_t)scene->plan.class_grid[0];
    out->graph = scene->use_graph ? 1 : 2;
    out->chunk = scene->wf_chunk;
    out->quota0 = scene->tuning.quota0;
    out->quota_max = scene->tuning.quota_max;
    return NRT_OK;
}

int nrt_scene_set_tuning(nrt_scene* scene, const nrt_wavefront_tuning* in) {
    if (!scene || !in) return fail(NRT_ERR_INVALID, "null argument");
    if (in->step_blocks > (1LL << 24) || in->scatter_blocks > (1LL << 24) || in->class_blocks > (1 << 24))
        return fail(NRT_ERR_INVALID, "block counts above 2^24");
    if (in->graph > 2) return fail(NRT_ERR_INVALID, "graph must be 1 (graph) or 2 (host-driven)");
    if (in->chunk > (1LL << 30)) return fail(NRT_ERR_INVALID, "chunk above 2^30 rays");
    if (in->quota0 > 8 || in->quota_max > 8) return fail(NRT_ERR_INVALID, "round quotas above 8");
    const int q0 = in->quota0 > 0 ? in->quota0 : scene->tuning.quota0;
    const int qm = in->quota_max > 0 ? in->quota_max : scene->tuning.quota_max;
    if (q0 > qm) return fail(NRT_ERR_INVALID, "quota0 %d above quota_max %d", q0, qm);
    if (in->step_blocks > 0) scene->tuning.step_blocks = in->step_blocks;
    if (in->scatter_blocks > 0) scene->tuning.scatter_blocks = in->scatter_blocks;
    if (in->class_blocks > 0) scene->tuning.class_blocks = in->class_blocks;
    if (in->graph > 0) scene->use_graph = in->graph == 1;
    if (in->chunk > 0) scene->wf_chunk = in->chunk;  // the scratch is re-carved on the next call
    scene->tuning.quota0 = q0;
    scene->tuning.quota_max = qm;
    return NRT_OK;
}

int nrt_autotune(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                 const nrt_hits* hits, int reps, nrt_wavefront_tuning* out, float* best_ms, void* stream) {
    if (!scene || !rays || !opts || !hits || !out) return fail(NRT_ERR_INVALID, "null argument");
    if (n <= 0) return fail(NRT_ERR_INVALID, "autotuning needs rays");
    if (reps < 1 || reps > 1000) return fail(NRT_ERR_INVALID, "reps %d outside 1..1000", reps);
    nrt_intersect_opts o = *opts;
    o.schedule = NRT_SCHED_WAVEFRONT;
    const int was_on = scene->counters_on;
    scene->counters_on = 0;  // time the plain launches
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != scene->device) NRT_CUDA(cudaSetDevice(scene->device), "cudaSetDevice");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    int status = ce == cudaSuccess ? NRT_OK : cuda_fail(ce, "cudaEventCreate");
    auto trial = [&](const nrt_wavefront_tuning& t, float& ms) -> int {
        int rc = nrt_scene_set_tuning(scene, &t);
        if (rc == NRT_OK) rc = nrt_intersect(scene, rays, n, &o, hits, stream);  // builds the graph, if any
        if (rc != NRT_OK) return rc;
        cudaError_t e = cudaEventRecord(e0, st);
        for (int k = 0; k < reps && rc == NRT_OK; ++k) rc = nrt_intersect(scene, rays, n, &o, hits, stream);
        if (rc != NRT_OK) return rc;
        if (e == cudaSuccess) e = cudaEventRecord(e1, st);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) return cuda_fail(e, "autotune timing");
        ms /= (float)reps;
        return NRT_OK;
    };
    nrt_wavefront_tuning best{};
    if (status == NRT_OK) status = nrt_scene_get_tuning(scene, &best);
    float best_t = 0.f;
    if (status == NRT_OK) status = trial(best, best_t);
    const long long rays_blocks = (n + 127) / 128;
    const int64_t steps[] = {148 * 4, 148 * 8, 148 * 16, 148 * 64};
    const int64_t scats[] = {148 * 4, 148 * 8, 148 * 16, 148 * 64};
    const int32_t classes[] = {148 * 2, 148 * 4, 148 * 8, 148 * 16};
    const int64_t chunks[] = {1LL << 21, 1LL << 22, 1LL << 23};
    const int32_t quotas[] = {1 << 8 | 8, 2 << 8 | 8, 4 << 8 | 8, 1 << 8 | 4};  // (first round, cap)
    for (int pass = 0; pass < 2 && status == NRT_OK; ++pass) {
        auto knob = [&](auto&& values, int count, auto&& set) {
            for (int k = 0; k < count && status == NRT_OK; ++k) {
                nrt_wavefront_tuning t = best;
                if (!set(t, values[k])) continue;
                float ms = 0.f;
                status = trial(t, ms);
                if (status == NRT_OK && ms < best_t) {
                    best_t = ms;
                    best = t;
                }
            }
        };
        knob(steps, 4, [&](nrt_wavefront_tuning& t, int64_t v) {
            if (v == t.step_blocks || (v > rays_blocks && t.step_blocks >= rays_blocks)) return false;
            t.step_blocks = v;
            return true;
        });
        knob(scats, 4, [&](nrt_wavefront_tuning& t, int64_t v) {
            if (v == t.scatter_blocks || (v > rays_blocks && t.scatter_blocks >= rays_blocks)) return false;
            t.scatter_blocks = v;
            return true;
        });
        knob(classes, 4, [&](nrt_wavefront_tuning& t, int32_t v) {
            if (v == t.class_blocks) return false;
            t.class_blocks = v;
            return true;
        });
        knob(quotas, 4, [&](nrt_wavefront_tuning& t, int32_t v) {
            const int q0 = v >> 8, qm = v & 255;
            if (q0 == t.quota0 && qm == t.quota_max) return false;
            t.quota0 = q0;
            t.quota_max = qm;
            return true;
        });
        knob(chunks, 3, [&](nrt_wavefront_tuning& t, int64_t v) {
            if (v == t.chunk || (v > n && t.chunk >= n)) return false;
            t.chunk = v;
            return true;
        });
    }
    if (status == NRT_OK) status = nrt_scene_set_tuning(scene, &best);
    scene->counters_on = was_on;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (prev != scene->device) cudaSetDevice(prev);
    if (status != NRT_OK) return status;
    *out = best;
    if (best_ms) *best_ms = best_t;
    return NRT_OK;
}

int nrt_enable_kernel_timing(nrt_scene* scene, int enable) {
    if (!scene) return fail(NRT_ERR_INVALID, "null scene");
    scene->timing_on = enable != 0;
    return NRT_OK;
}

int nrt_enable_counters(nrt_scene* scene, int enable) {
    if (!scene) return fail(NRT_ERR_INVALID, "null scene");
    scene->counters_on = enable ? 1 : 0;
    return NRT_OK;
}

int nrt_get_counters(nrt_scene* scene, nrt_counters* out, void* stream) {
    if (!scene || !out) return fail(NRT_ERR_INVALID, "null argument");
    unsigned long long h[dev::kCounterWords];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NRT_CUDA(cudaMemcpyAsync(h, scene->counters, sizeof(h), cudaMemcpyDeviceToHost, st), "counter read");
    NRT_CUDA(cudaStreamSynchronize(st), "counter sync");
    out->rays = h[dev::kRays];
    out->box_tests = h[dev::kBoxTests];
    out->patch_candidates = h[dev::kCandidates];
    out->patch_culled = h[dev::kCulled];
    out->newton_solves = h[dev::kSolves];
    out->newton_evals = h[dev::kEvals];
    out->fp64_solves = h[dev::kFp64Solves];
    out->fp64_final_steps = h[dev::kFp64Final];
    out->hits = h[dev::kHits];
    out->errors = h[dev::kErrors];
    out->learned_solves = h[dev::kLearned];
    out->learned_fallbacks = h[dev::kFallbacks];
    out->flat_skips = h[dev::kFlatSkips];
    if (scene->last_graph) {  // rounds counted on the device; kernels per pass and per round are fixed
        const uint64_t per_pass = 4 + (uint64_t)scene->plan.n_classes, per_round = 4 + (uint64_t)scene->plan.n_classes;
        out->rounds = h[dev::kRoundsDone];
        out->kernel_launches = (uint64_t)scene->wf_graph_passes * per_pass + out->rounds * per_round;
    } else {
        out->kernel_launches = (uint64_t)scene->last_launches;
        out->rounds = (uint64_t)scene->last_rounds;
    }
    out->newton_kernel_ms = scene->newton_ms;
    out->newton_kernel_launches = (uint64_t)scene->newton_launches;
    for (int k = 0; k < 64; ++k) {
        out->evals_by_degree[k] = h[dev::kEvalsByDegree + k];
        out->hull_tests_by_degree[k] = h[dev::kHullByDegree + k];
    }
    if (out->errors) return fail(NRT_ERR_DEVICE, "kernel reported %llu errors (traversal stack or degree)",
                                 (unsigned long long)out->errors);
    return NRT_OK;
}

size_t nrt_bounce_scratch_bytes(int64_t n) { return n > 0 ? (size_t)((n + 255) / 256 + 1) * sizeof(int32_t) : 0; }

int nrt_generate_bounce_rays(const nrt_rays* rays, const nrt_hits* hits, int64_t n, uint32_t seed, float offset,
                             const nrt_rays_out* out, int32_t* src_index, int64_t* n_out, void* user_scratch,
                             void* stream) {
    if (!rays || !hits || !out || !src_index || !n_out) return fail(NRT_ERR_INVALID, "null argument");
    if (!hits->patch || !hits->geom) return fail(NRT_ERR_INVALID, "bounce rays need hits->patch and hits->geom");
    if (!out->ox || !out->oy || !out->oz || !out->dx || !out->dy || !out->dz || !rays->dx || !rays->dy || !rays->dz)
        return fail(NRT_ERR_INVALID, "null ray array");
    if (n < 0 || n > (1LL << 31) - 256) return fail(NRT_ERR_INVALID, "ray count %lld outside 0..2^31-256", (long long)n);
    *n_out = 0;
    if (n == 0) return NRT_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long nb = (n + 255) / 256;
    int32_t* scratch = static_cast<int32_t*>(user_scratch);
    if (!scratch) NRT_CUDA(cudaMalloc(reinterpret_cast<void**>(&scratch), (nb + 1) * sizeof(int32_t)), "cudaMalloc");
    const nrt::dev::Rays r{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz};
    cudaError_t e = nrt::dev::launch_bounce_rays(r, hits->patch, hits->geom, n, seed, offset, out->ox, out->oy, out->oz,
                                                 out->dx, out->dy, out->dz, src_index, scratch, st);
    int32_t total = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, scratch + nb, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (!user_scratch) {
        const cudaError_t ef = cudaFree(scratch);
        if (e == cudaSuccess) e = ef;
    }
    if (e != cudaSuccess) return cuda_fail(e, "bounce rays");
    *n_out = total;
    return NRT_OK;
}

int nrt_generate_camera_rays(const nrt_camera* cam, const nrt_rays_out* out, void* stream) {
    if (!cam || !out || !out->ox || !out->oy || !out->oz || !out->dx || !out->dy || !out->dz)
        return fail(NRT_ERR_INVALID, "null argument");
    if (cam->width <= 0 || cam->height <= 0 || cam->spp <= 0) return fail(NRT_ERR_INVALID, "empty image");
    if (!(cam->fov_deg > 0.f && cam->fov_deg < 180.f)) return fail(NRT_ERR_INVALID, "fov outside (0,180)");
    // camera basis in double, unfused, as Transform::lookAt (src/math/transform.h:46-60)
    auto norm = [](double v[3]) {
        const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double il = 1.0 / l;
        v[0] = v[0] * il; v[1] = v[1] * il; v[2] = v[2] * il;
    };
    auto cross = [](const double a[3], const double b[3], double o[3]) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    dev::CameraParams cp{};
    double E[3] = {cam->eye[0], cam->eye[1], cam->eye[2]}, L[3] = {cam->look[0], cam->look[1], cam->look[2]},
           U[3] = {cam->up[0], cam->up[1], cam->up[2]};
    double f[3] = {L[0] - E[0], L[1] - E[1], L[2] - E[2]};
    norm(f);
    double rt[3];
    cross(U, f, rt);
    norm(rt);
    double up[3];
    cross(f, rt, up);
    for (int a = 0; a < 3; ++a) { cp.eye[a] = E[a]; cp.fwd[a] = f[a]; cp.right[a] = rt[a]; cp.up[a] = up[a]; }
    const double aspect = (double)cam->width / (double)cam->height;
    if (aspect > 1.0) { cp.x0 = -aspect; cp.x1 = aspect; cp.y0 = -1; cp.y1 = 1; }
    else { cp.x0 = -1; cp.x1 = 1; cp.y0 = -1.0 / aspect; cp.y1 = 1.0 / aspect; }
    cp.tan_half = std::tan((double)cam->fov_deg * (3.14159265358979323846 / 180.0) / 2.0);
    cp.width = cam->width;
    cp.height = cam->height;
    cp.spp = cam->spp;
    cp.seed = cam->seed;
    cudaError_t e = dev::launch_camera_rays(cp, out->ox, out->oy, out->oz, out->dx, out->dy, out->dz,
                                            static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "camera ray launch");
    return NRT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Views for nrt_intersect_noalloc (noalloc.cu): validates the arguments as
// nrt_intersect does and hands out the scene's device views; allocates nothing.
namespace nrt {

int noalloc_views(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                  const nrt_hits* hits, NoallocViews* v) {
    if (!scene || !rays || !opts || !hits || !v) return fail(NRT_ERR_INVALID, "null argument");
    if (n < 0) return fail(NRT_ERR_INVALID, "negative ray count");
    if (n > 0 && (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz))
        return fail(NRT_ERR_INVALID, "null ray array");
    if (n > 0 && (!hits->patch || !hits->t || !hits->u || !hits->v)) return fail(NRT_ERR_INVALID, "null hit array");
    const nrt_intersect_opts& o = *opts;
    if (o.max_iter < 1 || o.max_iter > 256) return fail(NRT_ERR_INVALID, "max_iter %d outside 1..256", o.max_iter);
    if (!(o.eps > 0.f)) return fail(NRT_ERR_INVALID, "eps must be positive");
    if (o.init_mode != NRT_INIT_MIDPOINT && o.init_mode != NRT_INIT_BILINEAR)
        return fail(NRT_ERR_UNSUPPORTED, "init mode %d not available without allocation", o.init_mode);
    if (o.flat_threshold > 0.f) return fail(NRT_ERR_UNSUPPORTED, "flat-skip runs on the per-pixel schedule only");
    v->scene = scene->view;
    v->plan = scene->plan;
    v->counters = scene->counters;
    v->device = scene->device;
    to_dev_opts(o, v->opts, scene->counters_on);
    return NRT_OK;
}

void noalloc_record(nrt_scene* scene, long long launches, long long rounds) {
    scene->last_launches = launches;
    scene->last_rounds = rounds;
    scene->last_graph = false;
}

}  // namespace nrt

extern "C" {

int nrt_scene_set_mlp(nrt_scene* scene, const nrt_mlp* mlp) {
    if (!scene || !mlp) return fail(NRT_ERR_INVALID, "null argument");
    if (mlp_device(mlp) != scene->device) return fail(NRT_ERR_INVALID, "network and scene are on different devices");
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != scene->device) cudaSetDevice(scene->device);
    cudaError_t e = cudaSuccess;
    if (!scene->mlp_blob) e = cudaMalloc(&scene->mlp_blob, mlp_blob_bytes());
    if (e == cudaSuccess) e = cudaMemcpy(scene->mlp_blob, mlp_device_blob(mlp), mlp_blob_bytes(), cudaMemcpyDeviceToDevice);
    if (prev != scene->device) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "scene network copy");
    return NRT_OK;
}

int nrt_collect_training_data(nrt_scene* scene, const nrt_rays* rays, int64_t n, const nrt_intersect_opts* opts,
                              float* features, float* targets, int64_t capacity, int64_t* count, void* stream) {
    if (!scene || !rays || !opts || !features || !targets || !count || n < 0 || capacity < 0)
        return fail(NRT_ERR_INVALID, "bad argument");
    if (opts->init_mode != NRT_INIT_MIDPOINT) return fail(NRT_ERR_INVALID, "training pairs come from the midpoint guess");
    *count = 0;
    if (n == 0) return NRT_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != scene->device) cudaSetDevice(scene->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // scratch outputs and the pair counter (this is a training-time call: it allocates)
    void* tmp = nullptr;
    const size_t out_bytes = (size_t)n * 16 + 256;
    cudaError_t e = cudaMalloc(&tmp, out_bytes);
    if (e != cudaSuccess) {
        if (prev != scene->device) cudaSetDevice(prev);
        return cuda_fail(e, "cudaMalloc(collection scratch)");
    }
    char* base = static_cast<char*>(tmp);
    unsigned long long* dcount = reinterpret_cast<unsigned long long*>(base);
    dev::Hits h{reinterpret_cast<int32_t*>(base + 256), reinterpret_cast<float*>(base + 256 + 4 * (size_t)n),
                reinterpret_cast<float*>(base + 256 + 8 * (size_t)n), reinterpret_cast<float*>(base + 256 + 12 * (size_t)n),
                nullptr, nullptr, nullptr};
    e = cudaMemsetAsync(dcount, 0, sizeof(unsigned long long), st);
    dev::Opts d;
    to_dev_opts(*opts, d, 0);
    d.col_feat = features;
    d.col_targ = targets;
    d.col_count = dcount;
    d.col_cap = capacity;
    const dev::Rays r{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz};
    const long long chunk = std::min<long long>(n, scene->wf_chunk);
    if (e == cudaSuccess && scene->wf_rays < chunk) {
        if (scene->wf_ws) cudaFree(scene->wf_ws);
        scene->wf_ws = nullptr;
        scene->wf_rays = 0;
        e = cudaMalloc(&scene->wf_ws, dev::wavefront_scratch_bytes(chunk, scene->plan.n_slots));
        if (e == cudaSuccess) scene->wf_rays = chunk;
        else scene->wf_ws = nullptr;
    }
    if (e == cudaSuccess && !scene->host_count) e = cudaMallocHost(&scene->host_count, sizeof(int32_t));
    long long launches = 0, rounds = 0;
    if (e == cudaSuccess) {
        const dev::WfBuffers wb = dev::wavefront_carve(scene->wf_ws, scene->wf_rays, scene->plan.n_slots);
        for (long long at = 0; at < n && e == cudaSuccess; at += chunk) {
            const long long m = std::min(chunk, (long long)n - at);
            dev::Rays rc{r.ox + at, r.oy + at, r.oz + at, r.dx + at, r.dy + at, r.dz + at};
            dev::Hits hc{h.patch + at, h.t + at, h.u + at, h.v + at, nullptr, nullptr, nullptr};
            dev::Opts dc = d;
            dc.seed_offset = d.seed_offset + (uint32_t)at;
            e = dev::launch_wavefront(scene->view, scene->plan, rc, m, dc, hc, wb, scene->host_count, scene->counters, st,
                                      &launches, &rounds);
        }
    }
    unsigned long long got = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&got, dcount, sizeof(got), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    if (prev != scene->device) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "training-pair collection");
    *count = (int64_t)got;
    return NRT_OK;
}

}  // extern "C"
