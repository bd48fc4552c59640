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
#include "scene_build.h"
#include "slot_pack.cuh"
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

int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? NRT_ERR_NOMEM : NRT_ERR_CUDA, "%s: %s (%s)", what,
                cudaGetErrorName(e), cudaGetErrorString(e));
}

#define NRT_CUDA(call, what)                               \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

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
    int last_guess_round = 0;    // ... and its guess kernels (learned mode): per round, and per pass
    int last_guess_pass = 0;
    dev::WfTuning tuning{};
    bool use_graph = true;       // false: host-driven rounds
    bool timing_on = false;      // events around the per-class Newton launches (host-driven rounds)
    cudaEvent_t tev[2] = {nullptr, nullptr};
    double newton_ms = 0.0;
    long long newton_launches = 0;
};

namespace nrt {

// The scene's device arena: one allocation, every array 256-byte aligned, in
// this order.  Both builders lay it out the same way.
ArenaLayout arena_layout(size_t n_wide, int N, size_t n_floats) {
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    ArenaLayout L{};
    size_t at = 0;
    auto take = [&](size_t bytes) { const size_t r = at; at += align(bytes); return r; };
    L.nodes = take(n_wide * sizeof(Node4));
    L.hdr = take(N * sizeof(int4));
    L.centre = take(N * sizeof(double4));
    L.cp = take(n_floats * sizeof(float));
    L.corners = take(4 * (size_t)N * sizeof(float4));
    L.delta = take(N * sizeof(float));
    L.counters = take(dev::kCounterWords * sizeof(unsigned long long));
    L.rank = take(N * sizeof(int32_t));
    L.frames = take(N * sizeof(dev::PatchFrame));
    L.obb = take(4 * (size_t)N * sizeof(float4));
    L.leafbox = take(2 * (size_t)N * sizeof(float4));
    L.total = at;
    return L;
}

// The wavefront's degree classes from the per-(p, q) patch counts: one class
// per degree pair present, in increasing p | q << 4, ranks assigned in that
// order (slots keep their order inside a class).
void plan_classes(const int* degree_hist, int N, dev::WfPlan& plan) {
    plan = dev::WfPlan{};
    plan.n_slots = N;
    int rank = 0;
    for (int key = 0; key < 256; ++key) {
        const int p = key & 15, q = key >> 4;
        if (p < 1 || q < 1 || p > NRT_MAX_DEGREE || q > NRT_MAX_DEGREE) continue;
        const int cnt = degree_hist[p * 8 + q];
        if (cnt == 0) continue;
        plan.class_pq[plan.n_classes] = key;
        plan.class_rank[plan.n_classes] = rank;
        plan.class_grid[plan.n_classes] = 148 * 4;
        ++plan.n_classes;
        rank += cnt;
    }
    plan.class_rank[plan.n_classes] = N;
}

// A scene object with its arena allocated (zero-filled) on the build's device.
int new_scene(const nrt_build_opts& o, const ArenaLayout& L, nrt_scene** out, char** arena) {
    nrt_scene* sc = new (std::nothrow) nrt_scene();
    if (!sc) return fail(NRT_ERR_NOMEM, "host allocation failed");
    sc->device = o.device;
    sc->wf_chunk = o.wavefront_chunk > 0 ? o.wavefront_chunk : (1LL << 23);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(o.device);
    if (e != cudaSuccess) { delete sc; return cuda_fail(e, "cudaSetDevice"); }
    e = cudaMalloc(&sc->arena, L.total);
    if (e == cudaSuccess) e = cudaMemset(sc->arena, 0, L.total);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        if (sc->arena) cudaFree(sc->arena);
        delete sc;
        return cuda_fail(e, "cudaMalloc(scene)");
    }
    sc->arena_bytes = L.total;
    *out = sc;
    *arena = static_cast<char*>(sc->arena);
    return NRT_OK;
}

// Points the scene's views at its filled arena and records the rest.
void finish_scene(nrt_scene* sc, const ArenaLayout& L, int N, dev::WfPlan plan, nrt_scene_info info, PatchSet&& ps,
                  int n_surfaces) {
    char* base = static_cast<char*>(sc->arena);
    sc->view.nodes = reinterpret_cast<const dev::Node4*>(base + L.nodes);
    sc->view.hdr = reinterpret_cast<const int4*>(base + L.hdr);
    sc->view.centre = reinterpret_cast<const double4*>(base + L.centre);
    sc->view.cp = reinterpret_cast<const float*>(base + L.cp);
    sc->view.corners = reinterpret_cast<const float4*>(base + L.corners);
    sc->view.delta = reinterpret_cast<const float*>(base + L.delta);
    sc->counters = reinterpret_cast<unsigned long long*>(base + L.counters);
    plan.rank_of = reinterpret_cast<const int32_t*>(base + L.rank);
    sc->view.frames = reinterpret_cast<const dev::PatchFrame*>(base + L.frames);
    sc->view.obb = reinterpret_cast<const float4*>(base + L.obb);
    sc->view.leafbox = reinterpret_cast<const float4*>(base + L.leafbox);
    sc->view.n_slots = N;
    sc->view.n_nodes = info.n_nodes;
    sc->plan = plan;
    info.n_patches = N;
    info.device_bytes = L.total;
    sc->info = info;
    sc->ps = std::move(ps);
    sc->n_surfaces = n_surfaces;
}

int build_scene(PatchSet&& ps, int n_surfaces, const nrt_build_opts* opts, nrt_scene** out, const BinaryBVH* given,
                const float* delta_by_patch) {
    if (!out) return fail(NRT_ERR_INVALID, "out is null");
    *out = nullptr;
    const int N = ps.count();
    if (N <= 0) return fail(NRT_ERR_INVALID, "scene has no patches");
    nrt_build_opts o{NRT_BVH_BINNED_SAH, 1, 0, 0};
    if (opts) o = *opts;
    if (o.wavefront_chunk < 0) return fail(NRT_ERR_INVALID, "negative wavefront_chunk");
    if (o.max_leaf < 1 || o.max_leaf > 8) return fail(NRT_ERR_INVALID, "max_leaf must be in 1..8");
    if (o.builder != NRT_BVH_BINNED_SAH && o.builder != NRT_BVH_EXACT_SAH)
        return fail(NRT_ERR_INVALID, "unknown BVH builder %d", o.builder);
    if (N >= (1 << 27)) return fail(NRT_ERR_INVALID, "too many patches (%d)", N);
    for (int k = 0; k < N; ++k) {
        const int p = ps.deg[2 * k], q = ps.deg[2 * k + 1];
        if (p < 1 || q < 1 || p > NRT_MAX_DEGREE || q > NRT_MAX_DEGREE)
            return fail(NRT_ERR_INVALID, "patch %d has degree (%d,%d) outside 1..%d", k, p, q, NRT_MAX_DEGREE);
    }
    // BVH over patch boxes (or the caller's tree)
    std::vector<Box3> boxes;
    patch_boxes(ps, boxes);
    BinaryBVH bin;
    if (given) bin = *given;
    else if (o.builder == NRT_BVH_EXACT_SAH) build_exact_sah(boxes, bin);
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
    size_t total_floats = 0;
    for (int s = 0; s < N; ++s) {
        const int k = bin.order[s];
        total_floats += 4 * (size_t)dev::padded_points(ps.deg[2 * k], ps.deg[2 * k + 1]);
    }
    if (total_floats >= ((size_t)1 << 31))
        return fail(NRT_ERR_INVALID, "scene too large (%zu block floats)", total_floats);
    blocks.assign(total_floats, 0.f);
    size_t off = 0;
    nrt_scene_info info{};
    for (int s = 0; s < N; ++s) {
        const int k = bin.order[s];
        const int p = ps.deg[2 * k], q = ps.deg[2 * k + 1];
        pack_slot(&ps.cp[4 * (size_t)ps.off[k]], p, q, boxes[k], k, ps.surf[k], (long long)off, &blocks[off], hdr[s],
                  centre[s], &corners[4 * (size_t)s], delta[s], frames[s], &obbs[4 * (size_t)s]);
        if (delta_by_patch) delta[s] = delta_by_patch[k];  // the caller's flatness values
        info.degree_hist[p * 8 + q] += 1;
        off += 4 * (size_t)dev::padded_points(p, q);
    }

    // wavefront plan: patches ranked by (p, q, slot)
    dev::WfPlan plan{};
    plan_classes(info.degree_hist, N, plan);
    std::vector<int32_t> rank_of(N);
    {
        int next[256] = {0};
        for (int c = 0; c < plan.n_classes; ++c) next[plan.class_pq[c]] = plan.class_rank[c];
        for (int s2 = 0; s2 < N; ++s2) rank_of[s2] = next[hdr[s2].y & 0xff]++;
    }
    const ArenaLayout L = arena_layout(wide.size(), N, blocks.size());
    nrt_scene* sc = nullptr;
    char* base = nullptr;
    if (int st = new_scene(o, L, &sc, &base)) return st;
    cudaError_t e = cudaSuccess;
    auto put = [&](size_t at, const void* src, size_t bytes) {
        if (bytes && e == cudaSuccess) e = cudaMemcpy(base + at, src, bytes, cudaMemcpyHostToDevice);
    };
    put(L.nodes, wide.data(), wide.size() * sizeof(Node4));
    put(L.hdr, hdr.data(), N * sizeof(int4));
    put(L.centre, centre.data(), N * sizeof(double4));
    put(L.cp, blocks.data(), blocks.size() * sizeof(float));
    put(L.corners, corners.data(), corners.size() * sizeof(float4));
    put(L.delta, delta.data(), N * sizeof(float));
    put(L.rank, rank_of.data(), N * sizeof(int32_t));
    put(L.frames, frames.data(), N * sizeof(dev::PatchFrame));
    put(L.obb, obbs.data(), obbs.size() * sizeof(float4));
    put(L.leafbox, leafbox.data(), leafbox.size() * sizeof(float4));
    if (e != cudaSuccess) {
        nrt_scene_destroy(sc);
        return cuda_fail(e, "scene upload");
    }
    info.n_surfaces = n_surfaces;
    info.n_nodes = (int)wide.size();
    info.bvh_depth = depth;
    finish_scene(sc, L, N, plan, info, std::move(ps), n_surfaces);
    *out = sc;
    return NRT_OK;
}

}  // namespace nrt

namespace {

void to_dev_opts(const nrt_intersect_opts& o, dev::Opts& d, int counters) {
    d.nw.max_iter = o.max_iter;
    d.nw.eps = o.eps;
    d.nw.det_eps = o.det_eps;
    d.nw.cond_fp64 = o.cond_fp64;
    d.nw.fp64_final = o.fp64_final;
    d.nw.fp64_band = o.fp64_final ? 1 : 0;  // the FP64 final-step mode decides convergence near eps in FP64
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
    if (opts && opts->builder == NRT_BVH_BINNED_SAH_DEVICE) return build_scene_device_surfaces(surfaces, n_surfaces, *opts, out);
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
    if (opts && opts->builder == NRT_BVH_BINNED_SAH_DEVICE)
        return build_scene_device_patches(cp, cp_offset, degrees, n_patches, *opts, out);
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
    const PatchSet& ps = scene->ps;
    if (ps.spans.empty()) {
        const int N = (int)ps.surf.size();
        if (surface_of) std::memcpy(surface_of, ps.surf.data(), sizeof(int32_t) * N);
        if (ranges) std::memcpy(ranges, ps.ranges.data(), sizeof(float) * 4 * N);
        return NRT_OK;
    }
    for (size_t si = 0; si < ps.spans.size(); ++si) {  // expanded from the per-surface breakpoints
        const PatchSet::Spans& sp = ps.spans[si];
        const float *bu = &ps.breaks[sp.bu], *bv = &ps.breaks[sp.bv];
        for (int i = 0; i < sp.nbU; ++i)
            for (int j = 0; j < sp.nbV; ++j) {
                const size_t k = (size_t)sp.patch0 + (size_t)i * sp.nbV + j;
                if (surface_of) surface_of[k] = (int32_t)si;
                if (ranges) {
                    ranges[4 * k] = bu[i]; ranges[4 * k + 1] = bu[i + 1];
                    ranges[4 * k + 2] = bv[j]; ranges[4 * k + 3] = bv[j + 1];
                }
            }
    }
    return NRT_OK;
}

int nrt_scene_copy_arena(const nrt_scene* scene, void* host_dst, size_t bytes) {
    if (!scene || !host_dst) return fail(NRT_ERR_INVALID, "null argument");
    if (bytes < scene->arena_bytes) return fail(NRT_ERR_INVALID, "buffer of %zu bytes, arena has %zu", bytes,
                                                scene->arena_bytes);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(scene->device);
    const cudaError_t e = cudaMemcpy(host_dst, scene->arena, scene->arena_bytes, cudaMemcpyDeviceToHost);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "nrt_scene_copy_arena");
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
                                          scene->tuning.quota0, scene->tuning.quota_max,
                                          scene->tuning.stage_nodes);
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
        scene->last_guess_round = o.init_mode == NRT_INIT_LEARNED ? 1 : 0;
        scene->last_guess_pass = (o.init_mode == NRT_INIT_LEARNED && hits->iters) ? 1 : 0;
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
    out->stage_nodes = scene->tuning.stage_nodes;
    return NRT_OK;
}

int nrt_scene_set_tuning(nrt_scene* scene, const nrt_wavefront_tuning* in) {
    if (!scene || !in) return fail(NRT_ERR_INVALID, "null argument");
    if (in->step_blocks > (1LL << 24) || in->scatter_blocks > (1LL << 24) || in->class_blocks > (1 << 24))
        return fail(NRT_ERR_INVALID, "block counts above 2^24");
    if (in->graph > 2) return fail(NRT_ERR_INVALID, "graph must be 1 (graph) or 2 (host-driven)");
    if (in->chunk > (1LL << 30)) return fail(NRT_ERR_INVALID, "chunk above 2^30 rays");
    if (in->quota0 > 8 || in->quota_max > 8) return fail(NRT_ERR_INVALID, "round quotas above 8");
    if (in->stage_nodes > dev::kMaxStagedNodes)
        return fail(NRT_ERR_INVALID, "stage_nodes %d above %d", in->stage_nodes, dev::kMaxStagedNodes);
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
    if (in->stage_nodes > 0) scene->tuning.stage_nodes = in->stage_nodes;
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
    const int32_t stages[] = {1, 21, 85, 341};  // whole top levels of the 4-wide tree: none (the root), 3, 4, 5
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
        knob(stages, 4, [&](nrt_wavefront_tuning& t, int32_t v) {
            if (v == t.stage_nodes) return false;
            t.stage_nodes = v;
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
    out->learned_converged = h[dev::kLearnedConverged];
    out->learned_fallback_converged = h[dev::kFallbackConverged];
    out->flat_skips = h[dev::kFlatSkips];
    if (scene->last_graph) {  // rounds counted on the device; kernels per pass and per round are fixed
        const uint64_t nc = (uint64_t)scene->plan.n_classes;
        const uint64_t per_pass = 4 + nc * (1 + scene->last_guess_pass), per_round = 4 + nc * (1 + scene->last_guess_round);
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
    v->scene = scene->view;
    v->plan = scene->plan;
    v->counters = scene->counters;
    v->device = scene->device;
    v->quota0 = scene->tuning.quota0;  // the round quotas and staged tree top nrt_intersect runs with
    v->quota_max = scene->tuning.quota_max;
    v->stage_nodes = scene->tuning.stage_nodes;
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
