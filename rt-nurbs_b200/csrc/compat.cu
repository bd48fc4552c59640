// compat.cu -- the reference's own C++ entry points over this engine.
//
// calculateIntersectWrapper and calculateRaysWrapper are exported with the
// reference's exact signatures (include/nrt_compat.h restates its types), so a
// program written against the reference (src/core/benchmark.cpp,
// src/core/main.cpp) links against libnrt.so unchanged.  The intersection
// reads the caller's array-of-structures patches and binary tree
// (bezierPatch, BVHNode; device, managed or host memory), packs them once into
// an engine scene that keeps the caller's tree, runs nrt_intersect with the
// reference's settings and writes the per-pixel surfaceInteraction records and
// idx_interact as the reference's kernel does (src/gpu/intersect.cu:20-194).
#include <cuda.h>  // CUdeviceptr / CUresult of the driver call looked up below (libcuda is not linked)
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/nrt_compat.h"
#include "scene_build.h"

static_assert(sizeof(bezierPatch) == 40, "bezierPatch layout (src/math/bezier_patch.h:10-16)");
static_assert(sizeof(BVHNode) == 32, "BVHNode layout (src/core/bvh.h:13-17)");
static_assert(sizeof(surfaceInteraction) == 72, "surfaceInteraction layout (src/gpu/interact.h:6-21)");
static_assert(sizeof(SoAQueue::ray_queue) == 56, "ray_queue layout (src/gpu/soa.h:6-14)");

namespace {

// ---------------------------------------------------------------------------
// Reading the caller's memory, wherever it lives.

using GetAddressRange = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);

// Bytes from p to the end of the CUDA allocation holding it (device or
// managed memory), or 0 when p is not in one (host memory: read directly).
size_t bytes_to_end(const void* p) {
    static GetAddressRange range = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            range = reinterpret_cast<GetAddressRange>(f);
    });
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return 0;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (!range || range(&base, &size, reinterpret_cast<CUdeviceptr>(p)) != CUDA_SUCCESS) return 0;
    return (size_t)(base + size - reinterpret_cast<CUdeviceptr>(p));
}

bool fetch(void* dst, const void* src, size_t bytes) {
    if (!bytes) return true;
    return cudaMemcpy(dst, src, bytes, cudaMemcpyDefault) == cudaSuccess;
}

uint64_t mix(uint64_t h, const void* data, size_t bytes) {  // FNV-1a over 8-byte words
    const unsigned char* c = static_cast<const unsigned char*>(data);
    size_t i = 0;
    for (; i + 8 <= bytes; i += 8) {
        uint64_t w;
        std::memcpy(&w, c + i, 8);
        h = (h ^ w) * 0x100000001b3ull;
    }
    for (; i < bytes; ++i) h = (h ^ c[i]) * 0x100000001b3ull;
    return h;
}

// The caller's scene, read back: tree, patches, points, flatness.
struct HostScene {
    std::vector<BVHNode> nodes;  // the nodes reachable from the root (indices kept)
    std::vector<bezierPatch> patches;
    nrt::PatchSet ps;
    std::vector<float> delta;
    bool leaves_fit = true;      // every leaf holds at most 8 patches
    uint64_t hash = 0;
};

int read_scene(const BVHNode* nodes, const bezierPatch* patches, const float* delta, bool want_delta, HostScene& hs) {
    // the tree: all nodes of its allocation in one copy, or node by node from host memory
    const size_t node_room = bytes_to_end(nodes) / sizeof(BVHNode);
    if (node_room) {
        hs.nodes.resize(std::min<size_t>(node_room, (size_t)1 << 26));
        if (!fetch(hs.nodes.data(), nodes, hs.nodes.size() * sizeof(BVHNode)))
            return nrt::fail(NRT_ERR_CUDA, "reading the BVH nodes");
    }
    auto node = [&](uint32_t i, BVHNode& out) {
        if (node_room) {
            if (i >= hs.nodes.size()) return false;
            out = hs.nodes[i];
            return true;
        }
        out = nodes[i];  // host memory
        return true;
    };
    uint32_t n_patches = 0, n_used = 1;
    std::vector<uint32_t> todo{0};
    size_t visited = 0;
    while (!todo.empty()) {
        const uint32_t i = todo.back();
        todo.pop_back();
        BVHNode nd;
        if (!node(i, nd) || ++visited > ((size_t)1 << 27))
            return nrt::fail(NRT_ERR_INVALID, "BVH node %u is outside the node array", i);
        n_used = std::max(n_used, i + 1);
        if (nd.prim_count > 0) {
            n_patches = std::max(n_patches, nd.left_first + nd.prim_count);
            if (nd.prim_count > 8) hs.leaves_fit = false;
        } else {
            if (nd.left_first <= i) return nrt::fail(NRT_ERR_INVALID, "BVH node %u points back to %u", i, nd.left_first);
            todo.push_back(nd.left_first);
            todo.push_back(nd.left_first + 1);
        }
    }
    if (!node_room) hs.nodes.assign(nodes, nodes + n_used);
    hs.nodes.resize(n_used);
    if (n_patches == 0) return nrt::fail(NRT_ERR_INVALID, "the BVH has no patches");
    // the patch records
    const size_t patch_room = bytes_to_end(patches);
    if (patch_room && patch_room < n_patches * sizeof(bezierPatch))
        return nrt::fail(NRT_ERR_INVALID, "the BVH references %u patches; the patch array holds %zu", n_patches,
                         patch_room / sizeof(bezierPatch));
    hs.patches.resize(n_patches);
    if (!fetch(hs.patches.data(), patches, n_patches * sizeof(bezierPatch)))
        return nrt::fail(NRT_ERR_CUDA, "reading the patch records");
    // their control points: one copy of the span they share, else one per patch
    const char* lo = nullptr;
    const char* hi = nullptr;
    size_t points = 0;
    for (uint32_t k = 0; k < n_patches; ++k) {
        const bezierPatch& b = hs.patches[k];
        if (b.p < 1 || b.q < 1 || b.p > NRT_MAX_DEGREE || b.q > NRT_MAX_DEGREE || !b.control_point)
            return nrt::fail(NRT_ERR_INVALID, "patch %u has degree (%d,%d) or no control points", k, b.p, b.q);
        const size_t np = (size_t)(b.p + 1) * (b.q + 1);
        const char* a = reinterpret_cast<const char*>(b.control_point);
        lo = (!lo || a < lo) ? a : lo;
        hi = (!hi || a + 16 * np > hi) ? a + 16 * np : hi;
        points += np;
    }
    nrt::PatchSet& ps = hs.ps;
    ps = nrt::PatchSet{};
    ps.off.resize(n_patches);
    ps.deg.resize(2 * (size_t)n_patches);
    ps.ranges.resize(4 * (size_t)n_patches);
    ps.surf.assign(n_patches, 0);
    const size_t span = (size_t)(hi - lo);
    bool shared = span <= 4 * 16 * points + (1u << 20);
    for (uint32_t k = 0; k < n_patches && shared; ++k)
        shared = (reinterpret_cast<const char*>(hs.patches[k].control_point) - lo) % 16 == 0;
    const size_t cp_room = bytes_to_end(lo);
    if (shared && (!cp_room || cp_room < span)) shared = false;  // host memory: patch by patch
    if (shared) {
        ps.cp.resize(span / 4);
        if (!fetch(ps.cp.data(), lo, span)) return nrt::fail(NRT_ERR_CUDA, "reading the control points");
    } else {
        ps.cp.resize(4 * points);
    }
    size_t at = 0;
    for (uint32_t k = 0; k < n_patches; ++k) {
        const bezierPatch& b = hs.patches[k];
        const size_t np = (size_t)(b.p + 1) * (b.q + 1);
        if (shared) {
            ps.off[k] = (int32_t)((reinterpret_cast<const char*>(b.control_point) - lo) / 16);
        } else {
            ps.off[k] = (int32_t)at;
            if (!fetch(&ps.cp[4 * at], b.control_point, 16 * np))
                return nrt::fail(NRT_ERR_CUDA, "reading the control points of patch %u", k);
            at += np;
        }
        ps.deg[2 * k] = b.p;
        ps.deg[2 * k + 1] = b.q;
        ps.ranges[4 * k + 0] = b.u0;
        ps.ranges[4 * k + 1] = b.u1;
        ps.ranges[4 * k + 2] = b.v0;
        ps.ranges[4 * k + 3] = b.v1;
    }
    hs.delta.clear();
    if (want_delta) {
        hs.delta.resize(n_patches);
        if (!delta || !fetch(hs.delta.data(), delta, n_patches * sizeof(float)))
            return nrt::fail(NRT_ERR_INVALID, "flat-skip needs the delta array (%u floats)", n_patches);
    }
    uint64_t h = 0xcbf29ce484222325ull;
    h = mix(h, hs.nodes.data(), hs.nodes.size() * sizeof(BVHNode));
    h = mix(h, hs.patches.data(), hs.patches.size() * sizeof(bezierPatch));
    h = mix(h, ps.cp.data(), ps.cp.size() * sizeof(float));
    h = mix(h, hs.delta.data(), hs.delta.size() * sizeof(float));
    hs.hash = h;
    return NRT_OK;
}

// The engine scene of the caller's patches, keeping the caller's tree (so the
// leaf boxes that flat-skip measures against are the reference's own).
int make_scene(HostScene& hs, int device, nrt_scene** out) {
    nrt::BinaryBVH bin;
    const size_t M = hs.nodes.size();
    bin.box.resize(M);
    bin.left_first.resize(M);
    bin.prim_count.resize(M);
    for (size_t i = 0; i < M; ++i) {
        const MathExtra::bounds3f& b = hs.nodes[i].node_bound;
        bin.box[i] = nrt::Box3{{b.p_min_x, b.p_min_y, b.p_min_z}, {b.p_max_x, b.p_max_y, b.p_max_z}};
        bin.left_first[i] = hs.nodes[i].left_first;
        bin.prim_count[i] = hs.nodes[i].prim_count;
    }
    const int N = hs.ps.count();
    bin.order.resize(N);
    for (int k = 0; k < N; ++k) bin.order[k] = k;  // the caller's patches are in leaf order already
    bin.used = (int)M;
    nrt_build_opts o{NRT_BVH_BINNED_SAH, 1, device, 0};
    // a leaf of more than 8 patches does not fit the engine's 4-wide nodes: such a tree is rebuilt
    // (the closest hit does not depend on the tree; flat-skip's leaf boxes do)
    nrt::PatchSet ps = hs.ps;
    return nrt::build_scene(std::move(ps), 1, &o, out, hs.leaves_fit ? &bin : nullptr,
                            hs.delta.empty() ? nullptr : hs.delta.data());
}

// One cached scene (the last one used) and the hit buffers.
struct Cache {
    std::mutex mu;
    const void* nodes = nullptr;
    const void* patches = nullptr;
    int device = -1;
    uint64_t hash = 0;
    nrt_scene* scene = nullptr;
    void* hits = nullptr;
    long long hit_cap = 0;
} g_cache;

// ---------------------------------------------------------------------------
// Kernels.

// Hit records as the reference's kernel writes them (src/gpu/intersect.cu:117-190):
// a hit sets t_hit, uv, dpdu, dpdv and idx_interact = the pixel index; a miss
// writes nothing; every pixel whose idx_interact is then not -1 gets wo = -d.
__global__ void k_compat_write(long long n, const int32_t* patch, const float* t, const float* u, const float* v,
                               const float* geom, SoAQueue::ray_queue q, surfaceInteraction* out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    surfaceInteraction& s = out[i];
    if (patch[i] >= 0) {
        s.t_hit = t[i];
        s.uv.v[0] = u[i];
        s.uv.v[1] = v[i];
        const float* g = geom + 9 * i;
        s.dpdu.v[0] = g[3]; s.dpdu.v[1] = g[4]; s.dpdu.v[2] = g[5];
        s.dpdv.v[0] = g[6]; s.dpdv.v[1] = g[7]; s.dpdv.v[2] = g[8];
        q.idx_interact[i] = (int)i;
    }
    if (q.idx_interact[i] != -1) {
        s.wo.v[0] = -q.direction_x[i];
        s.wo.v[1] = -q.direction_y[i];
        s.wo.v[2] = -q.direction_z[i];
    }
}

__global__ void k_compat_count(unsigned long long* newton, unsigned long long* skip, unsigned long long nv,
                               unsigned long long sv) {
    if (newton) atomicAdd(newton, nv);
    if (skip) atomicAdd(skip, sv);
}

// (column-major 4x4) x (x, y, z, w), summed left to right in round-to-nearest,
// as MatrixOps::multiply (src/math/matrix_ops.h:120-127) on the host.
__device__ __forceinline__ float mat_row(const MathTypes::matrix4x4f& m, int r, float x, float y, float z, float w) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m.m[r], x), __fmul_rn(m.m[4 + r], y)), __fmul_rn(m.m[8 + r], z)),
                     __fmul_rn(m.m[12 + r], w));
}

// Pixel-centre rays (CameraOps::calculateRay, src/core/camera.h:142-174).
template <bool PERSPECTIVE>
__global__ void k_compat_rays(MathTypes::matrix4x4f world_from_camera, MathTypes::matrix4x4f camera_from_raster,
                              int W, int H, SoAQueue::ray_queue q) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const long long i = (long long)y * W + x;
    const float rx = __fadd_rn((float)x, 0.5f), ry = __fadd_rn((float)y, 0.5f);
    const MathTypes::matrix4x4f& c = camera_from_raster;
    const float cx = mat_row(c, 0, rx, ry, 0.f, 1.f), cy = mat_row(c, 1, rx, ry, 0.f, 1.f);
    const float cz = mat_row(c, 2, rx, ry, 0.f, 1.f);
    const MathTypes::matrix4x4f& w = world_from_camera;
    if (PERSPECTIVE) {
        // normalize: times 1/sqrt(x*x + y*y + z*z) (VectorOps::normalize, src/math/vector_ops.h:104-113)
        const float l2 = __fadd_rn(__fadd_rn(__fmul_rn(cx, cx), __fmul_rn(cy, cy)), __fmul_rn(cz, cz));
        const float il = __fdiv_rn(1.0f, __fsqrt_rn(l2));
        const float px = __fmul_rn(cx, il), py = __fmul_rn(cy, il), pz = __fmul_rn(cz, il);
        q.origin_x[i] = w.m[12];
        q.origin_y[i] = w.m[13];
        q.origin_z[i] = w.m[14];
        q.direction_x[i] = mat_row(w, 0, px, py, pz, 0.f);
        q.direction_y[i] = mat_row(w, 1, px, py, pz, 0.f);
        q.direction_z[i] = mat_row(w, 2, px, py, pz, 0.f);
    } else {
        const float cw = mat_row(c, 3, rx, ry, 0.f, 1.f);
        q.origin_x[i] = mat_row(w, 0, cx, cy, cz, cw);
        q.origin_y[i] = mat_row(w, 1, cx, cy, cz, cw);
        q.origin_z[i] = mat_row(w, 2, cx, cy, cz, cw);
        q.direction_x[i] = w.m[8];
        q.direction_y[i] = w.m[9];
        q.direction_z[i] = w.m[10];
    }
    q.idx_interact[i] = -1;
}

void report(const char* where) { std::fprintf(stderr, "%s: %s\n", where, nrt_last_error()); }

int intersect(SoAQueue::ray_queue& q, BVHNode* nodes, bezierPatch* patches, surfaceInteraction* interact, int W, int H,
              float flat_threshold, float v_fov, float* delta, unsigned long long* newton_count,
              unsigned long long* skip_count) {
    if (!nodes || !patches || !interact || !q.origin_x || !q.origin_y || !q.origin_z || !q.direction_x ||
        !q.direction_y || !q.direction_z || !q.idx_interact)
        return nrt::fail(NRT_ERR_INVALID, "null argument");
    if (W <= 0 || H <= 0) return NRT_OK;
    const long long n = (long long)W * H;
    int device = 0;
    cudaGetDevice(&device);
    // the caller's last kernels may still write its arrays (the reference's calls are synchronous)
    if (cudaDeviceSynchronize() != cudaSuccess) return nrt::fail(NRT_ERR_CUDA, "device synchronisation failed");
    const bool flat = flat_threshold > 0.f;
    std::lock_guard<std::mutex> lock(g_cache.mu);
    HostScene hs;
    if (int st = read_scene(nodes, patches, delta, flat, hs)) return st;
    if (!g_cache.scene || g_cache.nodes != nodes || g_cache.patches != patches || g_cache.device != device ||
        g_cache.hash != hs.hash) {
        if (g_cache.scene) nrt_scene_destroy(g_cache.scene);
        g_cache.scene = nullptr;
        if (int st = make_scene(hs, device, &g_cache.scene)) return st;
        g_cache.nodes = nodes;
        g_cache.patches = patches;
        g_cache.device = device;
        g_cache.hash = hs.hash;
    }
    if (g_cache.hit_cap < n) {
        if (g_cache.hits) cudaFree(g_cache.hits);
        g_cache.hits = nullptr;
        g_cache.hit_cap = 0;
        if (cudaMalloc(&g_cache.hits, (size_t)n * 52) != cudaSuccess) return nrt::fail(NRT_ERR_NOMEM, "hit buffers");
        g_cache.hit_cap = n;
    }
    char* hb = static_cast<char*>(g_cache.hits);
    int32_t* patch = reinterpret_cast<int32_t*>(hb);
    float* t = reinterpret_cast<float*>(hb + 4 * n);
    float* u = reinterpret_cast<float*>(hb + 8 * n);
    float* v = reinterpret_cast<float*>(hb + 12 * n);
    float* geom = reinterpret_cast<float*>(hb + 16 * n);
    nrt_intersect_opts o;
    nrt_reference_opts(&o);
    o.flat_threshold = flat ? flat_threshold : 0.f;
    // cam_k as the reference forms it (src/gpu/intersect.cu:210)
    o.cam_k = 0.5 * (float)H / std::tan(v_fov / 2.0f);
    const bool counting = newton_count || skip_count;
    o.schedule = NRT_SCHED_WAVEFRONT;
    // the exact culls only drop pairs whose Newton cannot converge; without them the counters count
    // every pair the traversal tests, as the reference's do, and flat-skip sees every pair
    o.hull_cull = (flat || counting) ? 0 : 3;
    nrt_scene* sc = g_cache.scene;
    if (int st = nrt_enable_counters(sc, counting ? 1 : 0)) return st;
    const nrt_rays r{q.origin_x, q.origin_y, q.origin_z, q.direction_x, q.direction_y, q.direction_z};
    const nrt_hits h{patch, t, u, v, nullptr, nullptr, geom};
    if (int st = nrt_intersect(sc, &r, n, &o, &h, nullptr)) return st;
    k_compat_write<<<(unsigned)((n + 255) / 256), 256>>>(n, patch, t, u, v, geom, q, interact);
    if (counting) {
        nrt_counters c;
        if (int st = nrt_get_counters(sc, &c, nullptr)) return st;
        k_compat_count<<<1, 1>>>(newton_count, skip_count, c.newton_solves, c.flat_skips);
        nrt_enable_counters(sc, 0);
    }
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return nrt::fail(NRT_ERR_CUDA, "calculateIntersectWrapper: %s", cudaGetErrorString(e));
    return NRT_OK;
}

}  // namespace

// Exported with the reference's C++ signatures (src/gpu/intersect.h:9-13,
// src/gpu/generateRaysKernel.h:6).
void calculateIntersectWrapper(SoAQueue::ray_queue& ray_queue, BVHNode* nodes, bezierPatch* patches,
                               surfaceInteraction* interact, int screen_res_x, int screen_res_y, float flat_threshold,
                               float v_fov, float* delta, unsigned long long* newton_count,
                               unsigned long long* skip_count) {
    if (intersect(ray_queue, nodes, patches, interact, screen_res_x, screen_res_y, flat_threshold, v_fov, delta,
                  newton_count, skip_count) != NRT_OK)
        report("calculateIntersectWrapper");
}

void calculateRaysWrapper(SoAQueue::ray_queue& ray_queue, projection proj, camera_config& camera) {
    const int W = camera.screen_resolution_x, H = camera.screen_resolution_y;
    if (W <= 0 || H <= 0) return;
    if (!ray_queue.origin_x || !ray_queue.origin_y || !ray_queue.origin_z || !ray_queue.direction_x ||
        !ray_queue.direction_y || !ray_queue.direction_z || !ray_queue.idx_interact) {
        nrt::fail(NRT_ERR_INVALID, "null ray array");
        report("calculateRaysWrapper");
        return;
    }
    const dim3 block(16, 16), grid((W + 15) / 16, (H + 15) / 16);
    if (proj == perspective)
        k_compat_rays<true><<<grid, block>>>(camera.world_from_camera, camera.camera_from_raster, W, H, ray_queue);
    else
        k_compat_rays<false><<<grid, block>>>(camera.world_from_camera, camera.camera_from_raster, W, H, ray_queue);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        nrt::fail(NRT_ERR_CUDA, "ray generation: %s", cudaGetErrorString(e));
        report("calculateRaysWrapper");
    }
}
