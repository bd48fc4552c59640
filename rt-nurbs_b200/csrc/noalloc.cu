// noalloc.cu -- nrt_intersect_noalloc: the wavefront schedule with its scratch
// in a fixed device array instead of memory from cudaMalloc.
//
// Some callers cannot allocate GPU memory while they run: real-time or
// embedded loops with a fixed memory budget, or code running under a memory
// pool that owns the device.  For them this entry point allocates nothing: the
// scratch of the wavefront rounds (BVH stacks, candidate lists, work items,
// histograms) is carved from g_noalloc_scratch, a file-scope __device__ array
// of kNoallocScratchBytes that the library brings with it, and the per-round
// active count comes back through a static host word.  The caller still owns
// the rays, the hits and the scene (created beforehand with nrt_scene_create).
#include <cuda_runtime.h>

#include <mutex>

#include "kernels.h"
#include "nrt_internal.h"
#include "wavefront.h"

namespace {

// 64 MiB, held by every GPU that loads the library until the process exits.
constexpr size_t kNoallocScratchBytes = 64ull << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices];     // device address of g_noalloc_scratch, per device
int32_t g_round_count[kMaxDevices];    // host word for the per-round active count

// Once per device, with that device current: the array's device address.  In
// host code g_noalloc_scratch names a host-side stand-in, not device memory.
int scratch_address(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) return nrt::fail(NRT_ERR_INVALID, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return nrt::fail(NRT_ERR_CUDA, "cudaGetSymbolAddress(no-alloc scratch): %s", cudaGetErrorString(e));
        g_scratch_addr[device] = p;
    }
    *out = g_scratch_addr[device];
    return NRT_OK;
}

// Largest pass (rays) whose wavefront scratch fits the array for this scene.
long long rays_per_pass(int n_slots) {
    const size_t fixed = nrt::dev::wavefront_scratch_bytes(0, n_slots);
    if (fixed >= kNoallocScratchBytes) return 0;
    const size_t per_ray = nrt::dev::wavefront_scratch_bytes(1 << 20, n_slots) - fixed;  // for 2^20 rays
    long long m = (long long)((double)(kNoallocScratchBytes - fixed) / ((double)per_ray / (1 << 20)));
    while (m > 0 && nrt::dev::wavefront_scratch_bytes(m, n_slots) > kNoallocScratchBytes) m -= 256;
    return m;
}

}  // namespace

extern "C" int nrt_intersect_noalloc(nrt_scene* scene, const nrt_rays* rays, int64_t n,
                                     const nrt_intersect_opts* opts, const nrt_hits* hits, void* stream) {
    nrt::NoallocViews v;
    if (int st = nrt::noalloc_views(scene, rays, n, opts, hits, &v)) return st;
    if (n == 0) return NRT_OK;
    const long long pass = rays_per_pass(v.plan.n_slots);
    if (pass < 1024)
        return nrt::fail(NRT_ERR_INVALID,
                         "scene of %d patches is too large for the %zu-byte no-alloc scratch (it leaves room for %lld "
                         "rays per pass; at least 1024 are needed)",
                         v.plan.n_slots, kNoallocScratchBytes, pass);
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != v.device) {
        const cudaError_t e = cudaSetDevice(v.device);
        if (e != cudaSuccess) return nrt::fail(NRT_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    }
    void* scratch = nullptr;
    int st = scratch_address(v.device, &scratch);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const nrt::dev::WfBuffers wb = nrt::dev::wavefront_carve(scratch, pass, v.plan.n_slots);
    const nrt::dev::Rays r{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz};
    long long launches = 0, rounds = 0;
    cudaError_t e = cudaSuccess;
    if (st == NRT_OK && v.opts.counters)
        e = cudaMemsetAsync(v.counters, 0, nrt::dev::kCounterWords * sizeof(unsigned long long), s);
    for (long long at = 0; st == NRT_OK && e == cudaSuccess && at < n; at += pass) {
        const long long m = (n - at) < pass ? (n - at) : pass;
        const nrt::dev::Rays rc{r.ox + at, r.oy + at, r.oz + at, r.dx + at, r.dy + at, r.dz + at};
        const nrt::dev::Hits hc{hits->patch + at, hits->t + at, hits->u + at, hits->v + at,
                                hits->iters ? hits->iters + at : nullptr, hits->tests ? hits->tests + at : nullptr,
                                hits->geom ? hits->geom + 9 * at : nullptr};
        nrt::dev::Opts oc = v.opts;
        oc.seed_offset = v.opts.seed_offset + (uint32_t)at;  // seeds follow the global ray index
        e = nrt::dev::launch_wavefront(v.scene, v.plan, rc, m, oc, hc, wb, &g_round_count[v.device], v.counters, s,
                                       &launches, &rounds, nullptr, nullptr, nullptr, v.quota0, v.quota_max,
                                       v.stage_nodes);
    }
    if (prev != v.device) cudaSetDevice(prev);
    if (st != NRT_OK) return st;
    if (e != cudaSuccess) return nrt::fail(NRT_ERR_CUDA, "no-alloc intersect: %s", cudaGetErrorString(e));
    nrt::noalloc_record(scene, launches, rounds);
    return NRT_OK;
}
