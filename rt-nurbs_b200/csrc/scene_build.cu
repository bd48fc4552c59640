// scene_build.cu -- scene creation on the device (builder
// NRT_BVH_BINNED_SAH_DEVICE): knot-insertion decomposition, patch boxes, the
// 32-bin SAH, the 4-wide collapse and the per-slot packing all run as
// kernels, and the arena they fill is the one the host builder fills for
// NRT_BVH_BINNED_SAH, bit for bit.  That holds because
//   * every value is computed by the same function on both sides
//     (scene_math.h, slot_pack.cuh), this file being compiled with
//     -fmad=false so that no multiply-add is contracted;
//   * the decomposition of each line (one thread per net column in u, one per
//     strip row in v) runs the same sequential knot insertions as the host's
//     sweep over all lines at once (each line's arithmetic is independent);
//   * the SAH's inputs are order-free (centroid bounds and bin boxes are
//     min/max, bin counts are sums) and its partition is stable, so the tree
//     and its leaf order do not depend on the order in which nodes are
//     processed (here a level at a time, a warp per small node and a block
//     per large one);
//   * the wide collapse numbers nodes breadth-first, as the host's does.
// The reference builds on the host only (BezierPatchOps::getPatch,
// src/math/bezier_patch.h:86-139; BvhOps::buildBVH, src/core/bvh.h:148-179).
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#include "scene_build.h"
#include "slot_pack.cuh"

namespace nrt {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBigNode = 4096;   // nodes with more patches get a block, the rest a warp
constexpr int kSmallWarps = 8;

struct SurfDesc {
    long long net;       // first point of the net (row-major, n+1 rows of m+1)
    long long ku, kv;    // first u knot, first v knot
    long long strips;    // first point of the u pass's strips (nbU+1 strips of (p+1) x (m+1))
    long long cp;        // first point of the surface's patches (patch b*nbV + j: (p+1) x (q+1))
    int n, m, p, q, nbU, nbV;
    int patch0;          // global index of the first patch
    int line_u;          // first u-pass line (net column) of this surface
    int line_v;          // first v-pass line (strip row) of this surface
};

// Index of the last entry of the non-decreasing first[0..n) that is <= t.
__device__ int find_owner(const int* first, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Decomposition

__global__ void k_split_u(const SurfDesc* __restrict__ sd, const int* __restrict__ line_u, int n_surf, int n_lines,
                          const P4* __restrict__ nets, const float* __restrict__ knots, P4* strips, int* err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_lines) return;
    const SurfDesc s = sd[find_owner(line_u, n_surf, t)];
    const int r = t - s.line_u, cols = s.m + 1;
    const long strip = (long)(s.p + 1) * cols;
    const int nb = split_axis(nets + s.net + r, cols, 0, 1, s.p, knots + s.ku, s.n + s.p + 1,
                              View{strips + s.strips + r, cols, 0, strip});
    if (nb != s.nbU) atomicExch(err, 1);
}

__global__ void k_split_v(const SurfDesc* __restrict__ sd, const int* __restrict__ line_v, int n_surf, int n_lines,
                          const P4* __restrict__ strips, const float* __restrict__ knots, P4* cp, int* err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_lines) return;
    const SurfDesc s = sd[find_owner(line_v, n_surf, t)];
    const int local = t - s.line_v, b = local / (s.p + 1), r = local % (s.p + 1), cols = s.m + 1;
    const long strip = (long)(s.p + 1) * cols, piece = (long)(s.p + 1) * (s.q + 1);
    const int nb = split_axis(strips + s.strips + b * strip + (long)r * cols, 1, 0, 1, s.q, knots + s.kv,
                              s.m + s.q + 1, View{cp + s.cp + b * s.nbV * piece + r * (s.q + 1), 1, 0, piece});
    if (nb != s.nbV) atomicExch(err, 1);
}

// Per patch: first point, degrees, surface.
__global__ void k_patch_meta(const SurfDesc* __restrict__ sd, const int* __restrict__ patch0, int n_surf, int N,
                             long long* off, int* deg, int* surf) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const int si = find_owner(patch0, n_surf, k);
    const SurfDesc s = sd[si];
    off[k] = s.cp + (long long)(k - s.patch0) * (s.p + 1) * (s.q + 1);
    deg[2 * k] = s.p;
    deg[2 * k + 1] = s.q;
    surf[k] = si;
}

// Per patch: box, centroid, and the identity order.
__global__ void k_boxes(const P4* __restrict__ cp, const long long* __restrict__ off, const int* __restrict__ deg,
                        int N, Box3* box, float* cen, int32_t* order) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const Box3 b = patch_box(reinterpret_cast<const float*>(cp + off[k]), (deg[2 * k] + 1) * (deg[2 * k + 1] + 1));
    box[k] = b;
    for (int a = 0; a < 3; ++a) cen[3 * k + a] = centre(b, a);
    order[k] = k;
}

// Root box: one block joins every patch box.
__global__ void k_root_box(const Box3* __restrict__ box, int N, Box3* root) {
    __shared__ float s[6][32];
    float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int k = threadIdx.x; k < N; k += blockDim.x)
        for (int a = 0; a < 3; ++a) {
            v[a] = fminf(v[a], box[k].lo[a]);
            v[3 + a] = fmaxf(v[3 + a], box[k].hi[a]);
        }
    for (int o = 16; o > 0; o >>= 1)
        for (int a = 0; a < 3; ++a) {
            v[a] = fminf(v[a], __shfl_xor_sync(kFull, v[a], o));
            v[3 + a] = fmaxf(v[3 + a], __shfl_xor_sync(kFull, v[3 + a], o));
        }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (l == 0)
        for (int a = 0; a < 6; ++a) s[a][w] = v[a];
    __syncthreads();
    if (threadIdx.x == 0) {
        Box3 r = empty_box();
        for (int i = 0; i < nw; ++i)
            for (int a = 0; a < 3; ++a) {
                r.lo[a] = fminf(r.lo[a], s[a][i]);
                r.hi[a] = fmaxf(r.hi[a], s[3 + a][i]);
            }
        *root = r;
    }
}

// ---------------------------------------------------------------------------
// Binned SAH, one level per launch pair

// Floats as ints ordered like the floats (for atomicMin / atomicMax).
__device__ __forceinline__ int f2o(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// SahBins with its floats held as ordered ints while the bins fill.
union BinStore {
    SahBins f;
    struct {
        int lo[3][kSahBins][3];
        int hi[3][kSahBins][3];
        int cnt[3][kSahBins];
    } i;
};

__device__ __forceinline__ void bins_clear(BinStore& B, int t, int nt) {
    for (int e = t; e < 3 * kSahBins; e += nt) {
        const int a = e / kSahBins, k = e % kSahBins;
        B.i.cnt[a][k] = 0;
        for (int c = 0; c < 3; ++c) {
            B.i.lo[a][k][c] = f2o(INFINITY);
            B.i.hi[a][k][c] = f2o(-INFINITY);
        }
    }
}

__device__ __forceinline__ void bins_add(BinStore& B, const Box3& box, const float* c, const float* lo,
                                         const float* ext, const float* scale) {
    for (int a = 0; a < 3; ++a) {
        if (!(ext[a] > 0)) continue;
        const int b = sah_bin(c[a], lo[a], scale[a]);
        atomicAdd(&B.i.cnt[a][b], 1);
        for (int d = 0; d < 3; ++d) {  // NaN coordinates are skipped, as fminf / fmaxf skip them
            if (box.lo[d] == box.lo[d]) atomicMin(&B.i.lo[a][b][d], f2o(box.lo[d]));
            if (box.hi[d] == box.hi[d]) atomicMax(&B.i.hi[a][b][d], f2o(box.hi[d]));
        }
    }
}

// One bin per lane: lane k holds bin k of an axis.
struct LaneBin {
    float lo[3], hi[3];
    int cnt;
};

__device__ __forceinline__ LaneBin lane_bin(const BinStore& B, int a, int k) {
    LaneBin b;
    for (int c = 0; c < 3; ++c) {
        b.lo[c] = o2f(B.i.lo[a][k][c]);
        b.hi[c] = o2f(B.i.hi[a][k][c]);
    }
    b.cnt = B.i.cnt[a][k];
    return b;
}

// sah_choose with a warp: prefix and suffix joins of the bins by shuffles
// (joins are min / max, so every partial box equals the sequential sweep's),
// each lane costs the split after its bin, and the cheapest split wins, the
// earliest (axis, bin) on ties: the sweep's choice.  All lanes return it,
// with the patch count left of the split.
__device__ __forceinline__ void warp_choose(const LaneBin (&b)[3], const float ext[3], int lane, int& axis,
                                            int& split, int& nl) {
    float best_c = INFINITY;
    int best_key = 0x7fffffff, best_nl = 0;
    for (int a = 0; a < 3; ++a) {
        if (!(ext[a] > 0)) continue;
        float L[6], R[6];
        int nL = b[a].cnt, nR = b[a].cnt;
        for (int c = 0; c < 3; ++c) {
            L[c] = R[c] = b[a].lo[c];
            L[3 + c] = R[3 + c] = b[a].hi[c];
        }
        for (int d = 1; d < 32; d <<= 1) {
            float t[6];
            for (int c = 0; c < 6; ++c) t[c] = __shfl_up_sync(kFull, L[c], d);
            const int tn = __shfl_up_sync(kFull, nL, d);
            if (lane >= d) {
                for (int c = 0; c < 3; ++c) { L[c] = fminf(L[c], t[c]); L[3 + c] = fmaxf(L[3 + c], t[3 + c]); }
                nL += tn;
            }
            for (int c = 0; c < 6; ++c) t[c] = __shfl_down_sync(kFull, R[c], d);
            const int rn = __shfl_down_sync(kFull, nR, d);
            if (lane + d < 32) {
                for (int c = 0; c < 3; ++c) { R[c] = fminf(R[c], t[c]); R[3 + c] = fmaxf(R[3 + c], t[3 + c]); }
                nR += rn;
            }
        }
        float Rn[6];
        for (int c = 0; c < 6; ++c) Rn[c] = __shfl_down_sync(kFull, R[c], 1);
        const int nRn = __shfl_down_sync(kFull, nR, 1);
        if (lane < kSahBins - 1 && nL != 0 && nRn != 0) {
            const Box3 lb = {{L[0], L[1], L[2]}, {L[3], L[4], L[5]}};
            const Box3 rb = {{Rn[0], Rn[1], Rn[2]}, {Rn[3], Rn[4], Rn[5]}};
            const float c = nL * half_area(lb) + nRn * half_area(rb);
            if (c < best_c) { best_c = c; best_key = a * 32 + lane; best_nl = nL; }
        }
    }
    for (int d = 16; d > 0; d >>= 1) {
        const float oc = __shfl_xor_sync(kFull, best_c, d);
        const int ok = __shfl_xor_sync(kFull, best_key, d), onl = __shfl_xor_sync(kFull, best_nl, d);
        if (oc < best_c || (oc == best_c && ok < best_key)) { best_c = oc; best_key = ok; best_nl = onl; }
    }
    if (best_key == 0x7fffffff) {
        axis = -1; split = 0; nl = 0;
    } else {
        axis = best_key / 32; split = best_key % 32 + 1; nl = best_nl;
    }
}

// The two sides' boxes of a split (sah_sides with a warp).
__device__ __forceinline__ void warp_sides(const LaneBin& b, int lane, int split, Box3& l, Box3& r) {
    for (int c = 0; c < 3; ++c) {
        float llo = lane < split ? b.lo[c] : INFINITY, lhi = lane < split ? b.hi[c] : -INFINITY;
        float rlo = lane < split ? INFINITY : b.lo[c], rhi = lane < split ? -INFINITY : b.hi[c];
        for (int d = 16; d > 0; d >>= 1) {
            llo = fminf(llo, __shfl_xor_sync(kFull, llo, d));
            lhi = fmaxf(lhi, __shfl_xor_sync(kFull, lhi, d));
            rlo = fminf(rlo, __shfl_xor_sync(kFull, rlo, d));
            rhi = fmaxf(rhi, __shfl_xor_sync(kFull, rhi, d));
        }
        l.lo[c] = llo; l.hi[c] = lhi;
        r.lo[c] = rlo; r.hi[c] = rhi;
    }
}

struct SahLevel {
    const Box3* prim;
    const float* cen;
    int32_t* order;
    int32_t* order2;
    Box3* nbox;
    uint32_t* lf;
    uint32_t* pc;
    const int32_t* list;    // this level's nodes of this size class
    int n_list;
    int32_t* next_big;
    int32_t* next_small;
    int* ctr;               // [0] next big count, [1] next small count, [2] nodes used, [3] largest unsplit leaf
    int max_leaf;
};

__device__ __forceinline__ void push_child(const SahLevel& L, int node, uint32_t count) {
    if ((int)count <= L.max_leaf) return;
    if (count > (uint32_t)kBigNode) L.next_big[atomicAdd(&L.ctr[0], 1)] = node;
    else L.next_small[atomicAdd(&L.ctr[1], 1)] = node;
}

// Records the split of node nd (first, count) with nl patches on the left.
__device__ __forceinline__ void make_children(const SahLevel& L, int nd, uint32_t first, uint32_t count, uint32_t nl,
                                              const Box3& bl, const Box3& br) {
    const int l = atomicAdd(&L.ctr[2], 2), r = l + 1;
    L.nbox[l] = bl;
    L.lf[l] = first;
    L.pc[l] = nl;
    L.nbox[r] = br;
    L.lf[r] = first + nl;
    L.pc[r] = count - nl;
    L.lf[nd] = (uint32_t)l;
    L.pc[nd] = 0;
    push_child(L, l, nl);
    push_child(L, r, count - nl);
}

// A warp per node (nodes of at most kBigNode patches).
__global__ void __launch_bounds__(32 * kSmallWarps) k_sah_small(SahLevel L) {
    __shared__ BinStore bins[kSmallWarps];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int a_idx = blockIdx.x * kSmallWarps + w;
    if (a_idx >= L.n_list) return;
    BinStore& B = bins[w];
    const int nd = L.list[a_idx];
    const uint32_t first = L.lf[nd], count = L.pc[nd];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = lane; i < count; i += 32) {
        const int id = L.order[first + i];
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(lo[a], L.cen[3 * id + a]);
            hi[a] = fmaxf(hi[a], L.cen[3 * id + a]);
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(lo[a], __shfl_xor_sync(kFull, lo[a], o));
            hi[a] = fmaxf(hi[a], __shfl_xor_sync(kFull, hi[a], o));
        }
    float ext[3], scale[3];
    for (int a = 0; a < 3; ++a) {
        ext[a] = hi[a] - lo[a];
        scale[a] = kSahBins / ext[a];
    }
    bins_clear(B, lane, 32);
    __syncwarp();
    for (uint32_t i = lane; i < count; i += 32) {
        const int id = L.order[first + i];
        const float c[3] = {L.cen[3 * id], L.cen[3 * id + 1], L.cen[3 * id + 2]};
        bins_add(B, L.prim[id], c, lo, ext, scale);
    }
    __syncwarp();
    const LaneBin b[3] = {lane_bin(B, 0, lane), lane_bin(B, 1, lane), lane_bin(B, 2, lane)};
    int axis, split, nl;
    warp_choose(b, ext, lane, axis, split, nl);
    if (axis < 0 || nl == 0 || (uint32_t)nl == count) {  // all centroids coincide: a leaf
        if (lane == 0 && count > 8) atomicMax(&L.ctr[3], (int)count);
        return;
    }
    Box3 bl, br;
    warp_sides(b[axis], lane, split, bl, br);
    const float alo = lo[axis], ascale = scale[axis];
    // stable partition through order2
    uint32_t lbase = 0;
    for (uint32_t i0 = 0; i0 < count; i0 += 32) {
        const uint32_t i = i0 + lane;
        const bool valid = i < count;
        const int id = valid ? L.order[first + i] : 0;
        const bool left = valid && sah_bin(L.cen[3 * id + axis], alo, ascale) < split;
        const unsigned m = __ballot_sync(kFull, left);
        const uint32_t before = __popc(m & ((1u << lane) - 1u));
        if (valid) L.order2[first + (left ? lbase + before : nl + (i - lbase - before))] = id;
        lbase += __popc(m);
    }
    __syncwarp();
    for (uint32_t i = lane; i < count; i += 32) L.order[first + i] = L.order2[first + i];
    if (lane == 0) make_children(L, nd, first, count, (uint32_t)nl, bl, br);
}

// Nodes of more than kBigNode patches are cut into chunks of kChunk patches,
// each handled by one block: bounds and bins meet in the node's state through
// atomics, one warp per node chooses the split, and each chunk scatters its
// patches after the left counts of the chunks before it (stable overall).
constexpr int kChunk = 4096;
constexpr int kChunkThreads = 256;

struct BigState {
    int bounds[6];   // centroid bounds, ordered ints: lo xyz, hi xyz
    int axis, split, nl, nch;
    uint32_t first, count;  // the node's patch range (its node record changes once it is split)
    BinStore bins;
};

struct BigLevel {
    SahLevel L;
    BigState* st;
    int* chunk_cnt;        // n_big + 1: chunks per node (last 0)
    int* chunk_off;        // n_big + 1: first chunk of each node, [n_big] = total
    int* chunk_left;       // per chunk: patches going left
    int* chunk_pre;        // per chunk: left patches of the node's earlier chunks
};

// Node j and the patch range [b, e) of chunk c.
__device__ __forceinline__ int chunk_range(const BigLevel& G, int c, uint32_t& b, uint32_t& e, uint32_t& first) {
    const int j = find_owner(G.chunk_off, G.L.n_list, c);
    first = G.st[j].first;
    b = (uint32_t)(c - G.chunk_off[j]) * kChunk;
    e = min(b + (uint32_t)kChunk, G.st[j].count);
    return j;
}

__global__ void k_big_init(BigLevel G) {
    const int j = blockIdx.x;
    BigState& s = G.st[j];
    bins_clear(s.bins, threadIdx.x, blockDim.x);
    if (threadIdx.x < 3) {
        s.bounds[threadIdx.x] = f2o(INFINITY);
        s.bounds[3 + threadIdx.x] = f2o(-INFINITY);
    }
    if (threadIdx.x == 0) {
        const int nd = G.L.list[j];
        const uint32_t count = G.L.pc[nd];
        s.first = G.L.lf[nd];
        s.count = count;
        s.nch = (int)((count + kChunk - 1) / kChunk);
        G.chunk_cnt[j] = s.nch;
        if (j == 0) G.chunk_cnt[G.L.n_list] = 0;
    }
}

__device__ __forceinline__ void node_frame(const BigState& s, float lo[3], float ext[3], float scale[3]) {
    for (int a = 0; a < 3; ++a) {
        lo[a] = o2f(s.bounds[a]);
        ext[a] = o2f(s.bounds[3 + a]) - lo[a];
        scale[a] = kSahBins / ext[a];
    }
}

__global__ void __launch_bounds__(kChunkThreads) k_big_bounds(BigLevel G) {
    __shared__ float red[6][kChunkThreads / 32];
    const int total = G.chunk_off[G.L.n_list];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        uint32_t b, e, first;
        const int j = chunk_range(G, c, b, e, first);
        float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = b + threadIdx.x; i < e; i += kChunkThreads) {
            const int id = G.L.order[first + i];
            for (int a = 0; a < 3; ++a) {
                v[a] = fminf(v[a], G.L.cen[3 * id + a]);
                v[3 + a] = fmaxf(v[3 + a], G.L.cen[3 * id + a]);
            }
        }
        for (int o = 16; o > 0; o >>= 1)
            for (int a = 0; a < 3; ++a) {
                v[a] = fminf(v[a], __shfl_xor_sync(kFull, v[a], o));
                v[3 + a] = fmaxf(v[3 + a], __shfl_xor_sync(kFull, v[3 + a], o));
            }
        if (lane == 0)
            for (int a = 0; a < 6; ++a) red[a][w] = v[a];
        __syncthreads();
        if (threadIdx.x < 6) {
            const int a = threadIdx.x;
            float r = red[a][0];
            for (int k = 1; k < kChunkThreads / 32; ++k) r = a < 3 ? fminf(r, red[a][k]) : fmaxf(r, red[a][k]);
            if (r == r) {  // an all-NaN chunk adds nothing
                if (a < 3) atomicMin(&G.st[j].bounds[a], f2o(r));
                else atomicMax(&G.st[j].bounds[a], f2o(r));
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kChunkThreads) k_big_bins(BigLevel G) {
    __shared__ BinStore B;
    const int total = G.chunk_off[G.L.n_list];
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        uint32_t b, e, first;
        const int j = chunk_range(G, c, b, e, first);
        float lo[3], ext[3], scale[3];
        node_frame(G.st[j], lo, ext, scale);
        bins_clear(B, threadIdx.x, kChunkThreads);
        __syncthreads();
        for (uint32_t i = b + threadIdx.x; i < e; i += kChunkThreads) {
            const int id = G.L.order[first + i];
            const float cc[3] = {G.L.cen[3 * id], G.L.cen[3 * id + 1], G.L.cen[3 * id + 2]};
            bins_add(B, G.L.prim[id], cc, lo, ext, scale);
        }
        __syncthreads();
        BinStore& S = G.st[j].bins;
        for (int t = threadIdx.x; t < 3 * kSahBins; t += kChunkThreads) {
            const int a = t / kSahBins, k = t % kSahBins;
            if (B.i.cnt[a][k] == 0) continue;
            atomicAdd(&S.i.cnt[a][k], B.i.cnt[a][k]);
            for (int d = 0; d < 3; ++d) {
                atomicMin(&S.i.lo[a][k][d], B.i.lo[a][k][d]);
                atomicMax(&S.i.hi[a][k][d], B.i.hi[a][k][d]);
            }
        }
        __syncthreads();
    }
}

// A warp per big node: the split, the children, the chunks' left-count prefix
// comes later (k_big_prefix).
__global__ void k_big_choose(BigLevel G) {
    const int j = blockIdx.x, lane = threadIdx.x;
    BigState& s = G.st[j];
    const int nd = G.L.list[j];
    const uint32_t first = s.first, count = s.count;
    float lo[3], ext[3], scale[3];
    node_frame(s, lo, ext, scale);
    const LaneBin b[3] = {lane_bin(s.bins, 0, lane), lane_bin(s.bins, 1, lane), lane_bin(s.bins, 2, lane)};
    int axis, split, nl;
    warp_choose(b, ext, lane, axis, split, nl);
    if (axis < 0 || nl == 0 || (uint32_t)nl == count) {
        if (lane == 0) {
            s.axis = -1;
            if (count > 8) atomicMax(&G.L.ctr[3], (int)count);
        }
        return;
    }
    Box3 bl, br;
    warp_sides(b[axis], lane, split, bl, br);
    if (lane == 0) {
        s.axis = axis;
        s.split = split;
        s.nl = nl;
        make_children(G.L, nd, first, count, (uint32_t)nl, bl, br);
    }
}

__global__ void __launch_bounds__(kChunkThreads) k_big_count(BigLevel G) {
    __shared__ int red[kChunkThreads / 32];
    const int total = G.chunk_off[G.L.n_list];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        uint32_t b, e, first;
        const int j = chunk_range(G, c, b, e, first);
        const BigState& s = G.st[j];
        if (s.axis < 0) continue;  // uniform over the block
        float lo[3], ext[3], scale[3];
        node_frame(s, lo, ext, scale);
        int n = 0;
        for (uint32_t i = b + threadIdx.x; i < e; i += kChunkThreads) {
            const int id = G.L.order[first + i];
            n += sah_bin(G.L.cen[3 * id + s.axis], lo[s.axis], scale[s.axis]) < s.split;
        }
        for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(kFull, n, o);
        if (lane == 0) red[w] = n;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int k = 0; k < kChunkThreads / 32; ++k) t += red[k];
            G.chunk_left[c] = t;
        }
        __syncthreads();
    }
}

__global__ void k_big_prefix(BigLevel G) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= G.L.n_list || G.st[j].axis < 0) return;
    int acc = 0;
    for (int c = G.chunk_off[j]; c < G.chunk_off[j + 1]; ++c) {
        G.chunk_pre[c] = acc;
        acc += G.chunk_left[c];
    }
}

__global__ void __launch_bounds__(kChunkThreads) k_big_scatter(BigLevel G) {
    constexpr int NW = kChunkThreads / 32;
    __shared__ uint32_t wcount[NW];
    const int total = G.chunk_off[G.L.n_list];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        uint32_t b, e, first;
        const int j = chunk_range(G, c, b, e, first);
        const BigState& s = G.st[j];
        if (s.axis < 0) continue;
        float lo[3], ext[3], scale[3];
        node_frame(s, lo, ext, scale);
        const uint32_t nl = (uint32_t)s.nl;
        uint32_t lbase = (uint32_t)G.chunk_pre[c];  // left patches before this position in the node
        for (uint32_t i0 = b; i0 < e; i0 += kChunkThreads) {
            const uint32_t i = i0 + threadIdx.x;
            const bool valid = i < e;
            const int id = valid ? G.L.order[first + i] : 0;
            const bool left = valid && sah_bin(G.L.cen[3 * id + s.axis], lo[s.axis], scale[s.axis]) < s.split;
            const unsigned m = __ballot_sync(kFull, left);
            if (lane == 0) wcount[w] = __popc(m);
            __syncthreads();
            uint32_t before = __popc(m & ((1u << lane) - 1u)), tot = 0;
            for (int k = 0; k < NW; ++k) {
                if (k < w) before += wcount[k];
                tot += wcount[k];
            }
            if (valid) G.L.order2[first + (left ? lbase + before : nl + (i - lbase - before))] = id;
            lbase += tot;
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kChunkThreads) k_big_copy(BigLevel G) {
    const int total = G.chunk_off[G.L.n_list];
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        uint32_t b, e, first;
        const int j = chunk_range(G, c, b, e, first);
        if (G.st[j].axis < 0) continue;
        for (uint32_t i = b + threadIdx.x; i < e; i += kChunkThreads) G.L.order[first + i] = G.L.order2[first + i];
    }
}

// ---------------------------------------------------------------------------
// 4-wide collapse, breadth first: queue[w] is the binary node of wide node w

__global__ void k_wide_count(const uint32_t* __restrict__ queue, int lb, int n, const Box3* __restrict__ nbox,
                             const uint32_t* __restrict__ lf, const uint32_t* __restrict__ pc, uint32_t* kids,
                             int* inner) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > n) return;
    if (t == n) {  // the scan's last entry becomes the level's total
        inner[n] = 0;
        return;
    }
    uint32_t k4[4];
    const int nk = wide_kids(queue[lb + t], nbox, lf, pc, k4);
    int ni = 0;
    for (int c = 0; c < 4; ++c) {
        kids[4 * t + c] = c < nk ? k4[c] : 0xffffffffu;
        if (c < nk && pc[k4[c]] == 0) ++ni;
    }
    inner[t] = ni;
}

__global__ void k_wide_write(uint32_t* queue, int lb, int n, const Box3* __restrict__ nbox,
                             const uint32_t* __restrict__ lf, const uint32_t* __restrict__ pc,
                             const uint32_t* __restrict__ kids, const int* __restrict__ inner_off, Node4* wide) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    Node4 nd;
    for (int c = 0; c < 4; ++c) {
        nd.lo_x[c] = nd.lo_y[c] = nd.lo_z[c] = INFINITY;
        nd.hi_x[c] = nd.hi_y[c] = nd.hi_z[c] = -INFINITY;
        nd.child[c] = -1;
        nd.count[c] = 0;
    }
    int next = lb + n + inner_off[t];
    for (int c = 0; c < 4; ++c) {
        const uint32_t b = kids[4 * t + c];
        if (b == 0xffffffffu) continue;
        const Box3& bx = nbox[b];
        nd.lo_x[c] = bx.lo[0]; nd.lo_y[c] = bx.lo[1]; nd.lo_z[c] = bx.lo[2];
        nd.hi_x[c] = bx.hi[0]; nd.hi_y[c] = bx.hi[1]; nd.hi_z[c] = bx.hi[2];
        if (pc[b] > 0) {
            nd.child[c] = ~(int32_t)lf[b];
            nd.count[c] = (int32_t)pc[b];
        } else {
            nd.child[c] = next;
            queue[next++] = b;
        }
    }
    wide[lb + t] = nd;
}

// ---------------------------------------------------------------------------
// Per-slot packing

__global__ void k_slot_sizes(const int32_t* __restrict__ order, const int* __restrict__ deg, int N, long long* sz) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > N) return;
    if (s == N) { sz[N] = 0; return; }
    const int k = order[s];
    sz[s] = 4 * (long long)dev::padded_points(deg[2 * k], deg[2 * k + 1]);
}

struct PackOut {
    float* blocks;
    int4* hdr;
    double4* centre;
    float4* corners;
    float* delta;
    dev::PatchFrame* frames;
    float4* obb;
    uint32_t* key;
    int* hist;
};

__global__ void __launch_bounds__(128) k_pack(const P4* __restrict__ cp, const long long* __restrict__ off,
                                              const int* __restrict__ deg, const int* __restrict__ surf,
                                              const Box3* __restrict__ box, const int32_t* __restrict__ order,
                                              const long long* __restrict__ boff, int N, PackOut o) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const int k = order[s], p = deg[2 * k], q = deg[2 * k + 1];
    const long long at = boff[s];
    pack_slot(reinterpret_cast<const float*>(cp + off[k]), p, q, box[k], k, surf[k], at, o.blocks + at, o.hdr[s],
              o.centre[s], o.corners + 4 * (size_t)s, o.delta[s], o.frames[s], o.obb + 4 * (size_t)s);
    o.key[s] = (uint32_t)(p | (q << 4));
    atomicAdd(&o.hist[p * 8 + q], 1);
}

__global__ void k_leafbox(const Node4* __restrict__ wide, int n_wide, float4* leafbox) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_wide) return;
    const Node4& nd = wide[w];
    for (int c = 0; c < 4; ++c)
        if (nd.child[c] < 0 && nd.count[c] > 0)
            for (int k = ~nd.child[c]; k < ~nd.child[c] + nd.count[c]; ++k) {
                leafbox[2 * (size_t)k] = make_float4(nd.lo_x[c], nd.lo_y[c], nd.lo_z[c], 0.f);
                leafbox[2 * (size_t)k + 1] = make_float4(nd.hi_x[c], nd.hi_y[c], nd.hi_z[c], 0.f);
            }
}

__global__ void k_iota(int32_t* v, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) v[i] = i;
}

__global__ void k_rank_of(const int32_t* __restrict__ by_rank, int N, int32_t* rank_of) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < N) rank_of[by_rank[r]] = r;
}

// ---------------------------------------------------------------------------
// Host side

// f(i) for i in [0, n) on up to 16 threads (inline for small n).
template <class F>
void parallel_for(int n, F f) {
    const int T = (int)std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
    if (n < 32 || T == 1) {
        for (int i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<int> next{0};
    auto work = [&] {
        for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) f(i);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < T; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
}

unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// Scratch carved from one allocation, 256-byte aligned pieces.
struct Scratch {
    char* base = nullptr;
    size_t at = 0, cap = 0;
    template <class T>
    T* take(size_t count) {
        T* p = reinterpret_cast<T*>(base + at);
        at += (count * sizeof(T) + 255) & ~(size_t)255;
        return p;
    }
};

// Everything after the patches exist on the device: cp (points), off/deg/surf
// per patch.  Host-side per-patch tables (ranges, surface ids) come in ps.
int build_from_device_patches(const nrt_build_opts& o, int N, int n_surfaces, const P4* cp, const long long* off,
                              const int* deg, const int* surf, long long n_floats, PatchSet&& ps, nrt_scene** out) {
    // scratch: boxes, centroids, order x2, binary nodes, lists, counters, wide
    // nodes and queue, kids, scan buffers, slot sizes/offsets, keys
    const size_t M = 2 * (size_t)N;
    size_t scan_bytes = 0, sort_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const long long*)nullptr, (long long*)nullptr, N + 1);
    size_t scan_i = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_i, (const int*)nullptr, (int*)nullptr, N + 1);
    scan_bytes = std::max(scan_bytes, scan_i);
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const int32_t*)nullptr, (int32_t*)nullptr, N, 0, 8);
    const size_t tmp_bytes = std::max(scan_bytes, sort_bytes);
    const size_t cap_big = (size_t)N / kBigNode + 2, cap_chunks = (size_t)N / kChunk + cap_big + 2;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t need = al(N * sizeof(Box3)) + al(3 * (size_t)N * sizeof(float)) + 2 * al(N * sizeof(int32_t)) +
                        al(M * sizeof(Box3)) + 2 * al(M * sizeof(uint32_t)) + 4 * al((N + 1) * sizeof(int32_t)) +
                        al(8 * sizeof(int)) + al((N + 1) * sizeof(Node4)) + al((N + 1) * sizeof(uint32_t)) +
                        al(4 * (size_t)(N + 1) * sizeof(uint32_t)) + 2 * al((N + 2) * sizeof(int)) +
                        2 * al((N + 1) * sizeof(long long)) + 2 * al(N * sizeof(uint32_t)) +
                        2 * al(N * sizeof(int32_t)) + al(64 * sizeof(int)) + al(tmp_bytes) +
                        al(cap_big * sizeof(BigState)) + 2 * al((cap_big + 1) * sizeof(int)) +
                        2 * al(cap_chunks * sizeof(int)) + 256;
    Scratch S;
    cudaError_t e = cudaMalloc(&S.base, need);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(scene build scratch)");
    S.cap = need;
    struct Guard {
        void* p;
        ~Guard() { cudaFree(p); }
    } guard{S.base};
    Box3* box = S.take<Box3>(N);
    float* cen = S.take<float>(3 * (size_t)N);
    int32_t* order = S.take<int32_t>(N);
    int32_t* order2 = S.take<int32_t>(N);
    Box3* nbox = S.take<Box3>(M);
    uint32_t* lf = S.take<uint32_t>(M);
    uint32_t* pc = S.take<uint32_t>(M);
    int32_t* lists[4] = {S.take<int32_t>(N + 1), S.take<int32_t>(N + 1), S.take<int32_t>(N + 1),
                         S.take<int32_t>(N + 1)};
    int* ctr = S.take<int>(8);
    Node4* wide = S.take<Node4>(N + 1);
    uint32_t* queue = S.take<uint32_t>(N + 1);
    uint32_t* kids = S.take<uint32_t>(4 * (size_t)(N + 1));
    int* inner = S.take<int>(N + 2);
    int* inner_off = S.take<int>(N + 2);
    long long* ssz = S.take<long long>(N + 1);
    long long* soff = S.take<long long>(N + 1);
    uint32_t* key = S.take<uint32_t>(N);
    uint32_t* key2 = S.take<uint32_t>(N);
    int32_t* slots = S.take<int32_t>(N);
    int32_t* by_rank = S.take<int32_t>(N);
    int* hist = S.take<int>(64);
    void* tmp = S.take<char>(tmp_bytes);
    BigState* big = S.take<BigState>(cap_big);
    int* chunk_cnt = S.take<int>(cap_big + 1);
    int* chunk_off = S.take<int>(cap_big + 1);
    int* chunk_left = S.take<int>(cap_chunks);
    int* chunk_pre = S.take<int>(cap_chunks);
    auto check = [&](const char* what) -> int {
        const cudaError_t k = cudaGetLastError();
        return k == cudaSuccess ? NRT_OK : cuda_fail(k, what);
    };

    // boxes, centroids, root
    k_boxes<<<blocks_for(N, 256), 256>>>(cp, off, deg, N, box, cen, order);
    k_root_box<<<1, 1024>>>(box, N, nbox);
    e = cudaMemset(lf, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpy(pc, &N, sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "scene build: root");
    if (int st = check("scene build: boxes")) return st;

    // binned SAH, a level at a time
    int h_ctr[4] = {0, 0, 1, 0};
    int n_big = 0, n_small = 0;
    const int32_t root = 0;
    if (N > o.max_leaf) {
        if (N > kBigNode) n_big = 1;
        else n_small = 1;
        e = cudaMemcpy(lists[n_big ? 0 : 1], &root, sizeof(root), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "scene build: SAH root");
    }
    e = cudaMemcpy(ctr, h_ctr, sizeof(h_ctr), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "scene build: SAH counters");
    int cur = 0;
    while (n_big + n_small > 0) {
        e = cudaMemset(ctr, 0, 2 * sizeof(int));
        if (e != cudaSuccess) return cuda_fail(e, "scene build: SAH level");
        SahLevel L{box, cen, order, order2, nbox, lf, pc, nullptr, 0, lists[2 * (cur ^ 1)], lists[2 * (cur ^ 1) + 1],
                   ctr, o.max_leaf};
        if (n_big) {
            L.list = lists[2 * cur];
            L.n_list = n_big;
            const BigLevel G{L, big, chunk_cnt, chunk_off, chunk_left, chunk_pre};
            k_big_init<<<n_big, 128>>>(G);
            size_t tb = tmp_bytes;
            e = cub::DeviceScan::ExclusiveSum(tmp, tb, chunk_cnt, chunk_off, n_big + 1);
            if (e != cudaSuccess) return cuda_fail(e, "scene build: chunk scan");
            const unsigned grid = (unsigned)std::min<long long>(148 * 4, (long long)N / kChunk + n_big + 1);
            k_big_bounds<<<grid, kChunkThreads>>>(G);
            k_big_bins<<<grid, kChunkThreads>>>(G);
            k_big_choose<<<n_big, 32>>>(G);
            k_big_count<<<grid, kChunkThreads>>>(G);
            k_big_prefix<<<blocks_for(n_big, 128), 128>>>(G);
            k_big_scatter<<<grid, kChunkThreads>>>(G);
            k_big_copy<<<grid, kChunkThreads>>>(G);
        }
        if (n_small) {
            L.list = lists[2 * cur + 1];
            L.n_list = n_small;
            k_sah_small<<<blocks_for(n_small, kSmallWarps), 32 * kSmallWarps>>>(L);
        }
        e = cudaMemcpy(h_ctr, ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "scene build: SAH level");
        n_big = h_ctr[0];
        n_small = h_ctr[1];
        cur ^= 1;
    }
    if (h_ctr[3] > 8) return fail(NRT_ERR_UNSUPPORTED, "BVH leaf with %d patches (limit 8)", h_ctr[3]);

    // 4-wide collapse, breadth first
    const uint32_t zero = 0;
    e = cudaMemcpy(queue, &zero, sizeof(zero), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "scene build: collapse");
    int lb = 0, le = 1, depth = 0;
    while (le > lb) {
        const int n = le - lb;
        ++depth;
        k_wide_count<<<blocks_for(n + 1, 256), 256>>>(queue, lb, n, nbox, lf, pc, kids, inner);
        size_t tb = tmp_bytes;
        e = cub::DeviceScan::ExclusiveSum(tmp, tb, inner, inner_off, n + 1);
        if (e != cudaSuccess) return cuda_fail(e, "scene build: collapse scan");
        k_wide_write<<<blocks_for(n, 256), 256>>>(queue, lb, n, nbox, lf, pc, kids, inner_off, wide);
        int total = 0;
        e = cudaMemcpy(&total, inner_off + n, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "scene build: collapse");
        lb = le;
        le = le + total;
    }
    const int n_wide = le;

    // slot block offsets
    k_slot_sizes<<<blocks_for(N + 1, 256), 256>>>(order, deg, N, ssz);
    {
        size_t tb = tmp_bytes;
        e = cub::DeviceScan::ExclusiveSum(tmp, tb, ssz, soff, N + 1);
        if (e != cudaSuccess) return cuda_fail(e, "scene build: block offsets");
    }
    if (int st = check("scene build: collapse")) return st;

    // the arena, filled in place
    const ArenaLayout A = arena_layout((size_t)n_wide, N, (size_t)n_floats);
    nrt_scene* sc = nullptr;
    char* base = nullptr;
    if (int st = new_scene(o, A, &sc, &base)) return st;
    auto fail_scene = [&](cudaError_t err, const char* what) {
        nrt_scene_destroy(sc);
        return cuda_fail(err, what);
    };
    e = cudaMemcpy(base + A.nodes, wide, n_wide * sizeof(Node4), cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return fail_scene(e, "scene build: nodes");
    e = cudaMemset(hist, 0, 64 * sizeof(int));
    if (e != cudaSuccess) return fail_scene(e, "scene build: packing");
    PackOut po{reinterpret_cast<float*>(base + A.cp), reinterpret_cast<int4*>(base + A.hdr),
               reinterpret_cast<double4*>(base + A.centre), reinterpret_cast<float4*>(base + A.corners),
               reinterpret_cast<float*>(base + A.delta), reinterpret_cast<dev::PatchFrame*>(base + A.frames),
               reinterpret_cast<float4*>(base + A.obb), key, hist};
    k_pack<<<blocks_for(N, 128), 128>>>(cp, off, deg, surf, box, order, soff, N, po);
    k_leafbox<<<blocks_for(n_wide, 128), 128>>>(reinterpret_cast<const Node4*>(base + A.nodes), n_wide,
                                                reinterpret_cast<float4*>(base + A.leafbox));
    // ranks: slots stably sorted by p | q << 4
    k_iota<<<blocks_for(N, 256), 256>>>(slots, N);
    {
        size_t tb = tmp_bytes;
        e = cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, slots, by_rank, N, 0, 8);
        if (e != cudaSuccess) return fail_scene(e, "scene build: rank sort");
    }
    k_rank_of<<<blocks_for(N, 256), 256>>>(by_rank, N, reinterpret_cast<int32_t*>(base + A.rank));
    nrt_scene_info info{};
    e = cudaMemcpy(info.degree_hist, hist, 64 * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail_scene(e, "scene build: packing");
    dev::WfPlan plan{};
    plan_classes(info.degree_hist, N, plan);
    info.n_surfaces = n_surfaces;
    info.n_nodes = n_wide;
    info.bvh_depth = depth;
    finish_scene(sc, A, N, plan, info, std::move(ps), n_surfaces);
    *out = sc;
    return NRT_OK;
}

struct DeviceGuard {
    int prev = 0;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
    }
    ~DeviceGuard() { cudaSetDevice(prev); }
};

int check_build_opts(const nrt_build_opts& o) {
    if (o.wavefront_chunk < 0) return fail(NRT_ERR_INVALID, "negative wavefront_chunk");
    if (o.max_leaf < 1 || o.max_leaf > 8) return fail(NRT_ERR_INVALID, "max_leaf must be in 1..8");
    return NRT_OK;
}

}  // namespace

int build_scene_device_surfaces(const nrt_nurbs_surface* surfaces, int n_surfaces, const nrt_build_opts& o,
                                nrt_scene** out) {
    *out = nullptr;
    if (int st = check_build_opts(o)) return st;
    std::vector<SurfDesc> sd(n_surfaces);
    std::vector<int> line_u(n_surfaces), line_v(n_surfaces), patch0(n_surfaces);
    PatchSet ps;
    long long pts_net = 0, pts_strip = 0, pts_cp = 0, n_knots = 0, n_floats = 0, lines_u = 0, lines_v = 0;
    long long N = 0;
    ps.spans.resize(n_surfaces);
    for (int si = 0; si < n_surfaces; ++si) {
        const nrt_nurbs_surface& s = surfaces[si];
        if (int st = check_surface(s)) {
            set_error("surface %d: %s", si, nrt_last_error());
            return st;
        }
        PatchSet::Spans& sp = ps.spans[si];
        sp.bu = ps.breaks.size();
        ps.breaks.resize(sp.bu + (s.n - s.p + 2));
        const int nbU = knot_spans(s.u_knots, s.n + s.p + 1, s.p, &ps.breaks[sp.bu]);
        ps.breaks.resize(sp.bu + nbU + 1);
        sp.bv = ps.breaks.size();
        ps.breaks.resize(sp.bv + (s.m - s.q + 2));
        const int nbV = knot_spans(s.v_knots, s.m + s.q + 1, s.q, &ps.breaks[sp.bv]);
        ps.breaks.resize(sp.bv + nbV + 1);
        sp.patch0 = (int)N;
        sp.nbU = nbU;
        sp.nbV = nbV;
        SurfDesc& d = sd[si];
        d.n = s.n; d.m = s.m; d.p = s.p; d.q = s.q; d.nbU = nbU; d.nbV = nbV;
        d.net = pts_net;
        d.ku = n_knots;
        d.kv = n_knots + s.n + s.p + 2;
        d.strips = pts_strip;
        d.cp = pts_cp;
        d.patch0 = (int)N;
        d.line_u = (int)lines_u;
        d.line_v = (int)lines_v;
        line_u[si] = d.line_u;
        line_v[si] = d.line_v;
        patch0[si] = d.patch0;
        pts_net += (long long)(s.n + 1) * (s.m + 1);
        n_knots += (s.n + s.p + 2) + (s.m + s.q + 2);
        pts_strip += (long long)(nbU + 1) * (s.p + 1) * (s.m + 1);
        pts_cp += (long long)nbU * nbV * (s.p + 1) * (s.q + 1);
        n_floats += (long long)nbU * nbV * 4 * dev::padded_points(s.p, s.q);
        lines_u += s.m + 1;
        lines_v += (long long)nbU * (s.p + 1);
        N += (long long)nbU * nbV;
        if (N >= (1 << 27) || lines_u >= (1LL << 31) || lines_v >= (1LL << 31))
            return fail(NRT_ERR_INVALID, "too many patches");
    }
    if (n_floats >= (1LL << 31)) return fail(NRT_ERR_INVALID, "scene too large (%lld block floats)", n_floats);
    // nets and knots, packed on the host (several threads: the first touch of
    // fresh pages dominates) and copied once
    std::unique_ptr<P4[]> nets(new (std::nothrow) P4[(size_t)pts_net]);
    std::unique_ptr<float[]> knots(new (std::nothrow) float[(size_t)n_knots]);
    if (!nets || !knots) return fail(NRT_ERR_NOMEM, "host allocation failed");
    parallel_for(n_surfaces, [&](int si) {
        const nrt_nurbs_surface& s = surfaces[si];
        const SurfDesc& d = sd[si];
        std::memcpy(&nets[d.net], s.control_points, sizeof(P4) * (size_t)(s.n + 1) * (s.m + 1));
        std::memcpy(&knots[d.ku], s.u_knots, sizeof(float) * (s.n + s.p + 2));
        std::memcpy(&knots[d.kv], s.v_knots, sizeof(float) * (s.m + s.q + 2));
    });
    DeviceGuard dg(o.device);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t need = al(sd.size() * sizeof(SurfDesc)) + 3 * al(n_surfaces * sizeof(int)) +
                        al((size_t)pts_net * sizeof(P4)) + al((size_t)n_knots * sizeof(float)) +
                        al((size_t)pts_strip * sizeof(P4)) + al((size_t)pts_cp * sizeof(P4)) +
                        al((size_t)N * sizeof(long long)) + al(2 * (size_t)N * sizeof(int)) +
                        al((size_t)N * sizeof(int)) + al(sizeof(int)) + 256;
    Scratch S;
    cudaError_t e = cudaMalloc(&S.base, need);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(decomposition scratch)");
    struct Guard {
        void* p;
        ~Guard() { cudaFree(p); }
    } guard{S.base};
    SurfDesc* d_sd = S.take<SurfDesc>(sd.size());
    int* d_line_u = S.take<int>(n_surfaces);
    int* d_line_v = S.take<int>(n_surfaces);
    int* d_patch0 = S.take<int>(n_surfaces);
    P4* d_nets = S.take<P4>((size_t)pts_net);
    float* d_knots = S.take<float>((size_t)n_knots);
    P4* d_strips = S.take<P4>((size_t)pts_strip);
    P4* d_cp = S.take<P4>((size_t)pts_cp);
    long long* d_off = S.take<long long>((size_t)N);
    int* d_deg = S.take<int>(2 * (size_t)N);
    int* d_surf = S.take<int>((size_t)N);
    int* d_err = S.take<int>(1);
    e = cudaMemcpy(d_sd, sd.data(), sd.size() * sizeof(SurfDesc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_line_u, line_u.data(), n_surfaces * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_line_v, line_v.data(), n_surfaces * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_patch0, patch0.data(), n_surfaces * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_nets, nets.get(), (size_t)pts_net * sizeof(P4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_knots, knots.get(), (size_t)n_knots * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_err, 0, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "scene build: upload");
    k_split_u<<<blocks_for(lines_u, 128), 128>>>(d_sd, d_line_u, n_surfaces, (int)lines_u, d_nets, d_knots, d_strips,
                                                 d_err);
    k_split_v<<<blocks_for(lines_v, 128), 128>>>(d_sd, d_line_v, n_surfaces, (int)lines_v, d_strips, d_knots, d_cp,
                                                 d_err);
    k_patch_meta<<<blocks_for(N, 256), 256>>>(d_sd, d_patch0, n_surfaces, (int)N, d_off, d_deg, d_surf);
    int h_err = 0;
    e = cudaMemcpy(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "scene build: decomposition");
    if (h_err) return fail(NRT_ERR_DEVICE, "scene build: decomposition gave an unexpected piece count");
    return build_from_device_patches(o, (int)N, n_surfaces, d_cp, d_off, d_deg, d_surf, n_floats, std::move(ps), out);
}

int build_scene_device_patches(const float* cp, const int32_t* cp_offset, const int32_t* degrees, int n_patches,
                               const nrt_build_opts& o, nrt_scene** out) {
    *out = nullptr;
    if (int st = check_build_opts(o)) return st;
    if (n_patches >= (1 << 27)) return fail(NRT_ERR_INVALID, "too many patches (%d)", n_patches);
    long long max_point = 0, n_floats = 0;
    std::vector<long long> off(n_patches);
    for (int k = 0; k < n_patches; ++k) {
        const int p = degrees[2 * k], q = degrees[2 * k + 1];
        if (p < 1 || q < 1 || p > NRT_MAX_DEGREE || q > NRT_MAX_DEGREE)
            return fail(NRT_ERR_INVALID, "patch %d has degree (%d,%d) outside 1..%d", k, p, q, NRT_MAX_DEGREE);
        if (cp_offset[k] < 0) return fail(NRT_ERR_INVALID, "negative control point offset");
        off[k] = cp_offset[k];
        max_point = std::max(max_point, (long long)cp_offset[k] + (p + 1) * (q + 1));
        n_floats += 4 * (long long)dev::padded_points(p, q);
    }
    if (n_floats >= (1LL << 31)) return fail(NRT_ERR_INVALID, "scene too large (%lld block floats)", n_floats);
    PatchSet ps;
    ps.ranges.assign(4 * (size_t)n_patches, 0.f);
    for (int k = 0; k < n_patches; ++k) { ps.ranges[4 * k + 1] = 1.f; ps.ranges[4 * k + 3] = 1.f; }
    ps.surf.assign(n_patches, 0);
    DeviceGuard dg(o.device);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t need = al((size_t)max_point * sizeof(P4)) + al((size_t)n_patches * sizeof(long long)) +
                        al(2 * (size_t)n_patches * sizeof(int)) + al((size_t)n_patches * sizeof(int)) + 256;
    Scratch S;
    cudaError_t e = cudaMalloc(&S.base, need);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(patch upload)");
    struct Guard {
        void* p;
        ~Guard() { cudaFree(p); }
    } guard{S.base};
    P4* d_cp = S.take<P4>((size_t)max_point);
    long long* d_off = S.take<long long>(n_patches);
    int* d_deg = S.take<int>(2 * (size_t)n_patches);
    int* d_surf = S.take<int>(n_patches);
    e = cudaMemcpy(d_cp, cp, (size_t)max_point * sizeof(P4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_off, off.data(), n_patches * sizeof(long long), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_deg, degrees, 2 * (size_t)n_patches * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_surf, 0, n_patches * sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "scene build: upload");
    return build_from_device_patches(o, n_patches, 1, d_cp, d_off, d_deg, d_surf, n_floats, std::move(ps), out);
}

}  // namespace nrt
