// refine_dev.cu -- curvature-driven refinement on the device
// (nrt_refine_surface_device): the refinement of refine.cpp
// (NurbsOps::curvatureRefinementU then V, src/math/nurbs.h:289-486) with its
// two costly parts as kernels, producing the same bits.
//
//  * Counts: one thread per (knot span, line of the net) evaluates the span's
//    count on that line (refine_math::knot_count, shared with the host); the
//    span's count is the maximum over lines (atomicMax).
//  * Insertions: the knots go in one at a time in ascending order by
//    Algorithm A5.1 (The NURBS Book, r = 1), one thread per line.  The host
//    walks the knot vector through the insertions once (the span k, the
//    multiplicity s and the p - s blending weights alpha, 1 - alpha of each
//    insertion depend on the knots only) and every line applies them.  An
//    insertion at span k rewrites points k-p+1 .. k-s and moves the rest one
//    place up; since insertions come in ascending order, each line keeps its
//    not-yet-reached points right-aligned at the end of a buffer of the final
//    length and pulls them forward only as insertions reach them, so an
//    insertion costs O(p) instead of O(n).  The blends are the same float
//    operations as A5.1's (alpha * R[i+1] + (1 - alpha) * R[i], no
//    contraction: this file is compiled with -fmad=false).
// Points are stored position-major ([position][line]), so the threads of a
// warp, which follow the same insertions, touch consecutive addresses.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "refine_math.h"
#include "scene_build.h"

namespace nrt {
namespace {

// One insertion: span k of the knot vector before it, the multiplicity s of
// the new knot there, and the blending weights of A5.1's loop.
struct InsertStep {
    int k, s;
    float alpha[NRT_MAX_DEGREE], beta[NRT_MAX_DEGREE];
};

__global__ void k_refine_counts(const float4* __restrict__ net, int len, int lines, const float* __restrict__ K,
                                int deg, float C, int* add) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int spans = len - deg;
    if (t >= (long long)spans * lines) return;
    const int i = deg + (int)(t / lines), l = (int)(t % lines);
    auto point = [&](int a) {
        const float4 q = net[(long long)a * lines + l];
        return refine_math::V3{q.x / q.w, q.y / q.w, q.z / q.w};
    };
    const int c = refine_math::knot_count(point, K, i, C, deg);
    if (c > 0) atomicMax(add + (i - deg), c);
}

// buf: (n_final + 1) positions x lines; on entry the line's n + 1 points sit at
// positions n_final - n .. n_final.
__global__ void k_refine_insert(float4* buf, int lines, int n, int n_final, int deg, const InsertStep* __restrict__ steps,
                                int n_steps) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= lines) return;
    auto B = [&](int pos) -> float4& { return buf[(long long)pos * lines + l]; };
    int h = 0;               // points [0, h) are the refined curve's head
    int tail = n_final - n;  // points [tail, n_final] are the original ones not yet reached
    for (int j = 0; j < n_steps; ++j) {
        const int k = steps[j].k, s = steps[j].s, L = k - deg + 1;
        while (h < k - s + 1) {  // bring the points this insertion reads into the head
            B(h) = B(tail);
            ++h;
            ++tail;
        }
        float4 R[NRT_MAX_DEGREE + 1];
        for (int i = 0; i <= deg - s; ++i) R[i] = B(k - deg + i);
        for (int i = 0; i <= deg - 1 - s; ++i) {
            const float a = steps[j].alpha[i], b = steps[j].beta[i];
            R[i] = make_float4(a * R[i + 1].x + b * R[i].x, a * R[i + 1].y + b * R[i].y, a * R[i + 1].z + b * R[i].z,
                               a * R[i + 1].w + b * R[i].w);
        }
        for (int i = h - 1; i >= k - s; --i) B(i + 1) = B(i);  // the points from k-s on move one place up
        for (int i = L; i <= k - s; ++i) B(i) = R[i - L];
        ++h;
    }
    while (tail <= n_final) {  // close the gap an insertion skipped by refine.cpp's rule leaves (else a no-op)
        B(h) = B(tail);
        ++h;
        ++tail;
    }
}

__global__ void k_transpose(const float4* __restrict__ in, float4* __restrict__ out, int rows, int cols) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)rows * cols) return;
    const int r = (int)(t / cols), c = (int)(t % cols);
    out[(long long)c * rows + r] = in[t];
}

}  // namespace
}  // namespace nrt

namespace nrt {
namespace {

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t bytes) {
        if (p) cudaFree(p);
        p = nullptr;
        return cudaMalloc(&p, bytes ? bytes : 1);
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

// One direction on the device.  net: len positions x lines, position-major;
// K: the knots of the direction (host, len + deg + 1 values), replaced by the
// refined ones; net is replaced by the refined net and len by its length.
int refine_dir_device(DevBuf& net, int& len, int lines, std::vector<float>& K, int deg, float C) {
    const int n = len - 1, spans = n - deg + 1;
    if (spans <= 0 || lines <= 0) return NRT_OK;
    DevBuf dK, dadd;
    cudaError_t e = dK.alloc(K.size() * sizeof(float));
    if (e == cudaSuccess) e = dadd.alloc(spans * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(dK.p, K.data(), K.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(dadd.p, 0, spans * sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "refinement set-up");
    const long long work = (long long)spans * lines;
    k_refine_counts<<<(unsigned)((work + 255) / 256), 256>>>(net.as<float4>(), len, lines, dK.as<float>(), deg, C,
                                                              dadd.as<int>());
    std::vector<int> add(spans);
    e = cudaMemcpy(add.data(), dadd.p, spans * sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "refinement counts");
    long long total = 0;
    for (int a : add) total += a;
    if (total == 0) return NRT_OK;
    if (n + total >= (1LL << 24)) return fail(NRT_ERR_INVALID, "refinement to %lld points per line", n + total);
    const int n_final = n + (int)total;
    // the knot vector through the insertions, on the host (as refine.cpp evolves it)
    std::vector<InsertStep> steps;
    steps.reserve((size_t)total);
    std::vector<float> U(K);
    int ncur = n;
    for (int i = deg; i <= n; ++i) {
        const int cnt = add[i - deg];
        const float lo = K[i], hi = K[i + 1];
        for (int j = 1; j <= cnt; ++j) {
            const float u = lo + (hi - lo) * j / (float)(cnt + 1);
            const int k = refine_math::find_span(ncur, deg, u, U.data());
            const int s = refine_math::multiplicity_at(U.data(), k, u);
            if (s >= deg) continue;  // as refine.cpp: A5.1's precondition
            InsertStep st{};
            st.k = k;
            st.s = s;
            const int L = k - deg + 1;
            for (int a = 0; a <= deg - 1 - s; ++a) {
                st.alpha[a] = (u - U[L + a]) / (U[a + k + 1] - U[L + a]);
                st.beta[a] = 1.0f - st.alpha[a];
            }
            steps.push_back(st);
            U.insert(U.begin() + k + 1, u);
            ++ncur;
        }
    }
    const int n_out = ncur;  // n_final unless an insertion was skipped (the kernel closes that gap)
    DevBuf out, dsteps;
    e = out.alloc((size_t)(n_final + 1) * lines * sizeof(float4));
    if (e == cudaSuccess) e = dsteps.alloc(steps.size() * sizeof(InsertStep));
    if (e == cudaSuccess)
        e = cudaMemcpy(dsteps.p, steps.data(), steps.size() * sizeof(InsertStep), cudaMemcpyHostToDevice);
    // the original points right-aligned
    if (e == cudaSuccess)
        e = cudaMemcpy(out.as<float4>() + (size_t)(n_final - n) * lines, net.p, (size_t)len * lines * sizeof(float4),
                       cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "refinement buffers");
    k_refine_insert<<<(unsigned)((lines + 127) / 128), 128>>>(out.as<float4>(), lines, n, n_final, deg,
                                                             dsteps.as<InsertStep>(), (int)steps.size());
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "refinement insertions");
    std::swap(net.p, out.p);  // the refined points are at positions 0 .. n_out
    len = n_out + 1;
    K.assign(U.begin(), U.begin() + n_out + deg + 2);
    return NRT_OK;
}

int refine_device(const nrt_nurbs_surface& s, float C, int device, std::vector<float4>& net_out,
                  std::vector<float>& U, std::vector<float>& V, int& n, int& m) {
    if (int st = check_surface(s)) return st;
    n = s.n;
    m = s.m;
    U.assign(s.u_knots, s.u_knots + n + s.p + 2);
    V.assign(s.v_knots, s.v_knots + m + s.q + 2);
    net_out.resize((size_t)(n + 1) * (m + 1));
    std::memcpy(net_out.data(), s.control_points, net_out.size() * sizeof(float4));
    if (!(C > 0.f)) return NRT_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    int st = NRT_OK;
    {
        DevBuf net, tmp;
        e = net.alloc(net_out.size() * sizeof(float4));
        if (e == cudaSuccess)
            e = cudaMemcpy(net.p, net_out.data(), net_out.size() * sizeof(float4), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = cuda_fail(e, "refinement upload");
        int rows = n + 1, cols = m + 1;
        // along u: the row-major net is position-major with one line per column
        if (st == NRT_OK) st = refine_dir_device(net, rows, cols, U, s.p, C);
        // along v: transposed, one line per row
        if (st == NRT_OK) {
            e = tmp.alloc((size_t)rows * cols * sizeof(float4));
            const long long t = (long long)rows * cols;
            if (e == cudaSuccess)
                k_transpose<<<(unsigned)((t + 255) / 256), 256>>>(net.as<float4>(), tmp.as<float4>(), rows, cols);
            if (e != cudaSuccess) st = cuda_fail(e, "refinement transpose");
            std::swap(net.p, tmp.p);
        }
        if (st == NRT_OK) st = refine_dir_device(net, cols, rows, V, s.q, C);
        if (st == NRT_OK) {
            e = tmp.alloc((size_t)rows * cols * sizeof(float4));
            const long long t = (long long)rows * cols;
            if (e == cudaSuccess)
                k_transpose<<<(unsigned)((t + 255) / 256), 256>>>(net.as<float4>(), tmp.as<float4>(), cols, rows);
            net_out.resize((size_t)rows * cols);
            if (e == cudaSuccess)
                e = cudaMemcpy(net_out.data(), tmp.p, net_out.size() * sizeof(float4), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) st = cuda_fail(e, "refinement read-back");
        }
        n = rows - 1;
        m = cols - 1;
    }
    cudaSetDevice(prev);
    return st;
}

}  // namespace
}  // namespace nrt

extern "C" int nrt_refine_surface_device(const nrt_nurbs_surface* surf, float C, int device, float* cp_out,
                                         int64_t cap_points, float* u_knots_out, int cap_u, float* v_knots_out,
                                         int cap_v, int* n_out, int* m_out) {
    if (!surf || !n_out || !m_out) return nrt::fail(NRT_ERR_INVALID, "null argument");
    std::vector<float4> net;
    std::vector<float> U, V;
    int n = 0, m = 0;
    if (int st = nrt::refine_device(*surf, C, device, net, U, V, n, m)) return st;
    *n_out = n;
    *m_out = m;
    if (!cp_out || !u_knots_out || !v_knots_out || (int64_t)net.size() > cap_points || (int64_t)U.size() > cap_u ||
        (int64_t)V.size() > cap_v)
        return nrt::fail(NRT_ERR_INVALID, "outputs too small for the refined surface (n = %d, m = %d: %zu points)", n,
                         m, net.size());
    std::memcpy(cp_out, net.data(), net.size() * sizeof(float4));
    std::memcpy(u_knots_out, U.data(), U.size() * sizeof(float));
    std::memcpy(v_knots_out, V.data(), V.size() * sizeof(float));
    return NRT_OK;
}
