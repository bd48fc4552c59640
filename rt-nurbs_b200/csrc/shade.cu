// shade.cu -- the output stage after intersection, headless: framebuffers
// from hit records (the reference's debug shading, src/gpu/testShading.cu:9-55),
// the per-ray error measures of its benchmark (src/core/benchmark.cpp:206-222)
// and a PPM writer (benchmark.cpp:82-120).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "kernels.h"
#include "nrt_internal.h"

namespace nrt {
namespace dev {

// mode 0: hit mask in red (redTestShading, testShading.cu:9-24);
// mode 1: (n + 1) / 2 with n = normalize(dS/dv x dS/du) (normalsTestShading,
// testShading.cu:27-55), black where the ray missed.
__global__ void __launch_bounds__(256) k_shade(const int32_t* __restrict__ patch, const float* __restrict__ geom,
                                               long long n, int mode, float* __restrict__ r, float* __restrict__ g,
                                               float* __restrict__ b) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const bool hit = patch[i] >= 0;
        float cr = 0.f, cg = 0.f, cb = 0.f;
        if (mode == 0) {
            cr = hit ? 1.f : 0.f;
        } else if (hit) {
            const float* q = geom + 9 * i;
            const float ux = q[3], uy = q[4], uz = q[5], vx = q[6], vy = q[7], vz = q[8];
            float nx = vy * uz - vz * uy, ny = vz * ux - vx * uz, nz = vx * uy - vy * ux;
            const float l = sqrtf(nx * nx + ny * ny + nz * nz);
            if (l > 0.f) { nx /= l; ny /= l; nz /= l; }
            cr = (nx + 1.f) * 0.5f;
            cg = (ny + 1.f) * 0.5f;
            cb = (nz + 1.f) * 0.5f;
        }
        r[i] = cr;
        g[i] = cg;
        b[i] = cb;
    }
}

// Per ray, against a reference hit set: the distance between the two hit
// points projected to pixels, |P_ref - P_test| * cam_k / t_ref, and the angle
// between the two normals in degrees (benchmark.cpp:206-222); NaN unless both
// hit; mismatch[i] = 1 where exactly one of them hit.
__global__ void __launch_bounds__(256) k_compare_hits(Rays rays, const int32_t* __restrict__ pr,
                                                      const float* __restrict__ tr, const float* __restrict__ gr,
                                                      const int32_t* __restrict__ pt, const float* __restrict__ tt,
                                                      const float* __restrict__ gt, long long n, float cam_k,
                                                      float* __restrict__ px_err, float* __restrict__ deg_err,
                                                      int32_t* __restrict__ mismatch) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const bool hr = pr[i] >= 0, ht = pt[i] >= 0;
        mismatch[i] = hr != ht;
        if (!(hr && ht)) {
            px_err[i] = NAN;
            deg_err[i] = NAN;
            continue;
        }
        const float dx = rays.dx[i], dy = rays.dy[i], dz = rays.dz[i];
        const float a = tr[i], c = tt[i];
        const float ex = (a - c) * dx, ey = (a - c) * dy, ez = (a - c) * dz;
        px_err[i] = a > 0.f ? sqrtf(ex * ex + ey * ey + ez * ez) * cam_k / a : 0.f;
        float n1[3], n2[3];
        const float* q[2] = {gr + 9 * i, gt + 9 * i};
        float* nn[2] = {n1, n2};
        for (int k = 0; k < 2; ++k) {
            const float ux = q[k][3], uy = q[k][4], uz = q[k][5], vx = q[k][6], vy = q[k][7], vz = q[k][8];
            float x = uy * vz - uz * vy, y = uz * vx - ux * vz, z = ux * vy - uy * vx;
            const float l = sqrtf(x * x + y * y + z * z);
            if (l > 0.f) { x /= l; y /= l; z /= l; }
            nn[k][0] = x; nn[k][1] = y; nn[k][2] = z;
        }
        // atan2(|n1 x n2|, |n1 . n2|): accurate near zero, where acos of the dot product is not
        const float cx = n1[1] * n2[2] - n1[2] * n2[1], cy = n1[2] * n2[0] - n1[0] * n2[2],
                    cz = n1[0] * n2[1] - n1[1] * n2[0];
        const float d = n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2];
        deg_err[i] = atan2f(sqrtf(cx * cx + cy * cy + cz * cz), fabsf(d)) * (180.f / 3.14159265358979f);
    }
}

}  // namespace dev
}  // namespace nrt

extern "C" {

int nrt_shade(const nrt_hits* hits, int64_t n, int mode, float* r, float* g, float* b, void* stream) {
    if (!hits || !hits->patch || !r || !g || !b) return nrt::fail(NRT_ERR_INVALID, "null argument");
    if (mode != 0 && mode != 1) return nrt::fail(NRT_ERR_INVALID, "shade mode %d is neither 0 (hit mask) nor 1 (normals)", mode);
    if (mode == 1 && !hits->geom) return nrt::fail(NRT_ERR_INVALID, "normal shading needs hits->geom");
    if (n <= 0) return NRT_OK;
    const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 32);
    nrt::dev::k_shade<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(hits->patch, hits->geom, n, mode,
                                                                                      r, g, b);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NRT_OK : nrt::fail(NRT_ERR_CUDA, "shade launch: %s", cudaGetErrorString(e));
}

int nrt_compare_hits(const nrt_rays* rays, const nrt_hits* ref, const nrt_hits* test, int64_t n, float cam_k,
                     float* px_err, float* deg_err, int32_t* mismatch, void* stream) {
    if (!rays || !ref || !test || !px_err || !deg_err || !mismatch) return nrt::fail(NRT_ERR_INVALID, "null argument");
    if (!ref->patch || !ref->t || !ref->geom || !test->patch || !test->t || !test->geom)
        return nrt::fail(NRT_ERR_INVALID, "hit comparison needs patch, t and geom of both hit sets");
    if (n <= 0) return NRT_OK;
    const nrt::dev::Rays r{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz};
    const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 32);
    nrt::dev::k_compare_hits<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        r, ref->patch, ref->t, ref->geom, test->patch, test->t, test->geom, n, cam_k, px_err, deg_err, mismatch);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NRT_OK : nrt::fail(NRT_ERR_CUDA, "compare launch: %s", cudaGetErrorString(e));
}

int nrt_write_ppm(const char* path, int width, int height, const float* r, const float* g, const float* b) {
    if (!path || !r || !g || !b || width <= 0 || height <= 0) return nrt::fail(NRT_ERR_INVALID, "bad argument");
    const size_t n = (size_t)width * height;
    std::vector<unsigned char> rgb(3 * n);
    auto byte = [](float c) { return (unsigned char)((c < 0.f ? 0.f : (c > 1.f ? 1.f : c)) * 255.999f); };
    for (size_t i = 0; i < n; ++i) {
        rgb[3 * i] = byte(r[i]);
        rgb[3 * i + 1] = byte(g[i]);
        rgb[3 * i + 2] = byte(b[i]);
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return nrt::fail(NRT_ERR_INVALID, "cannot open %s", path);
    std::fprintf(f, "P6\n%d %d\n255\n", width, height);
    const size_t w = std::fwrite(rgb.data(), 1, rgb.size(), f);
    std::fclose(f);
    return w == rgb.size() ? NRT_OK : nrt::fail(NRT_ERR_INVALID, "short write to %s", path);
}

}  // extern "C"
