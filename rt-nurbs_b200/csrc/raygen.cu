// raygen.cu -- pinhole primary rays into a SoA ray queue.
//
// The reference builds pbrt-style camera matrices on the host
// (CameraOps::init_camera / getPerspectiveCamera, src/core/camera.h:63-141) and
// evaluates calculateRay<perspective_projection> per pixel
// (src/core/camera.h:162-174, src/gpu/generateRaysKernel.cu:15-35).  Reduced to
// closed form that is: screen window [-a,a]x[-1,1] (a = W/H >= 1), camera-space
// direction normalize(sx*tan(fov/2), sy*tan(fov/2), 1), rotated by
// [right | up' | forward] of Transform::lookAt (src/math/transform.h:46-60),
// origin at the eye.  It is evaluated here in FP64 with unfused operations and
// rounded once to float.
#include <cuda_runtime.h>

#include "kernels.h"

namespace nrt {
namespace dev {

__global__ void __launch_bounds__(256) k_camera_rays(CameraParams cp, float* __restrict__ ox, float* __restrict__ oy,
                                                     float* __restrict__ oz, float* __restrict__ dx,
                                                     float* __restrict__ dy, float* __restrict__ dz) {
    const long long total = (long long)cp.width * cp.height * cp.spp;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < total;
         r += (long long)gridDim.x * blockDim.x) {
        const long long pix = r / cp.spp;
        const int px = (int)(pix % cp.width), py = (int)(pix / cp.width);
        double jx = 0.5, jy = 0.5;
        if (cp.spp > 1) {
            uint32_t h = pcg_hash(cp.seed ^ pcg_hash((uint32_t)r));
            jx = (double)(h >> 8) * (1.0 / 16777216.0);
            h = pcg_hash(h);
            jy = (double)(h >> 8) * (1.0 / 16777216.0);
        }
        const double sx = __dadd_rn(cp.x0, __ddiv_rn(__dmul_rn(__dadd_rn((double)px, jx), __dsub_rn(cp.x1, cp.x0)),
                                                     (double)cp.width));
        const double sy = __dsub_rn(cp.y1, __ddiv_rn(__dmul_rn(__dadd_rn((double)py, jy), __dsub_rn(cp.y1, cp.y0)),
                                                     (double)cp.height));
        const double cx = __dmul_rn(sx, cp.tan_half), cy = __dmul_rn(sy, cp.tan_half);
        const double len = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), 1.0));
        const double il = __ddiv_rn(1.0, len);
        const double ux = __dmul_rn(cx, il), uy = __dmul_rn(cy, il), uz = __dmul_rn(1.0, il);
        const double wx = __dadd_rn(__dadd_rn(__dmul_rn(cp.right[0], ux), __dmul_rn(cp.up[0], uy)), __dmul_rn(cp.fwd[0], uz));
        const double wy = __dadd_rn(__dadd_rn(__dmul_rn(cp.right[1], ux), __dmul_rn(cp.up[1], uy)), __dmul_rn(cp.fwd[1], uz));
        const double wz = __dadd_rn(__dadd_rn(__dmul_rn(cp.right[2], ux), __dmul_rn(cp.up[2], uy)), __dmul_rn(cp.fwd[2], uz));
        ox[r] = (float)cp.eye[0];
        oy[r] = (float)cp.eye[1];
        oz[r] = (float)cp.eye[2];
        dx[r] = (float)wx;
        dy[r] = (float)wy;
        dz[r] = (float)wz;
    }
}

cudaError_t launch_camera_rays(const CameraParams& cp, float* ox, float* oy, float* oz, float* dx, float* dy,
                               float* dz, cudaStream_t stream) {
    const long long total = (long long)cp.width * cp.height * cp.spp;
    if (total <= 0) return cudaSuccess;
    const int threads = 256;
    long long blocks = (total + threads - 1) / threads;
    if (blocks > 148LL * 64) blocks = 148LL * 64;
    k_camera_rays<<<(unsigned)blocks, threads, 0, stream>>>(cp, ox, oy, oz, dx, dy, dz);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Diffuse bounce rays from hits, compacted in ray order (deterministic):
// count hits per block of 256, scan the block counts, then every hit writes
// its bounce ray at (block offset + rank within the block).
__global__ void __launch_bounds__(256) k_bounce_count(const int32_t* __restrict__ patch, long long n,
                                                      int32_t* __restrict__ block_counts) {
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    const int hit = (i < n && patch[i] >= 0) ? 1 : 0;
    const int c = __syncthreads_count(hit);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = c;
}

// In-place exclusive scan of nb block counts; total into block_counts[nb].
__global__ void __launch_bounds__(1024) k_bounce_scan(int32_t* block_counts, int nb) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int per = (nb + 1023) / 1024;
    const int a = min(nb, t * per), b = min(nb, a + per);
    int s = 0;
    for (int k = a; k < b; ++k) s += block_counts[k];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - s;
    for (int k = a; k < b; ++k) {
        const int c = block_counts[k];
        block_counts[k] = run;
        run += c;
    }
    if (t == 1023) block_counts[nb] = part[1023];
}

// Shading normal n = normalize(dS/dv x dS/du) (the reference's convention,
// src/gpu/testShading.cu:46), turned against the incoming direction; a
// cosine-weighted direction about n (Malley: a uniform disk point lifted to
// the hemisphere) from a PCG hash of (seed, ray index); origin S + offset n.
__global__ void __launch_bounds__(256) k_bounce_write(Rays in, const int32_t* __restrict__ patch,
                                                      const float* __restrict__ geom, long long n,
                                                      const int32_t* __restrict__ block_offsets, uint32_t seed,
                                                      float offset, float* __restrict__ ox, float* __restrict__ oy,
                                                      float* __restrict__ oz, float* __restrict__ dx,
                                                      float* __restrict__ dy, float* __restrict__ dz,
                                                      int32_t* __restrict__ src) {
    __shared__ int warp_base[8];
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    const bool hit = i < n && patch[i] >= 0;
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) warp_base[warp] = __popc(m);
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w) before += warp_base[w];
    if (!hit) return;
    const long long k = (long long)block_offsets[blockIdx.x] + before + __popc(m & ((1u << lane) - 1));
    const float* g = geom + 9 * i;
    const float sx = g[0], sy = g[1], sz = g[2];
    const float ux = g[3], uy = g[4], uz = g[5], vx = g[6], vy = g[7], vz = g[8];
    float nx = vy * uz - vz * uy, ny = vz * ux - vx * uz, nz = vx * uy - vy * ux;
    const float nl = sqrtf(nx * nx + ny * ny + nz * nz);
    const float rdx = in.dx[i], rdy = in.dy[i], rdz = in.dz[i];
    if (nl > 0.f) {
        nx /= nl; ny /= nl; nz /= nl;
    } else {  // degenerate tangents: bounce straight back
        const float rl = sqrtf(rdx * rdx + rdy * rdy + rdz * rdz);
        nx = -rdx / rl; ny = -rdy / rl; nz = -rdz / rl;
    }
    if (nx * rdx + ny * rdy + nz * rdz > 0.f) { nx = -nx; ny = -ny; nz = -nz; }
    // orthonormal basis about n (Duff et al. 2017, branchless)
    const float sgn = copysignf(1.f, nz);
    const float a = -1.f / (sgn + nz), b = nx * ny * a;
    const float t1x = 1.f + sgn * nx * nx * a, t1y = sgn * b, t1z = -sgn * nx;
    const float t2x = b, t2y = sgn + ny * ny * a, t2z = -ny;
    uint32_t h = pcg_hash(seed ^ pcg_hash((uint32_t)i));
    const float r1 = (float)(h >> 8) * (1.f / 16777216.f);
    h = pcg_hash(h);
    const float r2 = (float)(h >> 8) * (1.f / 16777216.f);
    const float rad = sqrtf(r1), phi = 6.2831853071795865f * r2;
    float sp, cp;
    sincosf(phi, &sp, &cp);
    const float lx = rad * cp, ly = rad * sp, lz = sqrtf(fmaxf(0.f, 1.f - r1));
    float wx = lx * t1x + ly * t2x + lz * nx, wy = lx * t1y + ly * t2y + lz * ny, wz = lx * t1z + ly * t2z + lz * nz;
    const float wl = sqrtf(wx * wx + wy * wy + wz * wz);
    wx /= wl; wy /= wl; wz /= wl;
    ox[k] = sx + offset * nx;
    oy[k] = sy + offset * ny;
    oz[k] = sz + offset * nz;
    dx[k] = wx;
    dy[k] = wy;
    dz[k] = wz;
    src[k] = (int32_t)i;
}

cudaError_t launch_bounce_rays(const Rays& in, const int32_t* patch, const float* geom, long long n, uint32_t seed,
                               float offset, float* ox, float* oy, float* oz, float* dx, float* dy, float* dz,
                               int32_t* src, int32_t* scratch, cudaStream_t stream) {
    const int nb = (int)((n + 255) / 256);
    k_bounce_count<<<nb, 256, 0, stream>>>(patch, n, scratch);
    k_bounce_scan<<<1, 1024, 0, stream>>>(scratch, nb);
    k_bounce_write<<<nb, 256, 0, stream>>>(in, patch, geom, n, scratch, seed, offset, ox, oy, oz, dx, dy, dz, src);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace nrt
