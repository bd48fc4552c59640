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

}  // namespace dev
}  // namespace nrt
