// kernels.h -- launchers of the engine's CUDA kernels (host-callable).
#pragma once

#include <cuda_runtime.h>

#include "device_scene.cuh"

// Every (p, q) with 1 <= p, q <= 7 gets its own specialised Newton.
#define NRT_FOR_EACH_DEGREE(X)                                                                             \
    X(1, 1) X(1, 2) X(1, 3) X(1, 4) X(1, 5) X(1, 6) X(1, 7) X(2, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 5) X(2, 6) \
    X(2, 7) X(3, 1) X(3, 2) X(3, 3) X(3, 4) X(3, 5) X(3, 6) X(3, 7) X(4, 1) X(4, 2) X(4, 3) X(4, 4) X(4, 5) \
    X(4, 6) X(4, 7) X(5, 1) X(5, 2) X(5, 3) X(5, 4) X(5, 5) X(5, 6) X(5, 7) X(6, 1) X(6, 2) X(6, 3) X(6, 4) \
    X(6, 5) X(6, 6) X(6, 7) X(7, 1) X(7, 2) X(7, 3) X(7, 4) X(7, 5) X(7, 6) X(7, 7)

namespace nrt {
namespace dev {

cudaError_t launch_intersect_pixel(const Scene& sc, const Rays& rays, long long n, const Opts& op, const Hits& out,
                                   unsigned long long* ctr, cudaStream_t stream);

struct CameraParams {
    double eye[3];
    double right[3], up[3], fwd[3];
    double x0, x1, y0, y1, tan_half;
    int width, height, spp;
    uint32_t seed;
};
cudaError_t launch_camera_rays(const CameraParams& cp, float* ox, float* oy, float* oz, float* dx, float* dy,
                               float* dz, cudaStream_t stream);
// Compacted diffuse bounce rays of the hits (scratch: (n + 255) / 256 + 1 ints).
cudaError_t launch_bounce_rays(const Rays& in, const int32_t* patch, const float* geom, long long n, uint32_t seed,
                               float offset, float* ox, float* oy, float* oz, float* dx, float* dy, float* dz,
                               int32_t* src, int32_t* scratch, cudaStream_t stream);

}  // namespace dev
}  // namespace nrt
