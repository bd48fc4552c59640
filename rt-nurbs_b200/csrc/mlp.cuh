// mlp.cuh -- the learned initial guess: features of a (ray, patch) pair and a
// 12 -> 64 -> 64 -> 2 MLP (SiLU) on BF16 tensor cores with FP32 accumulation.
//
// Features (12), all dimensionless, in the patch frame:
//   0-2  where the ray enters the patch's slab |h| <= H (clipped to its box)
//   3-5  where it leaves the slab (same clipping); h is given as h/H
//   6-8  ray direction, normalised
//   9,10 p/7, q/7
//   11   slab half-thickness H over the frame size (a flatness measure, the
//        role of patchDelta in src/core/main.cpp:18-43)
// The patch frame maps a point X to (s, t, h) with X = o + s*A + t*B + h*N:
// A and B are the tangents dS/du and dS/dv at the patch centre (u, v) =
// (1/2, 1/2), N the normal of A x B scaled by sqrt|A x B|, and
// o = S(1/2, 1/2) - A/2 - B/2, so that (s, t) equals (u, v) to first order
// (where the ray crosses the tangent plane is one Newton step from the
// midpoint) and the hit lies between the entry and exit points.  The network
// maps the features to a starting (u, v).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "patch_math.cuh"

namespace nrt {
namespace dev {

constexpr int kMlpIn = 12, kMlpInPad = 16, kMlpHidden = 64, kMlpOut = 2, kMlpOutPad = 8;
constexpr int kMlpLd = kMlpHidden + 8;    // padded row of hidden activations in shared memory (bf16)
constexpr int kMlpLdIn = kMlpInPad + 8;   // padded row of inputs

// Per patch slot: frame origin (patch-local coordinates), inverse frame
// (row-major 3x3), box in patch-local coordinates, flatness feature.
struct __align__(16) PatchFrame {
    float ox, oy, oz, flat;
    float m[9];
    float slab, pad1, pad2;   // slab: half-thickness H of the control net in h
    float lo[3], hi_x;
    float hi_y, hi_z, pad3, pad4;
};
static_assert(sizeof(PatchFrame) == 96, "PatchFrame layout");

// Device parameters: bf16 weights stored transposed (row n holds the weights
// into output n), FP32 biases.  One contiguous blob.
struct MlpParams {
    const __nv_bfloat16* w1t;  // [64][16]  (inputs 12..15 zero)
    const __nv_bfloat16* w2t;  // [64][64]
    const __nv_bfloat16* w3t;  // [8][64]   (outputs 2..7 zero)
    const float* b1;           // [64]
    const float* b2;           // [64]
    const float* b3;           // [8]
};

__device__ __forceinline__ float silu(float x) { return x / (1.f + __expf(-x)); }
// Inference: x * sigmoid(x) = h + h * tanh(h) with h = x / 2, on the hardware
// tanh approximation (relative error about 2^-11, below the BF16 rounding of
// the stored activation).
__device__ __forceinline__ float silu_fast(float x) {
    const float h = 0.5f * x;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
    return fmaf(h, t, h);
}
__device__ __forceinline__ float dsilu_f(float z) {
    const float s = 1.f / (1.f + __expf(-z));
    return s * (1.f + z * (1.f - s));
}

__device__ __forceinline__ void features(const PatchFrame& f, int p, int q, const RayFrame& r, const PatchRay& pr,
                                         double cx, double cy, double cz, float (&x)[kMlpIn]) {
    // ray origin in patch-local coordinates (FP64 difference, then rounded)
    const float lox = (float)((double)r.ox - cx), loy = (float)((double)r.oy - cy), loz = (float)((double)r.oz - cz);
    const float rdx = __frcp_rn(r.dx), rdy = __frcp_rn(r.dy), rdz = __frcp_rn(r.dz);
    const float t0x = (f.lo[0] - lox) * rdx, t1x = (f.hi_x - lox) * rdx;
    const float t0y = (f.lo[1] - loy) * rdy, t1y = (f.hi_y - loy) * rdy;
    const float t0z = (f.lo[2] - loz) * rdz, t1z = (f.hi_z - loz) * rdz;
    float bin = fmaxf(fmaxf(fminf(t0x, t1x), fmaxf(fminf(t0y, t1y), fminf(t0z, t1z))), 0.f);
    float bout = fminf(fmaxf(t0x, t1x), fminf(fmaxf(t0y, t1y), fmaxf(t0z, t1z)));
    if (!(bout >= bin)) {  // grazing the box: the point of closest approach to its centre
        bin = fmaxf(-(lox * r.dx + loy * r.dy + loz * r.dz), 0.f);
        bout = bin;
    }
    // origin and direction in the frame
    const float ax = lox - f.ox, ay = loy - f.oy, az = loz - f.oz;
    const float os = f.m[0] * ax + f.m[1] * ay + f.m[2] * az;
    const float ot = f.m[3] * ax + f.m[4] * ay + f.m[5] * az;
    const float oh = f.m[6] * ax + f.m[7] * ay + f.m[8] * az;
    const float ds = f.m[0] * r.dx + f.m[1] * r.dy + f.m[2] * r.dz;
    const float dt = f.m[3] * r.dx + f.m[4] * r.dy + f.m[5] * r.dz;
    const float dh = f.m[6] * r.dx + f.m[7] * r.dy + f.m[8] * r.dz;
    // the slab |h| <= H, clipped to the box segment
    float tin = bin, tout = bout;
    if (fabsf(dh) > 1e-20f) {
        const float ta = (-f.slab - oh) / dh, tb = (f.slab - oh) / dh;
        const float sin_ = fmaxf(fminf(ta, tb), bin), sout = fminf(fmaxf(ta, tb), bout);
        if (sout >= sin_) { tin = sin_; tout = sout; }
    }
    const float ih = 1.f / fmaxf(f.slab, 1e-30f);
    x[0] = os + tin * ds;
    x[1] = ot + tin * dt;
    x[2] = (oh + tin * dh) * ih;
    x[3] = os + tout * ds;
    x[4] = ot + tout * dt;
    x[5] = (oh + tout * dh) * ih;
    const float il = rsqrtf(fmaxf(ds * ds + dt * dt + dh * dh, 1e-30f));
    x[6] = ds * il;
    x[7] = dt * il;
    x[8] = dh * il;
    x[9] = (float)p * (1.f / 7.f);
    x[10] = (float)q * (1.f / 7.f);
    x[11] = f.flat;
#pragma unroll
    for (int k = 0; k < 6; ++k) x[k] = fminf(fmaxf(x[k], -8.f), 8.f);  // keep far-outside inputs bounded
}

// Forward + backward of one training batch on the tcgen05 tensor cores
// (mlp_tc.cu): gradients added to grad (public parameter order), the batch
// loss to *loss; *err set if a tensor-core step did not complete.
cudaError_t launch_mlp_fwd_bwd_tc(const MlpParams& P, const float* X, const float* T, const int32_t* perm,
                                  long long begin, long long count, float inv_batch, float* grad, float* loss, int* err,
                                  cudaStream_t st);

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Shared memory of one block for inference (dynamic shared memory, about
// 65 KB for 8 warps): weights (transposed, padded rows) and per-warp tiles.
struct MlpSmem {
    __nv_bfloat16 w1t[kMlpHidden][kMlpLdIn];
    __nv_bfloat16 w2t[kMlpHidden][kMlpLd];
    __nv_bfloat16 w3t[kMlpOutPad][kMlpLd];
    float b1[kMlpHidden], b2[kMlpHidden], b3[kMlpOutPad];
    __nv_bfloat16 x[8][32][kMlpLdIn];   // per warp: inputs
    __nv_bfloat16 h[8][32][kMlpLd];     // per warp: hidden activations (reused by both layers)
    float y[8][32][2];
};

// All threads of the block: copy the parameters into shared memory.
__device__ __forceinline__ void mlp_load(MlpSmem& s, const MlpParams& P) {
    for (int k = threadIdx.x; k < kMlpHidden * kMlpInPad; k += blockDim.x)
        s.w1t[k / kMlpInPad][k % kMlpInPad] = P.w1t[k];
    for (int k = threadIdx.x; k < kMlpHidden * kMlpHidden; k += blockDim.x)
        s.w2t[k / kMlpHidden][k % kMlpHidden] = P.w2t[k];
    for (int k = threadIdx.x; k < kMlpOutPad * kMlpHidden; k += blockDim.x)
        s.w3t[k / kMlpHidden][k % kMlpHidden] = P.w3t[k];
    for (int k = threadIdx.x; k < kMlpHidden; k += blockDim.x) {
        s.b1[k] = P.b1[k];
        s.b2[k] = P.b2[k];
    }
    for (int k = threadIdx.x; k < kMlpOutPad; k += blockDim.x) s.b3[k] = P.b3[k];
}

// One dense layer for the warp's 32 rows: out[32][N] = act(in[32][K] * W + b),
// written back as bf16 into `out` (row stride kMlpLd).  K in {16, 64}.
template <int K, int LDA, int N, bool ACT>
__device__ __forceinline__ void mlp_layer(const __nv_bfloat16 (*in)[LDA], const __nv_bfloat16 (*wt)[LDA],
                                          const float* bias, __nv_bfloat16 (*out)[kMlpLd], float (*yout)[2], int lane) {
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
        for (int nt = 0; nt < N / 8; ++nt) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ks = 0; ks < K / 16; ++ks) {
                const int r0 = mt * 16, c0 = ks * 16;
                const uint32_t a0 = *reinterpret_cast<const uint32_t*>(&in[r0 + g][c0 + 2 * t]);
                const uint32_t a1 = *reinterpret_cast<const uint32_t*>(&in[r0 + g + 8][c0 + 2 * t]);
                const uint32_t a2 = *reinterpret_cast<const uint32_t*>(&in[r0 + g][c0 + 2 * t + 8]);
                const uint32_t a3 = *reinterpret_cast<const uint32_t*>(&in[r0 + g + 8][c0 + 2 * t + 8]);
                const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&wt[nt * 8 + g][c0 + 2 * t]);
                const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&wt[nt * 8 + g][c0 + 2 * t + 8]);
                mma_bf16(d, a0, a1, a2, a3, b0, b1);
            }
            const int col = nt * 8 + 2 * t, row = mt * 16 + g;
            const float v0 = d[0] + bias[col], v1 = d[1] + bias[col + 1];
            const float v2 = d[2] + bias[col], v3 = d[3] + bias[col + 1];
            if (ACT) {
                *reinterpret_cast<uint32_t*>(&out[row][col]) = pack_bf16(silu_fast(v0), silu_fast(v1));
                *reinterpret_cast<uint32_t*>(&out[row + 8][col]) = pack_bf16(silu_fast(v2), silu_fast(v3));
            } else if (col == 0) {  // the two real outputs live in columns 0 and 1
                yout[row][0] = v0;
                yout[row][1] = v1;
                yout[row + 8][0] = v2;
                yout[row + 8][1] = v3;
            }
        }
    }
}

// Warp-synchronous inference: every lane of the warp passes its features and
// receives the network's raw (u, v).  All 32 lanes must call it together.
__device__ __forceinline__ void mlp_infer_warp(MlpSmem& s, int warp, int lane, const float (&x)[kMlpIn], float& u,
                                               float& v) {
#pragma unroll
    for (int k = 0; k < kMlpInPad; k += 2)
        *reinterpret_cast<uint32_t*>(&s.x[warp][lane][k]) =
            pack_bf16(k < kMlpIn ? x[k] : 0.f, k + 1 < kMlpIn ? x[k + 1] : 0.f);
    __syncwarp();
    mlp_layer<kMlpInPad, kMlpLdIn, kMlpHidden, true>(s.x[warp], s.w1t, s.b1, s.h[warp], nullptr, lane);
    __syncwarp();
    // layer 2 reads h and writes h in place, one 16-row block at a time: a
    // block's products only read its own rows, so its accumulators (32 floats
    // per lane) are written back once every lane has read those rows.
    __nv_bfloat16 (*h)[kMlpLd] = s.h[warp];
    {
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            float acc[8][4];
            const int r0 = mt * 16;
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
                for (int ks = 0; ks < 4; ++ks) {
                    const int c0 = ks * 16;
                    const uint32_t a0 = *reinterpret_cast<const uint32_t*>(&h[r0 + g][c0 + 2 * t]);
                    const uint32_t a1 = *reinterpret_cast<const uint32_t*>(&h[r0 + g + 8][c0 + 2 * t]);
                    const uint32_t a2 = *reinterpret_cast<const uint32_t*>(&h[r0 + g][c0 + 2 * t + 8]);
                    const uint32_t a3 = *reinterpret_cast<const uint32_t*>(&h[r0 + g + 8][c0 + 2 * t + 8]);
                    const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&s.w2t[nt * 8 + g][c0 + 2 * t]);
                    const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&s.w2t[nt * 8 + g][c0 + 2 * t + 8]);
                    mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
                }
            }
            __syncwarp();
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int col = nt * 8 + 2 * t, row = r0 + g;
                *reinterpret_cast<uint32_t*>(&h[row][col]) =
                    pack_bf16(silu_fast(acc[nt][0] + s.b2[col]), silu_fast(acc[nt][1] + s.b2[col + 1]));
                *reinterpret_cast<uint32_t*>(&h[row + 8][col]) =
                    pack_bf16(silu_fast(acc[nt][2] + s.b2[col]), silu_fast(acc[nt][3] + s.b2[col + 1]));
            }
        }
    }
    __syncwarp();
    mlp_layer<kMlpHidden, kMlpLd, kMlpOutPad, false>(h, s.w3t, s.b3, nullptr, s.y[warp], lane);
    __syncwarp();
    u = s.y[warp][lane][0];
    v = s.y[warp][lane][1];
    __syncwarp();
}

}  // namespace dev
}  // namespace nrt
