// mlp_tc.cu -- forward and backward of the learned guess's MLP
// (12 -> 64 -> 64 -> 2, SiLU, mean-squared error) for training, on the
// Blackwell tensor cores: tcgen05.mma kind::f16 with BF16 operands in the
// CTA's own shared memory and FP32 accumulators in tensor memory (TMEM), one
// 128-sample tile per step, one CTA of 4 warps (thread r owns sample row r of
// the tile).  The rounding points are those of the CPU oracle
// (oracle/mlp_oracle.py) and of the mma.sync inference path: every tensor-core
// operand is BF16 (inputs, weights, activations, output and hidden
// gradients); pre-activations, biases, bias gradients and the weight-gradient
// accumulation are FP32.
//
// Per tile, the GEMMs (M = 128 rows, K in steps of 16):
//   forward   Z1 = X W1^T (K 16), H1 = silu(Z1 + b1); Z2 = H1 W2^T (K 64),
//             H2 = silu(Z2 + b2); Y = H2 W3^T + b3 (N 16, 2 used)
//   backward  dY = 2 (Y - T) / B; dH2 = dY W3 (K 16); dZ2 = dH2 silu'(Z2);
//             dH1 = dZ2 W2 (K 64); dZ1 = dH1 silu'(Z1)
//   gradients dW3^T += H2^T dY, dW2^T += H1^T dZ2, dW1 += dZ1^T X (K = the 128
//             samples), accumulated in TMEM over all tiles of the CTA and
//             added to the global gradient once at the end.
// The weight-gradient GEMMs have 64 useful rows; they run with M = 128 and
// rows 64..127 read whatever follows their operand in shared memory (the
// layout below puts 18 KB of other operands there), and those rows of the
// result are never read.  Every operand is K-major (tc05.cuh); the operands
// whose K is the sample index are written transposed by the epilogues, with
// core matrices 144 bytes apart along K so that the 32 rows a warp writes at
// once fall in different banks.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "mlp.cuh"
#include "nrt_internal.h"
#include "tc05.cuh"

namespace nrt {
namespace dev {
namespace {

using tc05::kmajor_offset;

// Public parameter order: W1[64][12], b1[64], W2[64][64], b2[64], W3[2][64], b3[2].
constexpr int kW1 = 0, kB1 = kW1 + 64 * 12, kW2 = kB1 + 64, kB2 = kW2 + 64 * 64, kW3 = kB2 + 64, kB3 = kW3 + 2 * 64;
static_assert(kB3 + 2 == NRT_MLP_PARAMS, "parameter order");

// Operands whose K is the 128 samples: core matrices 144 bytes apart along K
// (LBO), 8-row groups 2304 bytes apart (SBO).
constexpr uint32_t kTLbo = 144, kTSbo = 2304;
__device__ __forceinline__ uint32_t tpos(int r, int s) {  // element (row r, sample s)
    return (uint32_t)((r >> 3) * kTSbo + (s >> 3) * kTLbo + (r & 7) * 16 + (s & 7) * 2);
}

// Shared-memory layout (bytes from a 1024-aligned base).
constexpr uint32_t kOffW1 = 0;                        // [64 out][16 in]      B of Z1
constexpr uint32_t kOffW2 = kOffW1 + 64 * 16 * 2;     // [64 out][64 in]      B of Z2
constexpr uint32_t kOffW3 = kOffW2 + 64 * 64 * 2;     // [16 out][64 in]      B of Y
constexpr uint32_t kOffW2T = kOffW3 + 16 * 64 * 2;    // [64 in][64 out]      B of dH1
constexpr uint32_t kOffW3T = kOffW2T + 64 * 64 * 2;   // [64 in][16 out]      B of dH2
constexpr uint32_t kOffX = kOffW3T + 64 * 16 * 2;     // [128][16]            A of Z1
constexpr uint32_t kOffDY = kOffX + 128 * 16 * 2;     // [128][16]            A of dH2
constexpr uint32_t kOffH1 = kOffDY + 128 * 16 * 2;    // [128][64]            A of Z2
constexpr uint32_t kOffH2 = kOffH1 + 128 * 64 * 2;    // [128][64]            A of Y
constexpr uint32_t kOffDZ2 = kOffH2 + 128 * 64 * 2;   // [128][64]            A of dH1
constexpr uint32_t kTBytes = 8 * kTSbo;               // 64 rows, transposed layout
constexpr uint32_t kOffH1T = kOffDZ2 + 128 * 64 * 2;  // [64 in][128 s]       A of dW2^T (M 128)
constexpr uint32_t kOffH2T = kOffH1T + kTBytes;       // [64 in][128 s]       A of dW3^T (M 128)
constexpr uint32_t kOffDZ1T = kOffH2T + kTBytes;      // [64 out][128 s]      A of dW1   (M 128)
constexpr uint32_t kOffDZ2T = kOffDZ1T + kTBytes;     // [64 out][128 s]      B of dW2^T
constexpr uint32_t kOffXT = kOffDZ2T + kTBytes;       // [16 in][128 s]       B of dW1
constexpr uint32_t kOffDYT = kOffXT + 2 * kTSbo;      // [16 out][128 s]      B of dW3^T
constexpr uint32_t kSmemUsed = kOffDYT + 2 * kTSbo;
static_assert(kOffDZ2T - kOffDZ1T >= kTBytes && kSmemUsed - kOffDZ1T >= 2 * kTBytes,
              "the padding rows of an M = 128 gradient operand must stay inside the layout");
constexpr uint32_t kSmemBytes = kSmemUsed + 1024;     // plus the alignment of the base

// TMEM columns (FP32 accumulators, lane = row).
constexpr uint32_t kColZ1 = 0, kColZ2 = 64, kColY = 128, kColDH2 = 160, kColDH1 = 224, kColG3 = 288, kColG2 = 320,
                   kColG1 = 384, kTmemCols = 512;
constexpr uint32_t kWaitLimit = 1u << 24;  // polls of an MMA completion (about a second) before giving up

__device__ __forceinline__ void put_bf16(unsigned char* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// Eight values of row r, columns c0..c0+7, of a K-major operand with K columns.
__device__ __forceinline__ void put_row8(unsigned char* base, int r, int c0, int K, const float* v) {
    uint4 q;
    q.x = pack_bf16(v[0], v[1]);
    q.y = pack_bf16(v[2], v[3]);
    q.z = pack_bf16(v[4], v[5]);
    q.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4*>(base + kmajor_offset(r, c0, K)) = q;
}

// Sums of 64 per-row values over the 32 rows of a warp: after the exchange
// lane l holds the sums of columns 2l and 2l + 1 (in s[0], s[1]).
__device__ __forceinline__ void warp_column_sums(float (&v)[64], int lane) {
#pragma unroll
    for (int m = 16, c = 64; m >= 1; m >>= 1, c >>= 1) {
        const bool upper = lane & m;
#pragma unroll
        for (int j = 0; j < c / 2; ++j) {
            const float send = upper ? v[j] : v[j + c / 2];
            const float keep = upper ? v[j + c / 2] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
    }
}

// The weights in their operand layouts, the biases, and zeroed padding.
__device__ void stage_weights(const MlpParams& P, unsigned char* sm, float* b1, float* b2, float* b3) {
    for (int k = threadIdx.x; k < 64 * 16; k += blockDim.x) {
        const int n = k / 16, i = k % 16;
        *reinterpret_cast<__nv_bfloat16*>(sm + kOffW1 + kmajor_offset(n, i, 16)) = P.w1t[n * 16 + i];
        // W3^T: row = input (64), column = output (16, 2 used; rows 2..7 of w3t are zero)
        const int o = i, in = n;
        *reinterpret_cast<__nv_bfloat16*>(sm + kOffW3T + kmajor_offset(in, o, 16)) =
            o < 8 ? P.w3t[o * 64 + in] : __float2bfloat16_rn(0.f);
    }
    for (int k = threadIdx.x; k < 64 * 64; k += blockDim.x) {
        const int n = k / 64, i = k % 64;
        *reinterpret_cast<__nv_bfloat16*>(sm + kOffW2 + kmajor_offset(n, i, 64)) = P.w2t[n * 64 + i];
        *reinterpret_cast<__nv_bfloat16*>(sm + kOffW2T + kmajor_offset(i, n, 64)) = P.w2t[n * 64 + i];
    }
    for (int k = threadIdx.x; k < 16 * 64; k += blockDim.x) {
        const int n = k / 64, i = k % 64;
        *reinterpret_cast<__nv_bfloat16*>(sm + kOffW3 + kmajor_offset(n, i, 64)) =
            n < 8 ? P.w3t[n * 64 + i] : __float2bfloat16_rn(0.f);
    }
    // rows 2..15 of dY^T stay zero: they are columns of the dW3^T product that are never read
    for (int k = threadIdx.x; k < (int)(2 * kTSbo / 4); k += blockDim.x)
        reinterpret_cast<uint32_t*>(sm + kOffDYT)[k] = 0u;
    for (int k = threadIdx.x; k < 64; k += blockDim.x) {
        b1[k] = P.b1[k];
        b2[k] = P.b2[k];
    }
    if (threadIdx.x < 2) b3[threadIdx.x] = P.b3[threadIdx.x];
}

// The whole forward + backward over `count` samples from `begin` (through perm
// if given).  Gradients of mean((Y - T)^2) with 1/B = inv_batch are added to
// grad (public order) and the batch loss to *loss.  A tensor-core completion
// that does not come within the poll limit sets *err and ends the kernel
// (after freeing its tensor memory).
__global__ void __launch_bounds__(128, 1) k_mlp_fwd_bwd_tc(MlpParams P, const float* __restrict__ X,
                                                           const float* __restrict__ T,
                                                           const int32_t* __restrict__ perm, long long begin,
                                                           long long count, float inv_batch, float* grad, float* loss,
                                                           int* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    __shared__ float b1[64], b2[64], b3[2], gb1[64], gb2[64], gb3[2], sloss;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    stage_weights(P, sm, b1, b2, b3);
    for (int k = tid; k < 64; k += blockDim.x) gb1[k] = gb2[k] = 0.f;
    if (tid < 2) gb3[tid] = 0.f;
    if (tid == 0) {
        sloss = 0.f;
        tc05::mbar_init(tc05::smem_addr(&bar), 1);
    }
    if (warp == 0) tc05::tmem_alloc(&tmem_slot, kTmemCols);
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    const uint32_t tmem = tmem_slot;
    const uint32_t my_lanes = (uint32_t)(32 * warp) << 16;  // this warp's TMEM lanes
    const uint32_t bar_a = tc05::smem_addr(&bar);
    const uint32_t base = tc05::smem_addr(sm);
    uint32_t phase = 0;
    bool failed = false;
    // MMAs issued by thread 0; every thread waits for their completion
    auto issue_and_wait = [&](auto&& issue) {
        tc05::fence_smem_to_async();  // this thread's operand writes, visible to the tensor cores
        tc05::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc05::fence_after_sync();
            issue();
            tc05::commit(bar_a);
        }
        const bool ok = tc05::mbar_wait(bar_a, phase, kWaitLimit);
        phase ^= 1u;
        tc05::fence_after_sync();
        failed = __syncthreads_or(!ok) != 0;
    };
    auto desc = [&](uint32_t off, uint32_t lbo, uint32_t sbo) { return tc05::smem_desc(base + off, lbo, sbo); };
    const long long tiles = (count + 127) / 128;
    bool first = true;
    float my_loss = 0.f;
    for (long long tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
        const long long row = tile * 128 + tid;
        const bool valid = row < count;
        const long long smp = valid ? (perm ? (long long)perm[begin + row] : begin + row) : 0;
        // ---- inputs: X row (bf16, features 12..15 zero) and its transpose; targets
        {
            float x[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = (valid && k < 12) ? X[smp * 12 + k] : 0.f;
            put_row8(sm + kOffX, tid, 0, 16, x);
            put_row8(sm + kOffX, tid, 8, 16, x + 8);
#pragma unroll
            for (int k = 0; k < 16; ++k) put_bf16(sm + kOffXT, tpos(k, tid), x[k]);
        }
        const float t0 = valid ? T[smp * 2] : 0.f, t1 = valid ? T[smp * 2 + 1] : 0.f;
        // ---- Z1 = X W1^T
        issue_and_wait([&] {
            tc05::mma_bf16(tmem + kColZ1, desc(kOffX, 128, 256), desc(kOffW1, 128, 256), tc05::idesc_bf16(128, 64), 0);
        });
        if (failed) break;
        // ---- H1 = silu(Z1 + b1), row-major and transposed
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16], h[16];
            tc05::tmem_ld16(tmem + my_lanes + kColZ1 + 16 * q, z);
#pragma unroll
            for (int j = 0; j < 16; ++j) h[j] = silu(z[j] + b1[16 * q + j]);
            put_row8(sm + kOffH1, tid, 16 * q, 64, h);
            put_row8(sm + kOffH1, tid, 16 * q + 8, 64, h + 8);
#pragma unroll
            for (int j = 0; j < 16; ++j) put_bf16(sm + kOffH1T, tpos(16 * q + j, tid), h[j]);
        }
        // ---- Z2 = H1 W2^T
        issue_and_wait([&] {
            for (int ks = 0; ks < 4; ++ks)
                tc05::mma_bf16(tmem + kColZ2, desc(kOffH1 + 256 * ks, 128, 1024), desc(kOffW2 + 256 * ks, 128, 1024),
                               tc05::idesc_bf16(128, 64), ks > 0);
        });
        if (failed) break;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z[16], h[16];
            tc05::tmem_ld16(tmem + my_lanes + kColZ2 + 16 * q, z);
#pragma unroll
            for (int j = 0; j < 16; ++j) h[j] = silu(z[j] + b2[16 * q + j]);
            put_row8(sm + kOffH2, tid, 16 * q, 64, h);
            put_row8(sm + kOffH2, tid, 16 * q + 8, 64, h + 8);
#pragma unroll
            for (int j = 0; j < 16; ++j) put_bf16(sm + kOffH2T, tpos(16 * q + j, tid), h[j]);
        }
        // ---- Y = H2 W3^T + b3, dY = 2 (Y - T) / B
        issue_and_wait([&] {
            for (int ks = 0; ks < 4; ++ks)
                tc05::mma_bf16(tmem + kColY, desc(kOffH2 + 256 * ks, 128, 1024), desc(kOffW3 + 256 * ks, 128, 1024),
                               tc05::idesc_bf16(128, 16), ks > 0);
        });
        if (failed) break;
        {
            float y[16];
            tc05::tmem_ld16(tmem + my_lanes + kColY, y);
            const float e0 = valid ? y[0] + b3[0] - t0 : 0.f, e1 = valid ? y[1] + b3[1] - t1 : 0.f;
            my_loss += e0 * e0 + e1 * e1;
            float d[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) d[j] = 0.f;
            d[0] = 2.f * e0 * inv_batch;
            d[1] = 2.f * e1 * inv_batch;
            put_row8(sm + kOffDY, tid, 0, 16, d);
            put_row8(sm + kOffDY, tid, 8, 16, d + 8);
            put_bf16(sm + kOffDYT, tpos(0, tid), d[0]);
            put_bf16(sm + kOffDYT, tpos(1, tid), d[1]);
            float g0 = d[0], g1 = d[1];
#pragma unroll
            for (int m = 16; m >= 1; m >>= 1) {
                g0 += __shfl_xor_sync(0xffffffffu, g0, m);
                g1 += __shfl_xor_sync(0xffffffffu, g1, m);
            }
            if (lane == 0) {
                atomicAdd(&gb3[0], g0);
                atomicAdd(&gb3[1], g1);
            }
        }
        // ---- dH2 = dY W3; dW3^T += H2^T dY
        issue_and_wait([&] {
            tc05::mma_bf16(tmem + kColDH2, desc(kOffDY, 128, 256), desc(kOffW3T, 128, 256), tc05::idesc_bf16(128, 64),
                           0);
            for (int ks = 0; ks < 8; ++ks)
                tc05::mma_bf16(tmem + kColG3, desc(kOffH2T + 2 * kTLbo * ks, kTLbo, kTSbo),
                               desc(kOffDYT + 2 * kTLbo * ks, kTLbo, kTSbo), tc05::idesc_bf16(128, 16),
                               (!first || ks > 0) ? 1u : 0u);
        });
        if (failed) break;
        // ---- dZ2 = dH2 silu'(Z2), row-major and transposed; bias gradient
        {
            float dz[64];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float dh[16], z[16];
                tc05::tmem_ld16(tmem + my_lanes + kColDH2 + 16 * q, dh);
                tc05::tmem_ld16(tmem + my_lanes + kColZ2 + 16 * q, z);
#pragma unroll
                for (int j = 0; j < 16; ++j) dz[16 * q + j] = dh[j] * dsilu_f(z[j] + b2[16 * q + j]);
            }
#pragma unroll
            for (int c = 0; c < 64; c += 8) put_row8(sm + kOffDZ2, tid, c, 64, dz + c);
#pragma unroll
            for (int c = 0; c < 64; ++c) put_bf16(sm + kOffDZ2T, tpos(c, tid), dz[c]);
            warp_column_sums(dz, lane);
            atomicAdd(&gb2[2 * lane], dz[0]);
            atomicAdd(&gb2[2 * lane + 1], dz[1]);
        }
        // ---- dH1 = dZ2 W2; dW2^T += H1^T dZ2
        issue_and_wait([&] {
            for (int ks = 0; ks < 4; ++ks)
                tc05::mma_bf16(tmem + kColDH1, desc(kOffDZ2 + 256 * ks, 128, 1024),
                               desc(kOffW2T + 256 * ks, 128, 1024), tc05::idesc_bf16(128, 64), ks > 0);
            for (int ks = 0; ks < 8; ++ks)
                tc05::mma_bf16(tmem + kColG2, desc(kOffH1T + 2 * kTLbo * ks, kTLbo, kTSbo),
                               desc(kOffDZ2T + 2 * kTLbo * ks, kTLbo, kTSbo), tc05::idesc_bf16(128, 64),
                               (!first || ks > 0) ? 1u : 0u);
        });
        if (failed) break;
        // ---- dZ1 = dH1 silu'(Z1), transposed; bias gradient
        {
            float dz[64];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float dh[16], z[16];
                tc05::tmem_ld16(tmem + my_lanes + kColDH1 + 16 * q, dh);
                tc05::tmem_ld16(tmem + my_lanes + kColZ1 + 16 * q, z);
#pragma unroll
                for (int j = 0; j < 16; ++j) dz[16 * q + j] = dh[j] * dsilu_f(z[j] + b1[16 * q + j]);
            }
#pragma unroll
            for (int c = 0; c < 64; ++c) put_bf16(sm + kOffDZ1T, tpos(c, tid), dz[c]);
            warp_column_sums(dz, lane);
            atomicAdd(&gb1[2 * lane], dz[0]);
            atomicAdd(&gb1[2 * lane + 1], dz[1]);
        }
        // ---- dW1 += dZ1^T X
        issue_and_wait([&] {
            for (int ks = 0; ks < 8; ++ks)
                tc05::mma_bf16(tmem + kColG1, desc(kOffDZ1T + 2 * kTLbo * ks, kTLbo, kTSbo),
                               desc(kOffXT + 2 * kTLbo * ks, kTLbo, kTSbo), tc05::idesc_bf16(128, 16),
                               (!first || ks > 0) ? 1u : 0u);
        });
        first = false;
    }
    if (failed) {
        if (tid == 0) atomicExch(err, 1);
    } else if (!first) {
        // the accumulated weight gradients: rows 0..63 of each, in warps 0 and 1
        if (warp < 2) {
            const int r = tid;  // TMEM lane r = row r
            float v[16];
            tc05::tmem_ld16(tmem + my_lanes + kColG3, v);  // dW3^T[in = r][out]
            atomicAdd(grad + kW3 + r, v[0]);
            atomicAdd(grad + kW3 + 64 + r, v[1]);
#pragma unroll
            for (int q = 0; q < 4; ++q) {                  // dW2^T[in = r][out]
                tc05::tmem_ld16(tmem + my_lanes + kColG2 + 16 * q, v);
#pragma unroll
                for (int j = 0; j < 16; ++j) atomicAdd(grad + kW2 + (16 * q + j) * 64 + r, v[j]);
            }
            tc05::tmem_ld16(tmem + my_lanes + kColG1, v);  // dW1[out = r][in]
#pragma unroll
            for (int j = 0; j < 12; ++j) atomicAdd(grad + kW1 + r * 12 + j, v[j]);
        }
        float l = my_loss;
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) l += __shfl_xor_sync(0xffffffffu, l, m);
        if (lane == 0) atomicAdd(&sloss, l);
        __syncthreads();
        for (int k = tid; k < 64; k += blockDim.x) {
            atomicAdd(grad + kB1 + k, gb1[k]);
            atomicAdd(grad + kB2 + k, gb2[k]);
        }
        if (tid < 2) atomicAdd(grad + kB3 + tid, gb3[tid]);
        if (tid == 0) atomicAdd(loss, sloss * inv_batch);
    }
    tc05::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc05::tmem_free(tmem, kTmemCols);
}

}  // namespace

// Launcher (mlp.cu): one CTA per 128-sample tile, at most one per SM.
cudaError_t launch_mlp_fwd_bwd_tc(const MlpParams& P, const float* X, const float* T, const int32_t* perm,
                                  long long begin, long long count, float inv_batch, float* grad, float* loss, int* err,
                                  cudaStream_t st) {
    static bool attr_set = false;
    if (!attr_set) {
        const cudaError_t e =
            cudaFuncSetAttribute(k_mlp_fwd_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    const long long tiles = (count + 127) / 128;
    const unsigned blocks = (unsigned)(tiles < 148 ? tiles : 148);
    k_mlp_fwd_bwd_tc<<<blocks, 128, kSmemBytes, st>>>(P, X, T, perm, begin, count, inv_batch, grad, loss, err);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace nrt
