// mlp.cu -- training and inference entry points of the learned-initial-guess
// MLP (12 -> 64 -> 64 -> 2, SiLU) with FP32 master weights and Adam.
// Training forward + backward runs on the tcgen05 tensor cores (mlp_tc.cu,
// FP32 accumulators in tensor memory); inference on BF16 mma.sync m16n8k16
// (mlp.cuh), FP32 accumulation.
//
// Rounding points (mirrored by the CPU oracle, oracle/mlp_oracle.py): every
// tensor-core operand is bfloat16 (inputs, weights, hidden activations, output
// and hidden gradients); pre-activations, biases, bias gradients and weight
// gradient accumulation are FP32.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "mlp.cuh"
#include "nrt_internal.h"

using namespace nrt::dev;

namespace {

constexpr int kP_W1 = 0, kP_B1 = kP_W1 + 64 * 12, kP_W2 = kP_B1 + 64, kP_B2 = kP_W2 + 64 * 64, kP_W3 = kP_B2 + 64,
              kP_B3 = kP_W3 + 2 * 64, kNumParams = kP_B3 + 2;
static_assert(kNumParams == NRT_MLP_PARAMS, "parameter count");

// Byte offsets inside the device blob used by the kernels.
constexpr size_t kB_W1 = 0, kB_W2 = kB_W1 + 64 * 16 * 2, kB_W3 = kB_W2 + 64 * 64 * 2, kB_B1 = kB_W3 + 8 * 64 * 2,
                 kB_B2 = kB_B1 + 64 * 4, kB_B3 = kB_B2 + 64 * 4, kBlobBytes = kB_B3 + 8 * 4;

}  // namespace

namespace nrt {
dev::MlpParams blob_params(const void* blob) {
    const char* b = static_cast<const char*>(blob);
    dev::MlpParams p;
    p.w1t = reinterpret_cast<const __nv_bfloat16*>(b + kB_W1);
    p.w2t = reinterpret_cast<const __nv_bfloat16*>(b + kB_W2);
    p.w3t = reinterpret_cast<const __nv_bfloat16*>(b + kB_W3);
    p.b1 = reinterpret_cast<const float*>(b + kB_B1);
    p.b2 = reinterpret_cast<const float*>(b + kB_B2);
    p.b3 = reinterpret_cast<const float*>(b + kB_B3);
    return p;
}
size_t mlp_blob_bytes() { return kBlobBytes; }
}  // namespace nrt

struct nrt_mlp {
    int device = 0;
    float* master = nullptr;  // device, public order
    float* m = nullptr;
    float* v = nullptr;
    float* grad = nullptr;
    float* loss = nullptr;    // device scalar
    int* err = nullptr;       // device word: the training kernel gave up waiting for its tensor cores
    void* blob = nullptr;     // device, kernel layout
    long long step = 0;
    std::vector<float> host_m, host_v;  // only used by save/load staging
};

namespace {

// public index -> blob element, or -1 for none
__device__ __forceinline__ void put_blob(char* blob, int k, float w) {
    if (k < kP_B1) {
        const int n = k / 12, i = k % 12;
        reinterpret_cast<__nv_bfloat16*>(blob + kB_W1)[n * 16 + i] = __float2bfloat16_rn(w);
    } else if (k < kP_W2) {
        reinterpret_cast<float*>(blob + kB_B1)[k - kP_B1] = w;
    } else if (k < kP_B2) {
        reinterpret_cast<__nv_bfloat16*>(blob + kB_W2)[k - kP_W2] = __float2bfloat16_rn(w);
    } else if (k < kP_W3) {
        reinterpret_cast<float*>(blob + kB_B2)[k - kP_B2] = w;
    } else if (k < kP_B3) {
        reinterpret_cast<__nv_bfloat16*>(blob + kB_W3)[k - kP_W3] = __float2bfloat16_rn(w);
    } else {
        reinterpret_cast<float*>(blob + kB_B3)[k - kP_B3] = w;
    }
}

__global__ void k_mlp_to_blob(const float* master, char* blob) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < kNumParams) put_blob(blob, k, master[k]);
}

__global__ void k_mlp_adam(float* master, float* m, float* v, float* grad, char* blob, float lr, float b1, float b2,
                           float eps, float bc1, float bc2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kNumParams) return;
    const float g = grad[k];
    const float mk = b1 * m[k] + (1.f - b1) * g;
    const float vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    const float w = master[k] - lr * (mk / bc1) / (sqrtf(vk / bc2) + eps);
    master[k] = w;
    grad[k] = 0.f;
    put_blob(blob, k, w);
}

// Inference on feature rows (n x 12) -> outputs (n x 2), unclamped.
__global__ void __launch_bounds__(256) k_mlp_forward(MlpParams P, const float* __restrict__ X, long long n,
                                                     float* __restrict__ Y) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmem& s = *reinterpret_cast<MlpSmem*>(smem_raw);
    mlp_load(s, P);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (long long base = ((long long)blockIdx.x * 8 + warp) * 32; base < n; base += (long long)gridDim.x * 256) {
        const long long r = base + lane;
        float x[kMlpIn];
#pragma unroll
        for (int k = 0; k < kMlpIn; ++k) x[k] = r < n ? X[r * 12 + k] : 0.f;
        float u, v;
        mlp_infer_warp(s, warp, lane, x, u, v);
        if (r < n) {
            Y[2 * r] = u;
            Y[2 * r + 1] = v;
        }
    }
}

int cuda_fail(cudaError_t e, const char* what) {
    return nrt::fail(e == cudaErrorMemoryAllocation ? NRT_ERR_NOMEM : NRT_ERR_CUDA, "%s: %s", what,
                     cudaGetErrorString(e));
}

uint32_t crc32(const void* data, size_t n) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    uint32_t c = 0xFFFFFFFFu;
    for (size_t i = 0; i < n; ++i) {
        c ^= p[i];
        for (int k = 0; k < 8; ++k) c = (c >> 1) ^ (0xEDB88320u & (0u - (c & 1u)));
    }
    return ~c;
}

int upload_blob(nrt_mlp* m) {
    k_mlp_to_blob<<<(kNumParams + 255) / 256, 256>>>(m->master, static_cast<char*>(m->blob));
    const cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? NRT_OK : cuda_fail(e, "mlp weights");
}

struct DeviceGuard {
    int prev = 0;
    bool changed = false;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) {
            cudaSetDevice(dev);
            changed = true;
        }
    }
    ~DeviceGuard() {
        if (changed) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" {

size_t nrt_mlp_param_count(void) { return kNumParams; }

int nrt_mlp_create(int device, uint32_t seed, nrt_mlp** out) {
    if (!out) return nrt::fail(NRT_ERR_INVALID, "out is null");
    *out = nullptr;
    nrt_mlp* m = new (std::nothrow) nrt_mlp();
    if (!m) return nrt::fail(NRT_ERR_NOMEM, "host allocation failed");
    m->device = device;
    DeviceGuard dg(device);
    const size_t pbytes = sizeof(float) * kNumParams;
    cudaError_t e = cudaMalloc(&m->master, pbytes);
    if (e == cudaSuccess) e = cudaMalloc(&m->m, pbytes);
    if (e == cudaSuccess) e = cudaMalloc(&m->v, pbytes);
    if (e == cudaSuccess) e = cudaMalloc(&m->grad, pbytes);
    if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&m->blob, kBlobBytes);
    if (e == cudaSuccess) e = cudaMemset(m->blob, 0, kBlobBytes);
    if (e == cudaSuccess) e = cudaMemset(m->m, 0, pbytes);
    if (e == cudaSuccess) e = cudaMemset(m->v, 0, pbytes);
    if (e == cudaSuccess) e = cudaMemset(m->grad, 0, pbytes);
    if (e != cudaSuccess) {
        nrt_mlp_destroy(m);
        return cuda_fail(e, "mlp allocation");
    }
    // Glorot-uniform weights from a seeded generator, zero biases
    std::vector<float> w(kNumParams, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_out, int fan_in) {
        const float a = std::sqrt(6.f / (float)(fan_in + fan_out));
        std::uniform_real_distribution<float> U(-a, a);
        for (int k = 0; k < fan_out * fan_in; ++k) w[off + k] = U(rng);
    };
    fill(kP_W1, 64, 12);
    fill(kP_W2, 64, 64);
    fill(kP_W3, 2, 64);
    w[kP_B3] = 0.5f;  // outputs start at the patch midpoint
    w[kP_B3 + 1] = 0.5f;
    e = cudaMemcpy(m->master, w.data(), pbytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        nrt_mlp_destroy(m);
        return cuda_fail(e, "mlp upload");
    }
    if (int st = upload_blob(m)) {
        nrt_mlp_destroy(m);
        return st;
    }
    *out = m;
    return NRT_OK;
}

int nrt_mlp_destroy(nrt_mlp* m) {
    if (!m) return NRT_OK;
    DeviceGuard dg(m->device);
    cudaFree(m->master);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->grad);
    cudaFree(m->loss);
    cudaFree(m->err);
    cudaFree(m->blob);
    delete m;
    return NRT_OK;
}

int nrt_mlp_get_params(const nrt_mlp* m, float* host_out) {
    if (!m || !host_out) return nrt::fail(NRT_ERR_INVALID, "null argument");
    DeviceGuard dg(m->device);
    const cudaError_t e = cudaMemcpy(host_out, m->master, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? NRT_OK : cuda_fail(e, "mlp params");
}

int nrt_mlp_set_params(nrt_mlp* m, const float* host_in) {
    if (!m || !host_in) return nrt::fail(NRT_ERR_INVALID, "null argument");
    DeviceGuard dg(m->device);
    const cudaError_t e = cudaMemcpy(m->master, host_in, sizeof(float) * kNumParams, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "mlp params");
    return upload_blob(m);
}

int nrt_mlp_forward(const nrt_mlp* m, const float* features, int64_t n, float* out_uv, void* stream) {
    if (!m || (n > 0 && (!features || !out_uv)) || n < 0) return nrt::fail(NRT_ERR_INVALID, "bad argument");
    if (n == 0) return NRT_OK;
    DeviceGuard dg(m->device);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmem));
        attr_set = true;
    }
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_mlp_forward<<<(unsigned)blocks, 256, sizeof(MlpSmem), static_cast<cudaStream_t>(stream)>>>(
        nrt::blob_params(m->blob), features, n, out_uv);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NRT_OK : cuda_fail(e, "mlp forward");
}

// Forward + backward of one batch on the tcgen05 tensor cores (mlp_tc.cu).
static int fwd_bwd(nrt_mlp* m, const float* X, const float* T, const int32_t* perm, long long begin, long long count,
                   long long batch, cudaStream_t st) {
    const cudaError_t e = nrt::dev::launch_mlp_fwd_bwd_tc(nrt::blob_params(m->blob), X, T, perm, begin, count,
                                                          1.f / (float)batch, m->grad, m->loss, m->err, st);
    return e == cudaSuccess ? NRT_OK : cuda_fail(e, "mlp fwd/bwd");
}

// After a synchronisation: did a training kernel give up waiting for its tensor cores?
static int check_err(nrt_mlp* m) {
    int h = 0;
    const cudaError_t e = cudaMemcpy(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "mlp error word");
    if (h) {
        cudaMemset(m->err, 0, sizeof(int));
        return nrt::fail(NRT_ERR_DEVICE, "mlp training: a tensor-core step did not complete within its wait limit");
    }
    return NRT_OK;
}

int nrt_mlp_gradients(nrt_mlp* m, const float* features, const float* targets, int64_t n, float* host_grads,
                      float* host_loss, void* stream) {
    if (!m || !features || !targets || n <= 0 || !host_grads) return nrt::fail(NRT_ERR_INVALID, "bad argument");
    DeviceGuard dg(m->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(m->grad, 0, sizeof(float) * kNumParams, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->loss, 0, sizeof(float), st);
    if (e != cudaSuccess) return cuda_fail(e, "mlp grad reset");
    if (int s2 = fwd_bwd(m, features, targets, nullptr, 0, n, n, st)) return s2;
    e = cudaMemcpyAsync(host_grads, m->grad, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost, st);
    float loss = 0.f;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->grad, 0, sizeof(float) * kNumParams, st);
    if (e != cudaSuccess) return cuda_fail(e, "mlp gradients");
    if (int s3 = check_err(m)) return s3;
    if (host_loss) *host_loss = loss;
    return NRT_OK;
}

int nrt_mlp_train(nrt_mlp* m, const float* features, const float* targets, int64_t n, const nrt_train_opts* o,
                  float* host_epoch_loss, void* stream) {
    if (!m || !features || !targets || n <= 0 || !o) return nrt::fail(NRT_ERR_INVALID, "bad argument");
    if (o->epochs < 1 || o->batch < 32 || !(o->lr > 0.f)) return nrt::fail(NRT_ERR_INVALID, "bad training options");
    if (n > (int64_t)INT32_MAX) return nrt::fail(NRT_ERR_INVALID, "too many samples");
    DeviceGuard dg(m->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int32_t* perm = nullptr;
    cudaError_t e = cudaMalloc(&perm, sizeof(int32_t) * n);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(permutation)");
    std::vector<int32_t> idx(n);
    for (int64_t k = 0; k < n; ++k) idx[k] = (int32_t)k;
    std::mt19937_64 rng(o->seed);
    int status = NRT_OK;
    const float b1 = o->beta1 > 0 ? o->beta1 : 0.9f, b2 = o->beta2 > 0 ? o->beta2 : 0.999f,
                ep = o->eps > 0 ? o->eps : 1e-8f;
    for (int epoch = 0; epoch < o->epochs && status == NRT_OK; ++epoch) {
        std::shuffle(idx.begin(), idx.end(), rng);
        e = cudaMemcpyAsync(perm, idx.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(m->loss, 0, sizeof(float), st);
        if (e != cudaSuccess) { status = cuda_fail(e, "epoch setup"); break; }
        long long batches = 0;
        for (long long b = 0; b < n && status == NRT_OK; b += o->batch) {
            const long long cnt = std::min<long long>(o->batch, n - b);
            status = fwd_bwd(m, features, targets, perm, b, cnt, cnt, st);
            ++m->step;
            const float bc1 = 1.f - std::pow(b1, (float)m->step), bc2 = 1.f - std::pow(b2, (float)m->step);
            k_mlp_adam<<<(kNumParams + 255) / 256, 256, 0, st>>>(m->master, m->m, m->v, m->grad,
                                                                 static_cast<char*>(m->blob), o->lr, b1, b2, ep, bc1,
                                                                 bc2);
            ++batches;
        }
        float loss = 0.f;
        e = cudaMemcpyAsync(&loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { status = cuda_fail(e, "epoch loss"); break; }
        if ((status = check_err(m)) != NRT_OK) break;
        if (host_epoch_loss) host_epoch_loss[epoch] = loss / (float)batches;
    }
    cudaFree(perm);
    return status;
}

// File: "NRTMLP01", u32 version 1, u32 dims 12/64/64/2, u32 parameter count,
// i64 Adam step, master weights, Adam m, Adam v (float32), u32 CRC-32 of all
// preceding bytes.
int nrt_mlp_save(const nrt_mlp* m, const char* path) {
    if (!m || !path) return nrt::fail(NRT_ERR_INVALID, "null argument");
    DeviceGuard dg(m->device);
    std::vector<float> w(kNumParams), mm(kNumParams), vv(kNumParams);
    cudaError_t e = cudaMemcpy(w.data(), m->master, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(mm.data(), m->m, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(vv.data(), m->v, sizeof(float) * kNumParams, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "mlp save");
    std::vector<unsigned char> buf;
    auto put = [&](const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        buf.insert(buf.end(), c, c + n);
    };
    const uint32_t hdr[6] = {1, 12, 64, 64, 2, (uint32_t)kNumParams};
    put("NRTMLP01", 8);
    put(hdr, sizeof(hdr));
    const int64_t step = m->step;
    put(&step, sizeof(step));
    put(w.data(), sizeof(float) * kNumParams);
    put(mm.data(), sizeof(float) * kNumParams);
    put(vv.data(), sizeof(float) * kNumParams);
    const uint32_t crc = crc32(buf.data(), buf.size());
    put(&crc, sizeof(crc));
    FILE* f = std::fopen(path, "wb");
    if (!f) return nrt::fail(NRT_ERR_INVALID, "cannot open %s for writing", path);
    const size_t wrote = std::fwrite(buf.data(), 1, buf.size(), f);
    const int closed = std::fclose(f);
    if (wrote != buf.size() || closed != 0) return nrt::fail(NRT_ERR_INVALID, "short write to %s", path);
    return NRT_OK;
}

int nrt_mlp_load(const char* path, int device, nrt_mlp** out) {
    if (!path || !out) return nrt::fail(NRT_ERR_INVALID, "null argument");
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return nrt::fail(NRT_ERR_INVALID, "cannot open %s", path);
    std::vector<unsigned char> buf;
    unsigned char tmp[65536];
    size_t got;
    while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
    std::fclose(f);
    const size_t expect = 8 + 24 + 8 + 3 * sizeof(float) * kNumParams + 4;
    if (buf.size() != expect || std::memcmp(buf.data(), "NRTMLP01", 8) != 0)
        return nrt::fail(NRT_ERR_INVALID, "%s is not an nrt MLP file", path);
    uint32_t crc;
    std::memcpy(&crc, buf.data() + buf.size() - 4, 4);
    if (crc != crc32(buf.data(), buf.size() - 4)) return nrt::fail(NRT_ERR_INVALID, "%s: checksum mismatch", path);
    uint32_t hdr[6];
    std::memcpy(hdr, buf.data() + 8, sizeof(hdr));
    if (hdr[0] != 1 || hdr[1] != 12 || hdr[2] != 64 || hdr[3] != 64 || hdr[4] != 2 || hdr[5] != (uint32_t)kNumParams)
        return nrt::fail(NRT_ERR_INVALID, "%s: unsupported version or shape", path);
    nrt_mlp* m = nullptr;
    if (int st = nrt_mlp_create(device, 0, &m)) return st;
    int64_t step;
    std::memcpy(&step, buf.data() + 32, 8);
    m->step = step;
    const unsigned char* p = buf.data() + 40;
    DeviceGuard dg(device);
    cudaError_t e = cudaMemcpy(m->master, p, sizeof(float) * kNumParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(m->m, p + sizeof(float) * kNumParams, sizeof(float) * kNumParams, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(m->v, p + 2 * sizeof(float) * kNumParams, sizeof(float) * kNumParams, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        nrt_mlp_destroy(m);
        return cuda_fail(e, "mlp load");
    }
    if (int st = upload_blob(m)) {
        nrt_mlp_destroy(m);
        return st;
    }
    *out = m;
    return NRT_OK;
}

}  // extern "C"

namespace nrt {
const void* mlp_device_blob(const nrt_mlp* m) { return m ? m->blob : nullptr; }
int mlp_device(const nrt_mlp* m) { return m ? m->device : -1; }
}  // namespace nrt
