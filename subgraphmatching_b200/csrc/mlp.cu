// Learned matching-order cost model: a 64-256-256-1 MLP with ReLU, BF16
// weights and activations, FP32 accumulation, trained with Adam on FP32
// master weights.  No counterpart in the reference (its orders come from
// fixed rules, order.h:1138-1281, and analytic cost models, order.h:1391-1645);
// the model only ranks candidate orders, so it never changes a count.
//
// Device buffers (one allocation per model):
//   P  fp32 master parameters, layout W1[256][64] b1[256] W2[256][256] b2[256] W3[256] b3[1]
//   G  fp32 gradients, same layout;  M, V  Adam moments, same layout
//   Wb bf16 copies of W1, W2, W3 (same offsets as in P, biases unused)
//   per batch row: X (bf16, 64), H1, H2 (bf16, 256 each), Y, T, dY (fp32),
//   dH1, dH2 (fp32, 256 each), plus the fp32 input staging area.
//
// The GEMMs are small (at most max_batch x 256 x 256) and latency-bound;
// they are one generic strided kernel with 32 x 32 output tiles staged
// through shared memory in FP32.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "smx_internal.h"

#ifndef SMX_EMU
#include <cuda_bf16.h>
#endif

namespace smx {
namespace {

#ifndef SMX_EMU
typedef __nv_bfloat16 bf16;
__device__ __forceinline__ float bf2f(bf16 x) { return __bfloat162float(x); }
__device__ __forceinline__ bf16 f2bf(float x) { return __float2bfloat16_rn(x); }
#else
// emulator: bfloat16 as the top half of an IEEE binary32, rounded to
// nearest even (the format's definition)
struct bf16 {
    uint16_t v;
};
inline float bf2f(bf16 x) {
    uint32_t u = (uint32_t)x.v << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline bf16 f2bf(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return bf16{(uint16_t)((u >> 16) | 0x40u)};
    u += 0x7fffu + ((u >> 16) & 1u);
    return bf16{(uint16_t)(u >> 16)};
}
#endif

constexpr uint32_t kIn = SMX_MLP_INPUTS, kHid = SMX_MLP_HIDDEN;
constexpr size_t oW1 = 0, ob1 = oW1 + (size_t)kHid * kIn, oW2 = ob1 + kHid, ob2 = oW2 + (size_t)kHid * kHid,
                 oW3 = ob2 + kHid, ob3 = oW3 + kHid, kParams = ob3 + 1;
static_assert(kParams == SMX_MLP_PARAMS, "parameter layout");

template <class T>
__device__ __forceinline__ float ld(const T* p, size_t i);
template <>
__device__ __forceinline__ float ld<float>(const float* p, size_t i) {
    return p[i];
}
template <>
__device__ __forceinline__ float ld<bf16>(const bf16* p, size_t i) {
    return bf2f(p[i]);
}

enum Epi : int {
    kBiasReluBf16 = 0,  // out bf16 = relu(acc + bias[n])
    kBiasF32 = 1,       // out fp32 = acc + bias[n]
    kMaskF32 = 2,       // out fp32 = acc * (mask[m][n] > 0)
    kStoreF32 = 3       // out fp32 = acc
};

constexpr int kTile = 32;

// C[m][n] = sum_k A(m, k) * B(n, k), A(m, k) = A[m*sam + k*sak], B(n, k) =
// B[n*sbn + k*sbk]; 256 threads, each 4 outputs of a 32 x 32 tile.
template <class TA, class TB, int EPI>
__global__ void __launch_bounds__(256) gemm_kernel(const TA* __restrict__ A, size_t sam, size_t sak,
                                                   const TB* __restrict__ B, size_t sbn, size_t sbk, uint32_t M,
                                                   uint32_t N, uint32_t K, const float* __restrict__ bias,
                                                   const bf16* __restrict__ mask, void* __restrict__ out) {
    SMX_SHARED_ARRAY(float, sa, kTile * (kTile + 1));
    SMX_SHARED_ARRAY(float, sb, kTile * (kTile + 1));
    const uint32_t t = threadIdx.x;
    const uint32_t m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
    const uint32_t tm = t / 16, tn = t % 16;  // outputs (m0 + tm*2 + i, n0 + tn*2 + j)
    float acc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
    for (uint32_t k0 = 0; k0 < K; k0 += kTile) {
        for (uint32_t i = t; i < kTile * kTile; i += 256) {
            const uint32_t r = i / kTile, c = i % kTile;
            const uint32_t m = m0 + r, n = n0 + r, k = k0 + c;
            sa[r * (kTile + 1) + c] = (m < M && k < K) ? ld(A, (size_t)m * sam + (size_t)k * sak) : 0.f;
            sb[r * (kTile + 1) + c] = (n < N && k < K) ? ld(B, (size_t)n * sbn + (size_t)k * sbk) : 0.f;
        }
        __syncthreads();
        for (uint32_t c = 0; c < kTile; ++c) {
            const float a0 = sa[(tm * 2) * (kTile + 1) + c], a1 = sa[(tm * 2 + 1) * (kTile + 1) + c];
            const float b0 = sb[(tn * 2) * (kTile + 1) + c], b1 = sb[(tn * 2 + 1) * (kTile + 1) + c];
            acc[0][0] = fmaf(a0, b0, acc[0][0]);
            acc[0][1] = fmaf(a0, b1, acc[0][1]);
            acc[1][0] = fmaf(a1, b0, acc[1][0]);
            acc[1][1] = fmaf(a1, b1, acc[1][1]);
        }
        __syncthreads();
    }
    for (uint32_t i = 0; i < 2; ++i)
        for (uint32_t j = 0; j < 2; ++j) {
            const uint32_t m = m0 + tm * 2 + i, n = n0 + tn * 2 + j;
            if (m >= M || n >= N) continue;
            const size_t o = (size_t)m * N + n;
            float v = acc[i][j];
            if (EPI == kBiasReluBf16) {
                v += bias[n];
                static_cast<bf16*>(out)[o] = f2bf(v > 0.f ? v : 0.f);
            } else if (EPI == kBiasF32) {
                static_cast<float*>(out)[o] = v + bias[n];
            } else if (EPI == kMaskF32) {
                static_cast<float*>(out)[o] = bf2f(mask[o]) > 0.f ? v : 0.f;
            } else {
                static_cast<float*>(out)[o] = v;
            }
        }
}

__global__ void cast_kernel(const float* __restrict__ x, size_t n, bf16* __restrict__ y) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = f2bf(x[i]);
}

// bf16 copies of the three weight matrices from the fp32 masters
__global__ void weights_kernel(const float* __restrict__ P, bf16* __restrict__ Wb) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += (size_t)gridDim.x * blockDim.x) {
        const bool w = i < ob1 || (i >= oW2 && i < ob2) || (i >= oW3 && i < ob3);
        if (w) Wb[i] = f2bf(P[i]);
    }
}

// dY = (Y - T) / n, loss = sum (Y - T)^2 / (2n); one block, fixed order
__global__ void loss_kernel(const float* __restrict__ Y, const float* __restrict__ T, uint32_t n,
                            float* __restrict__ dY, float* __restrict__ loss) {
    SMX_SHARED_ARRAY(float, red, 256);
    float s = 0.f;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float d = Y[i] - T[i];
        dY[i] = d / (float)n;
        s += d * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (uint32_t w = 128; w; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] / (2.f * (float)n);
}

// db[j] = sum_m d[m][j] (columns of a row-major n x cols fp32 matrix)
__global__ void colsum_kernel(const float* __restrict__ d, uint32_t n, uint32_t cols, float* __restrict__ db) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.f;
    for (uint32_t m = 0; m < n; ++m) s += d[(size_t)m * cols + j];
    db[j] = s;
}

__global__ void adam_kernel(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ Mo,
                            float* __restrict__ Vo, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += (size_t)gridDim.x * blockDim.x) {
        const float g = G[i];
        const float m = b1 * Mo[i] + (1.f - b1) * g;
        const float v = b2 * Vo[i] + (1.f - b2) * g * g;
        Mo[i] = m;
        Vo[i] = v;
        P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
}

template <class TA, class TB, int EPI>
void gemm(cudaStream_t s, const TA* A, size_t sam, size_t sak, const TB* B, size_t sbn, size_t sbk, uint32_t M,
          uint32_t N, uint32_t K, const float* bias, const bf16* mask, void* out) {
    const dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
    auto kern = gemm_kernel<TA, TB, EPI>;
    SMX_LAUNCH(kern, grid, 256, 0, s, A, sam, sak, B, sbn, sbk, M, N, K, bias, mask, out);
}

}  // namespace
}  // namespace smx

struct smx_mlp {
    int device = 0;
    uint32_t max_batch = 0;
    cudaStream_t stream = nullptr;
    void* mem = nullptr;
    float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
    smx::bf16* Wb = nullptr;
    smx::bf16 *X = nullptr, *H1 = nullptr, *H2 = nullptr;
    float *Xf = nullptr, *Y = nullptr, *T = nullptr, *dY = nullptr, *dH1 = nullptr, *dH2 = nullptr, *loss = nullptr;
    uint64_t steps = 0;
};

namespace smx {
namespace {

int mlp_device_ok(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(SMX_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= n) return fail(SMX_BAD_ARGUMENT, "device index out of range");
    return SMX_OK;
}

// forward pass of rows [0, n) already in m->X; leaves Y, H1, H2
int mlp_forward_dev(smx_mlp* m, uint32_t n) {
    cudaStream_t s = m->stream;
    gemm<bf16, bf16, kBiasReluBf16>(s, m->X, kIn, 1, m->Wb + oW1, kIn, 1, n, kHid, kIn, m->P + ob1, nullptr, m->H1);
    gemm<bf16, bf16, kBiasReluBf16>(s, m->H1, kHid, 1, m->Wb + oW2, kHid, 1, n, kHid, kHid, m->P + ob2, nullptr,
                                    m->H2);
    gemm<bf16, bf16, kBiasF32>(s, m->H2, kHid, 1, m->Wb + oW3, kHid, 1, n, 1, kHid, m->P + ob3, nullptr, m->Y);
    SMX_CUDA_TRY(cudaGetLastError());
    return SMX_OK;
}

// gradients of the mean squared error / 2 into G (forward already done)
int mlp_backward_dev(smx_mlp* m, uint32_t n) {
    cudaStream_t s = m->stream;
    SMX_LAUNCH(loss_kernel, 1, 256, 0, s, m->Y, m->T, n, m->dY, m->loss);
    // layer 3: dW3[j] = sum_m dY[m] H2[m][j]; db3; dH2 = dY W3 * (H2 > 0)
    gemm<float, bf16, kStoreF32>(s, m->dY, 0, 1, m->H2, 1, kHid, 1, kHid, n, nullptr, nullptr, m->G + oW3);
    SMX_LAUNCH(colsum_kernel, 1, 32, 0, s, m->dY, n, 1u, m->G + ob3);
    gemm<float, bf16, kMaskF32>(s, m->dY, 1, 1, m->Wb + oW3, 1, 1, n, kHid, 1, nullptr, m->H2, m->dH2);
    // layer 2: dW2 = dH2^T H1; db2; dH1 = dH2 W2 * (H1 > 0)
    gemm<float, bf16, kStoreF32>(s, m->dH2, 1, kHid, m->H1, 1, kHid, kHid, kHid, n, nullptr, nullptr, m->G + oW2);
    SMX_LAUNCH(colsum_kernel, (kHid + 255) / 256, 256, 0, s, m->dH2, n, kHid, m->G + ob2);
    gemm<float, bf16, kMaskF32>(s, m->dH2, kHid, 1, m->Wb + oW2, 1, kHid, n, kHid, kHid, nullptr, m->H1, m->dH1);
    // layer 1: dW1 = dH1^T X; db1
    gemm<float, bf16, kStoreF32>(s, m->dH1, 1, kHid, m->X, 1, kIn, kHid, kIn, n, nullptr, nullptr, m->G + oW1);
    SMX_LAUNCH(colsum_kernel, (kHid + 255) / 256, 256, 0, s, m->dH1, n, kHid, m->G + ob1);
    SMX_CUDA_TRY(cudaGetLastError());
    return SMX_OK;
}

int mlp_load_inputs(smx_mlp* m, const float* x, const float* t, uint32_t n) {
    if (n == 0 || n > m->max_batch)
        return fail(SMX_TOO_LARGE, "batch of " + std::to_string(n) + " rows; this model takes 1.." +
                                       std::to_string(m->max_batch));
    SMX_CUDA_TRY(cudaSetDevice(m->device));
    SMX_CUDA_TRY(cudaMemcpyAsync(m->Xf, x, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, m->stream));
    if (t) SMX_CUDA_TRY(cudaMemcpyAsync(m->T, t, (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    SMX_LAUNCH(cast_kernel, 64, 256, 0, m->stream, m->Xf, (size_t)n * kIn, m->X);
    SMX_CUDA_TRY(cudaGetLastError());
    return SMX_OK;
}

int mlp_refresh_weights(smx_mlp* m) {
    SMX_LAUNCH(weights_kernel, 128, 256, 0, m->stream, m->P, m->Wb);
    SMX_CUDA_TRY(cudaGetLastError());
    return SMX_OK;
}

}  // namespace
}  // namespace smx

using namespace smx;

extern "C" {

size_t smx_mlp_param_count(void) { return kParams; }

int smx_mlp_create(int device, uint32_t max_batch, uint64_t seed, smx_mlp** out) {
    if (!out) return fail(SMX_BAD_ARGUMENT, "null argument");
    *out = nullptr;
    if (max_batch == 0 || max_batch > (1u << 20)) return fail(SMX_BAD_ARGUMENT, "max_batch must be 1 .. 2^20");
    int rc = mlp_device_ok(device);
    if (rc != SMX_OK) return rc;
    SMX_CUDA_TRY(cudaSetDevice(device));
    smx_mlp* m = new smx_mlp();
    m->device = device;
    m->max_batch = max_batch;
    const size_t B = max_batch;
    // byte layout, every array 256-byte aligned
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t o = at;
        at = (at + bytes + 255) & ~(size_t)255;
        return o;
    };
    const size_t oP = take(kParams * 4), oG = take(kParams * 4), oM = take(kParams * 4), oV = take(kParams * 4);
    const size_t oWb = take(kParams * 2), oX = take(B * kIn * 2), oH1 = take(B * kHid * 2), oH2 = take(B * kHid * 2);
    const size_t oXf = take(B * kIn * 4), oY = take(B * 4), oT = take(B * 4), odY = take(B * 4);
    const size_t odH1 = take(B * kHid * 4), odH2 = take(B * kHid * 4), oL = take(4);
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&m->mem, at) != cudaSuccess) {
        cudaGetLastError();
        smx_mlp_destroy(m);
        return fail(SMX_CUDA_ERROR, "model allocation failed");
    }
    char* b = static_cast<char*>(m->mem);
    m->P = reinterpret_cast<float*>(b + oP);
    m->G = reinterpret_cast<float*>(b + oG);
    m->M = reinterpret_cast<float*>(b + oM);
    m->V = reinterpret_cast<float*>(b + oV);
    m->Wb = reinterpret_cast<bf16*>(b + oWb);
    m->X = reinterpret_cast<bf16*>(b + oX);
    m->H1 = reinterpret_cast<bf16*>(b + oH1);
    m->H2 = reinterpret_cast<bf16*>(b + oH2);
    m->Xf = reinterpret_cast<float*>(b + oXf);
    m->Y = reinterpret_cast<float*>(b + oY);
    m->T = reinterpret_cast<float*>(b + oT);
    m->dY = reinterpret_cast<float*>(b + odY);
    m->dH1 = reinterpret_cast<float*>(b + odH1);
    m->dH2 = reinterpret_cast<float*>(b + odH2);
    m->loss = reinterpret_cast<float*>(b + oL);
    // He-normal weights, zero biases, from a seeded generator (splitmix64 + Box-Muller)
    std::vector<float> p(kParams, 0.f);
    uint64_t st = seed ^ 0x5eed5eedULL;
    auto next = [&]() {
        st += 0x9e3779b97f4a7c15ULL;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return ((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    auto normal = [&]() {
        const double u1 = std::max(next(), 1e-300), u2 = next();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    for (size_t i = oW1; i < ob1; ++i) p[i] = (float)(normal() * std::sqrt(2.0 / kIn));
    for (size_t i = oW2; i < ob2; ++i) p[i] = (float)(normal() * std::sqrt(2.0 / kHid));
    for (size_t i = oW3; i < ob3; ++i) p[i] = (float)(normal() * std::sqrt(1.0 / kHid));
    rc = smx_mlp_set_params(m, p.data(), kParams);
    if (rc != SMX_OK) {
        smx_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return SMX_OK;
}

int smx_mlp_set_params(smx_mlp* m, const float* params, size_t n) {
    if (!m || !params) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (n != kParams) return fail(SMX_BAD_ARGUMENT, "parameter count must be SMX_MLP_PARAMS");
    SMX_CUDA_TRY(cudaSetDevice(m->device));
    SMX_CUDA_TRY(cudaMemcpyAsync(m->P, params, kParams * 4, cudaMemcpyHostToDevice, m->stream));
    SMX_CUDA_TRY(cudaMemsetAsync(m->M, 0, kParams * 4, m->stream));
    SMX_CUDA_TRY(cudaMemsetAsync(m->V, 0, kParams * 4, m->stream));
    m->steps = 0;
    int rc = mlp_refresh_weights(m);
    if (rc != SMX_OK) return rc;
    SMX_CUDA_TRY(cudaStreamSynchronize(m->stream));
    return SMX_OK;
}

int smx_mlp_get_params(const smx_mlp* m, float* params, size_t n) {
    if (!m || !params) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (n != kParams) return fail(SMX_BAD_ARGUMENT, "parameter count must be SMX_MLP_PARAMS");
    SMX_CUDA_TRY(cudaSetDevice(m->device));
    SMX_CUDA_TRY(cudaMemcpyAsync(params, m->P, kParams * 4, cudaMemcpyDeviceToHost, m->stream));
    SMX_CUDA_TRY(cudaStreamSynchronize(m->stream));
    return SMX_OK;
}

int smx_mlp_forward(smx_mlp* m, const float* x, uint32_t n, float* y) {
    if (!m || !x || !y) return fail(SMX_BAD_ARGUMENT, "null argument");
    int rc = mlp_load_inputs(m, x, nullptr, n);
    if (rc != SMX_OK) return rc;
    rc = mlp_forward_dev(m, n);
    if (rc != SMX_OK) return rc;
    SMX_CUDA_TRY(cudaMemcpyAsync(y, m->Y, (size_t)n * 4, cudaMemcpyDeviceToHost, m->stream));
    SMX_CUDA_TRY(cudaStreamSynchronize(m->stream));
    return SMX_OK;
}

int smx_mlp_gradients(smx_mlp* m, const float* x, const float* t, uint32_t n, float* grads, float* loss) {
    if (!m || !x || !t) return fail(SMX_BAD_ARGUMENT, "null argument");
    int rc = mlp_load_inputs(m, x, t, n);
    if (rc == SMX_OK) rc = mlp_forward_dev(m, n);
    if (rc == SMX_OK) rc = mlp_backward_dev(m, n);
    if (rc != SMX_OK) return rc;
    if (grads) SMX_CUDA_TRY(cudaMemcpyAsync(grads, m->G, kParams * 4, cudaMemcpyDeviceToHost, m->stream));
    if (loss) SMX_CUDA_TRY(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->stream));
    SMX_CUDA_TRY(cudaStreamSynchronize(m->stream));
    return SMX_OK;
}

int smx_mlp_train_step(smx_mlp* m, const float* x, const float* t, uint32_t n, float lr, float* loss) {
    if (!m || !x || !t) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (!(lr > 0.f)) return fail(SMX_BAD_ARGUMENT, "learning rate must be positive");
    int rc = mlp_load_inputs(m, x, t, n);
    if (rc == SMX_OK) rc = mlp_forward_dev(m, n);
    if (rc == SMX_OK) rc = mlp_backward_dev(m, n);
    if (rc != SMX_OK) return rc;
    m->steps++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - (float)std::pow(b1, (double)m->steps), c2 = 1.f - (float)std::pow(b2, (double)m->steps);
    SMX_LAUNCH(adam_kernel, 128, 256, 0, m->stream, m->P, m->G, m->M, m->V, lr, b1, b2, 1e-8f, c1, c2);
    SMX_CUDA_TRY(cudaGetLastError());
    rc = mlp_refresh_weights(m);
    if (rc != SMX_OK) return rc;
    if (loss) SMX_CUDA_TRY(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->stream));
    SMX_CUDA_TRY(cudaStreamSynchronize(m->stream));
    return SMX_OK;
}

void smx_mlp_destroy(smx_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    if (m->mem) cudaFree(m->mem);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

}  // extern "C"
