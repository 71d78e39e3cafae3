// sw2d_mlp.cu — the learned momentum-exchange closure: an MLP of 10 inputs -> 64 -> 64 -> 2
// (GELU) whose inference and training run on the 5th-generation tensor cores (tcgen05, BF16
// operands, FP32 accumulators in TMEM): one hand-written GEMM kernel for training and
// stand-alone inference, and the DIP cell-update kernel with the network inside
// (k_update_closure, further down) for the closure in a model's step.
//
// k_umma_gemm computes, for a tile of 128 rows per CTA, D = A * B^T with A [M x K] and B [N x K]
// (bf16, row-major, K contiguous), K looped in chunks of 64 through shared memory (K-major
// core-matrix layout of umma.cuh), N <= 256 in one MMA row, and an epilogue that reads D from
// TMEM (each thread one row) and applies one of:
//   kEpiStore     out = D + bias                       (fp32)
//   kEpiGelu      z = D + bias -> pre (fp32), gelu(z) -> act (bf16)      forward hidden layer
//   kEpiGeluGrad  g = D * gelu'(pre) -> act (bf16)                       backward hidden layer
// One layer's forward is one launch; the backward data gradients dH = dZ W are the same kernel
// with the transposed weights; the weight gradients dW = dZ^T H are the same kernel with K = the
// batch (operands transposed by k_transpose).  Every reduction runs in a fixed order: training
// is deterministic.
//
// Every wait on the tensor core is bounded; a wait that runs out sets the status word, waits
// once more (bounded) for the MMA in flight, frees the TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/sw2d_b200.h"
#include "sw2d_internal.cuh"
#include "umma.cuh"

namespace {

using namespace sw2d::umma;

constexpr int kKC = 64;                   // K chunk staged in shared memory
constexpr int kMaxN = 128;
constexpr long long kWaitPolls = 1LL << 26;  // ~ seconds of polling: far beyond any MMA here
constexpr unsigned kStatusTimeout = 1u;

enum { kEpiStore = 0, kEpiGelu = 1, kEpiGeluGrad = 2 };

struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    int M, N, K, lda, ldb;
    const float* bias;       // [N] or null
    float* out;              // fp32 [M x ldo] (kEpiStore: D + bias; kEpiGelu: pre-activation)
    __nv_bfloat16* act;      // bf16 [M x lda_out] (kEpiGelu, kEpiGeluGrad)
    const float* pre;        // kEpiGeluGrad: pre-activation [M x ldo]
    int ldo, ldact;
    int n_valid;             // columns written (<= N)
    uint32_t tmem_cols;      // power of two >= max(32, N)
    unsigned* status;
    long long first_wait;    // polls of a chunk's first wait on the tensor core (the drain wait: kWaitPolls)
};

// GELU in its tanh form, 0.5 x (1 + tanh(k0 (x + k1 x^3))), with the hardware tanh
// (tanh.approx.f32, relative error about 2^-11: below the BF16 rounding the activation gets
// next) and explicit FMAs, so that training and inference share one activation whatever the
// file's contraction flags
__device__ __forceinline__ float tanh_hw(float u)
{
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return t;
}

constexpr float kGeluK0 = 0.7978845608028654f, kGeluK1 = 0.044715f;

__device__ __forceinline__ float gelu(float x)
{
    const float u = x * __fmaf_rn(kGeluK0 * kGeluK1, x * x, kGeluK0);
    const float hx = 0.5f * x;
    return __fmaf_rn(hx, tanh_hw(u), hx);
}

// d/dx of gelu: 0.5 (1 + t) + 0.5 x (1 - t^2) k0 (1 + 3 k1 x^2), t = tanh(k0 (x + k1 x^3))
__device__ __forceinline__ float gelu_grad(float x)
{
    const float x2 = x * x;
    const float t = tanh_hw(x * __fmaf_rn(kGeluK0 * kGeluK1, x2, kGeluK0));
    const float du = __fmaf_rn(3.0f * kGeluK0 * kGeluK1, x2, kGeluK0);
    const float sech2 = __fmaf_rn(-t, t, 1.0f);
    return __fmaf_rn(0.5f * x * sech2, du, __fmaf_rn(0.5f, t, 0.5f));
}

// Two GELUs at once in packed FP32 (sm_100 add / mul / fma .rn.f32x2): per lane the same IEEE
// operations, in the same order, as gelu() above, so the results are the same bit for bit,
// with about half the FP32 instructions.
__device__ __forceinline__ unsigned long long pack2(float a, float b)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float& a, float& b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c)
{
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// gelu(z0 + b0), gelu(z1 + b1)
__device__ __forceinline__ void gelu_bias2(float z0, float z1, float b0, float b1, float& g0, float& g1)
{
    const unsigned long long x = add2(pack2(z0, z1), pack2(b0, b1));
    const unsigned long long p = fma2(pack2(kGeluK0 * kGeluK1, kGeluK0 * kGeluK1), mul2(x, x), pack2(kGeluK0, kGeluK0));
    float u0, u1;
    unpack2(mul2(x, p), u0, u1);
    const unsigned long long hx = mul2(pack2(0.5f, 0.5f), x);
    unpack2(fma2(hx, pack2(tanh_hw(u0), tanh_hw(u1)), hx), g0, g1);
}

template <int kMode>
__global__ void __launch_bounds__(128) k_umma_gemm(GemmArgs g)
{
    __shared__ __align__(1024) uint16_t sA[kTileM * kKC];
    __shared__ __align__(1024) uint16_t sB[kMaxN * kKC];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_holder;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row0 = blockIdx.x * kTileM;
    if (warp == 0) {
        tmem_alloc(&tmem_holder, g.tmem_cols);
        tmem_relinquish();
    }
    if (tid == 0) mbar_init(&bar, 1);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_holder;
    const uint32_t idesc = idesc_bf16_f32(kTileM, g.N);
    uint32_t phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < g.K; k0 += kKC) {
        const int kc = min(kKC, g.K - k0);  // a multiple of 16
        const int nv = kc >> 3;             // 16-byte vectors per row
        {
            const int r = row0 + tid;
            for (int c = 0; c < nv; c++) {
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (r < g.M) v = *reinterpret_cast<const uint4*>(g.A + (size_t)r * g.lda + k0 + c * 8);
                *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sA) + core_offset(tid, c * 8, kc)) = v;
            }
        }
        for (int i = tid; i < g.N * nv; i += 128) {
            const int n = i / nv, c = i - n * nv;
            const uint4 v = *reinterpret_cast<const uint4*>(g.B + (size_t)n * g.ldb + k0 + c * 8);
            *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sB) + core_offset(n, c * 8, kc)) = v;
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int s = 0; s < kc / 16; s++)
                mma_bf16(tmem, smem_desc(a0 + 256u * s, kc), smem_desc(b0 + 256u * s, kc), idesc,
                         (k0 > 0 || s > 0) ? 1u : 0u);
            mma_commit(&bar);
        }
        if (!mbar_wait(&bar, phase, g.first_wait)) {
            ok = false;
            mbar_wait(&bar, phase, kWaitPolls);  // the MMA still in flight: give it time once more
        }
        phase ^= 1u;
        // every thread past the wait before the tiles are overwritten; a failed wait stops all
        ok = __syncthreads_and(ok);
        if (!ok) break;
    }
    fence_after_sync();
    const int r = row0 + 32 * warp + lane;
    for (int c0 = 0; c0 < g.N; c0 += 16) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
        tmem_wait_ld();
        if (!ok || r >= g.M) continue;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int n = c0 + j;
            if (n >= g.n_valid) continue;
            const float d = __uint_as_float(v[j]);
            if (kMode == kEpiStore) {
                g.out[(size_t)r * g.ldo + n] = d + (g.bias ? g.bias[n] : 0.0f);
            } else if (kMode == kEpiGelu) {
                const float z = d + (g.bias ? g.bias[n] : 0.0f);
                g.out[(size_t)r * g.ldo + n] = z;
                g.act[(size_t)r * g.ldact + n] = __float2bfloat16_rn(gelu(z));
            } else {
                g.act[(size_t)r * g.ldact + n] = __float2bfloat16_rn(d * gelu_grad(g.pre[(size_t)r * g.ldo + n]));
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, g.tmem_cols);
    if (!ok && tid == 0) atomicOr(g.status, kStatusTimeout);
}

// out[c * ldo + r] = in[r * ldi + c] for r < rows, c < cols (bf16)
__global__ void k_transpose(const __nv_bfloat16* __restrict__ in, int ldi, int rows, int cols, __nv_bfloat16* out,
                            int ldo)
{
    __shared__ __nv_bfloat16 t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        t[j][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * ldi + c] : __float2bfloat16_rn(0.0f);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = bx + j, r = by + threadIdx.x;
        if (c < cols && r < rows) out[(size_t)c * ldo + r] = t[threadIdx.x][j];
    }
}

uint32_t tmem_cols_for(int n)
{
    uint32_t c = 32;
    while ((int)c < n) c <<= 1;
    return c;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// The MLP object
// ------------------------------------------------------------------------------------------
namespace sw2d {

constexpr int kIn = 10, kInPad = 16, kHid = 64, kOut = 2, kOutPad = 16;
// parameter vector: W1 [64 x 10], b1 [64], W2 [64 x 64], b2 [64], W3 [2 x 64], b3 [2]
constexpr int kNW1 = kHid * kIn, kNB1 = kHid, kNW2 = kHid * kHid, kNB2 = kHid, kNW3 = kOut * kHid, kNB3 = kOut;
constexpr int kNParams = kNW1 + kNB1 + kNW2 + kNB2 + kNW3 + kNB3;

}  // namespace sw2d

struct sw2d_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    std::string err;
    unsigned* status = nullptr;
    long long first_wait = kWaitPolls;  // sw2d_mlp_set_wait_polls
    // fp32 master parameters, Adam moments, gradients
    float *p = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr;
    // bf16 operand copies: W1 [64 x 16] (inputs padded), W2 [64 x 64], W3 [16 x 64] (outputs padded),
    // and the transposed W2t [64 x 64], W3t [64 x 16] for the backward data gradients
    __nv_bfloat16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr, *w2t = nullptr, *w3t = nullptr;
    float *b1 = nullptr, *b2 = nullptr, *b3 = nullptr;  // fp32 biases (b3 padded to 16)
    // feature normalisation (x - mean) / std, target scale y * ystd + ymean
    float xmean[sw2d::kIn], xstd[sw2d::kIn], ymean[sw2d::kOut], ystd[sw2d::kOut];
    // work buffers for a batch of up to cap rows
    int64_t cap = 0;
    __nv_bfloat16 *x = nullptr, *h1 = nullptr, *h2 = nullptr, *dy = nullptr, *dz2 = nullptr, *dz1 = nullptr;
    __nv_bfloat16 *tA = nullptr, *tB = nullptr;
    float *z1 = nullptr, *z2 = nullptr, *y = nullptr, *t = nullptr, *loss = nullptr;
    float *raw = nullptr;  // raw features [cap x 10]
    float *gw1 = nullptr, *gw2 = nullptr, *gw3 = nullptr, *gb = nullptr;  // weight and bias gradients
    int64_t step = 0;
};

namespace {

int mlp_fail(sw2d_mlp* m, int code, const std::string& msg)
{
    if (m) m->err = msg;
    return code;
}

#define MCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return mlp_fail(m, SW2D_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <class T>
int malloc_dev(sw2d_mlp* m, size_t n, T** p)
{
    void* q = nullptr;
    MCK(cudaMalloc(&q, std::max<size_t>(1, n) * sizeof(T)));
    m->allocs.push_back(q);
    MCK(cudaMemsetAsync(q, 0, std::max<size_t>(1, n) * sizeof(T), m->stream));
    *p = static_cast<T*>(q);
    return SW2D_OK;
}

// bf16 operand copies of the fp32 parameters (padded and transposed)
__global__ void k_refresh_weights(const float* __restrict__ p, __nv_bfloat16* w1, __nv_bfloat16* w2,
                                  __nv_bfloat16* w3, __nv_bfloat16* w2t, __nv_bfloat16* w3t, float* b1, float* b2,
                                  float* b3)
{
    using namespace sw2d;
    const float* W1 = p;
    const float* B1 = W1 + kNW1;
    const float* W2 = B1 + kNB1;
    const float* B2 = W2 + kNW2;
    const float* W3 = B2 + kNB2;
    const float* B3 = W3 + kNW3;
    for (int i = threadIdx.x; i < kHid * kInPad; i += blockDim.x) {
        const int o = i / kInPad, k = i % kInPad;
        w1[i] = __float2bfloat16_rn(k < kIn ? W1[o * kIn + k] : 0.0f);
    }
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) {
        const int o = i / kHid, k = i % kHid;
        w2[i] = __float2bfloat16_rn(W2[i]);
        w2t[k * kHid + o] = __float2bfloat16_rn(W2[i]);
    }
    for (int i = threadIdx.x; i < kOutPad * kHid; i += blockDim.x) {
        const int o = i / kHid, k = i % kHid;
        const float v = o < kOut ? W3[o * kHid + k] : 0.0f;
        w3[i] = __float2bfloat16_rn(v);
        w3t[k * kOutPad + o] = __float2bfloat16_rn(v);
    }
    for (int i = threadIdx.x; i < kHid; i += blockDim.x) {
        b1[i] = B1[i];
        b2[i] = B2[i];
    }
    for (int i = threadIdx.x; i < kOutPad; i += blockDim.x) b3[i] = i < kOut ? B3[i] : 0.0f;
}

struct Norm {
    float xmean[sw2d::kIn], xstd[sw2d::kIn], ymean[sw2d::kOut], ystd[sw2d::kOut];
};

// raw features [n x 10] -> normalised bf16 [n x 16]; rows >= n (up to the padded count) zero
__global__ void k_features(const float* __restrict__ raw, int64_t n, int64_t npad, Norm nm, __nv_bfloat16* x)
{
    using namespace sw2d;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad) return;
    for (int k = 0; k < kInPad; k++) {
        float v = 0.0f;
        if (i < n && k < kIn) v = (raw[i * kIn + k] - nm.xmean[k]) / nm.xstd[k];
        x[i * kInPad + k] = __float2bfloat16_rn(v);
    }
}

// normalised targets [n x 16 padded]; loss gradient dY = 2 (y - t) / (n * 2) and per-block
// squared-error partial sums (deterministic reduction on the host)
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ t, int64_t n, int64_t npad,
                       __nv_bfloat16* dy, float* partial)
{
    using namespace sw2d;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float se = 0.0f;
    if (i < npad) {
        for (int k = 0; k < kOutPad; k++) {
            float g = 0.0f;
            if (i < n && k < kOut) {
                const float d = y[i * kOutPad + k] - t[i * kOut + k];
                se += d * d;
                g = 2.0f * d / (float)(n * kOut);
            }
            dy[i * kOutPad + k] = __float2bfloat16_rn(g);
        }
    }
    __shared__ float s[256];
    s[threadIdx.x] = se;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

// column sums of a bf16 [n x ld] array (bias gradients), one thread per column, fixed order
__global__ void k_colsum(const __nv_bfloat16* __restrict__ a, int64_t n, int ld, int cols, float* out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int64_t i = 0; i < n; i++) s += __bfloat162float(a[i * ld + c]);
    out[c] = s;
}

// gradient vector from the weight-gradient GEMM outputs (fp32 [rows x cols] with padding)
__global__ void k_pack_grad(const float* __restrict__ gw1, const float* __restrict__ gw2,
                            const float* __restrict__ gw3, const float* __restrict__ gb, float* grad)
{
    using namespace sw2d;
    for (int i = threadIdx.x; i < kNW1; i += blockDim.x) grad[i] = gw1[(i / kIn) * kInPad + (i % kIn)];
    for (int i = threadIdx.x; i < kNB1; i += blockDim.x) grad[kNW1 + i] = gb[i];
    for (int i = threadIdx.x; i < kNW2; i += blockDim.x) grad[kNW1 + kNB1 + i] = gw2[i];
    for (int i = threadIdx.x; i < kNB2; i += blockDim.x) grad[kNW1 + kNB1 + kNW2 + i] = gb[kHid + i];
    for (int i = threadIdx.x; i < kNW3; i += blockDim.x) grad[kNW1 + kNB1 + kNW2 + kNB2 + i] = gw3[i];
    for (int i = threadIdx.x; i < kNB3; i += blockDim.x) grad[kNParams - kNB3 + i] = gb[2 * kHid + i];
}

__global__ void k_adam(float* p, float* m1, float* m2, const float* __restrict__ g, int n, float lr, float b1,
                       float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

int gemm(sw2d_mlp* m, int mode, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
         const float* bias, float* out, int ldo, __nv_bfloat16* act, int ldact, const float* pre, int n_valid,
         cudaStream_t stream = nullptr)
{
    if (!stream) stream = m->stream;
    if (N % 16 || N > kMaxN || K % 16 || K <= 0 || M <= 0 || (lda % 8) || (ldb % 8))
        return mlp_fail(m, SW2D_E_ARG, "gemm: shape outside the kernel's contract");
    GemmArgs g{A, B, M, N, K, lda, ldb, bias, out, act, pre, ldo, ldact, n_valid, tmem_cols_for(N), m->status,
               m->first_wait};
    const unsigned grid = (unsigned)((M + kTileM - 1) / kTileM);
    if (mode == kEpiStore) k_umma_gemm<kEpiStore><<<grid, 128, 0, stream>>>(g);
    else if (mode == kEpiGelu) k_umma_gemm<kEpiGelu><<<grid, 128, 0, stream>>>(g);
    else k_umma_gemm<kEpiGeluGrad><<<grid, 128, 0, stream>>>(g);
    MCK(cudaGetLastError());
    return SW2D_OK;
}

int ensure_cap(sw2d_mlp* m, int64_t n)
{
    using namespace sw2d;
    const int64_t npad = (n + kTileM - 1) / kTileM * kTileM;
    if (npad <= m->cap) return SW2D_OK;
    int rc;
    if ((rc = malloc_dev(m, npad * kInPad, &m->x)) || (rc = malloc_dev(m, npad * kHid, &m->h1)) ||
        (rc = malloc_dev(m, npad * kHid, &m->h2)) || (rc = malloc_dev(m, npad * kOutPad, &m->dy)) ||
        (rc = malloc_dev(m, npad * kHid, &m->dz2)) || (rc = malloc_dev(m, npad * kHid, &m->dz1)) ||
        (rc = malloc_dev(m, npad * kHid, &m->tA)) || (rc = malloc_dev(m, npad * kHid, &m->tB)) ||
        (rc = malloc_dev(m, npad * kHid, &m->z1)) || (rc = malloc_dev(m, npad * kHid, &m->z2)) ||
        (rc = malloc_dev(m, npad * kOutPad, &m->y)) || (rc = malloc_dev(m, npad * kOut, &m->t)) ||
        (rc = malloc_dev(m, npad / 256 + 2, &m->loss)) || (rc = malloc_dev(m, npad * kIn, &m->raw)))
        return rc;
    m->cap = npad;
    return SW2D_OK;
}

Norm norm_of(const sw2d_mlp* m)
{
    Norm nm;
    std::memcpy(nm.xmean, m->xmean, sizeof(nm.xmean));
    std::memcpy(nm.xstd, m->xstd, sizeof(nm.xstd));
    std::memcpy(nm.ymean, m->ymean, sizeof(nm.ymean));
    std::memcpy(nm.ystd, m->ystd, sizeof(nm.ystd));
    return nm;
}

// forward of n rows already normalised in m->x (padded to a multiple of 128): Z1, H1, Z2, H2, Y
int forward(sw2d_mlp* m, int64_t npad)
{
    using namespace sw2d;
    int rc;
    if ((rc = gemm(m, kEpiGelu, m->x, kInPad, m->w1, kInPad, (int)npad, kHid, kInPad, m->b1, m->z1, kHid, m->h1, kHid,
                   nullptr, kHid)))
        return rc;
    if ((rc = gemm(m, kEpiGelu, m->h1, kHid, m->w2, kHid, (int)npad, kHid, kHid, m->b2, m->z2, kHid, m->h2, kHid,
                   nullptr, kHid)))
        return rc;
    return gemm(m, kEpiStore, m->h2, kHid, m->w3, kHid, (int)npad, kOutPad, kHid, m->b3, m->y, kOutPad, nullptr, 0,
                nullptr, kOutPad);
}

}  // namespace

extern "C" {

int sw2d_mlp_create(int device, const float* params, const float* norm, sw2d_mlp** out)
{
    using namespace sw2d;
    if (!params || !norm || !out) return SW2D_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return SW2D_E_NO_DEVICE;
    sw2d_mlp* m = new sw2d_mlp();
    m->device = device;
    auto bail = [&](int code) {
        sw2d_mlp_destroy(m);
        return code;
    };
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(SW2D_E_CUDA);
    for (int k = 0; k < kIn; k++) {
        m->xmean[k] = norm[k];
        m->xstd[k] = norm[kIn + k];
        if (!(m->xstd[k] > 0.0f)) return bail(SW2D_E_ARG);
    }
    for (int k = 0; k < kOut; k++) {
        m->ymean[k] = norm[2 * kIn + k];
        m->ystd[k] = norm[2 * kIn + kOut + k];
        if (!(m->ystd[k] > 0.0f)) return bail(SW2D_E_ARG);
    }
    int rc;
    if ((rc = malloc_dev(m, kNParams, &m->p)) || (rc = malloc_dev(m, kNParams, &m->m1)) ||
        (rc = malloc_dev(m, kNParams, &m->m2)) || (rc = malloc_dev(m, kNParams, &m->grad)) ||
        (rc = malloc_dev(m, kHid * kInPad, &m->w1)) || (rc = malloc_dev(m, kHid * kHid, &m->w2)) ||
        (rc = malloc_dev(m, kOutPad * kHid, &m->w3)) || (rc = malloc_dev(m, kHid * kHid, &m->w2t)) ||
        (rc = malloc_dev(m, kHid * kOutPad, &m->w3t)) || (rc = malloc_dev(m, kHid, &m->b1)) ||
        (rc = malloc_dev(m, kHid, &m->b2)) || (rc = malloc_dev(m, kOutPad, &m->b3)) ||
        (rc = malloc_dev(m, 1, &m->status)) || (rc = malloc_dev(m, kHid * kInPad, &m->gw1)) ||
        (rc = malloc_dev(m, kHid * kHid, &m->gw2)) || (rc = malloc_dev(m, kOutPad * kHid, &m->gw3)) ||
        (rc = malloc_dev(m, 2 * kHid + kOutPad, &m->gb)))
        return bail(rc);
    if (cudaMemcpyAsync(m->p, params, kNParams * sizeof(float), cudaMemcpyHostToDevice, m->stream) != cudaSuccess)
        return bail(SW2D_E_CUDA);
    k_refresh_weights<<<1, 256, 0, m->stream>>>(m->p, m->w1, m->w2, m->w3, m->w2t, m->w3t, m->b1, m->b2, m->b3);
    if (cudaStreamSynchronize(m->stream) != cudaSuccess) return bail(SW2D_E_CUDA);
    *out = m;
    return SW2D_OK;
}

int sw2d_mlp_destroy(sw2d_mlp* m)
{
    if (!m) return SW2D_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    for (void* p : m->allocs) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return SW2D_OK;
}

const char* sw2d_mlp_last_error(sw2d_mlp* m) { return m ? m->err.c_str() : ""; }

int sw2d_mlp_set_wait_polls(sw2d_mlp* m, int64_t polls)
{
    if (!m) return SW2D_E_ARG;
    m->first_wait = polls < 0 ? kWaitPolls : (long long)polls;
    return SW2D_OK;
}

int sw2d_mlp_get_params(sw2d_mlp* m, float* params)
{
    using namespace sw2d;
    if (!m || !params) return SW2D_E_ARG;
    MCK(cudaSetDevice(m->device));
    MCK(cudaMemcpyAsync(params, m->p, kNParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCK(cudaStreamSynchronize(m->stream));
    return SW2D_OK;
}

// Outputs of n raw feature rows (host [n x 10]) in physical units (host [n x 2]).  With `layers`
// non-null it also returns the hidden activations for checks: Z1, H1, Z2, H2 [n x 64] each.
int sw2d_mlp_infer(sw2d_mlp* m, const float* features, int64_t n, float* outputs, float* layers)
{
    using namespace sw2d;
    if (!m || !features || !outputs || n <= 0) return SW2D_E_ARG;
    MCK(cudaSetDevice(m->device));
    int rc = ensure_cap(m, n);
    if (rc) return rc;
    const int64_t npad = (n + kTileM - 1) / kTileM * kTileM;
    MCK(cudaMemcpyAsync(m->raw, features, n * kIn * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    k_features<<<(unsigned)((npad + 255) / 256), 256, 0, m->stream>>>(m->raw, n, npad, norm_of(m), m->x);
    if ((rc = forward(m, npad))) return rc;
    std::vector<float> y((size_t)n * kOutPad);
    MCK(cudaMemcpyAsync(y.data(), m->y, n * kOutPad * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    if (layers) {
        std::vector<__nv_bfloat16> hb((size_t)n * kHid);
        MCK(cudaMemcpyAsync(layers, m->z1, n * kHid * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        MCK(cudaMemcpyAsync(layers + 2 * n * kHid, m->z2, n * kHid * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
        MCK(cudaMemcpyAsync(hb.data(), m->h1, n * kHid * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost, m->stream));
        MCK(cudaStreamSynchronize(m->stream));
        for (int64_t i = 0; i < n * kHid; i++) layers[n * kHid + i] = __bfloat162float(hb[i]);
        MCK(cudaMemcpyAsync(hb.data(), m->h2, n * kHid * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost, m->stream));
        MCK(cudaStreamSynchronize(m->stream));
        for (int64_t i = 0; i < n * kHid; i++) layers[3 * n * kHid + i] = __bfloat162float(hb[i]);
    }
    MCK(cudaStreamSynchronize(m->stream));
    unsigned st = 0;
    MCK(cudaMemcpy(&st, m->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (st) {
        // reported once: the kernel that ran out freed its TMEM, and the object stays usable
        MCK(cudaMemset(m->status, 0, sizeof(unsigned)));
        return mlp_fail(m, SW2D_E_CUDA, "tensor-core wait ran out");
    }
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < kOut; k++) outputs[i * kOut + k] = y[i * kOutPad + k] * m->ystd[k] + m->ymean[k];
    return SW2D_OK;
}

// One pass of gradient computation on a batch (host features [n x 10], targets [n x 2] in
// physical units): the loss (mean squared error of the normalised outputs) and its gradient
// with respect to the parameter vector (host [kNParams], may be null).
int sw2d_mlp_loss_grad(sw2d_mlp* m, const float* features, const float* targets, int64_t n, double* loss,
                       float* grad_out)
{
    using namespace sw2d;
    if (!m || !features || !targets || n <= 0) return SW2D_E_ARG;
    MCK(cudaSetDevice(m->device));
    int rc = ensure_cap(m, n);
    if (rc) return rc;
    const int64_t npad = (n + kTileM - 1) / kTileM * kTileM;
    std::vector<float> tn((size_t)n * kOut);
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < kOut; k++) tn[i * kOut + k] = (targets[i * kOut + k] - m->ymean[k]) / m->ystd[k];
    MCK(cudaMemcpyAsync(m->raw, features, n * kIn * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MCK(cudaMemcpyAsync(m->t, tn.data(), n * kOut * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    k_features<<<(unsigned)((npad + 255) / 256), 256, 0, m->stream>>>(m->raw, n, npad, norm_of(m), m->x);
    if ((rc = forward(m, npad))) return rc;
    const unsigned lb = (unsigned)((npad + 255) / 256);
    k_loss<<<lb, 256, 0, m->stream>>>(m->y, m->t, n, npad, m->dy, m->loss);
    // backward data gradients on the tensor cores: dZ2 = (dY W3) * gelu'(Z2), dZ1 = (dZ2 W2) * gelu'(Z1)
    if ((rc = gemm(m, kEpiGeluGrad, m->dy, kOutPad, m->w3t, kOutPad, (int)npad, kHid, kOutPad, nullptr, nullptr, kHid,
                   m->dz2, kHid, m->z2, kHid)))
        return rc;
    if ((rc = gemm(m, kEpiGeluGrad, m->dz2, kHid, m->w2t, kHid, (int)npad, kHid, kHid, nullptr, nullptr, kHid, m->dz1,
                   kHid, m->z1, kHid)))
        return rc;
    // weight gradients on the tensor cores with K = the batch: dW = dZ^T H
    float *gw1 = m->gw1, *gw2 = m->gw2, *gw3 = m->gw3, *gb = m->gb;
    const int K = (int)npad;
    dim3 tb(32, 8);
    auto transpose = [&](const __nv_bfloat16* a, int cols, __nv_bfloat16* o) {
        dim3 gr((unsigned)((cols + 31) / 32), (unsigned)((npad + 31) / 32));
        k_transpose<<<gr, tb, 0, m->stream>>>(a, cols, (int)npad, cols, o, (int)npad);
    };
    transpose(m->dy, kOutPad, m->tA);
    transpose(m->h2, kHid, m->tB);
    if ((rc = gemm(m, kEpiStore, m->tA, K, m->tB, K, kOutPad, kHid, K, nullptr, gw3, kHid, nullptr, 0, nullptr, kHid)))
        return rc;
    transpose(m->dz2, kHid, m->tA);
    transpose(m->h1, kHid, m->tB);
    if ((rc = gemm(m, kEpiStore, m->tA, K, m->tB, K, kHid, kHid, K, nullptr, gw2, kHid, nullptr, 0, nullptr, kHid)))
        return rc;
    transpose(m->dz1, kHid, m->tA);
    transpose(m->x, kInPad, m->tB);
    if ((rc = gemm(m, kEpiStore, m->tA, K, m->tB, K, kHid, kInPad, K, nullptr, gw1, kInPad, nullptr, 0, nullptr,
                   kInPad)))
        return rc;
    k_colsum<<<1, 64, 0, m->stream>>>(m->dz1, npad, kHid, kHid, gb);
    k_colsum<<<1, 64, 0, m->stream>>>(m->dz2, npad, kHid, kHid, gb + kHid);
    k_colsum<<<1, 64, 0, m->stream>>>(m->dy, npad, kOutPad, kOutPad, gb + 2 * kHid);
    k_pack_grad<<<1, 256, 0, m->stream>>>(gw1, gw2, gw3, gb, m->grad);
    MCK(cudaGetLastError());
    std::vector<float> part(lb);
    MCK(cudaMemcpyAsync(part.data(), m->loss, lb * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    if (grad_out) MCK(cudaMemcpyAsync(grad_out, m->grad, kNParams * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCK(cudaStreamSynchronize(m->stream));
    unsigned st = 0;
    MCK(cudaMemcpy(&st, m->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (st) {
        // reported once: the kernel that ran out freed its TMEM, and the object stays usable
        MCK(cudaMemset(m->status, 0, sizeof(unsigned)));
        return mlp_fail(m, SW2D_E_CUDA, "tensor-core wait ran out");
    }
    double s = 0.0;
    for (float v : part) s += v;
    if (loss) *loss = s / (double)(n * kOut);
    return SW2D_OK;
}

// Adam step (learning rate lr, beta1 0.9, beta2 0.999, eps 1e-8) on the gradient of the last
// sw2d_mlp_loss_grad call, then refresh of the bf16 operand copies.
int sw2d_mlp_adam_step(sw2d_mlp* m, float lr)
{
    using namespace sw2d;
    if (!m) return SW2D_E_ARG;
    MCK(cudaSetDevice(m->device));
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
    k_adam<<<(kNParams + 255) / 256, 256, 0, m->stream>>>(m->p, m->m1, m->m2, m->grad, kNParams, lr, b1, b2, 1e-8f,
                                                           c1, c2);
    k_refresh_weights<<<1, 256, 0, m->stream>>>(m->p, m->w1, m->w2, m->w3, m->w2t, m->w3t, m->b1, m->b2, m->b3);
    MCK(cudaGetLastError());
    MCK(cudaStreamSynchronize(m->stream));
    return SW2D_OK;
}

int sw2d_mlp_param_count(void) { return sw2d::kNParams; }

}  // extern "C"

// ------------------------------------------------------------------------------------------
// The closure inside a model's step.  With a network attached (sw2d_set_closure), the DIP cell
// update runs as k_update_closure: per tile of 128 cells it forms the flux balance of every
// cell as the plain update does, then the ten features of the cell from the state at the step's
// start and the balanced one, runs the network on the tensor cores and adds the momentum
// correction it outputs where the features lie in the training hull, at the place where the
// plain momentum-dissipation closure acts (dip/swDipHyp.cpp:295-324, before the round-off
// flush and the sources).  Elsewhere the plain closure is applied as the update applies it when
// the model has one.  No launch is added to the step.
// ------------------------------------------------------------------------------------------
namespace sw2d {

struct ClosureState {
    sw2d_mlp* net = nullptr;
    float lo[kIn], hi[kIn];
    float scale = 1.0f;  // factor on the network's correction
    float* phig_min = nullptr;
    float* rec = nullptr;  // [nc x 12] features and outputs of the last step, or null
    unsigned grid = 0;     // persistent grid of the update kernel
    int sms = 0, per_sm_max = 1;  // SMs, resident CTAs per SM the kernel's resources allow
    int64_t ntiles = 0;
    std::vector<void*> allocs;
};

// the ten features of a cell from the state at the start of the step (a) and after the flux
// balance (b): depth, unit discharges, their increments, storage porosity, the smallest
// connectivity porosity of the cell's internal edges, dt and the speed at the start
SW2D_HD void closure_features(double4 a, double4 b, double phiw, double phig_min, double dt, double* f)
{
    f[0] = a.x;
    f[1] = a.y;
    f[2] = a.z;
    f[3] = b.x - a.x;
    f[4] = b.y - a.y;
    f[5] = b.z - a.z;
    f[6] = phiw;
    f[7] = phig_min;
    f[8] = dt;
    f[9] = sqrt(a.y * a.y + a.z * a.z) / fmax(a.x, 1e-3);
}

}  // namespace sw2d

namespace {

using namespace sw2d;

constexpr int kRec = kIn + kOut;  // floats per cell in the feature record

struct ClosureNorm {
    float xmean[kIn], xstd[kIn], lo[kIn], hi[kIn], ymean[kOut], ystd[kOut], scale;
};

struct ClosureArgs {
    const float* phig_min;
    ClosureNorm cn;
    const __nv_bfloat16 *w1, *w2, *w3;
    const float *b1, *b2, *b3;
    float* rec;
    int dissip;
    unsigned* status;
};

__global__ void k_closure_phig_min(DevMesh m, float* out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int k0 = m.coff[c].x, k1 = m.coff[c + 1].x;
    double g = 1.0;
    for (int k = k0; k < k1; k++) g = fmin(g, m.phig[m.cint[k].x >> 1]);
    out[c] = (float)g;
}

// The DIP cell update with the network at the closure site, persistent over tiles of 128 cells
// (thread i of the CTA owns cell i of the tile, which is TMEM lane i).  Per tile: the flux
// balance (as k_update: swSpHyp.cpp:214-273), the features as the first layer's BF16 A operand
// in shared memory, then per layer one round of MMAs into TMEM whose epilogue (bias, GELU,
// BF16) writes the next layer's A operand back to shared memory; the three accumulators share
// TMEM columns [0, 64), each layer's MMAs issued after every lane has read the previous one
// out.  Then the correction (in the hull) or the plain closure, the round-off flush, the
// negative-depth rule, friction and head loss, and the new state.  The weights are staged once
// per CTA.  The MMAs, their order and the epilogue arithmetic are those of the GEMM kernel, so
// the outputs equal sw2d_mlp_infer's on the same features bit for bit.
template <int kFriction, bool kHeadLoss>
__global__ void __launch_bounds__(128) k_update_closure(DevMesh m, ClosureArgs a)
{
    __shared__ __align__(1024) uint16_t sX[kTileM * kInPad];
    __shared__ __align__(1024) uint16_t sH[kTileM * kHid];
    __shared__ __align__(1024) uint16_t sW1[kHid * kInPad];
    __shared__ __align__(1024) uint16_t sW2[kHid * kHid];
    __shared__ __align__(1024) uint16_t sW3[kOutPad * kHid];
    __shared__ float sb1[kHid], sb2[kHid], sb3[kOutPad];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_holder;
    Ctrl* ctrl = m.ctrl;
    if (!ctrl->go) return;  // uniform over the grid: nothing allocated yet
    const double dt = ctrl->dt;
    const int tid = threadIdx.x, warp = tid >> 5;
    if (blockIdx.x == 0 && tid == 0) {
        ctrl->t = ctrl->t + dt;  // swSp.cpp:592; no other thread of this kernel reads t
        ctrl->steps += 1;
    }
    const uint32_t ncols = 64;
    if (warp == 0) {
        tmem_alloc(&tmem_holder, ncols);
        tmem_relinquish();
    }
    if (tid == 0) mbar_init(&bar, 1);
    // weights in the K-major core-matrix layout, biases
    for (int i = tid; i < kHid * (kInPad / 8); i += 128) {
        const int n = i / (kInPad / 8), c = i % (kInPad / 8);
        *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sW1) + core_offset(n, c * 8, kInPad)) =
            *reinterpret_cast<const uint4*>(a.w1 + n * kInPad + c * 8);
    }
    for (int i = tid; i < kHid * (kHid / 8); i += 128) {
        const int n = i / (kHid / 8), c = i % (kHid / 8);
        *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sW2) + core_offset(n, c * 8, kHid)) =
            *reinterpret_cast<const uint4*>(a.w2 + n * kHid + c * 8);
    }
    for (int i = tid; i < kOutPad * (kHid / 8); i += 128) {
        const int n = i / (kHid / 8), c = i % (kHid / 8);
        *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sW3) + core_offset(n, c * 8, kHid)) =
            *reinterpret_cast<const uint4*>(a.w3 + n * kHid + c * 8);
    }
    if (tid < kHid) {
        sb1[tid] = a.b1[tid];
        sb2[tid] = a.b2[tid];
    }
    if (tid < kOutPad) sb3[tid] = a.b3[tid];
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_holder;
    const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
    const uint32_t id64 = idesc_bf16_f32(kTileM, kHid), id16 = idesc_bf16_f32(kTileM, kOutPad);
    const uint32_t aX = smem_u32(sX), aH = smem_u32(sH), aW1 = smem_u32(sW1), aW2 = smem_u32(sW2),
                   aW3 = smem_u32(sW3);
    const ClosureNorm& cn = a.cn;
    uint32_t phase = 0;
    bool ok = true;
    const int ntiles = (m.nc + kTileM - 1) / kTileM;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int c = tile * kTileM + tid;
        const bool valid = c < m.nc;
        double4 s0 = make_double4(0, 0, 0, 0);
        double hh = 0, qq = 0, rr = 0;
        bool in = false;
        float f32[kIn];
        {
            float xv[kInPad];
            for (int k = 0; k < kInPad; k++) xv[k] = 0.0f;
            if (valid) {
                s0 = m.st[c];
                hh = s0.x;
                qq = s0.y;
                rr = s0.z;
                // hypComputeBalance (swSpHyp.cpp:214-273), the slots in the reference's order
                const int k0 = ld(&m.coff[c].y), k1 = ld(&m.coff[c + 1].y);
                for (int k = k0; k < k1; k++) {
                    const Slot v = m.slot[k];
                    hh += v.a * dt;
                    qq += v.b * dt;
                    rr += v.c * dt;
                }
                double f[kIn];
                closure_features(s0, make_double4(hh, qq, rr, 0.0), ld(&m.cst[c].z), a.phig_min[c], dt, f);
                in = true;
                for (int k = 0; k < kIn; k++) {
                    f32[k] = (float)f[k];
                    in = in && (f32[k] >= cn.lo[k]) && (f32[k] <= cn.hi[k]);
                    xv[k] = (f32[k] - cn.xmean[k]) / cn.xstd[k];
                }
            }
            for (int cc = 0; cc < kInPad / 8; cc++) {
                uint32_t pk[4];
                for (int j = 0; j < 4; j++) {
                    const __nv_bfloat162 pr = __floats2bfloat162_rn(xv[cc * 8 + 2 * j], xv[cc * 8 + 2 * j + 1]);
                    pk[j] = *reinterpret_cast<const uint32_t*>(&pr);
                }
                *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sX) + core_offset(tid, cc * 8, kInPad)) =
                    make_uint4(pk[0], pk[1], pk[2], pk[3]);
            }
        }
        // the network runs only for tiles with a cell inside the training hull (or while the
        // closure's inputs and outputs are recorded): elsewhere its outputs are not used
        fence_proxy_async();
        const bool net = __syncthreads_or((int)(valid && in)) != 0 || a.rec != nullptr;
        uint32_t v[16];
        for (int j = 0; j < 16; j++) v[j] = 0u;
        if (net) {
            // layer 1: one MMA of K = 16
            if (tid == 0) {
                fence_after_sync();
                mma_bf16(tmem, smem_desc(aX, kInPad), smem_desc(aW1, kInPad), id64, 0u);
                mma_commit(&bar);
            }
            if (!mbar_wait(&bar, phase, kWaitPolls)) {
                ok = false;
                mbar_wait(&bar, phase, kWaitPolls);
            }
            phase ^= 1u;
            fence_after_sync();
            // the hidden layers' epilogues, each followed by the next layer's four MMAs of K = 16
            for (int layer = 0; layer < 2; layer++) {
                const float* bias = layer == 0 ? sb1 : sb2;
                for (int c0 = 0; c0 < kHid; c0 += 16) {
                    uint32_t v[16];
                    tmem_ld16(lane_base + (uint32_t)c0, v);
                    tmem_wait_ld();
                    uint32_t hv[8];  // bf16 pairs
                    for (int j = 0; j < 8; j++) {
                        float g0, g1;
                        gelu_bias2(__uint_as_float(v[2 * j]), __uint_as_float(v[2 * j + 1]), bias[c0 + 2 * j],
                                   bias[c0 + 2 * j + 1], g0, g1);
                        const __nv_bfloat162 pr = __floats2bfloat162_rn(g0, g1);
                        hv[j] = *reinterpret_cast<const uint32_t*>(&pr);
                    }
                    *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sH) + core_offset(tid, c0, kHid)) =
                        make_uint4(hv[0], hv[1], hv[2], hv[3]);
                    *reinterpret_cast<uint4*>(reinterpret_cast<char*>(sH) + core_offset(tid, c0 + 8, kHid)) =
                        make_uint4(hv[4], hv[5], hv[6], hv[7]);
                }
                fence_before_sync();
                fence_proxy_async();
                __syncthreads();
                if (tid == 0) {
                    fence_after_sync();
                    const uint32_t bw = layer == 0 ? aW2 : aW3;
                    const uint32_t id = layer == 0 ? id64 : id16;
                    for (int s2 = 0; s2 < kHid / 16; s2++)
                        mma_bf16(tmem, smem_desc(aH + 256u * s2, kHid), smem_desc(bw + 256u * s2, kHid), id,
                                 s2 > 0 ? 1u : 0u);
                    mma_commit(&bar);
                }
                if (!mbar_wait(&bar, phase, kWaitPolls)) {
                    ok = false;
                    mbar_wait(&bar, phase, kWaitPolls);
                }
                phase ^= 1u;
                fence_after_sync();
            }
            tmem_ld16(lane_base, v);
            tmem_wait_ld();
        }
        if (valid && ok) {
            // the network's outputs in physical units, as sw2d_mlp_infer gives them
            const float y0 = (__uint_as_float(v[0]) + sb3[0]) * cn.ystd[0] + cn.ymean[0];
            const float y1 = (__uint_as_float(v[1]) + sb3[1]) * cn.ystd[1] + cn.ymean[1];
            if (a.rec) {
                float* r = a.rec + (size_t)c * kRec;
                for (int k = 0; k < kIn; k++) r[k] = f32[k];
                r[kIn] = y0;
                r[kIn + 1] = y1;
            }
            if (in) {
                qq += (double)(cn.scale * y0);
                rr += (double)(cn.scale * y1);
            } else if (a.dissip) {  // the plain closure (dip/swDipHyp.cpp:295-324)
                const double4 mu = ld(&m.mu[c]);
                momentum_dissipation(mu.x, mu.y, mu.z, mu.w, s0.x, s0.y, s0.z, hh, qq, rr);
            }
            if (fabs(hh) < kSmallReal) hh = 0.;
            if (fabs(qq) < kSmallReal) qq = 0.;
            if (fabs(rr) < kSmallReal) rr = 0.;
            // negative depth (swSpHyp.cpp:182-210)
            if (m.neg_detect) {
                if (hh < 0) atomicOr(&ctrl->status, kStatusNegDepth);
            } else if (hh < 0.) {
                hh = 0.;
                qq = 0.;
                rr = 0.;
            }
            cell_sources<kFriction, kHeadLoss>(m, c, dt, hh, qq, rr);
            m.st[c] = make_double4(hh, qq, rr, hh + ld(&m.zbv[c]));
        }
        fence_before_sync();
        ok = __syncthreads_and(ok);  // every lane read out before the next tile's MMAs overwrite TMEM
        if (!ok) break;
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, ncols);
    if (!ok && tid == 0) atomicOr(a.status, kStatusTimeout);
}

// the largest shared-memory carveout for every instance, so that the resident CTAs the
// occupancy query counts on fit
template <int kF>
cudaError_t closure_carveout()
{
    cudaError_t e = cudaFuncSetAttribute(k_update_closure<kF, false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_update_closure<kF, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    return e;
}

template <int kF>
void launch_closure_f(sw2d_handle* h, const DevMesh& m, const ClosureArgs& a, unsigned g)
{
    if (h->p.singular_head_loss) k_update_closure<kF, true><<<g, 128, 0, h->stream>>>(m, a);
    else k_update_closure<kF, false><<<g, 128, 0, h->stream>>>(m, a);
}

ClosureNorm closure_norm(const ClosureState* c)
{
    ClosureNorm cn;
    const sw2d_mlp* n = c->net;
    std::memcpy(cn.xmean, n->xmean, sizeof(cn.xmean));
    std::memcpy(cn.xstd, n->xstd, sizeof(cn.xstd));
    std::memcpy(cn.lo, c->lo, sizeof(cn.lo));
    std::memcpy(cn.hi, c->hi, sizeof(cn.hi));
    std::memcpy(cn.ymean, n->ymean, sizeof(cn.ymean));
    std::memcpy(cn.ystd, n->ystd, sizeof(cn.ystd));
    cn.scale = c->scale;
    return cn;
}

void closure_free(ClosureState* c)
{
    if (!c) return;
    for (void* p : c->allocs) cudaFree(p);
    delete c;
}

}  // namespace

namespace sw2d {

void closure_update(sw2d_handle* h, const DevMesh& m)
{
    ClosureState* c = h->closure;
    sw2d_mlp* net = c->net;
    ClosureArgs a;
    a.phig_min = c->phig_min;
    a.cn = closure_norm(c);
    a.w1 = net->w1;
    a.w2 = net->w2;
    a.w3 = net->w3;
    a.b1 = net->b1;
    a.b2 = net->b2;
    a.b3 = net->b3;
    a.rec = c->rec;
    a.dissip = h->dissipation && m.mu ? 1 : 0;
    a.status = net->status;
    switch (h->p.friction) {
        case SW2D_FRICTION_CHEZY: launch_closure_f<SW2D_FRICTION_CHEZY>(h, m, a, c->grid); break;
        case SW2D_FRICTION_MANNING: launch_closure_f<SW2D_FRICTION_MANNING>(h, m, a, c->grid); break;
        case SW2D_FRICTION_STRICKLER: launch_closure_f<SW2D_FRICTION_STRICKLER>(h, m, a, c->grid); break;
        default: launch_closure_f<SW2D_FRICTION_NONE>(h, m, a, c->grid); break;
    }
}

void closure_release(sw2d_handle* h)
{
    closure_free(h->closure);
    h->closure = nullptr;
}

int closure_set_ctas(sw2d_handle* h, int per_sm)
{
    ClosureState* c = h->closure;
    const int k = per_sm <= 0 ? c->per_sm_max : std::min(per_sm, c->per_sm_max);
    c->grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(c->ntiles, (int64_t)k * c->sms));
    return SW2D_OK;
}

int closure_record(sw2d_handle* h, int on)
{
    ClosureState* c = h->closure;
    if (on && !c->rec) {
        void* p = nullptr;
        const size_t bytes = (size_t)std::max<int64_t>(h->nc, 1) * kRec * sizeof(float);
        if (cudaMalloc(&p, bytes) != cudaSuccess) return fail(h, SW2D_E_CUDA, "closure record buffer");
        c->allocs.push_back(p);
        if (cudaMemset(p, 0, bytes) != cudaSuccess) return fail(h, SW2D_E_CUDA, "closure record buffer");
        c->rec = static_cast<float*>(p);
    } else if (!on) {
        c->rec = nullptr;  // the buffer stays allocated until the closure is detached
    }
    return SW2D_OK;
}

}  // namespace sw2d

using sw2d::fail;
using sw2d::grid_for;
using sw2d::kBlock;
using sw2d::kModelDip;

extern "C" {

int sw2d_set_closure(sw2d_handle* h, sw2d_mlp* net, const float* hull_lo, const float* hull_hi, float scale)
{
    using namespace sw2d;
    if (!h) return SW2D_E_ARG;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    closure_release(h);
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    if (!net) return SW2D_OK;
    if (h->model != sw2d::kModelDip) return fail(h, SW2D_E_UNSUPPORTED, "the learned closure runs on the DIP model");
    if (net->device != h->device) return fail(h, SW2D_E_ARG, "network and model on different devices");
    if (!hull_lo || !hull_hi) return fail(h, SW2D_E_ARG, "training hull missing");
    ClosureState* c = new ClosureState();
    c->net = net;
    std::memcpy(c->lo, hull_lo, sizeof(c->lo));
    std::memcpy(c->hi, hull_hi, sizeof(c->hi));
    c->scale = scale;
    void* p = nullptr;
    if (cudaMalloc(&p, (size_t)std::max<int64_t>(h->nc, 1) * sizeof(float)) != cudaSuccess) {
        closure_free(c);
        return fail(h, SW2D_E_CUDA, "closure buffers");
    }
    c->allocs.push_back(p);
    c->phig_min = static_cast<float*>(p);
    // persistent grid: every CTA resident at once (each holds 64 TMEM columns of the SM's 512)
    // resident CTAs per SM from the kernel's registers and shared memory (1 KB of it reserved per
    // CTA), at most 8: 8 x 64 TMEM columns fill the SM's 512
    cudaError_t e = closure_carveout<SW2D_FRICTION_NONE>();
    if (e == cudaSuccess) e = closure_carveout<SW2D_FRICTION_CHEZY>();
    if (e == cudaSuccess) e = closure_carveout<SW2D_FRICTION_MANNING>();
    if (e == cudaSuccess) e = closure_carveout<SW2D_FRICTION_STRICKLER>();
    cudaFuncAttributes fa;
    cudaDeviceProp prop;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_update_closure<SW2D_FRICTION_MANNING, true>);
    if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, h->device);
    if (e != cudaSuccess) {
        closure_free(c);
        return fail(h, SW2D_E_CUDA, std::string("closure launch set-up: ") + cudaGetErrorString(e));
    }
    c->sms = prop.multiProcessorCount;
    const int by_regs = prop.regsPerMultiprocessor / std::max(1, ((fa.numRegs * 32 + 255) / 256 * 256) * 4);
    const int by_smem = (int)(prop.sharedMemPerMultiprocessor / (fa.sharedSizeBytes + 1024));
    const int by_threads = prop.maxThreadsPerMultiProcessor / 128;
    c->per_sm_max = std::max(1, std::min(std::min(by_regs, by_smem), std::min(by_threads, 8)));
    c->ntiles = (h->nc + kTileM - 1) / kTileM;
    h->closure = c;
    closure_set_ctas(h, 0);
    k_closure_phig_min<<<grid_for(h->nc), kBlock, 0, h->stream>>>(h->m, c->phig_min);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return SW2D_OK;
}

// Features and network outputs of every cell in the last step taken with recording on
// (sw2d_set_option "closure_record"), in the caller's cell order: [n_cells x 12] floats, the
// ten features then the two outputs in physical units (before the scale factor and the hull
// test).  Returns the number of floats written.
int64_t sw2d_closure_record(sw2d_handle* h, float* out, int64_t capacity)
{
    using namespace sw2d;
    if (!h || !out) return SW2D_E_ARG;
    if (!h->closure || !h->closure->rec) return fail(h, SW2D_E_ARG, "closure recording is off");
    const int64_t n = h->nc * kRec;
    if (capacity < n) return fail(h, SW2D_E_ARG, "output buffer too small");
    CK(cudaSetDevice(h->device));
    std::vector<float> buf((size_t)n);
    CK(cudaMemcpyAsync(buf.data(), h->closure->rec, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int64_t i = 0; i < h->nc; i++)
        std::memcpy(out + (int64_t)h->cell_perm[i] * kRec, buf.data() + i * kRec, kRec * sizeof(float));
    return n;
}

}  // extern "C"
