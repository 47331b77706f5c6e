// Learned block-match proposals: a small MLP that reads coarse features of
// an anchor's neighbourhood and scores every offset of its search window, so
// that exact SSD runs only on a shortlist of the best-scored offsets.  It has
// no counterpart in the reference (whose matcher always searches the whole
// window, src/cuda/block_match.cu); it is the chosen form's learned part.
//
// Network: inputs -> hidden (ReLU) x layers -> outputs (one logit per offset
// (dx, dy, scheduled frame) of the window).  Weights are kept in FP32 for the
// optimiser and in BF16 for the forward and backward products, which
// accumulate in FP32.  Loss: softmax cross-entropy against the exact matcher's
// K nearest offsets, each weighted 1 / (their count).
//
// Kernels (all hand-written): a tiled GEMM C = op(A) op(B) (+ bias, ReLU) with
// FP32 or BF16 operands, the softmax loss and its gradient, the ReLU
// gradient, column sums (bias gradients), Adam; for inference the output
// layer on the 5th-generation tensor cores (tcgen05.mma, BF16 operands in
// shared memory, FP32 accumulators in tensor memory) and a per-row top-k of
// the logits by radix select for the shortlist.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>

#include "learned.h"

namespace vnlbgpu {
namespace {

constexpr int kTileM = 64, kTileN = 64, kTileK = 16;
constexpr int kGemmThreads = 256;  // 16 x 16 threads, 4 x 4 outputs each

template <typename T> __device__ __forceinline__ float to_f32(T v);
template <> __device__ __forceinline__ float to_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// C[M][N] (ldc) = alpha * op(A)[M][K] * op(B)[K][N] (+ bias[N]) (ReLU), with
// op(A)(i, k) = TA ? A[k * lda + i] : A[i * lda + k] and
// op(B)(k, j) = TB ? B[j * ldb + k] : B[k * ldb + j].
template <bool TA, bool TB, typename TypeA, typename TypeB>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(int M, int N, int K, const TypeA* A, int lda,
                                                             const TypeB* B, int ldb, float* C, int ldc,
                                                             const float* bias, int relu, float alpha,
                                                             int accumulate) {
    __shared__ float As[kTileK][kTileM + 4];
    __shared__ float Bs[kTileK][kTileN + 4];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * kTileM, n0 = blockIdx.x * kTileN;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += kTileK) {
        for (int e = tid; e < kTileK * kTileM; e += kGemmThreads) {
            int kk, i;
            if (TA) { i = e % kTileM; kk = e / kTileM; } else { kk = e % kTileK; i = e / kTileK; }
            const int gi = m0 + i, gk = k0 + kk;
            float v = 0.0f;
            if (gi < M && gk < K) v = to_f32(TA ? A[static_cast<size_t>(gk) * lda + gi] : A[static_cast<size_t>(gi) * lda + gk]);
            As[kk][i] = v;
        }
        for (int e = tid; e < kTileK * kTileN; e += kGemmThreads) {
            int kk, j;
            if (TB) { kk = e % kTileK; j = e / kTileK; } else { j = e % kTileN; kk = e / kTileN; }
            const int gj = n0 + j, gk = k0 + kk;
            float v = 0.0f;
            if (gj < N && gk < K) v = to_f32(TB ? B[static_cast<size_t>(gj) * ldb + gk] : B[static_cast<size_t>(gk) * ldb + gj]);
            Bs[kk][j] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kTileK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = As[kk][ty + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = Bs[kk][tx + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = fmaf(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int gi = m0 + ty + 16 * r;
        if (gi >= M) continue;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int gj = n0 + tx + 16 * c;
            if (gj >= N) continue;
            float v = alpha * acc[r][c];
            if (bias) v += bias[gj];
            if (relu) v = fmaxf(v, 0.0f);
            float* out = C + static_cast<size_t>(gi) * ldc + gj;
            *out = accumulate ? *out + v : v;
        }
    }
}

template <bool TA, bool TB, typename TypeA, typename TypeB>
cudaError_t gemm(int M, int N, int K, const TypeA* A, int lda, const TypeB* B, int ldb, float* C, int ldc,
                 const float* bias, bool relu, float alpha, bool accumulate, cudaStream_t stream) {
    if (M <= 0 || N <= 0) return cudaSuccess;
    const dim3 grid((N + kTileN - 1) / kTileN, (M + kTileM - 1) / kTileM);
    gemm_kernel<TA, TB, TypeA, TypeB><<<grid, kGemmThreads, 0, stream>>>(M, N, K, A, lda, B, ldb, C, ldc, bias,
                                                                        relu ? 1 : 0, alpha, accumulate ? 1 : 0);
    return cudaGetLastError();
}

// Softmax cross-entropy of each row of logits against its targets (up to
// `tk` class ids, -1 = none, each weighted 1 / count), one block per row.
// The logits become the gradient of the mean loss: (softmax - target) /
// rows.  loss[row] receives the row's loss.
__global__ void softmax_xent_kernel(float* logits, int classes, const int* targets, int tk, int rows,
                                    float* loss) {
    __shared__ float red[32];
    const int row = blockIdx.x;
    float* z = logits + static_cast<size_t>(row) * classes;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, warps = blockDim.x >> 5;
    float mx = -FLT_MAX;
    for (int i = tid; i < classes; i += blockDim.x) mx = fmaxf(mx, z[i]);
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    if (tid < 32) {
        float v = tid < warps ? red[tid] : -FLT_MAX;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (tid == 0) red[0] = v;
    }
    __syncthreads();
    mx = red[0];
    __syncthreads();
    float sum = 0.0f;
    for (int i = tid; i < classes; i += blockDim.x) sum += expf(z[i] - mx);
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) red[warp] = sum;
    __syncthreads();
    if (tid < 32) {
        float v = tid < warps ? red[tid] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (tid == 0) red[0] = v;
    }
    __syncthreads();
    const float lse = mx + logf(red[0]);
    const int* t = targets + static_cast<size_t>(row) * tk;
    int count = 0;
    for (int k = 0; k < tk; ++k) count += t[k] >= 0 && t[k] < classes;
    const float share = count > 0 ? 1.0f / static_cast<float>(count) : 0.0f;
    if (tid == 0 && loss) {
        float l = 0.0f;
        for (int k = 0; k < tk; ++k)
            if (t[k] >= 0 && t[k] < classes) l += share * (lse - z[t[k]]);
        loss[row] = l;
    }
    __syncthreads();  // the loss read z before it becomes the gradient
    const float inv_rows = 1.0f / static_cast<float>(rows);
    for (int i = tid; i < classes; i += blockDim.x) {
        float target = 0.0f;
        for (int k = 0; k < tk; ++k) target += (t[k] == i) ? share : 0.0f;
        z[i] = (expf(z[i] - lse) - target) * inv_rows;
    }
}

// dz = da * (a > 0): the gradient through a ReLU from its output a.
__global__ void relu_grad_kernel(float* da, const float* a, size_t n) {
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        if (!(a[i] > 0.0f)) da[i] = 0.0f;
}

// out[j] = sum over rows of x[row][j] (bias gradients).
__global__ void column_sums_kernel(const float* x, int rows, int cols, float* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += x[static_cast<size_t>(r) * cols + j];
    out[j] = s;
}

// Adam on FP32 master weights, then their BF16 copy.
__global__ void adam_kernel(float* w, __nv_bfloat16* w16, const float* g, float* m, float* v, size_t n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (w16) w16[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void to_bf16_kernel(const float* w, __nv_bfloat16* w16, size_t n) {
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
        w16[i] = __float2bfloat16_rn(w[i]);
}

// The `k` largest logits of each row, as class ids (ties by the lower id):
// one block per row loads the row's order-preserving keys into shared
// memory and bisects on the key bits for the k-th largest, counting the keys
// at or above the midpoint with a block reduction; it stops early when
// exactly k keys are at or above it (continuous logits: after about 15 of
// the 32 steps), else it resolves the ties at the k-th key in id order.
constexpr int kTopkThreads = 256;
constexpr int kTopkWarps = kTopkThreads / 32;

__device__ __forceinline__ unsigned order_key(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);  // larger float -> larger key
}

__global__ void __launch_bounds__(kTopkThreads) topk_kernel(const float* logits, int classes, int k, int* out) {
    extern __shared__ unsigned keys[];  // [classes]
    __shared__ int warp_count[2][kTopkWarps];
    __shared__ int s_pos;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float* z = logits + static_cast<size_t>(blockIdx.x) * classes;
    for (int i = tid; i < classes; i += kTopkThreads) keys[i] = order_key(z[i]);
    __syncthreads();
    // keys >= mid, summed over the block (double-buffered partial sums: one
    // barrier per step)
    int parity = 0;
    auto count_at_least = [&](unsigned mid) {
        int c = 0;
        for (int i = tid; i < classes; i += kTopkThreads) c += keys[i] >= mid;
        c = __reduce_add_sync(0xffffffffu, c);
        if (lane == 0) warp_count[parity][warp] = c;
        __syncthreads();
        int total = 0;
#pragma unroll
        for (int w = 0; w < kTopkWarps; ++w) total += warp_count[parity][w];
        parity ^= 1;
        return total;
    };
    unsigned lo = 0u, hi = 0xffffffffu;  // the k-th largest key lies in [lo, hi]
    bool exact = false;                  // exactly k keys are >= lo
    while (lo < hi) {
        const unsigned mid = static_cast<unsigned>((static_cast<unsigned long long>(lo) + hi + 1ull) / 2ull);
        const int count = count_at_least(mid);
        if (count == k) {
            lo = mid;
            exact = true;
            break;
        }
        if (count > k) lo = mid; else hi = mid - 1u;
    }
    if (tid == 0) s_pos = 0;
    __syncthreads();
    int* o = out + static_cast<size_t>(blockIdx.x) * k;
    if (exact) {
        for (int i = tid; i < classes; i += kTopkThreads)
            if (keys[i] >= lo) o[atomicAdd(&s_pos, 1)] = i;
        return;
    }
    const unsigned kth = lo;
    for (int i = tid; i < classes; i += kTopkThreads)
        if (keys[i] > kth) o[atomicAdd(&s_pos, 1)] = i;
    __syncthreads();
    const int above = s_pos;
    const int need = k - above;
    // the ties, in id order: chunks of 256 ids, ordered positions by ballots
    int taken = 0;
    for (int base = 0; base < classes && taken < need; base += kTopkThreads) {
        const int i = base + tid;
        const bool tie = i < classes && keys[i] == kth;
        const unsigned b = __ballot_sync(0xffffffffu, tie);
        if (lane == 0) warp_count[0][warp] = __popc(b);
        __syncthreads();
        int before = taken, total = 0;
        for (int w = 0; w < kTopkWarps; ++w) {
            if (w < warp) before += warp_count[0][w];
            total += warp_count[0][w];
        }
        const int pos = before + __popc(b & ((1u << lane) - 1u));
        if (tie && pos < need) o[above + pos] = i;
        taken += total;
        __syncthreads();
    }
}

int grid_for(size_t n) { return static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 16)); }

// The output layer for inference on the 5th-generation tensor cores: logits
// [M][N] = bf16(act)[M][K] * W16[N][K]^T + bias, FP32 accumulation in tensor
// memory.  One CTA of 4 warps takes 128 rows x 256 outputs: the rows'
// activations, rounded to BF16, and the 256 weight rows go to shared memory
// as no-swizzle K-major core matrices (8 rows x 16 bytes; core matrix (kc,
// g) of an operand with R rows at ((kc * R / 8) + g) * 128 bytes), one
// thread issues the K / 16 MMAs (M = 128, N = 256, K = 16) and commits them
// to an mbarrier, and each warp reads its 32 accumulator lanes back 32
// columns at a time, adds the bias and writes its rows through a shared
// transpose so that every store is a coalesced 128-byte row segment.
constexpr int kTcM = 128, kTcNOut = 256, kTcThreadsL = 128, kTcMaxK = 128;
constexpr int kTcSpin = 1 << 22;  // mbarrier polls before the wait gives up
constexpr uint32_t kLogitsIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                                  (static_cast<uint32_t>(kTcNOut >> 3) << 17) | (static_cast<uint32_t>(kTcM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

__global__ void __launch_bounds__(kTcThreadsL) tc_logits_kernel(int M, int N, int K, const float* act,
                                                                 const __nv_bfloat16* w16, const float* bias,
                                                                 float* logits, int* status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) unsigned long long done_bar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcNOut;
    unsigned char* a_s = smem;                                   // [K / 8][16][8 rows][16 B]
    unsigned char* b_s = smem + static_cast<size_t>(kTcM) * K * 2;  // [K / 8][32][8 rows][16 B]
    const uint32_t bar = smem_u32(&done_bar);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kTcNOut)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // A: row m0 + tid, 8 activations per core-matrix row, rounded to BF16
    {
        const int r = tid, m = m0 + r;
        for (int kc = 0; kc < K / 8; ++kc) {
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (m < M) {
                const float4* src = reinterpret_cast<const float4*>(act + static_cast<size_t>(m) * K + 8 * kc);
                const float4 lo = src[0], hi = src[1];
                __nv_bfloat162 p0 = __floats2bfloat162_rn(lo.x, lo.y), p1 = __floats2bfloat162_rn(lo.z, lo.w);
                __nv_bfloat162 p2 = __floats2bfloat162_rn(hi.x, hi.y), p3 = __floats2bfloat162_rn(hi.z, hi.w);
                v = make_uint4(*reinterpret_cast<uint32_t*>(&p0), *reinterpret_cast<uint32_t*>(&p1),
                               *reinterpret_cast<uint32_t*>(&p2), *reinterpret_cast<uint32_t*>(&p3));
            }
            *reinterpret_cast<uint4*>(a_s + ((kc * (kTcM / 8) + (r >> 3)) * 128 + (r & 7) * 16)) = v;
        }
    }
    // B: weight rows n0 + tid and n0 + tid + 128
    for (int h = 0; h < 2; ++h) {
        const int r = tid + kTcThreadsL * h, n = n0 + r;
        for (int kc = 0; kc < K / 8; ++kc) {
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (n < N) v = *reinterpret_cast<const uint4*>(w16 + static_cast<size_t>(n) * K + 8 * kc);
            *reinterpret_cast<uint4*>(b_s + ((kc * (kTcNOut / 8) + (r >> 3)) * 128 + (r & 7) * 16)) = v;
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    if (warp == 0) {
        const uint32_t leader = lane == 0 ? 1u : 0u;
        const uint32_t a0 = smem_u32(a_s), b0 = smem_u32(b_s);
        for (int s = 0; s < K / 16; ++s) {
            const uint64_t ad = kmajor_desc(a0 + 2 * s * (kTcM / 8) * 128, (kTcM / 8) * 128, 128);
            const uint64_t bd = kmajor_desc(b0 + 2 * s * (kTcNOut / 8) * 128, (kTcNOut / 8) * 128, 128);
            asm volatile(
                "{\n\t.reg .pred p, e;\n\tsetp.ne.b32 p, %4, 0;\n\tsetp.ne.b32 e, %5, 0;\n\t"
                "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                "l"(ad), "l"(bd), "r"(kLogitsIdesc), "r"(s > 0 ? 1u : 0u), "r"(leader)
                : "memory");
        }
        asm volatile(
            "{\n\t.reg .pred e;\n\tsetp.ne.b32 e, %1, 0;\n\t"
            "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}\n" ::"r"(bar),
            "r"(leader)
            : "memory");
        __syncwarp();
    }
    // the accumulators are complete once the commit arrives (bounded wait)
    int polls = 0;
    bool ok = true;
    while (!bar_try_wait(bar, 0)) {
        if (++polls >= kTcSpin) {
            ok = false;
            break;
        }
    }
    ok = __all_sync(0xffffffffu, ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (lane == 0 && status) atomicCAS(status, 0, kStatusLogitsTimeout);
    } else {
        // epilogue: 32 columns at a time through a [128][33] transpose in the
        // (now free) operand memory; warp w owns rows 32 w .. 32 w + 31
        float* tile = reinterpret_cast<float*>(smem) + warp * 32 * 33;
        for (int c0 = 0; c0 < kTcNOut; c0 += 32) {
            if (n0 + c0 >= N) break;  // uniform
            uint32_t v[32];
            const uint32_t ta = tmem + (static_cast<uint32_t>(32 * warp) << 16) + static_cast<uint32_t>(c0);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];\n\ttcgen05.wait::ld.sync.aligned;"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(ta)
                : "memory");
#pragma unroll
            for (int c = 0; c < 32; ++c) tile[lane * 33 + c] = __uint_as_float(v[c]);
            __syncwarp();
            const int n = n0 + c0 + lane;
            const float bn = n < N && bias ? bias[n] : 0.0f;
            for (int r = 0; r < 32; ++r) {
                const int m = m0 + 32 * warp + r;
                if (m < M && n < N) logits[static_cast<size_t>(m) * N + n] = tile[r * 33 + lane] + bn;
            }
            __syncwarp();
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        // after a wait that ran out, a bounded second wait for the MMAs
        // before the tensor memory goes
        if (!ok) {
            for (int i = 0; i < kTcSpin && !bar_try_wait(bar, 0); ++i) {
            }
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcNOut) : "memory");
    }
}

}  // namespace

cudaError_t mlp_forward(const MlpDevice& net, const float* x, int batch, float* const* acts, float* logits,
                        cudaStream_t stream) {
    const float* in = x;
    int width = net.inputs;
    for (int l = 0; l < net.layers; ++l) {
        cudaError_t e = gemm<false, true>(batch, net.hidden, width, in, width, net.w16[l], width, acts[l], net.hidden,
                                          net.b[l], true, 1.0f, false, stream);
        if (e != cudaSuccess) return e;
        in = acts[l];
        width = net.hidden;
    }
    return gemm<false, true>(batch, net.outputs, width, in, width, net.w16[net.layers], width, logits, net.outputs,
                             net.b[net.layers], false, 1.0f, false, stream);
}

cudaError_t mlp_infer(const MlpDevice& net, const float* x, int batch, float* const* acts, float* logits,
                      int* status, cudaStream_t stream) {
    const int K = net.layers > 0 ? net.hidden : net.inputs;
    if (K % 16 != 0 || K > kTcMaxK || batch <= 0)
        return mlp_forward(net, x, batch, acts, logits, stream);  // the CUDA-core GEMM for other widths
    const float* in = x;
    int width = net.inputs;
    for (int l = 0; l < net.layers; ++l) {
        cudaError_t e = gemm<false, true>(batch, net.hidden, width, in, width, net.w16[l], width, acts[l], net.hidden,
                                          net.b[l], true, 1.0f, false, stream);
        if (e != cudaSuccess) return e;
        in = acts[l];
        width = net.hidden;
    }
    const int smem = (kTcM + kTcNOut) * K * 2;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(tc_logits_kernel), smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((net.outputs + kTcNOut - 1) / kTcNOut, (batch + kTcM - 1) / kTcM);
    tc_logits_kernel<<<grid, kTcThreadsL, smem, stream>>>(batch, net.outputs, K, in, net.w16[net.layers],
                                                         net.b[net.layers], logits, status);
    return cudaGetLastError();
}

cudaError_t mlp_backward(const MlpDevice& net, const float* x, int batch, float* const* acts, float* dlogits,
                         const int* targets, int tk, float* loss, float* const* dacts, float* const* gw,
                         float* const* gb, cudaStream_t stream) {
    softmax_xent_kernel<<<batch, 256, 0, stream>>>(dlogits, net.outputs, targets, tk, batch, loss);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const float* grad = dlogits;
    int width = net.outputs;
    for (int l = net.layers; l >= 0; --l) {
        const int fan_in = l == 0 ? net.inputs : net.hidden;
        const float* in = l == 0 ? x : acts[l - 1];
        // dW[l] = grad^T in : [width][fan_in]
        if ((e = gemm<true, false>(width, fan_in, batch, grad, width, in, fan_in, gw[l], fan_in, nullptr, false,
                                   1.0f, false, stream)) != cudaSuccess)
            return e;
        column_sums_kernel<<<(width + 255) / 256, 256, 0, stream>>>(grad, batch, width, gb[l]);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (l == 0) break;
        // d(in) = grad W[l] : [batch][fan_in], then through the ReLU of layer l - 1
        if ((e = gemm<false, false>(batch, fan_in, width, grad, width, net.w16[l], fan_in, dacts[l - 1], fan_in,
                                    nullptr, false, 1.0f, false, stream)) != cudaSuccess)
            return e;
        const size_t n = static_cast<size_t>(batch) * fan_in;
        relu_grad_kernel<<<grid_for(n), 256, 0, stream>>>(dacts[l - 1], acts[l - 1], n);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        grad = dacts[l - 1];
        width = fan_in;
    }
    return cudaSuccess;
}

cudaError_t mlp_adam(const MlpDevice& net, float* const* gw, float* const* gb, float* const* mw, float* const* vw,
                     float* const* mb, float* const* vb, float* const* wmaster, float lr, int step,
                     cudaStream_t stream) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - powf(b1, static_cast<float>(step)), c2 = 1.0f - powf(b2, static_cast<float>(step));
    for (int l = 0; l <= net.layers; ++l) {
        const int fan_in = l == 0 ? net.inputs : net.hidden;
        const int fan_out = l == net.layers ? net.outputs : net.hidden;
        const size_t nw = static_cast<size_t>(fan_out) * fan_in;
        adam_kernel<<<grid_for(nw), 256, 0, stream>>>(wmaster[l], net.w16[l], gw[l], mw[l], vw[l], nw, lr, b1, b2,
                                                      eps, c1, c2);
        adam_kernel<<<grid_for(fan_out), 256, 0, stream>>>(net.b[l], nullptr, gb[l], mb[l], vb[l], fan_out, lr, b1,
                                                           b2, eps, c1, c2);
    }
    return cudaGetLastError();
}

cudaError_t weights_to_bf16(const float* w, __nv_bfloat16* w16, size_t n, cudaStream_t stream) {
    to_bf16_kernel<<<grid_for(n), 256, 0, stream>>>(w, w16, n);
    return cudaGetLastError();
}

cudaError_t logits_topk(const float* logits, int rows, int classes, int k, int* out, cudaStream_t stream) {
    if (rows <= 0) return cudaSuccess;
    if (k <= 0 || k > classes) return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(classes) * sizeof(unsigned);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(topk_kernel),
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    topk_kernel<<<rows, kTopkThreads, smem, stream>>>(logits, classes, k, out);
    return cudaGetLastError();
}

}  // namespace vnlbgpu

namespace vnlbgpu {
namespace {

// Coarse frames: the mean of each kFeatureCell x kFeatureCell box (partial
// boxes at the edges over their pixels), of every scheduled frame and search
// channel.
__global__ void cells_kernel(LearnedLaunch L) {
    const int n = L.slots_max * L.search_channels * L.cells_h * L.cells_w;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int cx = i % L.cells_w;
        const int cy = (i / L.cells_w) % L.cells_h;
        const int c = (i / (L.cells_w * L.cells_h)) % L.search_channels;
        const int k = i / (L.cells_w * L.cells_h * L.search_channels);
        float mean = 0.0f;
        if (k < L.schedule_len) {
            const float* plane = L.video + (static_cast<size_t>(L.schedule[k] % L.ring) * L.channels + c) *
                                               L.height * static_cast<size_t>(L.width);
            const int x0 = cx * kFeatureCell, y0 = cy * kFeatureCell;
            const int x1 = min(L.width, x0 + kFeatureCell), y1 = min(L.height, y0 + kFeatureCell);
            float s = 0.0f;
            for (int y = y0; y < y1; ++y)
                for (int x = x0; x < x1; ++x) s += __ldg(plane + static_cast<size_t>(y) * L.width + x);
            mean = s / static_cast<float>((x1 - x0) * (y1 - y0));
        }
        L.cells[i] = mean;
    }
}

// Features of each anchor: for every scheduled frame (zeros past the
// schedule) and search channel, the 3 x 3 coarse cells around the cell of the
// patch centre, minus that cell in the anchor frame, times feature_scale.
__global__ void features_kernel(LearnedLaunch L) {
    const int per = L.slots_max * L.search_channels * 9;
    const size_t n = static_cast<size_t>(L.anchor_count) * per;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int g = static_cast<int>(i / per);
        const int f = static_cast<int>(i - static_cast<size_t>(g) * per);
        const int k = f / (L.search_channels * 9);
        const int c = (f / 9) % L.search_channels;
        const int e = f % 9;
        const int2 a = L.anchors[g];
        const int cx0 = min((a.x + L.P / 2) / kFeatureCell, L.cells_w - 1);
        const int cy0 = min((a.y + L.P / 2) / kFeatureCell, L.cells_h - 1);
        const int cx = min(max(cx0 + e % 3 - 1, 0), L.cells_w - 1);
        const int cy = min(max(cy0 + e / 3 - 1, 0), L.cells_h - 1);
        float v = 0.0f;
        if (k < L.schedule_len) {
            const size_t plane = static_cast<size_t>(L.cells_h) * L.cells_w;
            const float here = L.cells[(static_cast<size_t>(k) * L.search_channels + c) * plane +
                                       static_cast<size_t>(cy) * L.cells_w + cx];
            const float centre = L.cells[static_cast<size_t>(c) * plane + static_cast<size_t>(cy0) * L.cells_w + cx0];
            v = (here - centre) * L.feature_scale;
        }
        L.features[static_cast<size_t>(g) * L.inputs + f] = v;
    }
}

// One warp per anchor: the exact SSD (for 8 x 8 patches in the plain
// matcher's arithmetic, so a shortlisted candidate gets the full search's
// distance bits) of every shortlisted candidate and of the anchor itself,
// then the plain matcher's selection on them: the K
// nearest by (distance, candidate order), threshold max(tau, d_K), at most
// soft_cap rows, nearest first; then the paste-mask victims.
__global__ void learned_match_kernel(LearnedLaunch L) {
    constexpr int kPer = kShortlistMax / 32 + 1;  // candidates per lane (the anchor is one more)
    const int lane = threadIdx.x & 31;
    const int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (g >= L.anchor_count) return;
    const int2 a = L.anchors[g];
    const int P = L.P, W = L.search_window;
    int xl, xh, yl, yh;
    spatial_range(a.x, L.width, P, W, xl, xh);
    spatial_range(a.y, L.height, P, W, yl, yh);
    const int Wx = xh - xl + 1, Wy = yh - yl + 1;
    const int cells = Wx * Wy;
    const size_t hw = static_cast<size_t>(L.height) * L.width;
    const float* ref = L.video + static_cast<size_t>(L.anchor_frame % L.ring) * L.channels * hw +
                       static_cast<size_t>(a.y) * L.width + a.x;
    __shared__ long long s_off[8][kShortlistMax + 1];  // candidate patch offsets in L.video (-1: none)
    __shared__ float s_dist[8][kShortlistMax + 1];
    const int wib = threadIdx.x >> 5;  // warp in block (blocks of 8 warps)
    float d[kPer];
    int id[kPer];
    const int n = L.shortlist_len + 1;
    // each lane's candidates: offset and the full search's candidate order
    for (int j = 0; j < kPer; ++j) {
        const int q = lane + 32 * j;
        d[j] = kInf;
        id[j] = 0x7fffffff;
        if (q >= n) continue;
        s_off[wib][q] = -1;
        int k, wx, wy;
        if (q == L.shortlist_len) {  // the anchor itself
            k = 0;
            wx = a.x - xl;
            wy = a.y - yl;
        } else {
            const int cls = L.shortlist[static_cast<size_t>(g) * L.shortlist_len + q];
            if (cls < 0) continue;
            k = cls / (W * W);
            wy = (cls / W) % W;
            wx = cls % W;
            if (k >= L.schedule_len || wx >= Wx || wy >= Wy) continue;
        }
        s_off[wib][q] = static_cast<long long>(static_cast<size_t>(L.schedule[k] % L.ring) * L.channels * hw +
                                               static_cast<size_t>(yl + wy) * L.width + xl + wx);
        id[j] = k * cells + wy * Wx + wx;
    }
    __syncwarp();
    if (P == 8) {
        // Exact SSD in the plain matcher's arithmetic (row_ssd8: each patch
        // row's 8 squared differences folded ((0+4)+(2+6))+((1+5)+(3+7)),
        // the rows added in order, planes (channel, t) in order): four
        // candidates a pass, an octet of lanes per candidate, lane r of the
        // octet folding patch row r, then the rows added in order.
        const int oct = lane >> 3, r = lane & 7;
        for (int base = 0; base < n; base += 4) {
            const int q = base + oct;
            const long long off = q < n ? s_off[wib][q] : -1;
            float dsum = 0.0f;
            for (int c = 0; c < L.search_channels; ++c)
                for (int t = 0; t < L.Pt; ++t) {
                    const size_t po = (static_cast<size_t>(t) * L.channels + c) * hw + static_cast<size_t>(r) * L.width;
                    float part = 0.0f;
                    if (off >= 0) {
                        const float* rr = ref + po;
                        const float* cr = L.video + static_cast<size_t>(off) + po;
                        float sq[8];
#pragma unroll
                        for (int i = 0; i < 8; ++i) {
                            const float df = __fsub_rn(__ldg(rr + i), __ldg(cr + i));
                            sq[i] = __fmul_rn(df, df);
                        }
                        part = __fadd_rn(__fadd_rn(__fadd_rn(sq[0], sq[4]), __fadd_rn(sq[2], sq[6])),
                                         __fadd_rn(__fadd_rn(sq[1], sq[5]), __fadd_rn(sq[3], sq[7])));
                    }
#pragma unroll
                    for (int row = 0; row < 8; ++row)
                        dsum = __fadd_rn(dsum, __shfl_sync(0xffffffffu, part, (oct << 3) + row));
                }
            if (r == 0 && off >= 0) s_dist[wib][q] = isfinite(dsum) ? dsum : kInf;
        }
        __syncwarp();
        for (int j = 0; j < kPer; ++j) {
            const int q = lane + 32 * j;
            if (q < n && id[j] != 0x7fffffff) d[j] = s_dist[wib][q];
        }
    } else {
        // other patch sizes: one lane per candidate, the samples in order
        for (int j = 0; j < kPer; ++j) {
            const int q = lane + 32 * j;
            if (q >= n || id[j] == 0x7fffffff) continue;
            const float* cand = L.video + static_cast<size_t>(s_off[wib][q]);
            float sum = 0.0f;
            for (int c = 0; c < L.search_channels; ++c)
                for (int t = 0; t < L.Pt; ++t) {
                    const size_t off = (static_cast<size_t>(t) * L.channels + c) * hw;
                    for (int py = 0; py < P; ++py)
                        for (int px = 0; px < P; ++px) {
                            const size_t o = off + static_cast<size_t>(py) * L.width + px;
                            const float diff = __fsub_rn(__ldg(ref + o), __ldg(cand + o));
                            sum = __fadd_rn(sum, __fmul_rn(diff, diff));
                        }
                }
            d[j] = isfinite(sum) ? sum : kInf;
        }
    }
    // duplicates (the anchor may also be shortlisted): keep the first copy
    for (int j = 0; j < kPer; ++j) {
        for (int jj = 0; jj < kPer; ++jj)
            for (int src = 0; src < 32; ++src) {
                const int other = __shfl_sync(0xffffffffu, id[jj], src);
                const int q_other = src + 32 * jj, q_me = lane + 32 * j;
                if (other == id[j] && q_other < q_me && id[j] != 0x7fffffff) d[j] = kInf;
            }
    }
    // rank of each candidate in (distance, id) order
    int rank[kPer];
    for (int j = 0; j < kPer; ++j) rank[j] = 0;
    for (int jj = 0; jj < kPer; ++jj)
        for (int src = 0; src < 32; ++src) {
            const float od = __shfl_sync(0xffffffffu, d[jj], src);
            const int oi = __shfl_sync(0xffffffffu, id[jj], src);
            for (int j = 0; j < kPer; ++j)
                rank[j] += (od < d[j] || (od == d[j] && oi < id[j])) ? 1 : 0;
        }
    // the K-th distance (threshold) and the count kept
    const int valid = __reduce_add_sync(0xffffffffu, [&] {
        int v = 0;
        for (int j = 0; j < kPer; ++j) v += d[j] < kInf;
        return v;
    }());
    const int selected = min(L.K, valid);
    float dk = 0.0f;
    for (int j = 0; j < kPer; ++j)
        if (rank[j] == selected - 1) dk = d[j];
    dk = __shfl_sync(0xffffffffu, dk, __ffs(__ballot_sync(0xffffffffu, [&] {
                                                 bool hit = false;
                                                 for (int j = 0; j < kPer; ++j) hit |= rank[j] == selected - 1;
                                                 return hit;
                                             }())) - 1);
    const float threshold = fmaxf(L.tau, dk);
    const int cap = min(min(L.soft_cap, L.max_rows), valid);
    MatchRow* out = L.rows + static_cast<size_t>(g) * L.max_rows;
    int kept = 0;
    for (int j = 0; j < kPer; ++j) {
        const bool keep = d[j] < kInf && d[j] <= threshold && rank[j] < cap;
        kept += keep;
        if (keep) {
            const int k = id[j] / cells;
            const int cell = id[j] - k * cells;
            MatchRow m;
            m.distance = d[j];
            m.x = xl + cell % Wx;
            m.y = yl + cell / Wx;
            m.frame = L.schedule[k];
            out[rank[j]] = m;
        }
    }
    const int S = __reduce_add_sync(0xffffffffu, kept);
    if (lane == 0) L.row_counts[g] = S;
    __syncwarp();
    // paste-mask victims (apply_frame_paste_mask, core.cpp:980-1008), as the
    // full matcher finds them
    int* vict = L.victims + static_cast<size_t>(g) * L.victim_stride;
    int nv = 0;
    for (int i0 = 0; i0 < S; i0 += 32) {
        const int i = i0 + lane;
        int found[5];
        int nf = 0;
        if (i < S) {
            const MatchRow m = out[i];
            if (m.frame == L.anchor_frame) {
                const int px[5] = {m.x, m.x, m.x, m.x - 1, m.x + 1};
                const int py[5] = {m.y, m.y - 1, m.y + 1, m.y, m.y};
                const bool use[5] = {true, m.y > 2 * P, m.y < L.height - 2 * P, m.x > 2 * P, m.x < L.width - 2 * P};
                for (int e = 0; e < 5; ++e) {
                    if (!use[e] || px[e] < 0 || px[e] >= L.width || py[e] < 0 || py[e] >= L.height) continue;
                    const int j = L.anchor_map[static_cast<size_t>(py[e]) * L.width + px[e]];
                    if (j > g) found[nf++] = j;
                }
            }
        }
        for (int e = 0; e < 5; ++e) {
            const unsigned has = __ballot_sync(0xffffffffu, e < nf);
            const int pos = nv + __popc(has & ((1u << lane) - 1u));
            if (e < nf && pos < L.victim_stride) vict[pos] = found[e];
            nv += __popc(has);
        }
    }
    if (lane == 0) L.victim_counts[g] = min(nv, L.victim_stride);
}

// Per tile: the recall of the full search's K nearest rows of its checked
// anchor among the learned matcher's K nearest; below the threshold the
// tile falls back to the full search.
__global__ void recall_kernel(LearnedLaunch L) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= L.tiles) return;
    const int g = L.check_anchor[t];
    const MatchRow* exact = L.check_rows + static_cast<size_t>(t) * L.max_rows;
    const MatchRow* got = L.rows + static_cast<size_t>(g) * L.max_rows;
    const int ne = min(L.K, L.check_counts[t]);
    const int ng = min(L.K, L.row_counts[g]);
    int hit = 0;
    for (int i = 0; i < ne; ++i)
        for (int j = 0; j < ng; ++j)
            if (exact[i].x == got[j].x && exact[i].y == got[j].y && exact[i].frame == got[j].frame) {
                ++hit;
                break;
            }
    const float recall = ne > 0 ? static_cast<float>(hit) / static_cast<float>(ne) : 1.0f;
    const int fail = recall < L.recall_threshold ? 1 : 0;
    L.tile_fail[t] = fail;
    atomicAdd(L.totals, 1ull);
    if (fail) atomicAdd(L.totals + 1, 1ull);
}

}  // namespace

cudaError_t launch_learned_features(const LearnedLaunch& L, cudaStream_t stream) {
    const int nc = L.slots_max * L.search_channels * L.cells_h * L.cells_w;
    cells_kernel<<<std::max(1, std::min((nc + 255) / 256, 148 * 8)), 256, 0, stream>>>(L);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t n = static_cast<size_t>(L.anchor_count) * L.inputs;
    features_kernel<<<grid_for(n), 256, 0, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_learned_match(const LearnedLaunch& L, cudaStream_t stream) {
    if (L.shortlist_len > kShortlistMax || L.anchor_count <= 0) return L.anchor_count <= 0 ? cudaSuccess
                                                                                              : cudaErrorInvalidValue;
    learned_match_kernel<<<(L.anchor_count + 7) / 8, 256, 0, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_learned_recall(const LearnedLaunch& L, cudaStream_t stream) {
    if (L.tiles <= 0) return cudaSuccess;
    recall_kernel<<<(L.tiles + 127) / 128, 128, 0, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace vnlbgpu
