// Shared device-side definitions of the B200 VNLB hot path.
//
// Every floating-point helper here reproduces one operation sequence of the
// reference CPU core exactly (same operands, same order, same roundings), so
// that the plain GPU form is bit-identical to the reference compiled with an
// 8-lane vector width (the pinned Highway semantics): a*b+c is written with
// __fmul_rn/__fadd_rn where the CPU rounds twice and with __fmaf_rn where the
// CPU uses a fused multiply-add.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vnlbgpu {

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`, never lowering it (smem_limit.cpp: concurrent sessions
// launch the same kernels with different amounts).
cudaError_t raise_smem_limit(const void* kernel, size_t bytes);

constexpr int kLanes = 8;          // CPU vector width the order is pinned to
constexpr float kInf = __builtin_huge_valf();

struct StageConfig {
    // vnlb::core::StageParameters (src/core/core.hpp:17-41), core units.
    float sigma;
    int patch_size;
    int patch_time;
    int search_window;
    int search_bwd;
    int search_fwd;
    int similar;        // K
    int rank;
    float similar_cap_factor;
    float model_cap_factor;
    float beta;
    float tau;
    float variance_threshold;
    float sigma_basic;
    float gamma;        // flat-area gamma
    float weight_alpha;
    float weight_beta;
    float weight_gamma;
    float weight_epsilon;
    float membership_noise_floor;
    int proc_step;
    int flat_areas;
    int couple_channels;
};

// Dimensions derived once per session.
struct Shape {
    int width, height, frames, channels;
    int stage;            // 0 Basic, 1 Final
    int P, Pt, patch_dim; // P*P*Pt
    int dim;              // estimator dimension (patch_dim * channels, coupled)
    int search_channels;  // 1 (Basic, luma) or channels (Final)
    int K;                // requested group size
    int soft_cap;         // ceil(K*cap_factor) (>= K), or INT_MAX
    int model_cap;        // ceil(K*model_cap_factor)
    int max_rows;         // largest retained row count S
    int slots;            // search_bwd + search_fwd + patch_time
    int window_w;         // spatial window width (search_window)
};

struct MatchRow {
    float distance;
    int x;
    int y;
    int frame;
};

// ---------------------------------------------------------------------------
// Pinned lane-structured arithmetic (src/core/distance_highway.hpp:11-58,
// src/linalg/kernels_highway.hpp).
__device__ __forceinline__ float reduce8(const float v[kLanes]) {
    const float a0 = __fadd_rn(v[0], v[4]);
    const float a1 = __fadd_rn(v[1], v[5]);
    const float a2 = __fadd_rn(v[2], v[6]);
    const float a3 = __fadd_rn(v[3], v[7]);
    return __fadd_rn(__fadd_rn(a0, a2), __fadd_rn(a1, a3));
}

// Packed pairs of FP32 (sm_100 add/sub/mul/fma .f32x2): one instruction
// computes two independent lanes, each rounded exactly as the scalar
// instruction with the same rounding mode, so a pairwise rewrite of a scalar
// sequence gives the same bits with half the FP32 instructions.
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

__device__ __forceinline__ float2 sub2_rn(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

__device__ __forceinline__ float2 fma2_rn(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

// Packed square d*d, rounded once.  It is fma(d, d, +0), not mul.rn.f32x2:
// ptxas contracts a mul.rn.f32x2 whose result feeds an add.rn.f32x2 into one
// fused multiply-add, even with --fmad=false, which changes the bits (every
// such mismatch measured on sm_100a equalled the fused result).  A square is
// never -0, so fma(d, d, +0) = round(d*d) exactly, and nothing fuses it.
__device__ __forceinline__ float2 sqr2_rn(float2 d) { return fma2_rn(d, d, make_float2(0.0f, 0.0f)); }

// row_ssd<8> on packed pairs: ref and cand hold samples (0,1) (2,3) (4,5)
// (6,7).  The fold ((v0+v4)+(v2+v6)) + ((v1+v5)+(v3+v7)) of reduce8 is two
// pair adds (a0,a1) (a2,a3), one pair add (a0+a2, a1+a3) and a scalar add.
__device__ __forceinline__ float row_ssd8_x2(float distance, const float2 ref[4], const float2 cand[4]) {
    float2 v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        v[i] = sqr2_rn(sub2_rn(ref[i], cand[i]));
    }
    const float2 t = add2_rn(add2_rn(v[0], v[2]), add2_rn(v[1], v[3]));
    return __fadd_rn(distance, __fadd_rn(t.x, t.y));
}

// add_squared_row_distance_highway: distance + SSD of one patch row of
// `count` samples, in the pinned order.  `ref` and `cand` may be any
// addressable memory (registers after unrolling, shared, global).
template <int Count, typename RefFn, typename CandFn>
__device__ __forceinline__ float row_ssd(float distance, RefFn ref, CandFn cand) {
    if constexpr (Count <= 0) {
        return distance;
    } else if constexpr (Count == kLanes) {
        float v[kLanes];
#pragma unroll
        for (int i = 0; i < kLanes; ++i) {
            const float d = __fsub_rn(ref(i), cand(i));
            v[i] = __fmul_rn(d, d);
        }
        return __fadd_rn(distance, reduce8(v));
    } else if constexpr (Count == 2 * kLanes) {
        float v[kLanes];
#pragma unroll
        for (int i = 0; i < kLanes; ++i) {
            const float d = __fsub_rn(ref(i), cand(i));
            v[i] = __fmul_rn(d, d);
        }
#pragma unroll
        for (int i = 0; i < kLanes; ++i) {
            const float d = __fsub_rn(ref(i + kLanes), cand(i + kLanes));
            v[i] = __fmaf_rn(d, d, v[i]);
        }
        return __fadd_rn(distance, reduce8(v));
    } else {
        constexpr int kFull = (Count / kLanes) * kLanes;
        if constexpr (kFull > 0) {
            float v[kLanes];
#pragma unroll
            for (int i = 0; i < kLanes; ++i) v[i] = 0.0f;
#pragma unroll
            for (int base = 0; base < kFull; base += kLanes) {
#pragma unroll
                for (int i = 0; i < kLanes; ++i) {
                    const float d = __fsub_rn(ref(base + i), cand(base + i));
                    v[i] = __fmaf_rn(d, d, v[i]);
                }
            }
            distance = __fadd_rn(distance, reduce8(v));
        }
        // (with no full chunk the CPU adds a zero vector sum: distance + 0,
        // which leaves a non-negative distance unchanged)
#pragma unroll
        for (int i = kFull; i < Count; ++i) {
            const float d = __fsub_rn(ref(i), cand(i));
            distance = __fadd_rn(distance, __fmul_rn(d, d));
        }
        return distance;
    }
}

// Runtime-count version of row_ssd for patch sizes without a specialised
// kernel.
__device__ __forceinline__ float row_ssd_dyn(float distance, const float* ref, const float* cand,
                                             int count) {
    float v[kLanes];
    if (count <= 0) return distance;
    if (count == kLanes) {
#pragma unroll
        for (int i = 0; i < kLanes; ++i) {
            const float d = __fsub_rn(ref[i], cand[i]);
            v[i] = __fmul_rn(d, d);
        }
        return __fadd_rn(distance, reduce8(v));
    }
    if (count == 2 * kLanes) {
#pragma unroll
        for (int i = 0; i < kLanes; ++i) {
            const float d = __fsub_rn(ref[i], cand[i]);
            v[i] = __fmul_rn(d, d);
        }
#pragma unroll
        for (int i = 0; i < kLanes; ++i) {
            const float d = __fsub_rn(ref[i + kLanes], cand[i + kLanes]);
            v[i] = __fmaf_rn(d, d, v[i]);
        }
        return __fadd_rn(distance, reduce8(v));
    }
#pragma unroll
    for (int i = 0; i < kLanes; ++i) v[i] = 0.0f;
    int index = 0;
    for (; index + kLanes <= count; index += kLanes) {
#pragma unroll
        for (int i = 0; i < kLanes; ++i) {
            const float d = __fsub_rn(ref[index + i], cand[index + i]);
            v[i] = __fmaf_rn(d, d, v[i]);
        }
    }
    distance = __fadd_rn(distance, reduce8(v));
    for (; index < count; ++index) {
        const float d = __fsub_rn(ref[index], cand[index]);
        distance = __fadd_rn(distance, __fmul_rn(d, d));
    }
    return distance;
}

// ---------------------------------------------------------------------------
// Elementary functions, correctly rounded to float: evaluated in double
// precision (error below one double ulp) and rounded once.  The reference
// calls std::exp/std::log/std::log1p/std::pow on floats; the oracle pins those
// to the same definition.
__host__ __device__ __forceinline__ float cr_expf(float x) { return static_cast<float>(exp(static_cast<double>(x))); }
__host__ __device__ __forceinline__ float cr_logf(float x) { return static_cast<float>(log(static_cast<double>(x))); }
__host__ __device__ __forceinline__ float cr_log1pf(float x) {
    return static_cast<float>(log1p(static_cast<double>(x)));
}

// std::max / std::min on floats (first operand wins ties and NaNs).
__host__ __device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ float std_min(float a, float b) { return (b < a) ? b : a; }

// compute_spatial_range (core.cpp:910-932)
__host__ __device__ __forceinline__ void spatial_range(int center, int axis, int P, int window, int& low, int& high) {
    const int max_origin = axis - P;
    const int half = (window - 1) / 2;
    const int start = center - half;
    const int end = center + half;
    const int shift = min(0, start) + max(0, end - max_origin);
    low = max(0, start - shift);
    high = min(max_origin, end - shift);
}

}  // namespace vnlbgpu
