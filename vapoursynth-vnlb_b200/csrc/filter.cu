// Bayesian PCA group filter and aggregation weights for the active groups of
// one anchor frame (plain form, dual-PCA model).
//
// Reference semantics: transform_vnlb_coupled_samples / transform_vnlb_group,
// filter_vnlb_samples, compute_filter_coefficients,
// accumulate_aggregation_model, finalize_aggregation_weights and
// project_bayes_estimate (src/core/core.cpp:190-412, 578-871, 276-294) on top
// of compute_mean, center_rows, compute_gram_centered,
// topk_symmetric_eigen_jacobi and map_dual_eigenvectors_to_basis
// (src/linalg/linalg.cpp).
//
// Three kernels, each shaped to its parallelism:
//   prepare  one warp per group: equality and flat-area tests, the means of
//            the first B rows, the centred model rows (shared memory) and the
//            B x B dual Gram, one pair per lane;
//   jacobi   the cyclic Jacobi of many groups per warp, one lane per matrix
//            row (a latency-bound chain of dependent rotations, so throughput
//            comes from the number of groups in flight);
//   apply    one CTA per group: dual -> primal basis, Wiener coefficients,
//            precision and volume, then every retained row streamed once per
//            warp for its membership score and its shrunken reconstruction,
//            and finally the aggregation weights.
// Samples are addressed through a per-launch table of column offsets
// (channel, t, py, px) -> video offset, so a gather is one add and one load.
// All dot products use the pinned 8-lane order (per-lane fused accumulators,
// then the fixed fold), elementwise updates the CPU's fused/unfused split, and
// the elementary functions are correctly rounded, so results are
// bit-identical to the CPU core -- with one stated exception: the flat-area
// variance (double sums) is reduced in a fixed parallel order, which can move
// its float value by one ulp; that changes the flat decision only when the
// variance lies within one ulp of gamma*sigma^2.
#include <cfloat>

#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr int kApplyThreads = 256;
constexpr int kApplyWarps = kApplyThreads / 32;
constexpr int kRecCols = 8;  // reconstruction columns held in registers per lane (blocks of 256)
constexpr int kPrepareWarps = 4;
constexpr float kEigenFloor = 128.0f * FLT_EPSILON;
constexpr size_t kFilterSharedLimit = 227 * 1024;  // dynamic shared memory of one CTA on sm_100

// dot_contiguous_highway (the pinned 8-lane order) computed by an octet of
// lanes (j = lane & 7): lane j owns accumulator j; the fold follows reduce8.  All 8 lanes return the dot.
// Every lane of the warp must call it.
__device__ __forceinline__ float octet_dot8(const float* l, const float* r, int count, int j) {
    float v = 0.0f;
    int index = 0;
    if (count == kLanes || count == 2 * kLanes) {
        v = __fmul_rn(l[j], r[j]);
        if (count == 2 * kLanes) v = __fmaf_rn(l[kLanes + j], r[kLanes + j], v);
        index = count;
    } else {
        for (; index + kLanes <= count; index += kLanes) v = __fmaf_rn(l[index + j], r[index + j], v);
    }
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 4, 8));
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 2, 8));
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 1, 8));
    float total = __shfl_sync(0xffffffffu, v, 0, 8);
    for (; index < count; ++index) total = __fadd_rn(total, __fmul_rn(l[index], r[index]));
    return total;
}

__device__ __forceinline__ bool fused_column(int col, int count) {
    return count == kLanes || count == 2 * kLanes || col < (count / kLanes) * kLanes;
}

// add_scaled_contiguous_highway element `col` of a row of `count`.
__device__ __forceinline__ float add_scaled_elem(float out, float in, float scale, int col, int count) {
    return fused_column(col, count) ? __fmaf_rn(scale, in, out) : __fadd_rn(out, __fmul_rn(scale, in));
}

// Offset of column col = (channel, t, py, px) from a patch origin.
__device__ __forceinline__ int column_offset(const FilterLaunch& L, int col) {
    const int pd = L.patch_dim;
    const int c = col / pd;
    const int pos = col - c * pd;
    const int pp = L.P * L.P;
    const int t = pos / pp;
    const int rem = pos - t * pp;
    const int py = rem / L.P;
    const int px = rem - py * L.P;
    return ((t * L.channels + c) * L.height + py) * L.width + px;
}

__device__ __forceinline__ size_t row_base(const FilterLaunch& L, const MatchRow& m) {
    return (static_cast<size_t>(m.frame % L.ring) * L.channels * L.height + m.y) * static_cast<size_t>(L.width) + m.x;
}

__device__ __forceinline__ int bmax_of(const FilterLaunch& L) { return min(L.model_cap, L.max_rows); }

// One m16n8k8 TF32 tensor-core MMA with FP32 accumulation (row-major A,
// column-major B): d += a * b.
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// Dual Gram X X^T / B of up to 16 centred rows (row stride ldx, D a multiple
// of 8) on the tensor cores, one warp: A = the rows (16 x 8 per step), B =
// their transpose in tiles of 8 columns; rows and columns past B are zero.
// Lane (g, q) = (lane / 4, lane % 4) holds A rows g, g + 8 at columns q, q + 4
// and the accumulators of rows g, g + 8 at columns 2q, 2q + 1.
__device__ __forceinline__ void gram_tf32(const float* X, int ldx, int B, int D, float scale, float* gram,
                                          int lane) {
    const int g = lane >> 2, q = lane & 3;
    for (int n0 = 0; n0 < B; n0 += 8) {
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int k0 = 0; k0 < D; k0 += 8) {
            uint32_t a[4], b[2];
            a[0] = g < B ? to_tf32(X[g * ldx + k0 + q]) : 0u;
            a[1] = g + 8 < B ? to_tf32(X[(g + 8) * ldx + k0 + q]) : 0u;
            a[2] = g < B ? to_tf32(X[g * ldx + k0 + q + 4]) : 0u;
            a[3] = g + 8 < B ? to_tf32(X[(g + 8) * ldx + k0 + q + 4]) : 0u;
            const int n = n0 + g;  // B's column n is row n of X
            b[0] = n < B ? to_tf32(X[n * ldx + k0 + q]) : 0u;
            b[1] = n < B ? to_tf32(X[n * ldx + k0 + q + 4]) : 0u;
            mma_tf32(acc, a, b);
        }
        const int c0 = n0 + 2 * q;
        const int rows[2] = {g, g + 8};
        for (int h = 0; h < 2; ++h) {
            const int r = rows[h];
            if (r >= B) continue;
            if (c0 < B) gram[r * B + c0] = acc[2 * h] * scale;
            if (c0 + 1 < B) gram[r * B + c0 + 1] = acc[2 * h + 1] * scale;
        }
    }
}

// ---------------------------------------------------------------------------
// prepare: W warps per group.  W = 1 runs four groups per CTA, one per warp;
// W = 4 gives a CTA to one group, for model rows too large for four copies in
// shared memory to leave room for more than a few warps per SM (block 7,
// patch_time 2, YUV: 16 rows of 294 values).  Every value is computed in the
// same order either way: the column sums and the centring by the thread that
// owns the column, each Gram pair by one octet of lanes, each channel's
// flat-area sums by one warp.
template <int W>
__global__ void __launch_bounds__(32 * kPrepareWarps) prepare_kernel(FilterLaunch L) {
    constexpr int kGroups = kPrepareWarps / W;  // groups per CTA
    constexpr int kT = 32 * W;                  // threads per group
    extern __shared__ __align__(16) float sm[];
    __shared__ double s_sums[2 * 4];            // flat-area sums per channel (W > 1)
    const int D = L.dim;
    const int Bmax = bmax_of(L);
    int* coloff = reinterpret_cast<int*>(sm);
    size_t* bases_all = reinterpret_cast<size_t*>(sm + ((D + 3) & ~3));  // kGroups * max_rows
    const int ldx = D + 8;  // padded row stride: octets on different rows hit different banks
    const int slot = threadIdx.x / kT;          // this group's slot in the CTA
    const int t = threadIdx.x - slot * kT;      // thread within the group
    float* X = reinterpret_cast<float*>(bases_all + kGroups * L.max_rows) + slot * Bmax * ldx;  // model rows
    size_t* bases = bases_all + slot * L.max_rows;
    for (int col = threadIdx.x; col < D; col += blockDim.x) coloff[col] = column_offset(L, col);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int gwarp = t >> 5;  // warp within the group
    auto group_sync = [] {
        if constexpr (W == 1) __syncwarp();
        else __syncthreads();
    };
    auto group_any = [](bool p) -> bool {
        if constexpr (W == 1) return __any_sync(0xffffffffu, p);
        else return __syncthreads_or(p) != 0;
    };
    const StageConfig& P = L.cfg;
    const bool final_stage = L.stage == 1;
    const float* model_video = final_stage ? L.basic : L.noisy;
    const bool weights_enabled = P.weight_alpha != 0.0f || P.weight_beta != 0.0f || P.weight_gamma != 0.0f;
    const int active_count = L.counters->active;
    // model v = (active group a, model channel mc): one model per group when
    // the channels are coupled (or the clip has one plane), one per plane
    // otherwise (transform_vnlb_channel, core.cpp:795-808)
    const int models = L.models;
    const size_t hw = static_cast<size_t>(L.height) * L.width;
    const int RD = L.row_dim;
    for (int v = blockIdx.x * kGroups + slot; v < active_count * models; v += gridDim.x * kGroups) {
        group_sync();  // the previous group is done with bases and X
        const int a = v / models;
        const int mc = v - a * models;
        const size_t cb = mc * hw;  // plane offset of this model's channel
        const int g = L.active[a];
        const int S = L.row_counts[g];
        const MatchRow* rows = L.rows + static_cast<size_t>(g) * L.max_rows;
        const int r0 = L.row_offset[a];
        const int B = min(S, L.model_cap);
        for (int i = t; i < S; i += kT) {
            const MatchRow m = rows[i];
            if (mc == 0) {
                L.row_info[r0 + i] = m;
                L.row_group[r0 + i] = a;
            }
            bases[i] = row_base(L, m);
        }
        group_sync();
        // equal group (samples_are_equal / group_is_equal): independent loads
        bool differs = S <= 1;
        if (S > 1) {
            for (int col = t; col < D * models; col += kT) {
                const int cm = col / D;  // plane of an uncoupled group (group_is_equal, core.cpp:516-531)
                const float* src = L.noisy + cm * hw + coloff[col - cm * D];
                const float v0 = __ldg(src + bases[0]);
                int i = 1;
                for (; i + 4 <= S; i += 4) {
                    const float x0 = __ldg(src + bases[i]), x1 = __ldg(src + bases[i + 1]);
                    const float x2 = __ldg(src + bases[i + 2]), x3 = __ldg(src + bases[i + 3]);
                    differs |= (x0 != v0) | (x1 != v0) | (x2 != v0) | (x3 != v0);
                }
                for (; i < S; ++i) differs |= __ldg(src + bases[i]) != v0;
            }
        }
        if (!group_any(differs)) {
            // filtered = input, default aggregation model (core.cpp:253-274)
            for (int i = 0; i < S; ++i) {
                const size_t b = bases[i];
                float* out = L.filtered + static_cast<size_t>(r0 + i) * RD + mc * D;
                for (int col = t; col < D; col += kT) out[col] = __ldg(L.noisy + b + cb + coloff[col]);
            }
            const float tau = __fadd_rn(P.weight_epsilon, __fdiv_rn(static_cast<float>(D), static_cast<float>(B)));
            const float lgw = P.weight_alpha == 0.0f ? 0.0f : __fmul_rn(-P.weight_alpha, cr_logf(tau));
            float w = 1.0f;
            if (weights_enabled) {
                float lw = __fadd_rn(0.0f, lgw);
                lw = lw < -80.0f ? -80.0f : (80.0f < lw ? 80.0f : lw);
                w = cr_expf(lw);
            }
            if (mc == 0)
                for (int i = t; i < S; i += kT) L.weights[r0 + i] = w;
            if (t == 0) L.flags[v] = kGroupDone;
            continue;
        }
        // flat area (Final): mean channel variance of the noisy rows; one warp
        // sums a channel (lane-strided, then a fixed shuffle tree)
        bool flat = false;
        if (final_stage && P.flat_areas) {
            const int pd = L.patch_dim;
            const int channels = models > 1 ? models : D / pd;
            const int per_channel = pd * S;
            float variance = 0.0f;
            for (int c0 = 0; c0 < channels; c0 += W) {
                const int c = c0 + gwarp;
                double sum = 0.0, sum2 = 0.0;
                if (c < channels) {
                    for (int i = 0; i < S; ++i) {
                        const float* src = L.noisy + bases[i];
                        for (int q = lane; q < pd; q += 32) {
                            const float x = __ldg(src + (models > 1 ? c * hw + coloff[q] : coloff[c * pd + q]));
                            sum += static_cast<double>(x);
                            sum2 += static_cast<double>(x) * static_cast<double>(x);
                        }
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sum += __shfl_xor_sync(0xffffffffu, sum, o);
                    sum2 += __shfl_xor_sync(0xffffffffu, sum2, o);
                }
                if constexpr (W > 1) {
                    if (lane == 0 && c < channels) {
                        s_sums[2 * gwarp] = sum;
                        s_sums[2 * gwarp + 1] = sum2;
                    }
                    group_sync();
                }
                // the channels of this round in order
                for (int k = 0; k < W && c0 + k < channels; ++k) {
                    double ks = sum, ks2 = sum2;
                    if constexpr (W > 1) {
                        ks = s_sums[2 * k];
                        ks2 = s_sums[2 * k + 1];
                    }
                    if (per_channel > 1) {
                        const double count = static_cast<double>(per_channel);
                        variance = __fadd_rn(variance, static_cast<float>((ks2 - (ks * ks / count)) / (count - 1.0)));
                    }
                }
                if constexpr (W > 1) group_sync();
            }
            if (per_channel > 1) variance = __fdiv_rn(variance, static_cast<float>(channels));
            flat = variance < __fmul_rn(__fmul_rn(P.sigma, P.sigma), P.gamma);
        }
        if (B < min(D, L.rank)) {
            if (t == 0) {
                atomicCAS(L.status, 0, kStatusRankNotCovered);
                L.flags[v] = kGroupSkip;
            }
            continue;
        }
        // model rows, means over the first B rows (compute_mean), centring
        if constexpr (W == 1) {
            for (int s2 = 0; s2 < B; ++s2) {
                const size_t b = bases[s2];
                for (int col = lane; col < D; col += 32) X[s2 * ldx + col] = __ldg(model_video + b + cb + coloff[col]);
            }
        } else {
            for (int e = t; e < B * D; e += kT) {
                const int s2 = e / D;
                const int col = e - s2 * D;
                X[s2 * ldx + col] = __ldg(model_video + bases[s2] + cb + coloff[col]);
            }
        }
        group_sync();
        const float inv_b = __fdiv_rn(1.0f, static_cast<float>(B));
        float* means = L.means + static_cast<size_t>(v) * 2 * D;
        for (int col = t; col < D; col += kT) {
            float mm = 0.0f;
            for (int s2 = 0; s2 < B; ++s2) mm = __fadd_rn(mm, X[s2 * ldx + col]);
            mm = __fmul_rn(mm, inv_b);
            float center = mm;  // Basic: noisy mean; Final flat: basic mean
            if (final_stage && !flat) {
                float mn = 0.0f;
                for (int s2 = 0; s2 < B; ++s2) mn = __fadd_rn(mn, __ldg(L.noisy + bases[s2] + cb + coloff[col]));
                center = __fmul_rn(mn, inv_b);
            }
            means[col] = mm;
            means[D + col] = center;
            for (int s2 = 0; s2 < B; ++s2) X[s2 * ldx + col] = __fsub_rn(X[s2 * ldx + col], mm);
        }
        group_sync();
        if (L.rank > 0) {
            const float scale = __fdiv_rn(1.0f, static_cast<float>(B));
            float* gram = L.gram + static_cast<size_t>(v) * L.nmax * L.nmax;
            if (D >= 64 && B < D && L.mixed && W == 1 && B <= 16 && D % 8 == 0) {
                // chosen forms: TF32 tensor-core Gram, FP32 accumulation
                gram_tf32(X, ldx, B, D, scale, gram, lane);
            } else if (D >= 64 && B < D) {
                // dual Gram (compute_gram_centered): octet k takes pair e0 + k;
                // lane j of the octet runs the pinned chain j (octet_dot8)
                const int pairs = B * (B + 1) / 2;
                const int oct = t >> 3;
                for (int e0 = 0; e0 < pairs; e0 += kT / 8) {
                    const int e = min(e0 + oct, pairs - 1);
                    int r = 0;
                    while ((r + 1) * (r + 2) / 2 <= e) ++r;
                    const int c = e - r * (r + 1) / 2;
                    const float val = __fmul_rn(scale, octet_dot8(X + r * ldx, X + c * ldx, D, lane & 7));
                    if ((lane & 7) == 0 && e0 + oct < pairs) {
                        gram[r * B + c] = val;
                        gram[c * B + r] = val;
                    }
                }
            } else {
                // covariance (compute_covariance_centered, linalg.cpp:378-412):
                // per sample, row r gets x[r] * x[r..] through
                // add_scaled_contiguous_highway, fused on the full 8-lane chunks of
                // the D - r columns it spans; then scaled, both triangles
                const int entries = D * (D + 1) / 2;
                for (int e = t; e < entries; e += kT) {
                    int r = 0, rem = e;
                    while (rem >= D - r) {
                        rem -= D - r;
                        ++r;
                    }
                    const int c = r + rem;
                    const bool fused = fused_column(rem, D - r);
                    float acc = 0.0f;
                    for (int s2 = 0; s2 < B; ++s2) {
                        const float left = X[s2 * ldx + r];
                        const float x = X[s2 * ldx + c];
                        acc = fused ? __fmaf_rn(left, x, acc) : __fadd_rn(acc, __fmul_rn(left, x));
                    }
                    const float val = __fmul_rn(acc, scale);
                    gram[r * D + c] = val;
                    gram[c * D + r] = val;
                }
            }
        }
        if (t == 0) L.flags[v] = 0;
    }
}

// ---------------------------------------------------------------------------
// jacobi: topk_symmetric_eigen_jacobi (linalg.cpp:447-519) for many groups per
// warp.  A group owns a segment of `seg` lanes (a power of two >= its rows,
// at most 32); lane r of the segment owns matrix rows r, r + seg, ...
__global__ void __launch_bounds__(256) jacobi_kernel(FilterLaunch L, int seg, int ld, int gstride) {
    extern __shared__ __align__(16) float sm[];
    const int N = L.nmax;  // largest matrix dimension (model rows, or the dimension for covariance models)
    const int D = L.dim;
    const int R = L.rank;
    const int lane = threadIdx.x & 31;
    const int groups_per_warp = 32 / seg;
    const int slot = (threadIdx.x >> 5) * groups_per_warp + lane / seg;  // group slot in the CTA
    const int r0 = lane % seg;
    const unsigned seg_mask = seg == 32 ? 0xffffffffu : (((1u << seg) - 1u) << ((lane / seg) * seg));
    float* m = sm + static_cast<size_t>(slot) * gstride;
    float* v = m + N * ld;
    int* order = reinterpret_cast<int*>(v + N * ld);
    const int models_total = L.counters->active * L.models;
    const int slots_per_cta = (blockDim.x >> 5) * groups_per_warp;
    for (int base = blockIdx.x * slots_per_cta; base < models_total; base += gridDim.x * slots_per_cta) {
        const int a = base + slot;  // model index (group x model channel)
        bool valid = a < models_total && R > 0;
        int B = 0;  // matrix dimension: the dual Gram's B, or the covariance's D
        if (valid) {
            valid = L.flags[a] == 0;
            const int Bm = min(L.row_counts[L.active[a / L.models]], L.model_cap);
            B = (D >= 64 && Bm < D) ? Bm : D;  // use_dual_pca (core.cpp:656-658)
        }
        if (!valid) B = 0;
        const float* gram = L.gram + static_cast<size_t>(max(a, 0)) * N * N;
        float mx = 0.0f;
        for (int r = r0; r < B; r += seg) {
            for (int c = 0; c < B; ++c) {
                const float x = gram[r * B + c];
                m[r * ld + c] = x;
                v[r * ld + c] = r == c ? 1.0f : 0.0f;
                mx = std_max(mx, fabsf(x));
            }
        }
        for (int o = seg / 2; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        const float threshold = std_max(0.0f, __fmul_rn(64.0f * FLT_EPSILON, std_max(1.0f, mx)));
        __syncwarp();
        if (__any_sync(0xffffffffu, B > 1)) {
            for (int sweep = 0; sweep < 64; ++sweep) {
                float off = 0.0f;
                for (int r = r0; r < B; r += seg)
                    for (int c = r + 1; c < B; ++c) off = std_max(off, fabsf(m[r * ld + c]));
                for (int o = seg / 2; o > 0; o >>= 1) off = fmaxf(off, __shfl_xor_sync(0xffffffffu, off, o));
                const bool busy = B > 1 && !(off <= threshold);
                if (!__any_sync(0xffffffffu, busy)) break;
                for (int p = 0; p + 1 < N; ++p) {
                    for (int q = p + 1; q < N; ++q) {
                        bool rot = false;
                        float app = 0.0f, aqq = 0.0f, apq = 0.0f;
                        if (busy && q < B) {
                            apq = m[p * ld + q];
                            rot = fabsf(apq) > threshold && apq != 0.0f;
                            if (rot) {
                                app = m[p * ld + p];
                                aqq = m[q * ld + q];
                            }
                        }
                        __syncwarp();
                        if (rot) {
                            // jacobi_rotate (linalg.cpp:152-196)
                            float c, s;
                            if (L.mixed) {
                                // chosen forms: the rotation angle in FP64, so that near-degenerate
                                // pairs (aqq - app tiny against apq) keep their angle
                                const double tau = (static_cast<double>(aqq) - static_cast<double>(app)) /
                                                   (2.0 * static_cast<double>(apq));
                                const double t_abs = 1.0 / (fabs(tau) + sqrt(1.0 + tau * tau));
                                const double t = tau < 0.0 ? -t_abs : t_abs;
                                const double cd = 1.0 / sqrt(1.0 + t * t);
                                c = static_cast<float>(cd);
                                s = static_cast<float>(t * cd);
                            } else {
                                const float tau = __fdiv_rn(__fsub_rn(aqq, app), __fmul_rn(2.0f, apq));
                                const float tau_abs = fabsf(tau);
                                const float t_abs = __fdiv_rn(
                                    1.0f, __fadd_rn(tau_abs, __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(tau, tau)))));
                                const float t = tau < 0.0f ? -t_abs : t_abs;
                                c = __fdiv_rn(1.0f, __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(t, t))));
                                s = __fmul_rn(t, c);
                            }
                            for (int r = r0; r < B; r += seg) {
                                if (r != p && r != q) {
                                    const float arp = m[r * ld + p];
                                    const float arq = m[r * ld + q];
                                    const float nrp = __fsub_rn(__fmul_rn(c, arp), __fmul_rn(s, arq));
                                    const float nrq = __fadd_rn(__fmul_rn(s, arp), __fmul_rn(c, arq));
                                    m[r * ld + p] = nrp;
                                    m[p * ld + r] = nrp;
                                    m[r * ld + q] = nrq;
                                    m[q * ld + r] = nrq;
                                }
                                const float vrp = v[r * ld + p];
                                const float vrq = v[r * ld + q];
                                v[r * ld + p] = __fsub_rn(__fmul_rn(c, vrp), __fmul_rn(s, vrq));
                                v[r * ld + q] = __fadd_rn(__fmul_rn(s, vrp), __fmul_rn(c, vrq));
                                const float cc = __fmul_rn(c, c), ss = __fmul_rn(s, s);
                                const float cs2 = __fmul_rn(2.0f, __fmul_rn(c, s));
                                if (r == p) {
                                    m[p * ld + p] = __fadd_rn(__fsub_rn(__fmul_rn(cc, app), __fmul_rn(cs2, apq)),
                                                                __fmul_rn(ss, aqq));
                                    m[p * ld + q] = 0.0f;
                                } else if (r == q) {
                                    m[q * ld + q] = __fadd_rn(__fadd_rn(__fmul_rn(ss, app), __fmul_rn(cs2, apq)),
                                                                __fmul_rn(cc, aqq));
                                    m[q * ld + p] = 0.0f;
                                }
                            }
                        }
                        __syncwarp();
                    }
                }
            }
        }
        // stable sort of the diagonal (descending), canonicalised top-rank
        // eigenvectors (canonicalize_vector_row, linalg.cpp:198-227)
        for (int r = r0; r < B; r += seg) {
            const float dr = m[r * ld + r];
            int pos = 0;
            for (int j = 0; j < B; ++j) {
                const float dj = m[j * ld + j];
                if (dj > dr || (j < r && !(dr > dj))) ++pos;
            }
            order[pos] = r;
        }
        __syncwarp();
        if (valid) {
            float* eig = L.eig + static_cast<size_t>(a) * R;
            float* dual = L.dual + static_cast<size_t>(a) * R * N;
            for (int out = r0; out < R; out += seg) {
                const int src = order[out];
                eig[out] = m[src * ld + src];
                float norm2 = 0.0f, best = 0.0f;
                int pivot = 0;
                for (int r = 0; r < B; ++r) {
                    const float x = v[r * ld + src];
                    norm2 = __fadd_rn(norm2, __fmul_rn(x, x));
                    const float ax = fabsf(x);
                    if (ax > best) {
                        best = ax;
                        pivot = r;
                    }
                }
                float sc = 1.0f;
                const bool scale = !(norm2 <= FLT_MIN);
                if (scale) {
                    sc = __fdiv_rn(1.0f, __fsqrt_rn(norm2));
                    if (v[pivot * ld + src] < 0.0f) sc = -sc;
                }
                for (int r = 0; r < B; ++r) {
                    const float x = v[r * ld + src];
                    dual[out * N + r] = scale ? __fmul_rn(x, sc) : x;
                }
            }
        }
        __syncwarp();
        (void)seg_mask;
    }
}

// One model's term of a row's log weight (accumulate_aggregation_model,
// core.cpp:326-412): the group weight, minus beta times the membership.
__device__ __forceinline__ float model_log_weight(const StageConfig& P, bool membership_on, float lgw, float volume,
                                                  float score, float min_score) {
    if (P.weight_alpha == 0.0f && P.weight_beta == 0.0f) return 0.0f;
    if (!membership_on) return lgw;
    const float diff = __fsub_rn(score, min_score);
    const float membership = __fadd_rn(diff > 0.0f ? diff : 0.0f, volume);
    return __fsub_rn(lgw, __fmul_rn(P.weight_beta, membership));
}

// ---------------------------------------------------------------------------
// apply: one CTA per group.  Shared layout (floats unless noted):
//   coloff[D] (int), means[2D], X[B][ldx] centred model rows, basis[R][ldb],
//   dual[R*Bmax], per-component scalars (5R), scores[max_rows],
//   per-warp scratch (3 rows of ldb), row bases[max_rows] (size_t).
// Row strides are padded (ldx = D + 1, ldb = D + 8) so that lanes reading
// different rows at the same column hit different banks.
// Row tiles of the tiled row loop: kTileRows rows per warp, at most
// kTileComps components, and per row the folded dot products in kTileSlots
// floats (membership dots [0, 16), reconstruction dots [16, 32), norm at 32).
constexpr int kTileRows = 2;
constexpr int kTileComps = 16;
constexpr int kTileSlots = 33;

struct ApplyLayout {
    int D, Bmax, R, ldx, ldb, ldu, colpad;
    size_t means, X, basis, dual, scal, scores, scratch, tile_floats, bases, bytes;
};

// tiled: the row loop of apply_kernel<true>, whose per-warp row tiles (the
// centred rows at stride ldu = 8 mod 32, and the Final stage's noisy rows)
// share their space with the model rows X, which are dead by then.
__host__ __device__ inline ApplyLayout apply_layout(int D, int Bmax, int R, int max_rows, int warps,
                                                    bool tiled = false, bool final_stage = false) {
    ApplyLayout a{};
    a.D = D;
    a.Bmax = Bmax;
    a.R = R;
    a.ldx = D + 1;
    a.ldu = ((D + 23) & ~31) + 8;  // smallest stride >= D that is 8 mod 32
    // basis rows: the tiled loop reads four components at one column, 8 banks apart
    a.ldb = tiled ? a.ldu : D + 8;
    a.colpad = (D + 3) & ~3;
    size_t off = static_cast<size_t>(a.colpad);
    a.means = off;   off += 2 * static_cast<size_t>(D);
    a.basis = off;   off += static_cast<size_t>(R) * a.ldb;
    a.dual = off;    off += static_cast<size_t>(R) * Bmax;
    a.scal = off;    off += 5 * static_cast<size_t>(R);
    a.scores = off;  off += static_cast<size_t>(max_rows);
    a.scratch = off;
    if (tiled) {
        a.tile_floats = static_cast<size_t>(final_stage ? 2 : 1) * kTileRows * a.ldu + kTileRows * kTileSlots;
        a.X = off;
        const size_t tiles = static_cast<size_t>(warps) * a.tile_floats;
        const size_t model = static_cast<size_t>(Bmax) * a.ldx;
        off += tiles > model ? tiles : model;
    } else {
        // the centred model rows are read only while the basis is built,
        // before any warp uses its row scratch: they share the space
        a.X = off;
        const size_t rows = static_cast<size_t>(warps) * (2 * a.ldb + R + 1);
        const size_t model = static_cast<size_t>(Bmax) * a.ldx;
        off += rows > model ? rows : model;
    }
    off = (off + 1) & ~static_cast<size_t>(1);
    a.bases = off;   off += 2 * static_cast<size_t>(max_rows);
    a.bytes = off * sizeof(float);
    return a;
}

// The pinned 8-lane fold of an octet's chains as an xor butterfly: every lane
// of the octet ends with ((v0 + v4) + (v2 + v6)) + ((v1 + v5) + (v3 + v7)),
// the same additions as reduce8 (each one commutative).
__device__ __forceinline__ float octet_fold(float v) {
    v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 4));
    v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 2));
    return __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 1));
}

// kTiled: rows in tiles of kTileRows per warp (rank <= kTileComps, dimension
// above 16), else one row per warp with the components four at a time.
template <bool kTiled>
__global__ void __launch_bounds__(kApplyThreads, 3) apply_kernel(FilterLaunch L) {
    extern __shared__ __align__(16) float sm[];
    const int D = L.dim;
    const int Bmax = bmax_of(L);
    const int R = L.rank;
    const ApplyLayout lay = apply_layout(D, Bmax, R, L.max_rows, kApplyWarps, kTiled, L.stage == 1);
    const int ldx = lay.ldx, ldb = lay.ldb;
    int* coloff = reinterpret_cast<int*>(sm);
    float* means = sm + lay.means;  // membership mean, reconstruction centre
    float* X = sm + lay.X;
    float* basis = sm + lay.basis;
    float* dual = sm + lay.dual;
    float* eig = sm + lay.scal;     // eigenvalues
    float* coef = eig + R;          // Wiener coefficients
    float* denom = coef + R;        // signal eigenvalue + membership noise
    float* inv_sqrt = denom + R;    // 1 / sqrt(eigenvalue)
    float* terms = inv_sqrt + R;    // log1p(signal / membership noise)
    float* scores = sm + lay.scores;
    float* scratch = sm + lay.scratch;
    size_t* bases = reinterpret_cast<size_t*>(sm + lay.bases);
    __shared__ float s_misc[4];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    for (int col = tid; col < D; col += kApplyThreads) coloff[col] = column_offset(L, col);
    const StageConfig& P = L.cfg;
    const bool final_stage = L.stage == 1;
    const float* model_video = final_stage ? L.basic : L.noisy;
    const bool weights_enabled = P.weight_alpha != 0.0f || P.weight_beta != 0.0f || P.weight_gamma != 0.0f;
    const float sigma2 = __fmul_rn(__fmul_rn(P.beta, P.sigma), P.sigma);
    const float model_noise2 = final_stage ? __fmul_rn(__fmul_rn(P.beta, P.sigma_basic), P.sigma_basic) : sigma2;
    const float match_sigma = final_stage ? P.sigma_basic : P.sigma;
    const float mem2 = std_max(__fmul_rn(match_sigma, match_sigma),
                               __fmul_rn(__fmul_rn(P.membership_noise_floor, P.sigma), P.sigma));
    const bool membership_on = P.weight_beta != 0.0f;
    const int active_count = L.counters->active;
    const int models = L.models;  // models per group (planes when uncoupled)
    const size_t hw = static_cast<size_t>(L.height) * L.width;
    __syncthreads();
    for (int mi = blockIdx.x; mi < active_count * models; mi += gridDim.x) {
        if (L.flags[mi] != 0) continue;  // uniform: equal groups are done, skipped ones reported
        const int a = mi / models;
        const int mc = mi - a * models;
        const int g = L.active[a];
        const int S = L.row_counts[g];
        const MatchRow* rows = L.rows + static_cast<size_t>(g) * L.max_rows;
        const int r0 = L.row_offset[a];
        const int B = min(S, L.model_cap);
        const float* gm = L.means + static_cast<size_t>(mi) * 2 * D;
        for (int i = tid; i < 2 * D; i += kApplyThreads) means[i] = gm[i];
        const int N = L.nmax;  // row stride of the eigenvector rows
        const bool dual_model = D >= 64 && B < D;  // use_dual_pca (core.cpp:656-658)
        for (int i = tid; i < R * Bmax; i += kApplyThreads)
            dual[i] = L.dual[static_cast<size_t>(mi) * R * N + (i / Bmax) * N + i % Bmax];
        // row bases of this model's plane
        for (int i = tid; i < S; i += kApplyThreads) bases[i] = row_base(L, rows[i]) + mc * hw;
        // per-component scalars, computed once per group (same operations as
        // the CPU, which recomputes them where it uses them)
        for (int c = tid; c < R; c += kApplyThreads) {
            const float lambda = L.eig[static_cast<size_t>(mi) * R + c];
            eig[c] = lambda;
            const float diff = __fsub_rn(lambda, model_noise2);
            const float signal = diff > 0.0f ? diff : 0.0f;
            denom[c] = __fadd_rn(signal, mem2);
            inv_sqrt[c] = lambda > kEigenFloor ? __fdiv_rn(1.0f, __fsqrt_rn(lambda)) : 0.0f;
            terms[c] = (membership_on && signal > 0.0f) ? cr_log1pf(__fdiv_rn(signal, mem2)) : 0.0f;
            const float sigma_basic2 = final_stage ? model_noise2 : sigma2;
            const float threshold = __fmul_rn(P.variance_threshold, sigma2);
            float variance = lambda;
            if (sigma_basic2 > 0.0f) variance = __fsub_rn(variance, std_min(variance, sigma_basic2));
            coef[c] = variance > threshold ? __fdiv_rn(1.0f, __fadd_rn(1.0f, __fdiv_rn(sigma2, variance))) : 0.0f;
        }
        __syncthreads();
        const float* member_mean = means;
        const float* center_vec = means + D;
        if (R > 0 && !dual_model) {
            // covariance model: the canonicalised eigenvectors are the basis
            for (int b = warp; b < R; b += kApplyWarps)
                for (int col = lane; col < D; col += 32)
                    basis[b * ldb + col] = L.dual[static_cast<size_t>(mi) * R * N + static_cast<size_t>(b) * N + col];
            __syncthreads();
        }
        if (R > 0 && dual_model) {
            // centred model rows (compute_mean + center_rows of the first B rows)
            for (int s = warp; s < B; s += kApplyWarps) {
                const float* src = model_video + bases[s];
                for (int col = lane; col < D; col += 32)
                    X[s * ldx + col] = __fsub_rn(__ldg(src + coloff[col]), member_mean[col]);
            }
            __syncthreads();
            // dual -> primal basis (map_dual_eigenvectors_to_basis): one output
            // per lane, the samples accumulated in order
            for (int b = warp; b < R; b += kApplyWarps) {
                const bool live = eig[b] > kEigenFloor;
                for (int col = lane; col < D; col += 32) {
                    float acc = 0.0f;
                    if (live) {
                        const bool fused = fused_column(col, D);
                        for (int s = 0; s < B; ++s) {
                            const float x = X[s * ldx + col];
                            const float w = dual[b * Bmax + s];
                            acc = fused ? __fmaf_rn(w, x, acc) : __fadd_rn(acc, __fmul_rn(w, x));
                        }
                        acc = __fmul_rn(acc, inv_sqrt[b]);
                    }
                    basis[b * ldb + col] = acc;
                }
            }
            __syncthreads();
            for (int b = warp; b < R; b += kApplyWarps) {
                if (!(eig[b] > kEigenFloor)) continue;
                float* row = basis + b * ldb;
                const float norm2 = octet_dot8(row, row, D, lane & 7);
                __syncwarp();
                if (norm2 <= kEigenFloor) {
                    for (int col = lane; col < D; col += 32) row[col] = 0.0f;
                } else {
                    const float sc = __fdiv_rn(1.0f, __fsqrt_rn(norm2));
                    for (int col = lane; col < D; col += 32) row[col] = __fmul_rn(row[col], sc);
                }
            }
        }
        // group precision and volume (group_precision_tau, core.cpp:222-241,
        // 346-358): the terms are ready, the sums run in component order
        if (tid == 0) {
            float trace = 0.0f, volume = 0.0f;
            for (int c = 0; c < R; ++c) {
                const float diff = __fsub_rn(eig[c], model_noise2);
                const float lambda = diff > 0.0f ? diff : 0.0f;
                if (lambda > 0.0f) {
                    trace = __fadd_rn(trace, __fdiv_rn(lambda, __fadd_rn(lambda, sigma2)));
                    volume = __fadd_rn(volume, terms[c]);
                }
            }
            const float tau = __fadd_rn(
                __fadd_rn(P.weight_epsilon, __fdiv_rn(static_cast<float>(D), static_cast<float>(B))), trace);
            s_misc[0] = P.weight_alpha == 0.0f ? 0.0f : __fmul_rn(-P.weight_alpha, cr_logf(tau));
            s_misc[1] = __fdiv_rn(volume, static_cast<float>(D));
        }
        __syncthreads();
        const float lgw = s_misc[0];
        const float volume = s_misc[1];
        if constexpr (kTiled) {
            // Rows in tiles of kTileRows per warp.  Lane (j, g) runs the pinned
            // chain j (elements j + 8m) of both tile rows against components
            // g, g + 4, g + 8 and g + 12, so one basis load feeds the membership
            // and the reconstruction chains of two rows; octet_fold folds the
            // chains, and one lane per (row, dot) adds the unfused tail
            // (dot_contiguous_highway: the operations of octet_dot8).
            float* U = scratch + warp * lay.tile_floats;  // centred membership rows
            float* V = U + kTileRows * lay.ldu;            // centred noisy rows (Final)
            float* res = U + (final_stage ? 2 : 1) * kTileRows * lay.ldu;  // [row][kTileSlots]
            const int ldu = lay.ldu;
            const int j = lane & 7;
            const int grp = lane >> 3;
            const int full = D / kLanes;
            const float score_scale = __fsqrt_rn(__fmul_rn(2.0f, static_cast<float>(D)));
            for (int t0 = warp * kTileRows; t0 < S; t0 += kApplyWarps * kTileRows) {
                const int nrows = min(kTileRows, S - t0);
                for (int r = 0; r < nrows; ++r) {
                    const size_t b = bases[t0 + r];
                    for (int col = lane; col < D; col += 32) {
                        const float xn = __ldg(L.noisy + b + coloff[col]);
                        if (final_stage) {
                            U[r * ldu + col] = __fsub_rn(__ldg(L.basic + b + coloff[col]), member_mean[col]);
                            V[r * ldu + col] = __fsub_rn(xn, center_vec[col]);
                        } else {
                            U[r * ldu + col] = __fsub_rn(xn, member_mean[col]);
                        }
                    }
                }
                __syncwarp();
                const int r1 = nrows > 1 ? 1 : 0;  // a missing second row repeats the first
                float am[kTileRows][4], ar[kTileRows][4], an[kTileRows];
#pragma unroll
                for (int r = 0; r < kTileRows; ++r) {
                    an[r] = 0.0f;
#pragma unroll
                    for (int k = 0; k < 4; ++k) am[r][k] = ar[r][k] = 0.0f;
                }
                for (int m = 0; m < full; ++m) {
                    const int col = j + kLanes * m;
                    const float u0 = U[col], u1 = U[r1 * ldu + col];
                    an[0] = __fmaf_rn(u0, u0, an[0]);
                    an[1] = __fmaf_rn(u1, u1, an[1]);
                    if (final_stage) {
                        const float v0 = V[col], v1 = V[r1 * ldu + col];
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (grp + 4 * k < R) {
                                const float bv = basis[(grp + 4 * k) * ldb + col];
                                am[0][k] = __fmaf_rn(u0, bv, am[0][k]);
                                am[1][k] = __fmaf_rn(u1, bv, am[1][k]);
                                ar[0][k] = __fmaf_rn(v0, bv, ar[0][k]);
                                ar[1][k] = __fmaf_rn(v1, bv, ar[1][k]);
                            }
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (grp + 4 * k < R) {
                                const float bv = basis[(grp + 4 * k) * ldb + col];
                                am[0][k] = __fmaf_rn(u0, bv, am[0][k]);
                                am[1][k] = __fmaf_rn(u1, bv, am[1][k]);
                            }
                    }
                }
                // fold; lane j of octet grp stores (row j / 4, component grp + 4 (j % 4))
#pragma unroll
                for (int r = 0; r < kTileRows; ++r) {
                    an[r] = octet_fold(an[r]);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        am[r][k] = octet_fold(am[r][k]);
                        if (final_stage) ar[r][k] = octet_fold(ar[r][k]);
                    }
                }
#pragma unroll
                for (int r = 0; r < kTileRows; ++r)
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (j == 4 * r + k && grp + 4 * k < R) {
                            res[r * kTileSlots + grp + 4 * k] = am[r][k];
                            if (final_stage) res[r * kTileSlots + 16 + grp + 4 * k] = ar[r][k];
                        }
                if (lane < kTileRows) res[lane * kTileSlots + 32] = lane == 0 ? an[0] : an[1];
                __syncwarp();
                if (full * kLanes < D) {
                    // the unfused tail of each dot: lane -> (row, slot)
                    for (int e = lane; e < kTileRows * kTileSlots; e += 32) {
                        const int r = e / kTileSlots;
                        const int slot = e - r * kTileSlots;
                        const bool norm = slot == 32;
                        const bool recon = slot >= 16 && !norm;
                        const int c = norm ? 0 : (recon ? slot - 16 : slot);
                        if (r >= nrows || (!norm && (c >= R || (recon && !final_stage)))) continue;
                        const float* l = (recon ? V : U) + r * ldu;
                        const float* rgt = norm ? U + r * ldu : basis + c * ldb;
                        float total = res[e];
                        for (int idx = full * kLanes; idx < D; ++idx)
                            total = __fadd_rn(total, __fmul_rn(l[idx], rgt[idx]));
                        res[e] = total;
                    }
                    __syncwarp();
                }
                // membership score of each row, components in order
                if (lane < nrows && membership_on) {
                    const float* rr = res + lane * kTileSlots;
                    float distance = 0.0f, projected = 0.0f;
                    for (int ck = 0; ck < R; ++ck) {
                        const float mk = rr[ck];
                        const float proj2 = __fmul_rn(mk, mk);
                        distance = __fadd_rn(distance, __fdiv_rn(proj2, denom[ck]));
                        projected = __fadd_rn(projected, proj2);
                    }
                    const float resid = __fsub_rn(rr[32], projected);
                    distance = __fadd_rn(distance, __fdiv_rn(resid > 0.0f ? resid : 0.0f, mem2));
                    scores[t0 + lane] = __fdiv_rn(__fsub_rn(distance, static_cast<float>(D)), score_scale);
                }
                // reconstruction (project_bayes_estimate) of the tile's rows,
                // components in order, in registers over blocks of 32 * kRecCols
                const int proj_slot = final_stage ? 16 : 0;
                for (int base = 0; base < D; base += 32 * kRecCols) {
                    float o[kTileRows][kRecCols];
#pragma unroll
                    for (int r = 0; r < kTileRows; ++r)
#pragma unroll
                        for (int jj = 0; jj < kRecCols; ++jj) o[r][jj] = 0.0f;
                    for (int c = 0; c < R; ++c) {
                        const float cf = coef[c];
                        if (cf == 0.0f) continue;
                        const float sc0 = __fmul_rn(cf, res[proj_slot + c]);
                        const float sc1 = __fmul_rn(cf, res[kTileSlots + proj_slot + c]);
                        const float* bc = basis + c * ldb;
#pragma unroll
                        for (int jj = 0; jj < kRecCols; ++jj) {
                            const int col = base + lane + 32 * jj;
                            if (col < D) {
                                const float bv = bc[col];
                                o[0][jj] = add_scaled_elem(o[0][jj], bv, sc0, col, D);
                                o[1][jj] = add_scaled_elem(o[1][jj], bv, sc1, col, D);
                            }
                        }
                    }
#pragma unroll
                    for (int r = 0; r < kTileRows; ++r) {
                        if (r >= nrows) break;
                        float* out = L.filtered + static_cast<size_t>(r0 + t0 + r) * L.row_dim + mc * D;
#pragma unroll
                        for (int jj = 0; jj < kRecCols; ++jj) {
                            const int col = base + lane + 32 * jj;
                            if (col < D) out[col] = __fadd_rn(o[r][jj], center_vec[col]);
                        }
                    }
                }
                __syncwarp();
            }
        } else {
            // per row: membership score and reconstruction.  In the Basic stage the
            // membership row and the reconstruction row are the same centred noisy
            // row, so its projections serve both.
            float* u = scratch + warp * (2 * ldb + R + 1);  // centred membership row
            float* v = u + ldb;                             // centred noisy row (Final)
            float* proj = v + ldb;                          // projections for the reconstruction
            const int j8 = lane & 7;
            const int oct = lane >> 3;
            const float score_scale = __fsqrt_rn(__fmul_rn(2.0f, static_cast<float>(D)));
            for (int i = warp; i < S; i += kApplyWarps) {
                const size_t b = bases[i];
                for (int col = lane; col < D; col += 32) {
                    const float xn = __ldg(L.noisy + b + coloff[col]);
                    if (final_stage) {
                        u[col] = __fsub_rn(__ldg(L.basic + b + coloff[col]), member_mean[col]);
                        v[col] = __fsub_rn(xn, center_vec[col]);
                    } else {
                        u[col] = __fsub_rn(xn, member_mean[col]);
                    }
                }
                __syncwarp();
                float distance = 0.0f, projected = 0.0f, norm2 = 0.0f;
                // pass over c0 = -1 (norm), 0, 4, ...: octet k computes component c0 + k
                for (int c0 = membership_on ? -1 : 0; c0 < R; c0 += 4) {
                    const int c = min(c0 + oct, R - 1);
                    const float dm = (membership_on || !final_stage) ? octet_dot8(u, c < 0 ? u : basis + c * ldb, D, j8)
                                                                     : 0.0f;
                    const float dr = final_stage ? octet_dot8(v, basis + max(c, 0) * ldb, D, j8) : dm;
                    for (int k = 0; k < 4; ++k) {
                        const int ck = c0 + k;
                        const float mk = __shfl_sync(0xffffffffu, dm, k * 8);
                        const float rk = __shfl_sync(0xffffffffu, dr, k * 8);
                        if (ck >= R) break;
                        if (ck < 0) {
                            norm2 = mk;
                            continue;
                        }
                        if (membership_on) {
                            const float proj2 = __fmul_rn(mk, mk);
                            distance = __fadd_rn(distance, __fdiv_rn(proj2, denom[ck]));
                            projected = __fadd_rn(projected, proj2);
                        }
                        if (lane == 0) proj[ck] = rk;
                    }
                }
                if (membership_on) {
                    const float res = __fsub_rn(norm2, projected);
                    distance = __fadd_rn(distance, __fdiv_rn(res > 0.0f ? res : 0.0f, mem2));
                    const float score = __fdiv_rn(__fsub_rn(distance, static_cast<float>(D)), score_scale);
                    if (lane == 0) scores[i] = score;
                }
                __syncwarp();
                // reconstruction (project_bayes_estimate), components in order,
                // accumulated in registers over blocks of 32 * kRecCols columns
                float* out = L.filtered + static_cast<size_t>(r0 + i) * L.row_dim + mc * D;
                for (int base = 0; base < D; base += 32 * kRecCols) {
                    float o[kRecCols];
#pragma unroll
                    for (int j = 0; j < kRecCols; ++j) o[j] = 0.0f;
                    for (int c = 0; c < R; ++c) {
                        if (coef[c] == 0.0f) continue;
                        const float scaled = __fmul_rn(coef[c], proj[c]);
                        const float* bc = basis + c * ldb;
#pragma unroll
                        for (int j = 0; j < kRecCols; ++j) {
                            const int col = base + lane + 32 * j;
                            if (col < D) o[j] = add_scaled_elem(o[j], bc[col], scaled, col, D);
                        }
                    }
#pragma unroll
                    for (int j = 0; j < kRecCols; ++j) {
                        const int col = base + lane + 32 * j;
                        if (col < D) out[col] = __fadd_rn(o[j], center_vec[col]);
                    }
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // aggregation weights (accumulate_aggregation_model + finalize)
        if (tid == 0) {
            float mn = kInf;
            if (membership_on)
                for (int i = 0; i < S; ++i) mn = std_min(mn, scores[i]);
            s_misc[2] = mn;
        }
        __syncthreads();
        const float min_score = s_misc[2];
        for (int i = tid; i < S; i += kApplyThreads) {
            if (models > 1) {
                // this plane's term of the row's log weight; combine_weights
                // sums the planes in order and finalises
                L.logw[static_cast<size_t>(r0 + i) * models + mc] =
                    model_log_weight(P, membership_on, lgw, volume, scores[i], min_score);
                continue;
            }
            float w = 1.0f;
            if (weights_enabled) {
                float lw;
                if (P.weight_alpha == 0.0f && P.weight_beta == 0.0f) {
                    lw = 0.0f;
                } else if (membership_on) {
                    const float diff = __fsub_rn(scores[i], min_score);
                    const float membership = __fadd_rn(diff > 0.0f ? diff : 0.0f, volume);
                    lw = __fadd_rn(0.0f, __fsub_rn(lgw, __fmul_rn(P.weight_beta, membership)));
                } else {
                    lw = __fadd_rn(0.0f, lgw);
                }
                lw = lw < -80.0f ? -80.0f : (80.0f < lw ? 80.0f : lw);
                w = cr_expf(lw);
            }
            L.weights[r0 + i] = w;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// apply, warp per group: the same arithmetic as apply_kernel, register-blocked
// for D % 32 == 0, rank <= 8 and at most 8 model rows (the shapes of the
// default parameter sets: 8x8 patches, one or three planes, rank 8, group 8).
//
// A lane owns columns lane + 32 jj for the elementwise work (centred model
// rows in registers, basis columns, the reconstruction and its store); for
// the dot products octet k = lane / 8 runs the pinned 8-lane chains j = lane
// % 8 over elements j + 8 m of components k and k + 4 at once, on packed
// pairs: the basis sits in shared memory as float2 (component p, p + 4), so
// one 8-byte load and one packed fused multiply-add advance both chains.
// Per warp (floats): basis [4][D] float2, u[D], v[D], dual [8][8],
// per-component scalars [5][8], scores[max_rows], row bases[max_rows] (size_t).
constexpr int kWarpApplyWarps = 4;

struct WarpApplyLayout {
    int basis, u, v, dual, scal, scores, recon, rw, bases, per_warp;
};

// scatter: also the rows' scaled projections [max_rows][8] and weights
// [max_rows], kept for the second pass that adds the rows into the stack
__host__ __device__ inline WarpApplyLayout warp_apply_layout(int D, int max_rows, bool scatter = false) {
    WarpApplyLayout w{};
    int off = 0;
    w.basis = off;  off += 8 * D;
    w.u = off;      off += D;
    w.v = off;      off += D;
    w.dual = off;   off += 64;
    w.scal = off;   off += 5 * 8;
    w.scores = off; off += max_rows;
    w.recon = off;  off += scatter ? 8 * max_rows : 0;
    w.rw = off;     off += scatter ? max_rows : 0;
    off = (off + 1) & ~1;
    w.bases = off;  off += 2 * max_rows;
    off = (off + 3) & ~3;
    w.per_warp = off;
    return w;
}

__device__ __forceinline__ float2 octet_reduce2(float2 v) {
    // the reduce8 fold of lanes 8k .. 8k+7 into lane 8k, for both halves
    v.x = __fadd_rn(v.x, __shfl_down_sync(0xffffffffu, v.x, 4, 8));
    v.y = __fadd_rn(v.y, __shfl_down_sync(0xffffffffu, v.y, 4, 8));
    v.x = __fadd_rn(v.x, __shfl_down_sync(0xffffffffu, v.x, 2, 8));
    v.y = __fadd_rn(v.y, __shfl_down_sync(0xffffffffu, v.y, 2, 8));
    v.x = __fadd_rn(v.x, __shfl_down_sync(0xffffffffu, v.x, 1, 8));
    v.y = __fadd_rn(v.y, __shfl_down_sync(0xffffffffu, v.y, 1, 8));
    return v;
}

__device__ __forceinline__ float octet_reduce(float v) {
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 4, 8));
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 2, 8));
    v = __fadd_rn(v, __shfl_down_sync(0xffffffffu, v, 1, 8));
    return v;
}

// resident blocks per SM the warp-per-group apply is compiled for (a register
// budget); a build parameter for comparisons
#ifndef VNLB_APPLY_MIN_BLOCKS
#define VNLB_APPLY_MIN_BLOCKS 4
#endif

// Chosen forms: a lane's columns of one filtered row added into the anchor
// frame's stack, weight cw times the window at each pixel; the weight plane
// gets the same once per pixel (the columns of plane 0).  Slots outside the
// window are dropped, as the stack tiles drop them.  The additions' order is
// not fixed, so these forms are not bit-reproducible in the stacks' last
// bits.
//
// Pixel-interleaved stacks (L.scatter_pack = C+1): with C = 3 and 64
// columns per plane, a lane's columns jj, jj + kCols/3 and jj + 2 kCols/3
// are the same pixel of planes 0, 1 and 2, so the pixel's three values and
// its weight go in one 16-byte vector addition (C = 1: value and weight in
// one 8-byte one); a quarter (half) of the scalar atomics, and no shuffles.
// (Vector reductions of an octet's patch row in the planar layout, tried,
// were slower: the shuffles that gather a row cost more than they save.)
template <int kCols>
__device__ __forceinline__ void scatter_row(const FilterLaunch& L, const MatchRow& m, const float (&o)[kCols],
                                            float cw, int lane) {
    const size_t plane = static_cast<size_t>(L.height) * L.width;
    const int C = L.channels;
    const int P = L.P;
    const size_t base = static_cast<size_t>(m.y) * L.width + m.x;
    const int slot0 = m.frame + L.search_bwd - L.anchor_frame;
    if constexpr (kCols % 3 == 0) {
        if (L.scatter_pack == 4) {
            constexpr int kpp = kCols / 3;  // columns per plane and lane
#pragma unroll
            for (int jj = 0; jj < kpp; ++jj) {
                const int pos = lane + 32 * jj;  // (layer t, py, px) within the plane's patch
                const int t = pos / (P * P);
                const int rem = pos - t * P * P;
                const int py = rem / P;
                const int slot = slot0 + t;
                if (slot < 0 || slot >= L.slots) continue;
                const float w = L.windowed ? cw * __ldg(L.window + rem) : cw;
                const size_t at = base + static_cast<size_t>(py) * L.width + (rem - py * P);
                atomicAdd(reinterpret_cast<float4*>(L.scatter) + static_cast<size_t>(slot) * plane + at,
                          make_float4(w * o[jj], w * o[jj + kpp], w * o[jj + 2 * kpp], w));
            }
            return;
        }
    }
    if (L.scatter_pack == 2) {
#pragma unroll
        for (int jj = 0; jj < kCols; ++jj) {
            const int pos = lane + 32 * jj;
            const int t = pos / (P * P);
            const int rem = pos - t * P * P;
            const int py = rem / P;
            const int slot = slot0 + t;
            if (slot < 0 || slot >= L.slots) continue;
            const float w = L.windowed ? cw * __ldg(L.window + rem) : cw;
            const size_t at = base + static_cast<size_t>(py) * L.width + (rem - py * P);
            atomicAdd(reinterpret_cast<float2*>(L.scatter) + static_cast<size_t>(slot) * plane + at,
                      make_float2(w * o[jj], w));
        }
        return;
    }
#pragma unroll
    for (int jj = 0; jj < kCols; ++jj) {
        // column (plane c, layer t, py, px)
        const int col = lane + 32 * jj;
        const int c = col / L.patch_dim;
        const int pos = col - c * L.patch_dim;
        const int t = pos / (P * P);
        const int rem = pos - t * P * P;
        const int py = rem / P;
        const int slot = slot0 + t;
        if (slot < 0 || slot >= L.slots) continue;
        const float w = L.windowed ? cw * __ldg(L.window + rem) : cw;
        const size_t at = base + static_cast<size_t>(py) * L.width + (rem - py * P);
        atomicAdd(L.scatter + (static_cast<size_t>(slot) * (C + 1) + c) * plane + at, w * o[jj]);
        if (c == 0) atomicAdd(L.scatter + (static_cast<size_t>(slot) * (C + 1) + C) * plane + at, w);
    }
}

template <int D, bool kScatter>
__global__ void __launch_bounds__(32 * kWarpApplyWarps, VNLB_APPLY_MIN_BLOCKS) apply_warp_kernel(FilterLaunch L) {
    static_assert(D % 32 == 0, "columns are owned in blocks of 32");
    constexpr int kCols = D / 32;
    constexpr int kChain = D / 8;
    extern __shared__ __align__(16) float sm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int j8 = lane & 7;
    const int oct = lane >> 3;
    const WarpApplyLayout lay = warp_apply_layout(D, L.max_rows, kScatter);
    int* coloff = reinterpret_cast<int*>(sm);
    float* wr = sm + D + warp * lay.per_warp;
    float2* basis2 = reinterpret_cast<float2*>(wr + lay.basis);
    const float* basis_f = wr + lay.basis;  // component c, column col at ((c & 3) * D + col) * 2 + (c >> 2)
    float* u = wr + lay.u;
    float* v = wr + lay.v;
    float* dual = wr + lay.dual;
    float* eig = wr + lay.scal;
    float* coef = eig + 8;
    float* denom = coef + 8;
    float* inv_sqrt = denom + 8;
    float* terms = inv_sqrt + 8;
    float* scores = wr + lay.scores;
    size_t* bases = reinterpret_cast<size_t*>(wr + lay.bases);
    for (int col = threadIdx.x; col < D; col += blockDim.x) coloff[col] = column_offset(L, col);

    const int Bmax = bmax_of(L);
    const int R = L.rank;
    const StageConfig& P = L.cfg;
    const bool final_stage = L.stage == 1;
    const float* model_video = final_stage ? L.basic : L.noisy;
    const bool weights_enabled = P.weight_alpha != 0.0f || P.weight_beta != 0.0f || P.weight_gamma != 0.0f;
    const float sigma2 = __fmul_rn(__fmul_rn(P.beta, P.sigma), P.sigma);
    const float model_noise2 = final_stage ? __fmul_rn(__fmul_rn(P.beta, P.sigma_basic), P.sigma_basic) : sigma2;
    const float match_sigma = final_stage ? P.sigma_basic : P.sigma;
    const float mem2 = std_max(__fmul_rn(match_sigma, match_sigma),
                               __fmul_rn(__fmul_rn(P.membership_noise_floor, P.sigma), P.sigma));
    const bool membership_on = P.weight_beta != 0.0f;
    const bool need_dm = membership_on || !final_stage;
    const float score_scale = __fsqrt_rn(__fmul_rn(2.0f, static_cast<float>(D)));
    const int active_count = L.counters->active;
    const int models = L.models;  // models per group (planes when uncoupled)
    const size_t hw = static_cast<size_t>(L.height) * L.width;
    __syncthreads();

    for (int mi = blockIdx.x * kWarpApplyWarps + warp; mi < active_count * models;
         mi += gridDim.x * kWarpApplyWarps) {
        if (L.flags[mi] != 0) {  // equal groups are done, skipped ones reported
            if constexpr (kScatter) {
                if (L.flags[mi] == kGroupDone) {
                    // the pass-through rows prepare wrote, with their weights
                    const int g0 = L.active[mi];
                    const int S0 = L.row_counts[g0];
                    const int q0 = L.row_offset[mi];
                    const MatchRow* rows0 = L.rows + static_cast<size_t>(g0) * L.max_rows;
                    for (int i = 0; i < S0; ++i) {
                        float o[kCols];
#pragma unroll
                        for (int jj = 0; jj < kCols; ++jj)
                            o[jj] = L.filtered[static_cast<size_t>(q0 + i) * L.row_dim + lane + 32 * jj];
                        scatter_row(L, rows0[i], o, L.weights[q0 + i], lane);
                    }
                }
            }
            continue;
        }
        const int a = mi / models;
        const int mc = mi - a * models;
        const int g = L.active[a];
        const int S = L.row_counts[g];
        const MatchRow* rows = L.rows + static_cast<size_t>(g) * L.max_rows;
        const int r0 = L.row_offset[a];
        const int B = min(S, L.model_cap);
        const float* gm = L.means + static_cast<size_t>(mi) * 2 * D;
        float mm[kCols], cc[kCols];
#pragma unroll
        for (int jj = 0; jj < kCols; ++jj) {
            mm[jj] = __ldg(gm + lane + 32 * jj);
            cc[jj] = __ldg(gm + D + lane + 32 * jj);
        }
        for (int i = lane; i < S; i += 32) bases[i] = row_base(L, rows[i]) + mc * hw;  // this model's plane
        for (int i = lane; i < R * Bmax; i += 32) {
            const int b = i / Bmax, s = i - b * Bmax;
            dual[b * 8 + s] = L.dual[static_cast<size_t>(mi) * R * Bmax + i];
        }
        if (lane < R) {
            const int c = lane;
            const float lambda = L.eig[static_cast<size_t>(mi) * R + c];
            eig[c] = lambda;
            const float diff = __fsub_rn(lambda, model_noise2);
            const float signal = diff > 0.0f ? diff : 0.0f;
            denom[c] = __fadd_rn(signal, mem2);
            inv_sqrt[c] = lambda > kEigenFloor ? __fdiv_rn(1.0f, __fsqrt_rn(lambda)) : 0.0f;
            terms[c] = (membership_on && signal > 0.0f) ? cr_log1pf(__fdiv_rn(signal, mem2)) : 0.0f;
            const float sigma_basic2 = final_stage ? model_noise2 : sigma2;
            const float threshold = __fmul_rn(P.variance_threshold, sigma2);
            float variance = lambda;
            if (sigma_basic2 > 0.0f) variance = __fsub_rn(variance, std_min(variance, sigma_basic2));
            coef[c] = variance > threshold ? __fdiv_rn(1.0f, __fadd_rn(1.0f, __fdiv_rn(sigma2, variance))) : 0.0f;
        }
        __syncwarp();

        if (R > 0) {
            // dual -> primal basis over blocks of this lane's columns: the
            // centred model rows of the block in registers, then every
            // component's samples accumulated in order (all columns fused)
            float* bf = wr + lay.basis;
            constexpr int kBlk = kCols % 3 == 0 ? 3 : (kCols % 2 == 0 ? 2 : 1);
#pragma unroll
            for (int j0 = 0; j0 < kCols; j0 += kBlk) {
                float xr[8][kBlk];
#pragma unroll
                for (int s = 0; s < 8; ++s) {
                    if (s < B) {
                        const float* src = model_video + bases[s];
#pragma unroll
                        for (int jj = 0; jj < kBlk; ++jj)
                            xr[s][jj] = __fsub_rn(__ldg(src + coloff[lane + 32 * (j0 + jj)]), mm[j0 + jj]);
                    } else {
#pragma unroll
                        for (int jj = 0; jj < kBlk; ++jj) xr[s][jj] = 0.0f;
                    }
                }
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    if (b >= R) break;
                    const bool live = eig[b] > kEigenFloor;
                    float acc[kBlk];
#pragma unroll
                    for (int jj = 0; jj < kBlk; ++jj) acc[jj] = 0.0f;
                    if (live) {
#pragma unroll
                        for (int s = 0; s < 8; ++s) {
                            if (s >= B) break;
                            const float w = dual[b * 8 + s];
#pragma unroll
                            for (int jj = 0; jj < kBlk; ++jj) acc[jj] = __fmaf_rn(w, xr[s][jj], acc[jj]);
                        }
                        const float is = inv_sqrt[b];
#pragma unroll
                        for (int jj = 0; jj < kBlk; ++jj) acc[jj] = __fmul_rn(acc[jj], is);
                    }
#pragma unroll
                    for (int jj = 0; jj < kBlk; ++jj)
                        bf[((b & 3) * D + lane + 32 * (j0 + jj)) * 2 + (b >> 2)] = acc[jj];
                }
            }
            __syncwarp();
            // unit norm: octet k normalises components k and k + 4
            {
                float2 nv = make_float2(0.0f, 0.0f);
                const float2* row = basis2 + oct * D;
#pragma unroll
                for (int m = 0; m < kChain; ++m) {
                    const float2 x = row[j8 + 8 * m];
                    nv = fma2_rn(x, x, nv);
                }
                nv = octet_reduce2(nv);
                const float n0 = __shfl_sync(0xffffffffu, nv.x, oct * 8);
                const float n1 = __shfl_sync(0xffffffffu, nv.y, oct * 8);
                const int c0 = oct, c1 = oct + 4;
                const bool live0 = c0 < R && eig[c0] > kEigenFloor;
                const bool live1 = c1 < R && eig[c1] > kEigenFloor;
                const float s0 = live0 && !(n0 <= kEigenFloor) ? __fdiv_rn(1.0f, __fsqrt_rn(n0)) : 0.0f;
                const float s1 = live1 && !(n1 <= kEigenFloor) ? __fdiv_rn(1.0f, __fsqrt_rn(n1)) : 0.0f;
                float2* wrow = basis2 + oct * D;
#pragma unroll
                for (int m = 0; m < kChain; ++m) {
                    float2 x = wrow[j8 + 8 * m];
                    if (live0) x.x = n0 <= kEigenFloor ? 0.0f : __fmul_rn(x.x, s0);
                    if (live1) x.y = n1 <= kEigenFloor ? 0.0f : __fmul_rn(x.y, s1);
                    wrow[j8 + 8 * m] = x;
                }
            }
            __syncwarp();
        }
        // group precision and volume, component order (every lane, uniform)
        float lgw, volume;
        {
            float trace = 0.0f, vol = 0.0f;
            for (int c = 0; c < R; ++c) {
                const float diff = __fsub_rn(eig[c], model_noise2);
                const float lambda = diff > 0.0f ? diff : 0.0f;
                if (lambda > 0.0f) {
                    trace = __fadd_rn(trace, __fdiv_rn(lambda, __fadd_rn(lambda, sigma2)));
                    vol = __fadd_rn(vol, terms[c]);
                }
            }
            const float tau = __fadd_rn(
                __fadd_rn(P.weight_epsilon, __fdiv_rn(static_cast<float>(D), static_cast<float>(B))), trace);
            lgw = P.weight_alpha == 0.0f ? 0.0f : __fmul_rn(-P.weight_alpha, cr_logf(tau));
            volume = __fdiv_rn(vol, static_cast<float>(D));
        }

        // rows: membership score and reconstruction; the next row's samples are
        // loaded while the current one is reduced
        float min_score = kInf;
        float nx[kCols], nb[kCols];
        if (S > 0) {
#pragma unroll
            for (int jj = 0; jj < kCols; ++jj) {
                const size_t off = bases[0] + coloff[lane + 32 * jj];
                nx[jj] = __ldg(L.noisy + off);
                nb[jj] = final_stage ? __ldg(L.basic + off) : 0.0f;
            }
        }
        for (int i = 0; i < S; ++i) {
#pragma unroll
            for (int jj = 0; jj < kCols; ++jj) {
                const int col = lane + 32 * jj;
                if (final_stage) {
                    u[col] = __fsub_rn(nb[jj], mm[jj]);
                    v[col] = __fsub_rn(nx[jj], cc[jj]);
                } else {
                    u[col] = __fsub_rn(nx[jj], mm[jj]);
                }
            }
            if (i + 1 < S) {
#pragma unroll
                for (int jj = 0; jj < kCols; ++jj) {
                    const size_t off = bases[i + 1] + coloff[lane + 32 * jj];
                    nx[jj] = __ldg(L.noisy + off);
                    nb[jj] = final_stage ? __ldg(L.basic + off) : 0.0f;
                }
            }
            __syncwarp();
            // octet chains: norm of u, u . basis and (Final) v . basis for
            // components oct and oct + 4
            float nrm = 0.0f;
            float2 pm = make_float2(0.0f, 0.0f), pr = make_float2(0.0f, 0.0f);
            const float2* brow = basis2 + oct * D;
#pragma unroll 8
            for (int m = 0; m < kChain; ++m) {
                const int e = j8 + 8 * m;
                const float ue = u[e];
                if (membership_on) nrm = __fmaf_rn(ue, ue, nrm);
                if (R > 0) {
                    const float2 bb = brow[e];
                    if (need_dm) pm = fma2_rn(make_float2(ue, ue), bb, pm);
                    if (final_stage) {
                        const float ve = v[e];
                        pr = fma2_rn(make_float2(ve, ve), bb, pr);
                    }
                }
            }
            if (membership_on) nrm = octet_reduce(nrm);
            if (need_dm) pm = octet_reduce2(pm);
            if (final_stage) pr = octet_reduce2(pr);
            // lane c < R gathers component c from its octet leader
            const int src = 8 * (lane & 3);
            const bool hi = (lane & 4) != 0;
            float mk = 0.0f, rk = 0.0f;
            {
                const float tx = __shfl_sync(0xffffffffu, pm.x, src);
                const float ty = __shfl_sync(0xffffffffu, pm.y, src);
                mk = hi ? ty : tx;
                if (final_stage) {
                    const float qx = __shfl_sync(0xffffffffu, pr.x, src);
                    const float qy = __shfl_sync(0xffffffffu, pr.y, src);
                    rk = hi ? qy : qx;
                } else {
                    rk = mk;
                }
            }
            if (membership_on) {
                const float norm2 = __shfl_sync(0xffffffffu, nrm, 0);
                const float proj2 = __fmul_rn(mk, mk);
                const float q = lane < R ? __fdiv_rn(proj2, denom[lane]) : 0.0f;
                float distance = 0.0f, projected = 0.0f;
                for (int c = 0; c < R; ++c) {
                    distance = __fadd_rn(distance, __shfl_sync(0xffffffffu, q, c));
                    projected = __fadd_rn(projected, __shfl_sync(0xffffffffu, proj2, c));
                }
                const float res = __fsub_rn(norm2, projected);
                distance = __fadd_rn(distance, __fdiv_rn(res > 0.0f ? res : 0.0f, mem2));
                const float score = __fdiv_rn(__fsub_rn(distance, static_cast<float>(D)), score_scale);
                if (lane == 0) scores[i] = score;
                min_score = std_min(min_score, score);
            }
            // reconstruction (project_bayes_estimate), components in order
            const float scaled = lane < R ? __fmul_rn(coef[lane], rk) : 0.0f;
            if constexpr (kScatter) {
                // kept for the pass after the weights
                if (lane < 8) wr[lay.recon + i * 8 + lane] = scaled;
                __syncwarp();
            } else {
            float o[kCols];
#pragma unroll
            for (int jj = 0; jj < kCols; ++jj) o[jj] = 0.0f;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                if (c >= R) break;
                const float sc = __shfl_sync(0xffffffffu, scaled, c);
                if (coef[c] == 0.0f) continue;
#pragma unroll
                for (int jj = 0; jj < kCols; ++jj)
                    o[jj] = __fmaf_rn(sc, basis_f[((c & 3) * D + lane + 32 * jj) * 2 + (c >> 2)], o[jj]);
            }
            float* out = L.filtered + static_cast<size_t>(r0 + i) * L.row_dim + mc * D;
#pragma unroll
            for (int jj = 0; jj < kCols; ++jj) out[lane + 32 * jj] = __fadd_rn(o[jj], cc[jj]);
            __syncwarp();
            }
        }
        // aggregation weights (accumulate_aggregation_model + finalize)
        for (int i = lane; i < S; i += 32) {
            if (models > 1) {
                L.logw[static_cast<size_t>(r0 + i) * models + mc] =
                    model_log_weight(P, membership_on, lgw, volume, scores[i], min_score);
                continue;
            }
            float w = 1.0f;
            if (weights_enabled) {
                float lw;
                if (P.weight_alpha == 0.0f && P.weight_beta == 0.0f) {
                    lw = 0.0f;
                } else if (membership_on) {
                    const float diff = __fsub_rn(scores[i], min_score);
                    const float membership = __fadd_rn(diff > 0.0f ? diff : 0.0f, volume);
                    lw = __fadd_rn(0.0f, __fsub_rn(lgw, __fmul_rn(P.weight_beta, membership)));
                } else {
                    lw = __fadd_rn(0.0f, lgw);
                }
                lw = lw < -80.0f ? -80.0f : (80.0f < lw ? 80.0f : lw);
                w = cr_expf(lw);
            }
            L.weights[r0 + i] = w;
            if constexpr (kScatter) wr[lay.rw + i] = w;
        }
        __syncwarp();
        if constexpr (kScatter) {
            // each row rebuilt from its scaled projections and added into the
            // stack with its weight
            for (int i = 0; i < S; ++i) {
                const float* sc = wr + lay.recon + i * 8;
                float o[kCols];
#pragma unroll
                for (int jj = 0; jj < kCols; ++jj) o[jj] = 0.0f;
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    if (c >= R) break;
                    if (coef[c] == 0.0f) continue;
                    const float scv = sc[c];
#pragma unroll
                    for (int jj = 0; jj < kCols; ++jj)
                        o[jj] = __fmaf_rn(scv, basis_f[((c & 3) * D + lane + 32 * jj) * 2 + (c >> 2)], o[jj]);
                }
#pragma unroll
                for (int jj = 0; jj < kCols; ++jj) o[jj] = __fadd_rn(o[jj], cc[jj]);
                scatter_row(L, rows[i], o, wr[lay.rw + i], lane);
            }
            __syncwarp();
        }
    }
}

// Weights of the rows of an uncoupled group: the log-weight terms of its
// plane models summed in plane order, times 1 / models, clamped and
// exponentiated (finalize_aggregation_weights, core.cpp:276-294).  Equal
// groups already hold their default-model weight.
__global__ void combine_weights_kernel(FilterLaunch L) {
    const StageConfig& P = L.cfg;
    const bool weights_enabled = P.weight_alpha != 0.0f || P.weight_beta != 0.0f || P.weight_gamma != 0.0f;
    const int models = L.models;
    const float inv_models = __fdiv_rn(1.0f, static_cast<float>(models));
    const int rows = L.counters->rows;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
        const int a = L.row_group[r];
        if (L.flags[static_cast<size_t>(a) * models] != 0) continue;
        float w = 1.0f;
        if (weights_enabled) {
            float acc = 0.0f;
            for (int c = 0; c < models; ++c) acc = __fadd_rn(acc, L.logw[static_cast<size_t>(r) * models + c]);
            float lw = __fmul_rn(acc, inv_models);
            lw = lw < -80.0f ? -80.0f : (80.0f < lw ? 80.0f : lw);
            w = cr_expf(lw);
        }
        L.weights[r] = w;
    }
}

// Segment width, row stride and per-group floats of the Jacobi kernel for
// matrices up to N x N.  A segment of `seg` lanes per group, each lane owning
// rows r0, r0 + seg, ...; two rows per lane from 8 rows up, which halves the
// rotation parameters every lane recomputes.  Rows are padded to N + 1 and
// groups to gstride floats: for N = 8 (segments of 4, 8 groups per warp,
// gstride = 4 mod 32) the lanes of a warp touch 32 distinct banks.  Wider
// segments when a warp's groups would not fit in shared memory (N > 119: one
// group per warp).
struct JacobiShape {
    int seg, ld, gstride;
};
JacobiShape jacobi_shape(int N) {
    int seg = 1;
    while (seg < N && seg < 32) seg <<= 1;
    if (seg >= 8) seg /= 2;
    seg = std::max(seg, 1);
    const int ld = N + 1;
    int gstride = 2 * N * ld + N;
    if (seg == 4) gstride += ((4 - gstride % 32) + 32) % 32;
    while (seg < 32 && static_cast<size_t>(32 / seg) * gstride * sizeof(float) > kFilterSharedLimit) seg <<= 1;
    return JacobiShape{seg, ld, gstride};
}

template <int D>
cudaError_t launch_apply_warp(const FilterLaunch& L, int max_groups, cudaStream_t stream) {
    const bool scatter = L.scatter != nullptr;
    const WarpApplyLayout lay = warp_apply_layout(D, L.max_rows, scatter);
    const size_t smem = (static_cast<size_t>(D) + static_cast<size_t>(kWarpApplyWarps) * lay.per_warp) * sizeof(float);
    auto kernel = scatter ? apply_warp_kernel<D, true> : apply_warp_kernel<D, false>;
    cudaError_t err = raise_smem_limit(reinterpret_cast<const void*>(kernel), static_cast<int>(smem));
    if (err != cudaSuccess) return err;
    const int ctas = std::max(1, std::min((max_groups + kWarpApplyWarps - 1) / kWarpApplyWarps, 148 * 8));
    kernel<<<ctas, 32 * kWarpApplyWarps, smem, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace

size_t filter_shared_bytes(const FilterLaunch& L) {
    const int D = L.dim;
    const int Bmax = std::min(L.model_cap, L.max_rows);
    const int R = L.rank;
    const size_t colpad = static_cast<size_t>((D + 3) & ~3);
    const size_t rows_bytes = static_cast<size_t>(Bmax) * (D + 8) * sizeof(float);
    const int groups_per_cta = rows_bytes > 8 * 1024 ? 1 : kPrepareWarps;
    size_t need = (colpad + static_cast<size_t>(groups_per_cta) * Bmax * (D + 8)) * sizeof(float) +
                  static_cast<size_t>(groups_per_cta) * L.max_rows * sizeof(size_t);
    if (R > 0) {
        const JacobiShape js = jacobi_shape(L.nmax);
        need = std::max(need, static_cast<size_t>(32 / js.seg) * js.gstride * sizeof(float));
    }
    const bool tiled = R >= 1 && R <= kTileComps && D > 16;
    need = std::max(need, apply_layout(D, Bmax, R, L.max_rows, kApplyWarps, tiled, L.stage == 1).bytes);
    return need;
}

size_t filter_shared_limit() { return kFilterSharedLimit; }

bool filter_can_scatter(const FilterLaunch& L) {
    const int D = L.dim;
    const int Bmax = std::min(L.model_cap, L.max_rows);
    return L.models == 1 && L.rank <= 8 && Bmax <= 8 && L.nmax == Bmax &&
           (D == 64 || D == 128 || D == 192 || D == 256);
}

int filter_scatter_pack(const FilterLaunch& L) {
    if (!filter_can_scatter(L)) return 0;
    if (L.channels == 1 && L.dim == L.patch_dim) return 2;
    if (L.channels == 3 && L.dim == 192 && L.patch_dim == 64) return 4;
    return 0;
}

cudaError_t launch_filter(const FilterLaunch& L, int max_groups_in, cudaStream_t stream) {
    if (max_groups_in <= 0) return cudaSuccess;
    const int max_groups = max_groups_in * L.models;  // models to filter at most
    const int D = L.dim;
    const int Bmax = std::min(L.model_cap, L.max_rows);
    const int R = L.rank;
    const size_t colpad = static_cast<size_t>((D + 3) & ~3);
    // prepare: a warp per group while a group's model rows take at most
    // 8 KB of shared memory, else a CTA per group
    {
        const size_t rows_bytes = static_cast<size_t>(Bmax) * (D + 8) * sizeof(float);
        const bool wide = rows_bytes > 8 * 1024;
        const int groups_per_cta = wide ? 1 : kPrepareWarps;
        const size_t smem = (colpad + static_cast<size_t>(groups_per_cta) * Bmax * (D + 8)) * sizeof(float) +
                            static_cast<size_t>(groups_per_cta) * L.max_rows * sizeof(size_t);
        auto kernel = wide ? prepare_kernel<kPrepareWarps> : prepare_kernel<1>;
        cudaError_t err = raise_smem_limit(reinterpret_cast<const void*>(kernel),
                                               static_cast<int>(smem));
        if (err != cudaSuccess) return err;
        const int ctas = std::min((max_groups + groups_per_cta - 1) / groups_per_cta, 148 * 16);
        kernel<<<ctas, 32 * kPrepareWarps, smem, stream>>>(L);
        if ((err = cudaGetLastError()) != cudaSuccess) return err;
    }
    // jacobi
    if (R > 0) {
        // a segment of `seg` lanes per group, each lane owning rows r0, r0 + seg,
        // ...; two rows per lane from 8 rows up, which halves the rotation
        // parameters every lane recomputes
        const int N = L.nmax;  // largest matrix: model rows, or the dimension of covariance models
        const JacobiShape js = jacobi_shape(N);
        const int seg = js.seg, ld = js.ld, gstride = js.gstride;
        const size_t per_group = static_cast<size_t>(gstride) * sizeof(float);
        int warps = 8;
        while (warps > 1 && static_cast<size_t>(warps) * (32 / seg) * per_group > 160 * 1024) warps /= 2;
        const size_t smem = static_cast<size_t>(warps) * (32 / seg) * per_group;
        cudaError_t err = raise_smem_limit(reinterpret_cast<const void*>(jacobi_kernel),
                                               static_cast<int>(smem));
        if (err != cudaSuccess) return err;
        const int per_cta = warps * (32 / seg);
        const int ctas = std::max(1, std::min((max_groups + per_cta - 1) / per_cta, 148 * 32));
        jacobi_kernel<<<ctas, 32 * warps, smem, stream>>>(L, seg, ld, gstride);
        if ((err = cudaGetLastError()) != cudaSuccess) return err;
    }
    // apply
#ifndef VNLB_APPLY_WARP
#define VNLB_APPLY_WARP 1  // the warp-per-group apply for its shapes; a build parameter for comparisons
#endif
    const bool warp_shape = R <= 8 && Bmax <= 8 && L.nmax == Bmax && (D == 64 || D == 128 || D == 192 || D == 256);
    if (L.scatter && !(warp_shape && L.models == 1)) return cudaErrorInvalidValue;  // see filter_can_scatter
    if (L.scatter && L.scatter_pack != 0 &&
        (L.scatter_pack != filter_scatter_pack(L) ||
         reinterpret_cast<uintptr_t>(L.scatter) % (L.scatter_pack * sizeof(float)) != 0))
        return cudaErrorInvalidValue;
    if ((VNLB_APPLY_WARP || L.scatter) && warp_shape && (!L.apply_general || L.scatter)) {
        cudaError_t err = D == 64    ? launch_apply_warp<64>(L, max_groups, stream)
                          : D == 128 ? launch_apply_warp<128>(L, max_groups, stream)
                          : D == 192 ? launch_apply_warp<192>(L, max_groups, stream)
                                     : launch_apply_warp<256>(L, max_groups, stream);
        if (err != cudaSuccess) return err;
    } else {
        // tiled rows for rank <= kTileComps above dimension 16 (the special
        // 8- and 16-element dot orders stay with the row-per-warp loop)
        const bool tiled = R >= 1 && R <= kTileComps && D > 16;
        const ApplyLayout lay = apply_layout(D, Bmax, R, L.max_rows, kApplyWarps, tiled, L.stage == 1);
        const size_t smem = lay.bytes;
        auto kernel = tiled ? apply_kernel<true> : apply_kernel<false>;
        cudaError_t err = raise_smem_limit(reinterpret_cast<const void*>(kernel),
                                               static_cast<int>(smem));
        if (err != cudaSuccess) return err;
        const int ctas = std::min(max_groups, 148 * 8);
        kernel<<<ctas, kApplyThreads, smem, stream>>>(L);
        if ((err = cudaGetLastError()) != cudaSuccess) return err;
    }
    if (L.models > 1) {
        const long long rows = static_cast<long long>(max_groups_in) * L.max_rows;
        const int ctas = static_cast<int>(std::max<long long>(1, std::min<long long>((rows + 255) / 256, 148 * 8)));
        combine_weights_kernel<<<ctas, 256, 0, stream>>>(L);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
}

}  // namespace vnlbgpu
