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
// One CTA (4 warps) per active group, groups taken from the device-side
// active list in a grid-stride loop.  The B model rows are gathered and
// centred into shared memory; the B x B Gram is built one pair per thread; the
// cyclic Jacobi runs on warp 0 with one matrix row per lane; every retained
// row is then streamed once per warp for its membership score and its
// shrunken reconstruction.  All dot products use the pinned 8-lane order
// (per-lane fused accumulators, then the fixed fold), elementwise updates the
// CPU's fused/unfused split, and the elementary functions are correctly
// rounded, so results are bit-identical to the CPU core -- with one stated
// exception: the flat-area variance (double sums) is reduced in a fixed
// parallel order, which can move its float value by one ulp; that changes
// the flat decision only when the variance lies within one ulp of
// gamma*sigma^2.
#include <cfloat>

#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;

// dot_contiguous_highway, one thread.
__device__ float thread_dot8(const float* l, const float* r, int count) {
    float v[kLanes];
    if (count == kLanes || count == 2 * kLanes) {
#pragma unroll
        for (int i = 0; i < kLanes; ++i) v[i] = __fmul_rn(l[i], r[i]);
        if (count == 2 * kLanes) {
#pragma unroll
            for (int i = 0; i < kLanes; ++i) v[i] = __fmaf_rn(l[i + kLanes], r[i + kLanes], v[i]);
        }
        return reduce8(v);
    }
#pragma unroll
    for (int i = 0; i < kLanes; ++i) v[i] = 0.0f;
    int index = 0;
    for (; index + kLanes <= count; index += kLanes) {
#pragma unroll
        for (int i = 0; i < kLanes; ++i) v[i] = __fmaf_rn(l[index + i], r[index + i], v[i]);
    }
    float total = reduce8(v);
    for (; index < count; ++index) total = __fadd_rn(total, __fmul_rn(l[index], r[index]));
    return total;
}

// dot_contiguous_highway computed by an octet of lanes (j = lane & 7): lane j
// owns accumulator j; the fold follows reduce8.  All 8 lanes return the dot.
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

struct Layout {
    int D, B, rank, S;
};

__device__ __forceinline__ float sample_at(const float* video, const FilterLaunch& L, const MatchRow& m, int col) {
    const int pd = L.patch_dim;
    const int c = col / pd;
    const int pos = col - c * pd;
    const int pp = L.P * L.P;
    const int t = pos / pp;
    const int rem = pos - t * pp;
    const int py = rem / L.P;
    const int px = rem - py * L.P;
    return __ldg(video + ((static_cast<size_t>(m.frame + t) * L.channels + c) * L.height + (m.y + py)) *
                             static_cast<size_t>(L.width) + (m.x + px));
}

__global__ void __launch_bounds__(kThreads) filter_kernel(FilterLaunch L) {
    extern __shared__ __align__(16) float sm[];
    const int D = L.dim;
    const int Bmax = min(L.model_cap, L.max_rows);
    const int R = L.rank;
    // shared layout
    float* Xm = sm;                               // Bmax * D   centred model rows
    float* mean_n = Xm + Bmax * D;                // D
    float* mean_b = mean_n + D;                   // D
    float* basis = mean_b + D;                    // R * D
    float* jm = basis + R * D;                    // Bmax^2
    float* jv = jm + Bmax * Bmax;                 // Bmax^2
    float* dual = jv + Bmax * Bmax;               // R * Bmax
    float* eig = dual + R * Bmax;                 // R
    float* coef = eig + R;                        // R
    float* scores = coef + R;                     // max_rows
    float* logw = scores + L.max_rows;            // max_rows
    float* scratch = logw + L.max_rows;           // kWarps * 3 * D
    int* order = reinterpret_cast<int*>(scratch + kWarps * 3 * D);  // Bmax
    __shared__ float s_misc[8];
    __shared__ double s_red[2 * kThreads];

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const StageConfig& P = L.cfg;
    const bool final_stage = L.stage == 1;
    const float* model_video = final_stage ? L.basic : L.noisy;
    const int active_count = L.counters->active;

    for (int a = blockIdx.x; a < active_count; a += gridDim.x) {
        const int g = L.active[a];
        const int S = L.row_counts[g];
        const MatchRow* rows = L.rows + static_cast<size_t>(g) * L.max_rows;
        const int r0 = L.row_offset[a];
        const int B = min(S, L.model_cap);
        for (int i = tid; i < S; i += kThreads) {
            L.row_info[r0 + i] = rows[i];
            L.row_group[r0 + i] = a;
        }
        // ---- equal group (samples_are_equal / group_is_equal)
        int differs = 0;
        if (S > 1) {
            for (int e = tid; e < (S - 1) * D; e += kThreads) {
                const int i = 1 + e / D;
                const int col = e - (i - 1) * D;
                if (sample_at(L.noisy, L, rows[i], col) != sample_at(L.noisy, L, rows[0], col)) differs = 1;
            }
        }
        const bool equal = S > 1 && !__syncthreads_or(differs);
        const bool weights_enabled = P.weight_alpha != 0.0f || P.weight_beta != 0.0f || P.weight_gamma != 0.0f;
        if (equal) {
            // filtered = input, default aggregation model (core.cpp:253-274)
            for (int e = tid; e < S * D; e += kThreads) {
                const int i = e / D;
                const int col = e - i * D;
                L.filtered[static_cast<size_t>(r0 + i) * D + col] = sample_at(L.noisy, L, rows[i], col);
            }
            const float tau = __fadd_rn(P.weight_epsilon, __fdiv_rn(static_cast<float>(D), static_cast<float>(B)));
            const float lgw = P.weight_alpha == 0.0f ? 0.0f : __fmul_rn(-P.weight_alpha, cr_logf(tau));
            float w = 1.0f;
            if (weights_enabled) {
                float lw = __fadd_rn(0.0f, lgw);
                lw = lw < -80.0f ? -80.0f : (80.0f < lw ? 80.0f : lw);
                w = cr_expf(lw);
            }
            for (int i = tid; i < S; i += kThreads) L.weights[r0 + i] = w;
            __syncthreads();
            continue;
        }
        // ---- flat area (Final): mean channel variance of the noisy rows
        bool flat = false;
        if (final_stage && P.flat_areas) {
            const int pd = L.patch_dim;
            const int channels = D / pd;
            const int per_channel = pd * S;
            float variance = 0.0f;
            for (int c = 0; c < channels; ++c) {
                double sum = 0.0, sum2 = 0.0;
                for (int e = tid; e < per_channel; e += kThreads) {
                    const int i = e / pd;
                    const int q = e - i * pd;
                    const float v = sample_at(L.noisy, L, rows[i], c * pd + q);
                    sum += static_cast<double>(v);
                    sum2 += static_cast<double>(v) * static_cast<double>(v);
                }
                s_red[tid] = sum;
                s_red[kThreads + tid] = sum2;
                __syncthreads();
                for (int half = kThreads / 2; half > 0; half >>= 1) {
                    if (tid < half) {
                        s_red[tid] += s_red[tid + half];
                        s_red[kThreads + tid] += s_red[kThreads + tid + half];
                    }
                    __syncthreads();
                }
                if (per_channel > 1) {
                    const double count = static_cast<double>(per_channel);
                    const double s1 = s_red[0], s2 = s_red[kThreads];
                    variance = __fadd_rn(variance, static_cast<float>((s2 - (s1 * s1 / count)) / (count - 1.0)));
                }
                __syncthreads();
            }
            if (per_channel > 1) variance = __fdiv_rn(variance, static_cast<float>(channels));
            flat = variance < __fmul_rn(__fmul_rn(P.sigma, P.sigma), P.gamma);
        }
        if (B < min(D, R)) {
            if (tid == 0) {
                atomicCAS(&L.counters->status, 0, kStatusRankNotCovered);
                L.counters->detail = g;
            }
            __syncthreads();
            continue;
        }
        // ---- means over the first B rows (compute_mean) and centred model rows
        const float inv_b = __fdiv_rn(1.0f, static_cast<float>(B));
        for (int col = tid; col < D; col += kThreads) {
            float mb = 0.0f, mn = 0.0f;
            if (final_stage) {
                for (int r = 0; r < B; ++r) mb = __fadd_rn(mb, sample_at(L.basic, L, rows[r], col));
                mb = __fmul_rn(mb, inv_b);
            }
            if (!final_stage || !flat) {
                for (int r = 0; r < B; ++r) mn = __fadd_rn(mn, sample_at(L.noisy, L, rows[r], col));
                mn = __fmul_rn(mn, inv_b);
            }
            mean_b[col] = mb;
            mean_n[col] = mn;
            const float mm = final_stage ? mb : mn;
            for (int r = 0; r < B; ++r) Xm[r * D + col] = __fsub_rn(sample_at(model_video, L, rows[r], col), mm);
        }
        __syncthreads();
        const float* center_vec = (final_stage && flat) ? mean_b : mean_n;
        const float* member_mean = final_stage ? mean_b : mean_n;

        // ---- model noise constants (core.cpp:190-241, 616-636)
        const float sigma2 = __fmul_rn(__fmul_rn(P.beta, P.sigma), P.sigma);
        const float model_noise2 = final_stage ? __fmul_rn(__fmul_rn(P.beta, P.sigma_basic), P.sigma_basic) : sigma2;
        const float match_sigma = final_stage ? P.sigma_basic : P.sigma;
        const float mem2 = std_max(__fmul_rn(match_sigma, match_sigma),
                                   __fmul_rn(__fmul_rn(P.membership_noise_floor, P.sigma), P.sigma));

        if (R > 0) {
            // ---- dual Gram (compute_gram_centered)
            const float scale = __fdiv_rn(1.0f, static_cast<float>(B));
            const int pairs = B * (B + 1) / 2;
            for (int e = tid; e < pairs; e += kThreads) {
                int r = static_cast<int>((sqrtf(8.0f * e + 1.0f) - 1.0f) * 0.5f);
                while ((r + 1) * (r + 2) / 2 <= e) ++r;
                while (r * (r + 1) / 2 > e) --r;
                const int c = e - r * (r + 1) / 2;
                const float v = __fmul_rn(scale, thread_dot8(Xm + r * D, Xm + c * D, D));
                jm[r * B + c] = v;
                jm[c * B + r] = v;
            }
            for (int e = tid; e < B * B; e += kThreads) jv[e] = (e / B == e % B) ? 1.0f : 0.0f;
            __syncthreads();
            // ---- cyclic Jacobi (topk_symmetric_eigen_jacobi), warp 0
            if (warp == 0) {
                float mx = 0.0f;
                for (int e = lane; e < B * B; e += 32) mx = std_max(mx, fabsf(jm[e]));
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                const float threshold = std_max(0.0f, __fmul_rn(64.0f * FLT_EPSILON, std_max(1.0f, mx)));
                if (B > 1) {
                    for (int sweep = 0; sweep < 64; ++sweep) {
                        float off = 0.0f;
                        for (int e = lane; e < B * B; e += 32) {
                            const int r = e / B, c = e - (e / B) * B;
                            if (c > r) off = std_max(off, fabsf(jm[e]));
                        }
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) off = fmaxf(off, __shfl_xor_sync(0xffffffffu, off, o));
                        if (off <= threshold) break;
                        for (int p = 0; p + 1 < B; ++p) {
                            for (int q = p + 1; q < B; ++q) {
                                const float apq = jm[p * B + q];
                                if (!(fabsf(apq) > threshold)) continue;
                                const float app = jm[p * B + p];
                                const float aqq = jm[q * B + q];
                                __syncwarp();
                                if (apq == 0.0f) continue;
                                const float tau = __fdiv_rn(__fsub_rn(aqq, app), __fmul_rn(2.0f, apq));
                                const float tau_abs = fabsf(tau);
                                const float t_abs = __fdiv_rn(
                                    1.0f, __fadd_rn(tau_abs, __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(tau, tau)))));
                                const float t = tau < 0.0f ? -t_abs : t_abs;
                                const float c = __fdiv_rn(1.0f, __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(t, t))));
                                const float s = __fmul_rn(t, c);
                                const float cc = __fmul_rn(c, c), ss = __fmul_rn(s, s), cs = __fmul_rn(c, s);
                                for (int r = lane; r < B; r += 32) {
                                    if (r == p || r == q) continue;
                                    const float arp = jm[r * B + p];
                                    const float arq = jm[r * B + q];
                                    const float nrp = __fsub_rn(__fmul_rn(c, arp), __fmul_rn(s, arq));
                                    const float nrq = __fadd_rn(__fmul_rn(s, arp), __fmul_rn(c, arq));
                                    jm[r * B + p] = nrp;
                                    jm[p * B + r] = nrp;
                                    jm[r * B + q] = nrq;
                                    jm[q * B + r] = nrq;
                                }
                                for (int r = lane; r < B; r += 32) {
                                    const float vrp = jv[r * B + p];
                                    const float vrq = jv[r * B + q];
                                    jv[r * B + p] = __fsub_rn(__fmul_rn(c, vrp), __fmul_rn(s, vrq));
                                    jv[r * B + q] = __fadd_rn(__fmul_rn(s, vrp), __fmul_rn(c, vrq));
                                }
                                if (lane == 0) {
                                    const float cs2 = __fmul_rn(2.0f, cs);
                                    jm[p * B + p] = __fadd_rn(__fsub_rn(__fmul_rn(cc, app), __fmul_rn(cs2, apq)),
                                                              __fmul_rn(ss, aqq));
                                    jm[q * B + q] = __fadd_rn(__fadd_rn(__fmul_rn(ss, app), __fmul_rn(cs2, apq)),
                                                              __fmul_rn(cc, aqq));
                                    jm[p * B + q] = 0.0f;
                                    jm[q * B + p] = 0.0f;
                                }
                                __syncwarp();
                            }
                        }
                    }
                }
                // stable sort of the diagonal, descending
                for (int i = lane; i < B; i += 32) {
                    const float di = jm[i * B + i];
                    int pos = 0;
                    for (int j = 0; j < B; ++j) {
                        const float dj = jm[j * B + j];
                        if (dj > di || (j < i && !(di > dj))) ++pos;
                    }
                    order[pos] = i;
                }
                __syncwarp();
                // canonicalised top-rank dual vectors (canonicalize_vector_row)
                for (int out = lane; out < R; out += 32) {
                    const int src = order[out];
                    eig[out] = jm[src * B + src];
                    float* row = dual + out * Bmax;
                    float norm2 = 0.0f, best = 0.0f;
                    int pivot = 0;
                    for (int r = 0; r < B; ++r) {
                        const float v = jv[r * B + src];
                        row[r] = v;
                        norm2 = __fadd_rn(norm2, __fmul_rn(v, v));
                        const float av = fabsf(v);
                        if (av > best) {
                            best = av;
                            pivot = r;
                        }
                    }
                    if (!(norm2 <= FLT_MIN)) {
                        float sc = __fdiv_rn(1.0f, __fsqrt_rn(norm2));
                        if (row[pivot] < 0.0f) sc = -sc;
                        for (int r = 0; r < B; ++r) row[r] = __fmul_rn(row[r], sc);
                    }
                }
            }
            __syncthreads();
            // ---- dual -> primal basis (map_dual_eigenvectors_to_basis)
            const float floor_value = 128.0f * FLT_EPSILON;
            for (int e = tid; e < R * D; e += kThreads) {
                const int b = e / D;
                const int col = e - b * D;
                float acc = 0.0f;
                const float lambda = eig[b];
                if (lambda > floor_value) {
                    for (int s = 0; s < B; ++s) acc = add_scaled_elem(acc, Xm[s * D + col], dual[b * Bmax + s], col, D);
                    acc = __fmul_rn(acc, __fdiv_rn(1.0f, __fsqrt_rn(lambda)));
                }
                basis[e] = acc;
            }
            __syncthreads();
            for (int b = warp; b < R; b += kWarps) {
                if (!(eig[b] > floor_value)) continue;
                float* row = basis + b * D;
                const float norm2 = octet_dot8(row, row, D, lane & 7);
                __syncwarp();
                if (norm2 <= floor_value) {
                    for (int col = lane; col < D; col += 32) row[col] = 0.0f;
                } else {
                    const float sc = __fdiv_rn(1.0f, __fsqrt_rn(norm2));
                    for (int col = lane; col < D; col += 32) row[col] = __fmul_rn(row[col], sc);
                }
            }
            // ---- Wiener coefficients (compute_filter_coefficients)
            if (tid < R) {
                const float sigma_basic2 = final_stage ? model_noise2 : sigma2;
                const float threshold = __fmul_rn(P.variance_threshold, sigma2);
                float variance = eig[tid];
                if (sigma_basic2 > 0.0f) variance = __fsub_rn(variance, std_min(variance, sigma_basic2));
                coef[tid] = variance > threshold
                                ? __fdiv_rn(1.0f, __fadd_rn(1.0f, __fdiv_rn(sigma2, variance)))
                                : 0.0f;
            }
            __syncthreads();
        }
        // ---- group precision and volume (group_precision_tau, core.cpp:222-241, 346-358)
        if (tid == 0) {
            const float estimate_noise2 = sigma2;
            float trace = 0.0f, volume = 0.0f;
            for (int c = 0; c < R; ++c) {
                const float diff = __fsub_rn(eig[c], model_noise2);
                const float lambda = diff > 0.0f ? diff : 0.0f;
                if (lambda > 0.0f) {
                    trace = __fadd_rn(trace, __fdiv_rn(lambda, __fadd_rn(lambda, estimate_noise2)));
                    volume = __fadd_rn(volume, cr_log1pf(__fdiv_rn(lambda, mem2)));
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
        const bool membership_on = P.weight_beta != 0.0f && !(P.weight_alpha == 0.0f && P.weight_beta == 0.0f);
        // ---- per row: membership score and reconstruction
        float* u = scratch + warp * 3 * D;  // centred membership row
        float* v = u + D;                   // centred noisy row
        float* o = v + D;                   // reconstruction accumulator
        const int j8 = lane & 7;
        const int oct = lane >> 3;
        for (int i = warp; i < S; i += kWarps) {
            const MatchRow m = rows[i];
            for (int col = lane; col < D; col += 32) {
                const float xn = sample_at(L.noisy, L, m, col);
                const float xu = final_stage ? sample_at(L.basic, L, m, col) : xn;
                u[col] = __fsub_rn(xu, member_mean[col]);
                v[col] = __fsub_rn(xn, center_vec[col]);
                o[col] = 0.0f;
            }
            __syncwarp();
            if (membership_on) {
                // norm2 and the rank projections of the membership row, four
                // dots per pass (one per octet), consumed in component order
                float distance = 0.0f, projected = 0.0f, norm2 = 0.0f;
                for (int c0 = -1; c0 < R; c0 += 4) {
                    const int c = min(c0 + oct, R - 1);
                    const float d = octet_dot8(u, c < 0 ? u : basis + c * D, D, j8);
                    for (int k = 0; k < 4; ++k) {
                        const int ck = c0 + k;
                        const float dk = __shfl_sync(0xffffffffu, d, k * 8);
                        if (ck >= R) break;
                        if (ck < 0) {
                            norm2 = dk;
                        } else {
                            const float proj2 = __fmul_rn(dk, dk);
                            const float diff = __fsub_rn(eig[ck], model_noise2);
                            const float lambda = diff > 0.0f ? diff : 0.0f;
                            distance = __fadd_rn(distance, __fdiv_rn(proj2, __fadd_rn(lambda, mem2)));
                            projected = __fadd_rn(projected, proj2);
                        }
                    }
                }
                const float res = __fsub_rn(norm2, projected);
                distance = __fadd_rn(distance, __fdiv_rn(res > 0.0f ? res : 0.0f, mem2));
                const float score = __fdiv_rn(__fsub_rn(distance, static_cast<float>(D)),
                                              __fsqrt_rn(__fmul_rn(2.0f, static_cast<float>(D))));
                if (lane == 0) scores[i] = score;
            }
            // reconstruction (project_bayes_estimate): components in order
            for (int c0 = 0; c0 < R; c0 += 4) {
                const int c = min(c0 + oct, R - 1);
                const float d = octet_dot8(v, basis + c * D, D, j8);
                for (int k = 0; k < 4; ++k) {
                    const int ck = c0 + k;
                    const float dk = __shfl_sync(0xffffffffu, d, k * 8);
                    if (ck >= R) break;
                    if (coef[ck] == 0.0f) continue;
                    const float scaled = __fmul_rn(coef[ck], dk);
                    const float* bc = basis + ck * D;
                    for (int col = lane; col < D; col += 32) o[col] = add_scaled_elem(o[col], bc[col], scaled, col, D);
                }
            }
            float* out = L.filtered + static_cast<size_t>(r0 + i) * D;
            for (int col = lane; col < D; col += 32) out[col] = __fadd_rn(o[col], center_vec[col]);
            __syncwarp();
        }
        __syncthreads();
        // ---- aggregation weights (accumulate_aggregation_model + finalize)
        if (tid == 0) {
            float mn = kInf;
            if (membership_on)
                for (int i = 0; i < S; ++i) mn = std_min(mn, scores[i]);
            s_misc[2] = mn;
        }
        __syncthreads();
        const float min_score = s_misc[2];
        for (int i = tid; i < S; i += kThreads) {
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

}  // namespace

size_t filter_shared_bytes(const FilterLaunch& L) {
    const size_t D = L.dim;
    const size_t Bmax = std::min(L.model_cap, L.max_rows);
    const size_t R = L.rank;
    const size_t floats = Bmax * D + 2 * D + R * D + 2 * Bmax * Bmax + R * Bmax + 2 * R + 2 * L.max_rows +
                          kWarps * 3 * D + Bmax;
    return floats * sizeof(float);
}

cudaError_t launch_filter(const FilterLaunch& L, int ctas, cudaStream_t stream) {
    const size_t smem = filter_shared_bytes(L);
    cudaError_t err = cudaFuncSetAttribute(filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem));
    if (err != cudaSuccess) return err;
    filter_kernel<<<ctas, kThreads, smem, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace vnlbgpu
