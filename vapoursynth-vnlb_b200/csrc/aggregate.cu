// Contribution stacks and their normalisation (plain form).
//
// Reference semantics: write_sample_contributions_coupled_* and
// write_group_contributions (src/core/core.cpp:1587-1795) accumulate, pixel
// by pixel, the weighted filtered patches of the processed groups in raster
// group order and row order; render_aggregate_frame (src/vs/plugin.cpp:
// 966-1045) sums the stacks of the contributing anchor frames in anchor order
// and divides.
//
// Owner-computes tiles instead of atomics: a CTA owns one (tile, slot) of the
// anchor frame's stack.  It finds the groups whose matches can reach the tile
// (anchors within the search reach, a contiguous range of the raster-ordered
// active list), collects the rows whose patch covers the tile in increasing
// global row order (= CPU order), and every thread applies them to its pixels
// in that order.  The result is bit-identical to the CPU's sequential
// accumulation, needs no clear, and writes every stack value exactly once.
#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr int kTileThreads = 256;
constexpr int kEntryCap = 1024;

struct Entry {
    int r;   // global row
    int t;   // temporal offset inside the patch
    int x, y;
    float w;
};

__device__ __forceinline__ int lower_bound_xy(const int2* xy, int n, int y, int x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const int2 v = xy[mid];
        if (v.y < y || (v.y == y && v.x < x)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kTileThreads) tile_kernel(TileLaunch L) {
    __shared__ Entry entries[kEntryCap];
    __shared__ int s_count;
    __shared__ int s_done;
    extern __shared__ float window[];

    const int T = L.tile;
    const int tx0 = blockIdx.x * T;
    const int ty0 = blockIdx.y * T;
    const int slot = blockIdx.z;
    const int P = L.P;
    const int C = L.channels;
    const int reach = L.search_window - 1;  // |match - anchor| bound per axis
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;

    for (int i = tid; i < P * P; i += blockDim.x) window[i] = L.window[i];
    const int active = L.counters->active;
    // groups whose anchor row can reach the tile: one contiguous range of the
    // raster-ordered active list; their anchor x is filtered on the fly
    const int ay_lo = ty0 - (P - 1) - reach;
    const int ay_hi = ty0 + T - 1 + reach;
    const int ax_lo = tx0 - (P - 1) - reach;
    const int ax_hi = tx0 + T - 1 + reach;
    int cur_g = 0, g_end = 0, cur_r = -1;  // warp-0 iterator state
    if (warp == 0) {
        cur_g = lower_bound_xy(L.active_xy, active, ay_lo, -0x7fffffff);
        g_end = lower_bound_xy(L.active_xy, active, ay_hi + 1, -0x7fffffff);
    }

    constexpr int kMaxPix = 4;
    const int pix_per_thread = (T * T + blockDim.x - 1) / blockDim.x;
    float num[kMaxPix][4];
    float wt[kMaxPix];
#pragma unroll
    for (int p = 0; p < kMaxPix; ++p) {
        wt[p] = 0.0f;
#pragma unroll
        for (int c = 0; c < 4; ++c) num[p][c] = 0.0f;
    }
    __syncthreads();

    const int fused_cols = (P == kLanes || P == 2 * kLanes) ? P : (P / kLanes) * kLanes;
    for (;;) {
        // ---- warp 0 collects the next batch of covering rows, in row order
        if (warp == 0) {
            int count = 0;
            bool full = false;
            while (cur_g < g_end && !full) {
                if (cur_r < 0) {
                    const int gi = cur_g + lane;
                    bool near = false;
                    if (gi < g_end) {
                        const int2 a = L.active_xy[gi];
                        near = a.x >= ax_lo && a.x <= ax_hi;
                    }
                    const unsigned ballot = __ballot_sync(0xffffffffu, near);
                    if (!ballot) {
                        cur_g += 32;
                        continue;
                    }
                    cur_g += __ffs(ballot) - 1;
                    cur_r = L.row_offset[cur_g];
                }
                const int rend = L.row_offset[cur_g + 1];
                while (cur_r < rend) {
                    const int r = cur_r + lane;
                    int hits = 0;
                    int t_hit[4];
                    MatchRow m = {0.0f, 0, 0, 0};
                    if (r < rend) {
                        m = L.row_info[r];
                        if (m.x <= tx0 + T - 1 && m.x + P - 1 >= tx0 && m.y <= ty0 + T - 1 && m.y + P - 1 >= ty0) {
                            for (int t = 0; t < L.Pt && hits < 4; ++t)
                                if (m.frame + t - L.anchor_frame + L.search_bwd == slot) t_hit[hits++] = t;
                        }
                    }
                    int prefix = hits;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int v = __shfl_up_sync(0xffffffffu, prefix, o);
                        if (lane >= o) prefix += v;
                    }
                    const int total = __shfl_sync(0xffffffffu, prefix, 31);
                    if (count + total > kEntryCap) {
                        full = true;
                        break;
                    }
                    const int start = count + prefix - hits;
                    for (int e = 0; e < hits; ++e) {
                        Entry en;
                        en.r = r;
                        en.t = t_hit[e];
                        en.x = m.x;
                        en.y = m.y;
                        en.w = L.weights[r];
                        entries[start + e] = en;
                    }
                    count += total;
                    cur_r += 32;
                }
                if (!full) {
                    cur_g += 1;
                    cur_r = -1;
                }
            }
            if (lane == 0) {
                s_count = count;
                s_done = full ? 0 : 1;
            }
        }
        __syncthreads();
        // ---- apply the batch to this thread's pixels, in order
        const int n = s_count;
        for (int p = 0; p < pix_per_thread && p < kMaxPix; ++p) {
            const int local = tid + p * blockDim.x;
            if (local >= T * T) break;
            const int px = tx0 + local % T;
            const int py = ty0 + local / T;
            for (int e = 0; e < n; ++e) {
                const Entry en = entries[e];
                const int dx = px - en.x;
                const int dy = py - en.y;
                if (dx < 0 || dx >= P || dy < 0 || dy >= P) continue;
                const int pos = (en.t * P + dy) * P + dx;
                const float* f = L.filtered + static_cast<size_t>(en.r) * L.dim;
                if (L.coupled && !L.windowed) {
                    const bool fused = dx < fused_cols;
                    for (int c = 0; c < C; ++c) {
                        const float x = __ldg(f + c * L.patch_dim + pos);
                        num[p][c] = fused ? __fmaf_rn(en.w, x, num[p][c]) : __fadd_rn(num[p][c], __fmul_rn(en.w, x));
                    }
                    wt[p] = __fadd_rn(wt[p], en.w);
                } else {
                    const float cw = __fmul_rn(en.w, window[dy * P + dx]);
                    for (int c = 0; c < C; ++c) {
                        const float x = __ldg(f + c * L.patch_dim + pos);
                        num[p][c] = __fadd_rn(num[p][c], __fmul_rn(cw, x));
                    }
                    wt[p] = __fadd_rn(wt[p], cw);
                }
            }
        }
        const bool done = s_done != 0;
        __syncthreads();
        if (done) break;
    }
    // ---- write the tile of this slot
    const size_t plane = static_cast<size_t>(L.width) * L.height;
    float* base = L.stack + static_cast<size_t>(slot) * (C + 1) * plane;
    for (int p = 0; p < pix_per_thread && p < kMaxPix; ++p) {
        const int local = tid + p * blockDim.x;
        if (local >= T * T) break;
        const int px = tx0 + local % T;
        const int py = ty0 + local / T;
        if (px >= L.width || py >= L.height) continue;
        const size_t i = static_cast<size_t>(py) * L.width + px;
        for (int c = 0; c < C; ++c) base[c * plane + i] = num[p][c];
        base[C * plane + i] = wt[p];
    }
}

__global__ void normalize_kernel(NormalizeLaunch L) {
    const size_t plane = static_cast<size_t>(L.width) * L.height;
    const int C = L.channels;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < plane;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        float num[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        float w = 0.0f;
        for (int k = 0; k < L.count; ++k) {
            const float* s = L.stacks[k] + static_cast<size_t>(L.slots[k]) * (C + 1) * plane;
            for (int c = 0; c < C; ++c) num[c] = __fadd_rn(num[c], s[c * plane + i]);
            w = __fadd_rn(w, s[C * plane + i]);
        }
        for (int c = 0; c < C; ++c)
            L.out[c * plane + i] = w > 0.0f ? __fdiv_rn(num[c], w) : L.source[c * plane + i];
    }
}

__global__ void pack_kernel(const float* stack, int width, int height, int channels, int slots, float* out) {
    const size_t plane = static_cast<size_t>(width) * height;
    const size_t total = plane * channels * slots * 2;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t pix = i % plane;
        const size_t rest = i / plane;
        const int is_weight = static_cast<int>(rest % 2);
        const int slot = static_cast<int>((rest / 2) % slots);
        const int c = static_cast<int>(rest / (2 * slots));
        const float* s = stack + static_cast<size_t>(slot) * (channels + 1) * plane;
        out[i] = is_weight ? s[channels * plane + pix] : s[c * plane + pix];
    }
}

__global__ void aggregate_stacks_kernel(AggregateLaunch L) {
    const size_t plane = static_cast<size_t>(L.width) * L.height;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < plane * L.channels;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(i / plane);
        const size_t pix = i - static_cast<size_t>(c) * plane;
        const size_t y = pix / L.width;
        const size_t x = pix - y * L.width;
        float num = 0.0f, w = 0.0f;
        for (int k = 0; k < L.count; ++k) {
            const float* s = L.stacks[k] + static_cast<size_t>(c) * L.slots * 2 * plane;
            const size_t row = static_cast<size_t>(L.slots_of[k]) * 2 * L.height + y;
            num = __fadd_rn(num, s[row * L.width + x]);
            w = __fadd_rn(w, s[(row + L.height) * L.width + x]);
        }
        L.out[i] = w > 0.0f ? __fdiv_rn(num, w) : L.source[i];
    }
}

}  // namespace

cudaError_t launch_aggregate_stacks(const AggregateLaunch& L, cudaStream_t stream) {
    const size_t total = static_cast<size_t>(L.width) * L.height * L.channels;
    const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, 148 * 16));
    aggregate_stacks_kernel<<<blocks, 256, 0, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_tiles(const TileLaunch& L, cudaStream_t stream) {
    if (L.tile * L.tile > kTileThreads * 4 || L.channels > 4) return cudaErrorInvalidValue;
    const dim3 grid(L.tiles_x, L.tiles_y, L.slots);
    const size_t smem = static_cast<size_t>(L.P) * L.P * sizeof(float);
    tile_kernel<<<grid, kTileThreads, smem, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_normalize(const NormalizeLaunch& L, cudaStream_t stream) {
    if (L.channels > 4 || L.count > kMaxContributors) return cudaErrorInvalidValue;
    const size_t plane = static_cast<size_t>(L.width) * L.height;
    const int blocks = static_cast<int>(std::min<size_t>((plane + 255) / 256, 148 * 16));
    normalize_kernel<<<blocks, 256, 0, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_pack_stack(const float* stack, int width, int height, int channels, int slots, float* out,
                              cudaStream_t stream) {
    const size_t total = static_cast<size_t>(width) * height * channels * slots * 2;
    const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, 148 * 16));
    pack_kernel<<<blocks, 256, 0, stream>>>(stack, width, height, channels, slots, out);
    return cudaGetLastError();
}

}  // namespace vnlbgpu
