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

constexpr int kTileThreads = kTile * kTile;
constexpr int kTileWarps = kTileThreads / 32;
constexpr int kMaxGridRows = 64;  // grid rows per collection round

struct Entry {
    int r;     // global row
    int xyt;   // x | y << 14 | layer (tile_kernel) or slot (tile_slots_kernel) << 28
    float w;   // row weight
};

// One CTA per (16x16 tile, slot), one pixel per thread.  The rows that can
// cover the tile form one contiguous row range per grid row in reach (reach
// tables, built per grid); their concatenation is in increasing global row
// order.  All threads test 256 rows at a time, an ordered block compaction
// keeps the covering ones in that order, and every thread applies them to
// its pixel before the next chunk: the CPU's accumulation order, with no
// atomics and one write per stack value.
__global__ void __launch_bounds__(kTileThreads) tile_kernel(TileLaunch L) {
    __shared__ Entry entries[kTileThreads];
    __shared__ int s_rbeg[kMaxGridRows];
    __shared__ int s_rpre[kMaxGridRows + 1];
    __shared__ int s_warp[kTileWarps + 1];
    extern __shared__ float window[];

    const int tx = blockIdx.x, ty = blockIdx.y, slot = blockIdx.z;
    const int tx0 = tx * kTile, ty0 = ty * kTile;
    const int P = L.P;
    const int C = L.channels;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    for (int i = tid; i < P * P; i += blockDim.x) window[i] = L.window[i];

    const int px = tx0 + (tid % kTile);
    const int py = ty0 + (tid / kTile);
    float num[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    float wt = 0.0f;
    const int fused_cols = (P == kLanes || P == 2 * kLanes) ? P : (P / kLanes) * kLanes;
    const int2 grid_rows = L.tile_grid_rows[ty];

    for (int k0 = grid_rows.x; k0 < grid_rows.y; k0 += kMaxGridRows) {
        const int nk = min(kMaxGridRows, grid_rows.y - k0);
        __syncthreads();
        if (tid < nk) {
            const int2 anchors = L.tile_anchors[static_cast<size_t>(k0 + tid) * L.tiles_x + tx];
            const int rb = L.row_offset[L.active_prefix[anchors.x]];
            const int re = L.row_offset[L.active_prefix[anchors.y]];
            s_rbeg[tid] = rb;
            s_rpre[tid + 1] = re - rb;
        }
        __syncthreads();
        if (tid == 0) {
            s_rpre[0] = 0;
            for (int k = 1; k <= nk; ++k) s_rpre[k] += s_rpre[k - 1];
        }
        __syncthreads();
        const int total = s_rpre[nk];
        for (int chunk = 0; chunk < total; chunk += kTileThreads) {
            // test one virtual row per thread
            const int vrow = chunk + tid;
            bool hit = false;
            Entry en;
            if (vrow < total) {
                int lo = 0, hi = nk - 1;  // last k with s_rpre[k] <= vrow
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (s_rpre[mid] <= vrow) lo = mid;
                    else hi = mid - 1;
                }
                const int r = s_rbeg[lo] + (vrow - s_rpre[lo]);
                const MatchRow m = L.row_info[r];
                if (m.x <= tx0 + kTile - 1 && m.x + P - 1 >= tx0 && m.y <= ty0 + kTile - 1 && m.y + P - 1 >= ty0) {
                    const int t = slot - L.search_bwd + L.anchor_frame - m.frame;
                    if (t >= 0 && t < L.Pt) {
                        hit = true;
                        en.r = r;
                        en.xyt = m.x | (m.y << 14) | (t << 28);
                        en.w = L.weights[r];
                    }
                }
            }
            // ordered block compaction
            const unsigned ballot = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) s_warp[warp + 1] = __popc(ballot);
            __syncthreads();
            if (tid == 0) {
                s_warp[0] = 0;
                for (int w = 1; w <= kTileWarps; ++w) s_warp[w] += s_warp[w - 1];
            }
            __syncthreads();
            if (hit) entries[s_warp[warp] + __popc(ballot & ((1u << lane) - 1u))] = en;
            const int n = s_warp[kTileWarps];
            __syncthreads();
            // apply, in order, to this thread's pixel
            for (int e = 0; e < n; ++e) {
                const Entry x = entries[e];
                const unsigned dx = static_cast<unsigned>(px - (x.xyt & 0x3fff));
                const unsigned dy = static_cast<unsigned>(py - ((x.xyt >> 14) & 0x3fff));
                if (dx >= static_cast<unsigned>(P) || dy >= static_cast<unsigned>(P)) continue;
                const int t = x.xyt >> 28;
                const int pos = (t * P + static_cast<int>(dy)) * P + static_cast<int>(dx);
                const float* f = L.filtered + static_cast<size_t>(x.r) * L.dim + pos;
                if (L.coupled && !L.windowed) {
                    const bool fused = static_cast<int>(dx) < fused_cols;
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        if (c >= C) break;
                        const float v = __ldg(f + c * L.patch_dim);
                        num[c] = fused ? __fmaf_rn(x.w, v, num[c]) : __fadd_rn(num[c], __fmul_rn(x.w, v));
                    }
                    wt = __fadd_rn(wt, x.w);
                } else {
                    const float cw = __fmul_rn(x.w, window[dy * P + dx]);
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        if (c >= C) break;
                        const float v = __ldg(f + c * L.patch_dim);
                        num[c] = __fadd_rn(num[c], __fmul_rn(cw, v));
                    }
                    wt = __fadd_rn(wt, cw);
                }
            }
            __syncthreads();
        }
    }
    // write this slot's tile: every pixel, so the stack needs no clearing
    if (px < L.width && py < L.height) {
        const size_t plane = static_cast<size_t>(L.width) * L.height;
        float* base = L.stack + static_cast<size_t>(slot) * (C + 1) * plane + static_cast<size_t>(py) * L.width + px;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (c < C) base[c * plane] = num[c];
        base[C * plane] = wt;
    }
}

// All slots in one scan: a covering row's temporal layer t lands in slot
// s0 + t, s0 its frame's offset in the window, so one CTA per tile scans the
// candidate rows once for all slots (at most kMaxTileSlots) and keeps one
// accumulator set per slot.  Each (pixel, slot) still sees its rows in
// increasing global row order: the same sums as tile_kernel.  kLayers: the
// patch spans more than one frame (patch_time > 1).
constexpr int kMaxTileSlots = 4;

template <bool kLayers>
__global__ void __launch_bounds__(kTileThreads) tile_slots_kernel(TileLaunch L) {
    __shared__ Entry entries[kTileThreads];
    __shared__ int s_rbeg[kMaxGridRows];
    __shared__ int s_rpre[kMaxGridRows + 1];
    __shared__ int s_warp[kTileWarps + 1];
    extern __shared__ float window[];

    const int tx = blockIdx.x, ty = blockIdx.y;
    const int tx0 = tx * kTile, ty0 = ty * kTile;
    const int P = L.P;
    const int C = L.channels;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    for (int i = tid; i < P * P; i += blockDim.x) window[i] = L.window[i];

    const int px = tx0 + (tid % kTile);
    const int py = ty0 + (tid / kTile);
    float num[kMaxTileSlots][4];
    float wt[kMaxTileSlots];
#pragma unroll
    for (int s = 0; s < kMaxTileSlots; ++s) {
        wt[s] = 0.0f;
#pragma unroll
        for (int c = 0; c < 4; ++c) num[s][c] = 0.0f;
    }
    const int fused_cols = (P == kLanes || P == 2 * kLanes) ? P : (P / kLanes) * kLanes;
    const int2 grid_rows = L.tile_grid_rows[ty];
    const int slot_base = L.search_bwd - L.anchor_frame;  // slot = frame + slot_base

    for (int k0 = grid_rows.x; k0 < grid_rows.y; k0 += kMaxGridRows) {
        const int nk = min(kMaxGridRows, grid_rows.y - k0);
        __syncthreads();
        if (tid < nk) {
            const int2 anchors = L.tile_anchors[static_cast<size_t>(k0 + tid) * L.tiles_x + tx];
            const int rb = L.row_offset[L.active_prefix[anchors.x]];
            const int re = L.row_offset[L.active_prefix[anchors.y]];
            s_rbeg[tid] = rb;
            s_rpre[tid + 1] = re - rb;
        }
        __syncthreads();
        if (tid == 0) {
            s_rpre[0] = 0;
            for (int k = 1; k <= nk; ++k) s_rpre[k] += s_rpre[k - 1];
        }
        __syncthreads();
        const int total = s_rpre[nk];
        for (int chunk = 0; chunk < total; chunk += kTileThreads) {
            const int vrow = chunk + tid;
            bool hit = false;
            Entry en;
            if (vrow < total) {
                int lo = 0, hi = nk - 1;  // last k with s_rpre[k] <= vrow
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (s_rpre[mid] <= vrow) lo = mid;
                    else hi = mid - 1;
                }
                const int r = s_rbeg[lo] + (vrow - s_rpre[lo]);
                const MatchRow m = L.row_info[r];
                if (m.x <= tx0 + kTile - 1 && m.x + P - 1 >= tx0 && m.y <= ty0 + kTile - 1 && m.y + P - 1 >= ty0) {
                    // slot of layer 0; with several layers it may lie before the
                    // window (the temporal windows shift at the clip's ends)
                    // while a later layer lands in it, so it is stored + 8
                    const int slot = m.frame + slot_base;
                    if (slot >= (kLayers ? 1 - L.Pt : 0) && slot < L.slots) {
                        hit = true;
                        en.r = r;
                        en.xyt = static_cast<int>(static_cast<unsigned>(m.x) | (static_cast<unsigned>(m.y) << 14) |
                                                  (static_cast<unsigned>(kLayers ? slot + 8 : slot) << 28));
                        en.w = L.weights[r];
                    }
                }
            }
            const unsigned ballot = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) s_warp[warp + 1] = __popc(ballot);
            __syncthreads();
            if (tid == 0) {
                s_warp[0] = 0;
                for (int w = 1; w <= kTileWarps; ++w) s_warp[w] += s_warp[w - 1];
            }
            __syncthreads();
            if (hit) entries[s_warp[warp] + __popc(ballot & ((1u << lane) - 1u))] = en;
            const int n = s_warp[kTileWarps];
            __syncthreads();
            for (int e = 0; e < n; ++e) {
                const Entry x = entries[e];
                const unsigned dx = static_cast<unsigned>(px - (x.xyt & 0x3fff));
                const unsigned dy = static_cast<unsigned>(py - ((x.xyt >> 14) & 0x3fff));
                if (dx >= static_cast<unsigned>(P) || dy >= static_cast<unsigned>(P)) continue;
                const int slot0 = static_cast<int>(static_cast<unsigned>(x.xyt) >> 28) - (kLayers ? 8 : 0);
                const int t_end = kLayers ? min(L.Pt, L.slots - slot0) : 1;
                for (int t = kLayers ? max(0, -slot0) : 0; t < t_end; ++t) {
                    const int slot = slot0 + t;
                    const int pos = (t * P + static_cast<int>(dy)) * P + static_cast<int>(dx);
                    const float* f = L.filtered + static_cast<size_t>(x.r) * L.dim + pos;
                    float val[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) val[c] = c < C ? __ldg(f + c * L.patch_dim) : 0.0f;
                    if (L.coupled && !L.windowed) {
                        const bool fused = static_cast<int>(dx) < fused_cols;
#pragma unroll
                        for (int s = 0; s < kMaxTileSlots; ++s) {
                            if (s != slot) continue;
#pragma unroll
                            for (int c = 0; c < 4; ++c) {
                                if (c >= C) break;
                                num[s][c] = fused ? __fmaf_rn(x.w, val[c], num[s][c])
                                                  : __fadd_rn(num[s][c], __fmul_rn(x.w, val[c]));
                            }
                            wt[s] = __fadd_rn(wt[s], x.w);
                        }
                    } else {
                        const float cw = __fmul_rn(x.w, window[dy * P + dx]);
#pragma unroll
                        for (int s = 0; s < kMaxTileSlots; ++s) {
                            if (s != slot) continue;
#pragma unroll
                            for (int c = 0; c < 4; ++c) {
                                if (c >= C) break;
                                num[s][c] = __fadd_rn(num[s][c], __fmul_rn(cw, val[c]));
                            }
                            wt[s] = __fadd_rn(wt[s], cw);
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    if (px < L.width && py < L.height) {
        const size_t plane = static_cast<size_t>(L.width) * L.height;
#pragma unroll
        for (int s = 0; s < kMaxTileSlots; ++s) {
            if (s >= L.slots) break;
            float* base = L.stack + static_cast<size_t>(s) * (C + 1) * plane + static_cast<size_t>(py) * L.width + px;
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (c < C) base[c * plane] = num[s][c];
            base[C * plane] = wt[s];
        }
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
            if (L.packed[k] == 4) {  // [H][W][C+1] with C = 3: one 16-byte load
                const float4 v = __ldg(reinterpret_cast<const float4*>(s) + i);
                num[0] = __fadd_rn(num[0], v.x);
                num[1] = __fadd_rn(num[1], v.y);
                num[2] = __fadd_rn(num[2], v.z);
                w = __fadd_rn(w, v.w);
            } else if (L.packed[k] == 2) {  // C = 1
                const float2 v = __ldg(reinterpret_cast<const float2*>(s) + i);
                num[0] = __fadd_rn(num[0], v.x);
                w = __fadd_rn(w, v.y);
            } else {
                for (int c = 0; c < C; ++c) num[c] = __fadd_rn(num[c], s[c * plane + i]);
                w = __fadd_rn(w, s[C * plane + i]);
            }
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

// The same packing from a pixel-interleaved stack [slots][H][W][kPack]
// (kPack = C+1 = 4 or 2): one thread per pixel and slot, one vector load,
// 2C coalesced stores.
template <int kPack>
__global__ void pack_interleaved_kernel(const float* stack, int width, int height, int slots, float* out) {
    constexpr int C = kPack - 1;
    const size_t plane = static_cast<size_t>(width) * height;
    const size_t total = plane * slots;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int slot = static_cast<int>(i / plane);
        const size_t pix = i - static_cast<size_t>(slot) * plane;
        const float* s = stack + (static_cast<size_t>(slot) * plane + pix) * kPack;
        float v[kPack];
        if constexpr (kPack == 4) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(s));
            v[0] = q.x;
            v[1] = q.y;
            v[2] = q.z;
            v[3] = q.w;
        } else {
            const float2 q = __ldg(reinterpret_cast<const float2*>(s));
            v[0] = q.x;
            v[1] = q.y;
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const size_t row = static_cast<size_t>(c * slots + slot) * 2;
            out[row * plane + pix] = v[c];
            out[(row + 1) * plane + pix] = v[C];
        }
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
    if (L.channels > 4 || L.width >= (1 << 14) || L.height >= (1 << 14) || L.Pt > 7) return cudaErrorInvalidValue;
    const size_t smem = static_cast<size_t>(L.P) * L.P * sizeof(float);
    if (L.slots <= kMaxTileSlots) {
        if (L.Pt == 1) tile_slots_kernel<false><<<dim3(L.tiles_x, L.tiles_y, 1), kTileThreads, smem, stream>>>(L);
        else tile_slots_kernel<true><<<dim3(L.tiles_x, L.tiles_y, 1), kTileThreads, smem, stream>>>(L);
    } else {
        const dim3 grid(L.tiles_x, L.tiles_y, L.slots);
        tile_kernel<<<grid, kTileThreads, smem, stream>>>(L);
    }
    return cudaGetLastError();
}

cudaError_t launch_normalize(const NormalizeLaunch& L, cudaStream_t stream) {
    if (L.channels > 4 || L.count > kMaxContributors) return cudaErrorInvalidValue;
    for (int k = 0; k < L.count; ++k) {
        // the vector layouts hold C = 3 (16-byte pixels) or C = 1 (8-byte pixels)
        const int p = L.packed[k];
        if (p != 0 && !(p == L.channels + 1 && (p == 2 || p == 4) &&
                        reinterpret_cast<uintptr_t>(L.stacks[k]) % (p * sizeof(float)) == 0))
            return cudaErrorInvalidValue;
    }
    const size_t plane = static_cast<size_t>(L.width) * L.height;
    const int blocks = static_cast<int>(std::min<size_t>((plane + 255) / 256, 148 * 16));
    normalize_kernel<<<blocks, 256, 0, stream>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_pack_stack(const float* stack, int packed, int width, int height, int channels, int slots,
                              float* out, cudaStream_t stream) {
    if (packed != 0 && !(packed == channels + 1 && (packed == 2 || packed == 4) &&
                         reinterpret_cast<uintptr_t>(stack) % (packed * sizeof(float)) == 0))
        return cudaErrorInvalidValue;
    if (packed != 0) {
        const size_t pixels = static_cast<size_t>(width) * height * slots;
        const int blocks = static_cast<int>(std::min<size_t>((pixels + 255) / 256, 148 * 16));
        if (packed == 4) pack_interleaved_kernel<4><<<blocks, 256, 0, stream>>>(stack, width, height, slots, out);
        else pack_interleaved_kernel<2><<<blocks, 256, 0, stream>>>(stack, width, height, slots, out);
        return cudaGetLastError();
    }
    const size_t total = static_cast<size_t>(width) * height * channels * slots * 2;
    const int blocks = static_cast<int>(std::min<size_t>((total + 255) / 256, 148 * 16));
    pack_kernel<<<blocks, 256, 0, stream>>>(stack, width, height, channels, slots, out);
    return cudaGetLastError();
}

}  // namespace vnlbgpu
