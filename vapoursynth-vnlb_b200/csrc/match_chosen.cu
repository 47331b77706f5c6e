// Block matching for one anchor frame, chosen form: tensor-core distances on a
// short list, exact FP32 re-rank.
//
// The selected rows feed the same filter and aggregation as the plain form.
// What changes is how the candidates are scored:
//
//   1. approximate distance ||a||^2 + ||b||^2 - 2 a.b for every candidate, the
//      dot products on BF16 tensor cores (mma.sync m16n8k16, FP32
//      accumulation), the norms in FP32 from the FP32 samples;
//   2. the CPU's sequential selection (find_similar_patches,
//      core.cpp:1277-1359: the K-smallest front and the capped buffer) run on
//      the approximate distances, frame by frame in the CPU's candidate order;
//   3. the exact FP32 SSD, in the CPU's arithmetic order (the bits the plain
//      form computes), of every buffer entry a frame brings in, while that
//      frame is still staged;
//   4. select_similar_patches (core.cpp:1200-1243) on those exact distances:
//      the K smallest, the threshold max(tau, d_K), the entries within it,
//      closest first, at most the cap.
//
// The buffer is the plain form's whenever the approximate distances order the
// candidates as the exact ones do.  Step 4 keeps the rows sorted by
// (distance, candidate order); the CPU leaves the rows past the K-th in the
// order its heap replay produces, which only changes the order in which
// contributions are summed.
//
// Work decomposition.  One CTA takes a strip of up to 8 consecutive anchors
// of one grid row: rows 0-7 of each m16n8k16 tile are their reference patches
// (rows 8-15 are zero), K runs over the patch samples two patch rows per k16
// step, and the 8 columns of a tile are 8 consecutive candidate positions of
// one window row, shared by all anchors of the strip (results outside an
// anchor's window are dropped).  Every scheduled frame's search region is
// staged once in shared memory in FP32 (B fragments are converted to BF16 as
// they are staged; norms and the exact re-rank read the FP32 samples).  Each
// warp then takes one anchor through the selection of the frame.
#include <cuda_bf16.h>

#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr int kChosenThreads = 32 * kChosenWarps;
constexpr int kPatch = 8;  // the chosen matcher is built for 8 x 8 patches

__device__ __forceinline__ void mma_bf16_16816(float c[4], const unsigned a[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int NCH>  // k16 steps per patch: planes * kPatch / 2
__global__ void __launch_bounds__(kChosenThreads, 2) match_chosen_kernel(MatchLaunch L) {
    extern __shared__ __align__(16) float smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2;  // MMA group: fragment row / column
    const int t = lane & 3;
    constexpr int P = kPatch;
    const Strip strip = L.strips[blockIdx.x];
    const int planes_n = L.search_channels * L.Pt;
    const int kd = planes_n * P * P;
    const int rows = L.region_rows;
    const int rs = L.region_stride;
    const int plane = rows * rs;
    const int tiles_x = L.tiles_x;
    const int ncols = 8 * tiles_x;  // candidate columns covered by the tiles
    int yl, yh;
    spatial_range(strip.y, L.height, P, L.search_window, yl, yh);
    const int Wy = yh - yl + 1;
    const ChosenLayout lay = chosen_layout(planes_n, rows, rs, tiles_x, L.window_rows, L.window_cells, kd);
    float* region = smem + lay.region;
    __nv_bfloat16* ebf = reinterpret_cast<__nv_bfloat16*>(smem + lay.ebf);
    __nv_bfloat16* obf = reinterpret_cast<__nv_bfloat16*>(smem + lay.obf);
    float* nb = smem + lay.nb;
    float* dist = smem + lay.dist;
    float* rowsum = dist;  // consumed before the distances are written
    __nv_bfloat16* abf = reinterpret_cast<__nv_bfloat16*>(smem + lay.abf);
    float* reff = smem + lay.reff;
    float* na = smem + lay.na;
    int* win_lo = reinterpret_cast<int*>(smem + lay.win);  // window columns relative to the strip origin
    int* win_wx = win_lo + kChosenAnchors;
    const int count = strip.count;
    const int rx0 = strip.region_x;  // first candidate column of the strip

    if (threadIdx.x < kChosenAnchors) {
        const int m = threadIdx.x;
        int xl = 0, xh = -1;
        if (m < count) {
            const int2 a = L.anchors[strip.first + m];
            spatial_range(a.x, L.width, P, L.search_window, xl, xh);
        }
        win_lo[m] = xl - rx0;
        win_wx[m] = xh - xl + 1;
    }
    unsigned afrag[NCH][2];  // rows g of the tile (rows g + 8 are zero)
    int my_lo = 0, my_wx = 0;
    float my_na = 0.0f;
    // selection state of this warp's anchor (the plain matcher's WarpSelect)
    const int K = L.K;
    struct {
        int count, cap, worst_idx, top_count;
        float worst, top_front;
    } s;
    s.count = 0;
    s.cap = min(L.soft_cap, L.search_window * L.search_window * L.schedule_len);
    s.worst_idx = 0;
    s.worst = kInf;
    s.top_count = 0;
    s.top_front = kInf;
    unsigned reg_d = 0u, reg_top = 0u;  // bits of non-negative distances
    int reg_id = 0;
    float reg_exact = 0.0f;

    for (int k = 0; k < L.schedule_len; ++k) {
        const int frame = L.schedule[k];
        __syncthreads();
        // Stage frame k's planes (channel, t) in FP32.
        for (int q = 0; q < planes_n; ++q) {
            const int c = q / L.Pt;
            const int tt = q % L.Pt;
            const float* src = L.video + (static_cast<size_t>(frame + tt) * L.channels + c) * L.height *
                                             static_cast<size_t>(L.width);
            for (int r = warp; r < rows; r += kChosenWarps) {
                const int gy = yl + r;
                const float* srow = src + static_cast<size_t>(gy) * L.width;
                for (int cx = lane; cx < rs; cx += 32) {
                    const int gx = rx0 + cx;
                    const float v = gx < L.width && gy < L.height ? __ldg(srow + gx) : 0.0f;
                    const int i = q * plane + r * rs + cx;
                    region[i] = v;
                    const __nv_bfloat16 b = __float2bfloat16_rn(v);
                    ebf[i] = b;
                    if (cx > 0) obf[i - 1] = b;
                }
            }
        }
        __syncthreads();
        if (k == 0) {
            // reference patches (the anchor frame is scheduled first)
            for (int i = threadIdx.x; i < kChosenAnchors * kd; i += kChosenThreads) {
                const int m = i / kd;
                const int e = i - m * kd;
                float v = 0.0f;
                if (m < count) {
                    const int2 a = L.anchors[strip.first + m];
                    const int q = e / (P * P);
                    const int rem = e - q * P * P;
                    const int py = rem / P;
                    const int px = rem - py * P;
                    v = region[q * plane + (a.y - yl + py) * rs + (a.x - rx0 + px)];
                }
                reff[i] = v;
                abf[i] = __float2bfloat16_rn(v);
            }
        }
        // row sums of squares over P columns, all planes (candidate norms)
        for (int r = warp; r < rows; r += kChosenWarps)
            for (int cx = lane; cx < ncols; cx += 32) {
                float acc = 0.0f;
                for (int q = 0; q < planes_n; ++q) {
                    const float* row = region + q * plane + r * rs + cx;
#pragma unroll
                    for (int ii = 0; ii < P; ++ii) acc = fmaf(row[ii], row[ii], acc);
                }
                rowsum[r * ncols + cx] = acc;
            }
        __syncthreads();
        if (k == 0) {
            if (warp < kChosenAnchors) {
                float acc = 0.0f;
                for (int e = lane; e < kd; e += 32) acc = fmaf(reff[warp * kd + e], reff[warp * kd + e], acc);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                if (lane == 0) na[warp] = acc;
            }
            const unsigned* a32 = reinterpret_cast<const unsigned*>(abf);
#pragma unroll
            for (int cq = 0; cq < NCH; ++cq) {
                afrag[cq][0] = a32[(g * kd + 16 * cq + 2 * t) >> 1];
                afrag[cq][1] = a32[(g * kd + 16 * cq + 2 * t + 8) >> 1];
            }
            my_lo = g < count ? win_lo[g] : 1 << 20;
            my_wx = g < count ? win_wx[g] : 0;
        }
        for (int y = warp; y < Wy; y += kChosenWarps)
            for (int cx = lane; cx < ncols; cx += 32) {
                float acc = 0.0f;
#pragma unroll
                for (int r = 0; r < P; ++r) acc += rowsum[(y + r) * ncols + cx];
                nb[y * ncols + cx] = acc;
            }
        __syncthreads();
        if (k == 0) my_na = na[g];
        // Approximate distances: tile = 8 anchors (rows g) x 8 candidates of one row.
        {
            // lane pairs (columns c, c + 1) as one aligned 32-bit load: from the
            // even copy for even c, from the shifted copy (index c - 1) for odd c
            const unsigned* src32 = reinterpret_cast<const unsigned*>((g & 1) ? obf : ebf);
            int y = 0, j = warp;  // tile (y, j) = y * tiles_x + j, strided by the warp count
            while (j >= tiles_x && y < Wy) {
                j -= tiles_x;
                ++y;
            }
            for (; y < Wy; j += kChosenWarps) {
                while (j >= tiles_x) {
                    j -= tiles_x;
                    ++y;
                }
                if (y >= Wy) break;
                const int base = (y * rs + 8 * j + g + 2 * t - (g & 1)) >> 1;  // 32-bit word of the pair
                float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int cq = 0; cq < NCH; ++cq) {
                    const int w = base + (((cq >> 2) * plane + 2 * (cq & 3) * rs) >> 1);
                    const unsigned a[4] = {afrag[cq][0], 0u, afrag[cq][1], 0u};
                    mma_bf16_16816(c, a, src32[w], src32[w + (rs >> 1)]);
                }
                // this lane's results: anchor g, candidate columns 8j + 2t and + 1
                const int cx = 8 * j + 2 * t - my_lo;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (cx + h < 0 || cx + h >= my_wx) continue;
                    dist[g * L.window_cells + y * my_wx + cx + h] =
                        my_na + nb[y * ncols + 8 * j + 2 * t + h] - 2.0f * c[h];
                }
            }
        }
        __syncthreads();
        // The CPU's sequential selection over frame k (raster order) on the
        // approximate distances: the K-smallest front and the capped buffer,
        // buffer slot i in lane i (the plain matcher's register replay).
        if (warp < count) {
            const int m = warp;
            const int cells = win_wx[m] * Wy;
            const float* dk = dist + m * L.window_cells;
            for (int base = 0; base < cells; base += 32) {
                const int idx = base + lane;
                // approximate distances can dip below zero; clamp so that they
                // order like their bit patterns
                const float mine = idx < cells ? fmaxf(dk[idx], 0.0f) : kInf;
                float limit = s.top_count >= K ? std_max(L.tau, s.top_front) : kInf;
                if (s.count >= s.cap) limit = std_min(limit, s.worst);
                unsigned pass = __ballot_sync(0xffffffffu, idx < cells && mine <= limit);
                while (pass) {
                    const int src_lane = __ffs(pass) - 1;
                    pass &= pass - 1;
                    const float d = __shfl_sync(0xffffffffu, mine, src_lane);
                    limit = s.top_count >= K ? std_max(L.tau, s.top_front) : kInf;
                    if (s.count >= s.cap) limit = std_min(limit, s.worst);
                    if (!(d <= limit)) continue;
                    const int id = (k << 20) | (base + src_lane);
                    if (s.count < s.cap) {
                        if (lane == s.count) {
                            reg_d = __float_as_uint(d);
                            reg_id = id;
                        }
                        s.count++;
                        if (s.count == s.cap) {
                            const unsigned w = __reduce_max_sync(0xffffffffu, reg_d);
                            s.worst_idx = __ffs(__ballot_sync(0xffffffffu, reg_d == w)) - 1;
                            s.worst = __uint_as_float(w);
                        }
                    } else if (d < s.worst) {
                        if (lane == s.worst_idx) {
                            reg_d = __float_as_uint(d);
                            reg_id = id;
                        }
                        const unsigned w = __reduce_max_sync(0xffffffffu, reg_d);
                        s.worst_idx = __ffs(__ballot_sync(0xffffffffu, reg_d == w)) - 1;
                        s.worst = __uint_as_float(w);
                    }
                    if (s.top_count < K) {
                        if (lane == s.top_count) reg_top = __float_as_uint(d);
                        s.top_count++;
                        if (s.top_count == K) s.top_front = __uint_as_float(__reduce_max_sync(0xffffffffu, reg_top));
                    } else if (d < s.top_front) {
                        const unsigned f = __float_as_uint(s.top_front);
                        const int owner = __ffs(__ballot_sync(0xffffffffu, lane < K && reg_top == f)) - 1;
                        if (lane == owner) reg_top = __float_as_uint(d);
                        s.top_front = __uint_as_float(__reduce_max_sync(0xffffffffu, reg_top));
                    }
                }
            }
            // exact FP32 distance of the buffer entries frame k brought in,
            // while frame k is staged: each lane re-ranks its own slot
            if (lane < s.count && (reg_id >> 20) == k) {
                const int i = reg_id & 0xfffff;
                const int Wx = win_wx[m];
                const int cy = i / Wx;
                const int col = win_lo[m] + (i - cy * Wx);
                const float* rf = reff + m * kd;
                float d = 0.0f;
                for (int q = 0; q < planes_n; ++q) {
#pragma unroll
                    for (int r = 0; r < P; ++r) {
                        const float* rr = rf + q * P * P + r * P;
                        const float* cr = region + q * plane + (cy + r) * rs + col;
                        float2 a2[4], b2[4];
#pragma unroll
                        for (int ii = 0; ii < 4; ++ii) {
                            a2[ii] = make_float2(rr[2 * ii], rr[2 * ii + 1]);
                            b2[ii] = make_float2(cr[2 * ii], cr[2 * ii + 1]);
                        }
                        d = row_ssd8_x2(d, a2, b2);
                    }
                }
                reg_exact = d;
            }
        }
    }
    if (warp >= count) return;

    // select_similar_patches on the exact distances of the buffer: the K
    // smallest, the threshold max(tau, d_K), the entries within it, closest
    // first (ties by candidate order), at most the cap
    const int m = warp;
    const int gi = strip.first + m;
    const int2 anchor = L.anchors[gi];
    const int Wx = win_wx[m];
    const int xl = win_lo[m] + rx0;
    float* sd = dist + m * L.window_cells;  // sorted buffer (free now)
    int* si = reinterpret_cast<int*>(sd + 32);
    const int n = s.count;
    int S;
    if (K <= 1) {
        // similar <= 1: the anchor itself (core.cpp:1253-1257)
        if (lane == 0) {
            sd[0] = 0.0f;
            si[0] = -1;
        }
        S = 1;
    } else {
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const float dj = __shfl_sync(0xffffffffu, reg_exact, j);
            const int ij = __shfl_sync(0xffffffffu, reg_id, j);
            rank += (dj < reg_exact || (dj == reg_exact && ij < reg_id)) ? 1 : 0;
        }
        if (lane < n) {
            sd[rank] = reg_exact;
            si[rank] = reg_id;
        }
        __syncwarp();
        const int selected = min(K, n);
        const float threshold = std_max(L.tau, sd[selected - 1]);
        const int within = __popc(__ballot_sync(0xffffffffu, lane < n && sd[lane] <= threshold));
        S = min(within, min(L.soft_cap, n));
    }
    __syncwarp();
    MatchRow* rows_out = L.rows + static_cast<size_t>(gi) * L.max_rows;
    for (int i = lane; i < S; i += 32) {
        const int id = si[i];
        MatchRow r;
        r.distance = sd[i];
        if (id < 0) {
            r.x = anchor.x;
            r.y = anchor.y;
            r.frame = L.anchor_frame;
        } else {
            const int kk = id >> 20;
            const int cell = id & 0xfffff;
            const int cy = cell / Wx;
            r.x = xl + (cell - cy * Wx);
            r.y = yl + cy;
            r.frame = L.schedule[kk];
        }
        rows_out[i] = r;
    }
    if (lane == 0) L.row_counts[gi] = S;
    __syncwarp();
    // Paste-mask victims (apply_frame_paste_mask, core.cpp:980-1008), as in
    // the plain matcher.
    int* vict = L.victims + static_cast<size_t>(gi) * L.victim_stride;
    int nvict = 0;
    for (int i0 = 0; i0 < S; i0 += 32) {
        const int i = i0 + lane;
        int found[5];
        int nf = 0;
        if (i < S) {
            const MatchRow r = rows_out[i];
            if (r.frame == L.anchor_frame) {
                const int px[5] = {r.x, r.x, r.x, r.x - 1, r.x + 1};
                const int py[5] = {r.y, r.y - 1, r.y + 1, r.y, r.y};
                const bool use[5] = {true, r.y > 2 * P, r.y < L.height - 2 * P, r.x > 2 * P, r.x < L.width - 2 * P};
#pragma unroll
                for (int e = 0; e < 5; ++e) {
                    if (!use[e] || px[e] < 0 || px[e] >= L.width || py[e] < 0 || py[e] >= L.height) continue;
                    const int j = L.anchor_map[static_cast<size_t>(py[e]) * L.width + px[e]];
                    if (j > gi) found[nf++] = j;
                }
            }
        }
        int prefix = nf;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, prefix, o);
            if (lane >= o) prefix += v;
        }
        const int total = __shfl_sync(0xffffffffu, prefix, 31);
        const int start = nvict + prefix - nf;
        for (int e = 0; e < nf; ++e)
            if (start + e < L.victim_stride) vict[start + e] = found[e];
        nvict += total;
    }
    if (lane == 0) L.victim_counts[gi] = min(nvict, L.victim_stride);
}

}  // namespace

bool chosen_match_supported(int P, int planes_n) {
    const int nch = planes_n * P / 2;
    return P == kPatch && (nch == 4 || nch == 8 || nch == 12);
}

size_t chosen_match_shared_bytes(const MatchLaunch& L) {
    const int planes_n = L.search_channels * L.Pt;
    const ChosenLayout lay = chosen_layout(planes_n, L.region_rows, L.region_stride, L.tiles_x, L.window_rows,
                                           L.window_cells, planes_n * L.P * L.P);
    return static_cast<size_t>(lay.floats) * sizeof(float);
}

cudaError_t launch_match_chosen(const MatchLaunch& L, int strips, cudaStream_t stream) {
    if (strips <= 0) return cudaSuccess;
    const int planes_n = L.search_channels * L.Pt;
    if (!chosen_match_supported(L.P, planes_n)) return cudaErrorInvalidValue;
    const size_t smem = chosen_match_shared_bytes(L);
    cudaError_t err = cudaSuccess;
    auto launch = [&](auto kernel) {
        err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (err != cudaSuccess) return;
        kernel<<<strips, kChosenThreads, smem, stream>>>(L);
        err = cudaGetLastError();
    };
    switch (planes_n * L.P / 2) {
        case 4: launch(match_chosen_kernel<4>); break;
        case 8: launch(match_chosen_kernel<8>); break;
        default: launch(match_chosen_kernel<12>); break;
    }
    return err;
}

}  // namespace vnlbgpu
