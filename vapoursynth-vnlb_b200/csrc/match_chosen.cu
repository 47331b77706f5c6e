// Block matching for one anchor frame, chosen form: tensor-core distances on a
// short list, exact FP32 re-rank.
//
// The selected rows feed the same filter and aggregation as the plain form.
// What changes is how the candidates are scored:
//
//   1. approximate distance ||a||^2 + ||b||^2 - 2 a.b for every candidate, the
//      dot products on BF16 tensor cores (mma.sync m16n8k16, FP32
//      accumulation), the norms in FP32 from the FP32 samples;
//   2. per scheduled frame and anchor, the `shortlist` smallest approximate
//      distances (a bisection on the value, ties broken by candidate order);
//   3. their exact FP32 SSD in the CPU's arithmetic order (the same bits the
//      plain form computes for those candidates);
//   4. select_similar_patches (core.cpp:1200-1243) on the exact distances of
//      the pooled short lists: the K smallest, the threshold max(tau, d_K),
//      the rows within it closest first, at most the cap.
//
// Step 4 keeps the rows sorted by (distance, candidate order); the CPU leaves
// the rows past the K-th in the order its heap replay produces, which only
// changes the order in which equal-weight contributions are summed.
//
// Work decomposition.  One CTA takes a strip of up to 16 consecutive anchors
// of one grid row: the 16 rows of the MMA are the 16 reference patches (K =
// patch samples, two patch rows per k16 step), the 8 columns of an MMA tile
// are 8 consecutive candidate positions of one window row.  Every scheduled
// frame's search region is staged once in shared memory as FP32 (norms and
// exact re-rank) and as BF16 twice -- as loaded, and shifted left by one
// column -- so that each lane's pair of B-fragment samples is one aligned
// 32-bit load whatever the parity of its candidate column.  The candidate
// columns of the strip are shared by all its anchors; results outside an
// anchor's window are dropped.
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

__device__ __forceinline__ float warp_min_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <int NCH>  // k16 steps per patch: planes * kPatch / 2
__global__ void __launch_bounds__(kChosenThreads, 1) match_chosen_kernel(MatchLaunch L) {
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
    const ChosenLayout lay = chosen_layout(planes_n, rows, rs, tiles_x, L.window_rows, L.window_cells, kd, L.pool_cap);
    float* region = smem + lay.region;
    __nv_bfloat16* ebf = reinterpret_cast<__nv_bfloat16*>(smem + lay.ebf);
    __nv_bfloat16* obf = reinterpret_cast<__nv_bfloat16*>(smem + lay.obf);
    float* nb = smem + lay.nb;
    float* dist = smem + lay.dist;
    float* rowsum = dist;  // consumed before the distances are written
    __nv_bfloat16* abf = reinterpret_cast<__nv_bfloat16*>(smem + lay.abf);
    float* reff = smem + lay.reff;
    float* na = smem + lay.na;
    int* win_xl = reinterpret_cast<int*>(smem + lay.win);
    int* win_wx = win_xl + kChosenAnchors;
    float* pool_d = smem + lay.pool_d;
    int* pool_i = reinterpret_cast<int*>(smem + lay.pool_i);
    int* pool_n = reinterpret_cast<int*>(smem + lay.pool_n);
    const int count = strip.count;
    const int rx0 = strip.region_x;  // first candidate column of the strip

    if (threadIdx.x < kChosenAnchors) {
        const int m = threadIdx.x;
        int xl = 0, xh = -1;
        if (m < count) {
            const int2 a = L.anchors[strip.first + m];
            spatial_range(a.x, L.width, P, L.search_window, xl, xh);
        }
        win_xl[m] = xl;
        win_wx[m] = xh - xl + 1;
        pool_n[m] = 0;
    }
    unsigned afrag[NCH][4];
    const unsigned* e32 = reinterpret_cast<const unsigned*>(ebf);
    const unsigned* o32 = reinterpret_cast<const unsigned*>(obf);

    for (int k = 0; k < L.schedule_len; ++k) {
        const int frame = L.schedule[k];
        __syncthreads();
        // Stage frame k's planes (channel, t): FP32, BF16, BF16 shifted by one.
        for (int q = 0; q < planes_n; ++q) {
            const int c = q / L.Pt;
            const int tt = q % L.Pt;
            const float* src = L.video + (static_cast<size_t>(frame + tt) * L.channels + c) * L.height *
                                             static_cast<size_t>(L.width);
            for (int i = threadIdx.x; i < rows * rs; i += kChosenThreads) {
                const int r = i / rs;
                const int cx = i - r * rs;
                const int gx = rx0 + cx;
                const int gy = yl + r;
                float v = 0.0f;
                if (gx < L.width && gy < L.height) v = __ldg(src + static_cast<size_t>(gy) * L.width + gx);
                region[q * plane + i] = v;
                const __nv_bfloat16 b = __float2bfloat16_rn(v);
                ebf[q * plane + i] = b;
                if (cx > 0) obf[q * plane + i - 1] = b;
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
        for (int i = threadIdx.x; i < rows * ncols; i += kChosenThreads) {
            const int r = i / ncols;
            const int cx = i - r * ncols;
            float acc = 0.0f;
            for (int q = 0; q < planes_n; ++q) {
                const float* row = region + q * plane + r * rs + cx;
#pragma unroll
                for (int ii = 0; ii < P; ++ii) acc = fmaf(row[ii], row[ii], acc);
            }
            rowsum[i] = acc;
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
                afrag[cq][1] = a32[((g + 8) * kd + 16 * cq + 2 * t) >> 1];
                afrag[cq][2] = a32[(g * kd + 16 * cq + 2 * t + 8) >> 1];
                afrag[cq][3] = a32[((g + 8) * kd + 16 * cq + 2 * t + 8) >> 1];
            }
        }
        for (int i = threadIdx.x; i < Wy * ncols; i += kChosenThreads) {
            const int y = i / ncols;
            const int cx = i - y * ncols;
            float acc = 0.0f;
#pragma unroll
            for (int r = 0; r < P; ++r) acc += rowsum[(y + r) * ncols + cx];
            nb[i] = acc;
        }
        __syncthreads();
        // Approximate distances: tile = 16 anchors x 8 candidates of one row.
        {
            const unsigned* src32 = (g & 1) ? o32 : e32;
            const int tiles = Wy * tiles_x;
            for (int tile = warp; tile < tiles; tile += kChosenWarps) {
                const int y = tile / tiles_x;
                const int j = tile - y * tiles_x;
                const int col = 8 * j + g + 2 * t - (g & 1);  // even index into the even or shifted copy
                float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int cq = 0; cq < NCH; ++cq) {
                    const int q = cq >> 2;
                    const int rp = cq & 3;
                    const int base = q * plane + (y + 2 * rp) * rs + col;
                    mma_bf16_16816(c, afrag[cq], src32[base >> 1], src32[(base + rs) >> 1]);
                }
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const int m = g + 8 * (h >> 1);
                    const int cn = 8 * j + 2 * t + (h & 1);  // candidate column relative to rx0
                    if (m >= count) continue;
                    const int cxw = rx0 + cn - win_xl[m];
                    if (cxw < 0 || cxw >= win_wx[m]) continue;
                    dist[m * L.window_cells + y * win_wx[m] + cxw] = na[m] + nb[y * ncols + cn] - 2.0f * c[h];
                }
            }
        }
        __syncthreads();
        // Short list of frame k per anchor, exact re-rank.
        if (warp < count) {
            const int m = warp;
            const int Wx = win_wx[m];
            const int n = Wx * Wy;
            const float* dm = dist + m * L.window_cells;
            const int want = min(n, L.shortlist);
            float lo = kInf, hi = -kInf;
            for (int i = lane; i < n; i += 32) {
                const float v = dm[i];
                lo = fminf(lo, v);
                hi = fmaxf(hi, v);
            }
            lo = warp_min_f(lo);
            hi = warp_max_f(hi);
            // invariant: at least `want` values are <= hi
            if (want < n) {
                for (int it = 0; it < 32; ++it) {
                    const float mid = lo + 0.5f * (hi - lo);
                    if (!(mid > lo && mid < hi)) break;
                    int cnt = 0;
                    for (int i = lane; i < n; i += 32) cnt += dm[i] <= mid ? 1 : 0;
                    cnt = __reduce_add_sync(0xffffffffu, cnt);
                    if (cnt >= want) {
                        hi = mid;
                        if (cnt <= want + 8) break;
                    } else {
                        lo = mid;
                    }
                }
            }
            const int budget = L.shortlist + 8;
            const int np0 = pool_n[m];
            float* pd = pool_d + m * L.pool_cap + np0;
            int* pi = pool_i + m * L.pool_cap + np0;
            int taken = 0;
            for (int base = 0; base < n && taken < budget; base += 32) {
                const int i = base + lane;
                const bool sel = i < n && dm[i] <= hi;
                const unsigned bal = __ballot_sync(0xffffffffu, sel);
                const int pos = taken + __popc(bal & ((1u << lane) - 1u));
                if (sel && pos < budget) {
                    const int cy = i / Wx;
                    const int col = win_xl[m] + (i - cy * Wx) - rx0;
                    float d = 0.0f;
                    for (int q = 0; q < planes_n; ++q) {
#pragma unroll
                        for (int r = 0; r < P; ++r) {
                            const float* rr = reff + m * kd + q * P * P + r * P;
                            const float* cr = region + q * plane + (cy + r) * rs + col;
                            d = row_ssd<P>(d, [&](int ii) { return rr[ii]; }, [&](int ii) { return cr[ii]; });
                        }
                    }
                    pd[pos] = d;
                    pi[pos] = (k << 20) | i;
                }
                taken = min(budget, taken + __popc(bal));
            }
            __syncwarp();
            if (lane == 0) pool_n[m] = np0 + taken;
        }
    }
    __syncthreads();
    if (warp >= count) return;

    // select_similar_patches on the pooled exact distances
    const int m = warp;
    const int gi = strip.first + m;
    const int2 anchor = L.anchors[gi];
    const int Wx = win_wx[m];
    const int xl = win_xl[m];
    const int np = pool_n[m];
    const float* pd = pool_d + m * L.pool_cap;
    const int* pi = pool_i + m * L.pool_cap;
    float* sd = dist + m * L.window_cells;  // sorted pool (free now)
    int* si = reinterpret_cast<int*>(sd + L.soft_cap);
    const int K = L.K;
    const int cap = min(L.soft_cap, L.search_window * L.search_window * L.schedule_len);
    const int nbuf = min(cap, np);
    int S;
    if (K <= 1) {
        // similar <= 1: the anchor itself (core.cpp:1253-1257)
        if (lane == 0) {
            sd[0] = 0.0f;
            si[0] = -1;
        }
        S = 1;
    } else {
        for (int i = lane; i < np; i += 32) {
            const float di = pd[i];
            const int ii = pi[i];
            int rank = 0;
            for (int j = 0; j < np; ++j) {
                const float dj = pd[j];
                rank += (dj < di || (dj == di && pi[j] < ii)) ? 1 : 0;
            }
            if (rank < nbuf) {
                sd[rank] = di;
                si[rank] = ii;
            }
        }
        __syncwarp();
        const int selected = min(K, nbuf);
        const float threshold = std_max(L.tau, sd[selected - 1]);
        int within = 0;
        for (int base = 0; base < nbuf; base += 32) {
            const int i = base + lane;
            within += __popc(__ballot_sync(0xffffffffu, i < nbuf && sd[i] <= threshold));
        }
        S = min(within, min(L.soft_cap, nbuf));
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
                                           L.window_cells, planes_n * L.P * L.P, L.pool_cap);
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
