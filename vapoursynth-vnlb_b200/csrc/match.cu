// Exact block matching for one anchor frame (plain form).
//
// Reference semantics: find_similar_patches / select_similar_patches and the
// distance scans of src/core/core.cpp:1033-1362, plus the paste-mask victims
// of apply_frame_paste_mask (core.cpp:980-1008).
//
// Work decomposition.  The host cuts the raster-ordered anchor grid into
// strips: runs of up to `warps` consecutive anchors of one grid row whose
// search windows fit in one shared-memory region.  One CTA owns a strip, one
// warp owns an anchor.  For every scheduled temporal frame (anchor, future
// ascending, past descending: the CPU's candidate order) the CTA stages the
// strip's search region of every needed plane in shared memory, each warp
// computes the SSD of all its candidates in that frame with a register-tiled
// sweep (lane task = one candidate column x KY candidate rows, reference patch
// plane in registers), and then replays the CPU's sequential selection over
// the frame's candidates in raster order.  The replay is exact: it keeps the
// CPU's K-smallest heap front and its capped match buffer (same replacement
// slot), and the 32 candidates of a chunk are first tested against the
// current limit with one ballot -- the limit only shrinks, so a candidate that
// fails it can never be recorded later.
//
// Outputs per anchor g: the retained rows in the CPU's row order (the order
// std::partial_sort leaves them in), their count, and the later grid anchors
// whose paste-mask position one of its anchor-frame matches clears.
#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr int kKY = 4;           // candidate rows per lane task
constexpr int kMaxTopPerLane = 4; // K <= 128

struct WarpSelect {
    int count;       // entries in the match buffer
    int cap;         // buffer capacity (CPU output_cap)
    int worst_idx;
    float worst;
    int top_count;   // entries in the K-smallest heap
    float top_front; // its maximum (valid when full)
};

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// First index holding the maximum of buf_d[0, n) (std::max_element).
__device__ __forceinline__ void refresh_worst(const float* buf_d, int n, int lane, int& worst_idx,
                                              float& worst) {
    float best = -kInf;
    int best_i = 0x7fffffff;
    for (int i = lane; i < n; i += 32) {
        const float v = buf_d[i];
        if (best_i == 0x7fffffff || best < v) {
            best = v;
            best_i = i;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, best_i, o);
        const bool take = (oi != 0x7fffffff) &&
                          (best_i == 0x7fffffff || best < ov || (!(ov < best) && oi < best_i));
        if (take) {
            best = ov;
            best_i = oi;
        }
    }
    worst = best;
    worst_idx = best_i;
}

// std::partial_sort(first, first + middle, first + last) on (distance, id)
// pairs, reproducing the heap operations of the oracle toolchain's C++
// library (Floyd sift to a leaf, then sift up).  Single thread.
__device__ void heap_adjust(float* d, int* id, int hole, int len, float vd, int vid) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (d[child] < d[child - 1]) child--;
        d[hole] = d[child];
        id[hole] = id[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        d[hole] = d[child - 1];
        id[hole] = id[child - 1];
        hole = child - 1;
    }
    int parent = (hole - 1) / 2;
    while (hole > top && d[parent] < vd) {
        d[hole] = d[parent];
        id[hole] = id[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    d[hole] = vd;
    id[hole] = vid;
}

__device__ void heap_pop_into(float* d, int* id, int len, int result) {
    const float vd = d[result];
    const int vid = id[result];
    d[result] = d[0];
    id[result] = id[0];
    heap_adjust(d, id, 0, len, vd, vid);
}

__device__ void partial_sort_pairs(float* d, int* id, int middle, int last) {
    if (middle >= 2) {
        for (int parent = (middle - 2) / 2;; --parent) {
            heap_adjust(d, id, parent, middle, d[parent], id[parent]);
            if (parent == 0) break;
        }
    }
    for (int i = middle; i < last; ++i)
        if (d[i] < d[0]) heap_pop_into(d, id, middle, i);
    for (int len = middle; len > 1; --len) heap_pop_into(d, id, len - 1, len - 1);
}


// Distances of one lane task (candidate column cx_rel, rows gy*KY .. +KY-1)
// against the warp's reference patch, for every plane of scheduled frame k.
// Planes in shared memory are ordered (channel, t); region row stride `rs`.
template <int P>
__device__ __forceinline__ void task_distances(const float* planes, int plane_values, int rs, int col0,
                                               int row0, const float* ref, int planes_n, int p_dyn,
                                               float dist[kKY]) {
    const int PP = P > 0 ? P : p_dyn;
#pragma unroll
    for (int j = 0; j < kKY; ++j) dist[j] = 0.0f;
    for (int q = 0; q < planes_n; ++q) {
        const float* plane = planes + q * plane_values + row0 * rs + col0;
        const float* ref_plane = ref + q * PP * PP;
        if constexpr (P == kLanes) {
            // packed pairs: half the FP32 instructions, the same bits
            float2 rv[P * P / 2];
#pragma unroll
            for (int i = 0; i < P * P / 2; ++i) rv[i] = make_float2(ref_plane[2 * i], ref_plane[2 * i + 1]);
#pragma unroll
            for (int r = 0; r < kKY + P - 1; ++r) {
                float2 cv[P / 2];
#pragma unroll
                for (int i = 0; i < P / 2; ++i) cv[i] = make_float2(plane[r * rs + 2 * i], plane[r * rs + 2 * i + 1]);
#pragma unroll
                for (int j = 0; j < kKY; ++j) {
                    const int y = r - j;
                    if (y >= 0 && y < P) dist[j] = row_ssd8_x2(dist[j], rv + y * (P / 2), cv);
                }
            }
        } else if constexpr (P > 0) {
            float rv[P * P];
#pragma unroll
            for (int i = 0; i < P * P; ++i) rv[i] = ref_plane[i];
#pragma unroll
            for (int r = 0; r < kKY + P - 1; ++r) {
                float cv[P];
#pragma unroll
                for (int i = 0; i < P; ++i) cv[i] = plane[r * rs + i];
#pragma unroll
                for (int j = 0; j < kKY; ++j) {
                    const int y = r - j;
                    if (y >= 0 && y < P) {
                        dist[j] = row_ssd<P>(dist[j], [&](int i) { return rv[y * P + i]; },
                                             [&](int i) { return cv[i]; });
                    }
                }
            }
        } else {
            for (int r = 0; r < kKY + PP - 1; ++r) {
#pragma unroll
                for (int j = 0; j < kKY; ++j) {
                    const int y = r - j;
                    if (y >= 0 && y < PP)
                        dist[j] = row_ssd_dyn(dist[j], ref_plane + y * PP, plane + r * rs, PP);
                }
            }
        }
    }
}

// Approximate distances of one lane task for 8x8 patches (chosen form):
// ||a||^2 + ||b||^2 - 2 a.b, the dot products as packed FP32 multiply-adds
// (four per patch row and candidate, against 13 instructions for the exact
// row SSD), the candidate norms from the per-frame norm table, clamped at 0
// so that the values order like their bit patterns.
__device__ __forceinline__ void task_distances_approx(const float* planes, int plane_values, int rs, int col0,
                                                      int row0, const float* ref, int planes_n, float ref_norm,
                                                      const float* norms, float dist[kKY]) {
    constexpr int P = kLanes;
    float2 acc[kKY];
#pragma unroll
    for (int j = 0; j < kKY; ++j) acc[j] = make_float2(0.0f, 0.0f);
    for (int q = 0; q < planes_n; ++q) {
        const float* plane = planes + q * plane_values + row0 * rs + col0;
        const float* ref_plane = ref + q * P * P;
        float2 rv[P * P / 2];
#pragma unroll
        for (int i = 0; i < P * P / 2; ++i) rv[i] = make_float2(ref_plane[2 * i], ref_plane[2 * i + 1]);
#pragma unroll
        for (int r = 0; r < kKY + P - 1; ++r) {
            float2 cv[P / 2];
#pragma unroll
            for (int i = 0; i < P / 2; ++i) cv[i] = make_float2(plane[r * rs + 2 * i], plane[r * rs + 2 * i + 1]);
#pragma unroll
            for (int j = 0; j < kKY; ++j) {
                const int y = r - j;
                if (y >= 0 && y < P) {
#pragma unroll
                    for (int i = 0; i < P / 2; ++i) acc[j] = fma2_rn(rv[y * (P / 2) + i], cv[i], acc[j]);
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kKY; ++j)
        dist[j] = fmaxf(ref_norm + norms[(row0 + j) * rs + col0] - 2.0f * (acc[j].x + acc[j].y), 0.0f);
}

// Exact SSD of one candidate (the plain form's arithmetic and bits).
__device__ __forceinline__ float exact_distance8(const float* planes, int plane_values, int rs, int col, int row,
                                                 const float* ref, int planes_n) {
    constexpr int P = kLanes;
    float d = 0.0f;
    for (int q = 0; q < planes_n; ++q) {
#pragma unroll
        for (int r = 0; r < P; ++r) {
            const float* rr = ref + q * P * P + r * P;
            const float* cr = planes + q * plane_values + (row + r) * rs + col;
            float2 a2[P / 2], b2[P / 2];
#pragma unroll
            for (int i = 0; i < P / 2; ++i) {
                a2[i] = make_float2(rr[2 * i], rr[2 * i + 1]);
                b2[i] = make_float2(cr[2 * i], cr[2 * i + 1]);
            }
            d = row_ssd8_x2(d, a2, b2);
        }
    }
    return d;
}

// Staging with the tensor memory accelerator: one thread arms an mbarrier
// with the byte count of the frame's planes and issues one 2-D tile load per
// plane (box = region_stride x region_rows, x a multiple of 4 floats, no
// multicast); every thread then waits on the barrier's phase.
constexpr int kTmaSpinLimit = 1 << 24;  // barrier polls before a staging wait gives up

__device__ __forceinline__ void stage_bar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void stage_bar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool stage_bar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void tma_load_tile(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

template <int P, bool kApprox, bool kFlow>  // kFlow: search centres from L.centers
__global__ void __launch_bounds__(256, 3) match_kernel(MatchLaunch L, const __grid_constant__ CUtensorMap tmap) {
    extern __shared__ __align__(128) float smem[];
    __shared__ __align__(8) unsigned long long stage_bar;
    __shared__ int stage_failed;
    if (L.tile_fail && !L.tile_fail[L.strip_tile[blockIdx.x]]) return;  // the learned rows stand
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const Strip strip = L.strips[blockIdx.x];
    const int Pd = L.P;
    const int Cs = L.search_channels;
    const int planes_n = Cs * L.Pt;
    const int plane_values = L.plane_floats;
    const bool tma = !kFlow && L.tma != 0;
    const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&stage_bar));
    uint32_t stage_phase = 0;
    if (tma && threadIdx.x == 0) {
        stage_bar_init(bar);
        stage_failed = 0;
    }

    float* planes = smem;
    // chosen form: per-frame norm table of every patch origin in the region,
    // and the row sums of squares it is built from
    float* norms = planes + planes_n * plane_values;
    float* rowsq = norms + (kApprox ? plane_values : 0);
    float* warp_base = planes + planes_n * plane_values + (kApprox ? 2 * plane_values : 0) + warp * L.warp_floats;
    float* dist = warp_base;                                  // window_cells
    float* ref = dist + L.window_cells;                        // planes_n * P * P
    float* buf_d = ref + planes_n * Pd * Pd;                   // buffer_cap
    int* buf_i = reinterpret_cast<int*>(buf_d + L.buffer_cap); // buffer_cap

    const bool active_warp = warp < strip.count;
    const int g = strip.first + warp;
    int ax = 0, ay = 0;
    if (active_warp) {
        const int2 a = L.anchors[g];
        ax = a.x;
        ay = a.y;
    }
    int xl, xh, yl, yh;
    spatial_range(ax, L.width, Pd, L.search_window, xl, xh);
    spatial_range(strip.y, L.height, Pd, L.search_window, yl, yh);
    const int Wx = xh - xl + 1;
    const int Wy = yh - yl + 1;
    const int cells = Wx * Wy;
    const int tasks = Wx * ((Wy + kKY - 1) / kKY);
    int rx0 = strip.region_x, ry0 = strip.region_y, rw = strip.region_w, rh = strip.region_h;

    WarpSelect s;
    s.count = 0;
    s.cap = min(L.soft_cap, L.search_window * L.search_window * L.schedule_len);
    s.worst_idx = 0;
    s.worst = kInf;
    s.top_count = 0;
    s.top_front = kInf;
    float my_top[kMaxTopPerLane];
#pragma unroll
    for (int i = 0; i < kMaxTopPerLane; ++i) my_top[i] = -kInf;
    const int K = L.K;
    // register-resident buffer and heap when both fit in a warp
    const bool fast = s.cap <= 32 && K <= 32;
    unsigned reg_d = 0u, reg_top = 0u;  // bits of non-negative distances (0 = empty)
    int reg_id = 0;
    float ref_norm = 0.0f;   // chosen form: ||reference||^2
    float reg_exact = 0.0f;  // chosen form: exact distance of this lane's buffer slot

    // Flow-guided search: every warp's window of frame k lies around its
    // anchor's search centre there (same size as the anchor-centred one).  The
    // strip's warps are taken in passes; a pass stages the bounding box of the
    // windows of its warps, grown in warp order while it fits the reservation
    // (region_w_max columns, region_rows rows), so a strip whose anchors move
    // alike stages frame k once.  pending = warps still to search frame k.
    __shared__ int2 window_origin[kFlow ? 8 : 1];
    unsigned pending = 0u;
    unsigned group = 0xffffffffu;  // warps searching in this pass
    for (int k = 0; k < L.schedule_len; k += pending == 0u ? 1 : 0) {
        const int frame = L.schedule[k];
        if constexpr (kFlow) {
            if (pending == 0u) {
                __syncthreads();  // the previous frame's passes are done with the table
                if (active_warp) {
                    const int2 c = L.centers[static_cast<size_t>(g) * L.schedule_len + k];
                    spatial_range(c.x, L.width, Pd, L.search_window, xl, xh);
                    spatial_range(c.y, L.height, Pd, L.search_window, yl, yh);
                    if (lane == 0) window_origin[warp] = make_int2(xl, yl);
                }
                __syncthreads();
                pending = (1u << strip.count) - 1u;
            }
            const int w0 = __ffs(pending) - 1;
            int2 o = window_origin[w0];
            int x0 = o.x & ~3, x1 = o.x + Wx - 1 + Pd - 1, y0 = o.y, y1 = o.y + Wy - 1 + Pd - 1;
            group = 1u << w0;
            for (int w = w0 + 1; w < strip.count; ++w) {
                if (!((pending >> w) & 1u)) continue;
                o = window_origin[w];
                const int nx0 = min(x0, o.x & ~3), nx1 = max(x1, o.x + Wx - 1 + Pd - 1);
                const int ny0 = min(y0, o.y), ny1 = max(y1, o.y + Wy - 1 + Pd - 1);
                if (nx1 - nx0 + 1 > L.region_w_max || ny1 - ny0 + kKY > L.region_rows) continue;
                x0 = nx0;
                x1 = nx1;
                y0 = ny0;
                y1 = ny1;
                group |= 1u << w;
            }
            pending &= ~group;
            rx0 = x0;
            ry0 = y0;
            rw = x1 - x0 + 1;
            rh = y1 - y0 + 1;
        }
        __syncthreads();
        // Stage the strip's region of every plane (channel, t) of frame k.
        const int rows = rh;
        const int cols = rw;
        if (tma) {
            // whole boxes (region_stride x region_rows) from row (slot, c, ry0)
            // of the store; rows and columns past the region are never read
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier reads of these planes
                stage_bar_expect(bar, static_cast<uint32_t>(planes_n) * L.region_rows * L.region_stride * 4u);
                for (int q = 0; q < planes_n; ++q) {
                    const int c = q / L.Pt;
                    const int t = q % L.Pt;
                    const int y = (((frame % L.ring) + t) * L.channels + c) * L.height + ry0;
                    tma_load_tile(static_cast<uint32_t>(__cvta_generic_to_shared(planes + q * plane_values)), &tmap,
                                  rx0, y, bar);
                }
            }
            int spins = 0;
            while (!stage_bar_try_wait(bar, stage_phase))
                if (++spins >= kTmaSpinLimit) break;
            stage_phase ^= 1u;
            if (spins >= kTmaSpinLimit) stage_failed = 1;
            __syncthreads();
            if (stage_failed) {
                // the load never completed: report it, and give it a bounded
                // second chance to land before the block's shared memory goes
                if (threadIdx.x == 0) {
                    atomicCAS(L.status, 0, kStatusTmaTimeout);
                    for (int i = 0; i < kTmaSpinLimit && !stage_bar_try_wait(bar, stage_phase ^ 1u); ++i) {
                    }
                }
                __syncthreads();
                return;
            }
        } else {
            for (int q = 0; q < planes_n; ++q) {
                const int c = q / L.Pt;
                const int t = q % L.Pt;
                const float* src = L.video + ((static_cast<size_t>(frame % L.ring + t) * L.channels + c) * L.height +
                                              ry0) * static_cast<size_t>(L.width) + rx0;
                float* dst = planes + q * plane_values;
                for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
                    const int r = i / cols;
                    const int cx = i - r * cols;
                    dst[r * L.region_stride + cx] = __ldg(src + static_cast<size_t>(r) * L.width + cx);
                }
            }
        }
        __syncthreads();
        if constexpr (kApprox) {
            const int rs = L.region_stride;
            for (int i = threadIdx.x; i < rows * (cols - P + 1); i += blockDim.x) {
                const int r = i / (cols - P + 1);
                const int cx = i - r * (cols - P + 1);
                float acc = 0.0f;
                for (int q = 0; q < planes_n; ++q) {
                    const float* row = planes + q * plane_values + r * rs + cx;
#pragma unroll
                    for (int ii = 0; ii < P; ++ii) acc = fmaf(row[ii], row[ii], acc);
                }
                rowsq[r * rs + cx] = acc;
            }
            __syncthreads();
            for (int i = threadIdx.x; i < (rows - P + 1) * (cols - P + 1); i += blockDim.x) {
                const int r = i / (cols - P + 1);
                const int cx = i - r * (cols - P + 1);
                float acc = 0.0f;
#pragma unroll
                for (int rr = 0; rr < P; ++rr) acc += rowsq[(r + rr) * rs + cx];
                norms[r * rs + cx] = acc;
            }
            __syncthreads();
        }
        if (!active_warp || !((group >> warp) & 1u)) continue;
        if (k == 0) {
            // Reference patch (anchor frame is scheduled first).
            for (int i = lane; i < planes_n * Pd * Pd; i += 32) {
                const int q = i / (Pd * Pd);
                const int rem = i - q * Pd * Pd;
                const int py = rem / Pd;
                const int px = rem - py * Pd;
                ref[i] = planes[q * plane_values + (ay - ry0 + py) * L.region_stride + (ax - rx0 + px)];
            }
            __syncwarp();
            if constexpr (kApprox) {
                float acc = 0.0f;
                for (int i = lane; i < planes_n * Pd * Pd; i += 32) acc = fmaf(ref[i], ref[i], acc);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                ref_norm = acc;
            }
        }
        // Distances of all candidates of frame k.
        for (int task = lane; task < tasks; task += 32) {
            const int cx = task % Wx;
            const int gy = task / Wx;
            float d[kKY];
            if constexpr (kApprox)
                task_distances_approx(planes, plane_values, L.region_stride, xl - rx0 + cx, yl - ry0 + gy * kKY, ref,
                                      planes_n, ref_norm, norms, d);
            else
                task_distances<P>(planes, plane_values, L.region_stride, xl - rx0 + cx, yl - ry0 + gy * kKY, ref,
                                  planes_n, Pd, d);
#pragma unroll
            for (int j = 0; j < kKY; ++j) {
                const int cy = gy * kKY + j;
                if (cy < Wy) dist[cy * Wx + cx] = d[j];
            }
        }
        __syncwarp();
        // Replay of the CPU's sequential selection over frame k, raster order.
        if (fast) {
            // buffer slot i and heap entry i live in lane i; non-negative float
            // distances order like their bit patterns, so the first maximum
            // (std::max_element) is a max-reduction and a ballot
            for (int base = 0; base < cells; base += 32) {
                const int idx = base + lane;
                const float mine = idx < cells ? dist[idx] : kInf;
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
                    // record_candidate_match
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
                    // record_candidate_distance: the K smallest so far
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
            if constexpr (kApprox) {
                // exact FP32 distance of the buffer slots frame k filled, while
                // frame k is staged: each lane re-ranks its own slot
                if (lane < s.count && (reg_id >> 20) == k) {
                    const int cell = reg_id & 0xfffff;
                    const int cy = cell / Wx;
                    reg_exact = exact_distance8(planes, plane_values, L.region_stride, xl - rx0 + (cell - cy * Wx),
                                                yl - ry0 + cy, ref, planes_n);
                }
            }
            continue;
        }
        // Replay of the CPU's sequential selection over frame k, raster order.
        for (int base = 0; base < cells; base += 32) {
            const int idx = base + lane;
            const float mine = idx < cells ? dist[idx] : kInf;
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
                // record_candidate_match
                if (s.count < s.cap) {
                    if (lane == 0) {
                        buf_d[s.count] = d;
                        buf_i[s.count] = id;
                    }
                    s.count++;
                    __syncwarp();
                    if (s.count == s.cap) refresh_worst(buf_d, s.count, lane, s.worst_idx, s.worst);
                } else if (d < s.worst) {
                    if (lane == 0) {
                        buf_d[s.worst_idx] = d;
                        buf_i[s.worst_idx] = id;
                    }
                    __syncwarp();
                    refresh_worst(buf_d, s.count, lane, s.worst_idx, s.worst);
                }
                // record_candidate_distance
                if (s.top_count < K) {
                    const int slot = s.top_count;
#pragma unroll
                    for (int i = 0; i < kMaxTopPerLane; ++i)
                        if (i * 32 + lane == slot) my_top[i] = d;
                    s.top_count++;
                    if (s.top_count == K) {
                        float m = -kInf;
#pragma unroll
                        for (int i = 0; i < kMaxTopPerLane; ++i) m = fmaxf(m, my_top[i]);
                        s.top_front = warp_max(m);
                    }
                } else if (d < s.top_front) {
                    // replace one entry equal to the maximum
                    int owner = 0x7fffffff;
#pragma unroll
                    for (int i = 0; i < kMaxTopPerLane; ++i)
                        if (owner == 0x7fffffff && my_top[i] == s.top_front) owner = i * 32 + lane;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) owner = min(owner, __shfl_xor_sync(0xffffffffu, owner, o));
#pragma unroll
                    for (int i = 0; i < kMaxTopPerLane; ++i)
                        if (i * 32 + lane == owner) my_top[i] = d;
                    float m = -kInf;
#pragma unroll
                    for (int i = 0; i < kMaxTopPerLane; ++i) m = fmaxf(m, my_top[i]);
                    s.top_front = warp_max(m);
                }
            }
        }
        __syncwarp();
    }
    if (!active_warp) return;
    int S = 0;
    bool selected_in_warp = false;
    if (kApprox && fast && K > 1) {
        // chosen form: select_similar_patches on the exact distances of the
        // buffer -- the K smallest, the threshold max(tau, d_K), the slots
        // within it, closest first (ties by candidate order), at most the cap
        const int n = s.count;
        int rank = 0;
        for (int j = 0; j < n; ++j) {
            const float dj = __shfl_sync(0xffffffffu, reg_exact, j);
            const int ij = __shfl_sync(0xffffffffu, reg_id, j);
            rank += (dj < reg_exact || (dj == reg_exact && ij < reg_id)) ? 1 : 0;
        }
        if (lane < n) {
            buf_d[rank] = reg_exact;
            buf_i[rank] = reg_id;
        }
        __syncwarp();
        const int M = min(K, n);
        const float threshold = std_max(L.tau, buf_d[M - 1]);
        const int within = __popc(__ballot_sync(0xffffffffu, lane < n && buf_d[lane] <= threshold));
        S = min(within, min(L.soft_cap, n));
        selected_in_warp = true;
    } else if (fast) {
        // select_similar_patches with pairwise distinct buffered distances:
        // the heap replay below has a unique outcome, computed warp-wide.
        // partial_sort(first, first + M, first + n) keeps in [0, M) the M
        // smallest in ascending order; tail slot i (M <= i < n) ends up with
        // the heap's maximum at the time element i arrived when that element
        // is smaller (it is swapped in), else with the element itself.
        const int n = s.count;
        const unsigned key = lane < n ? reg_d : (0x80000000u | static_cast<unsigned>(lane));
        const bool tie = __any_sync(0xffffffffu, __popc(__match_any_sync(0xffffffffu, key)) > 1);
        if (K > 1 && !tie) {
            const int M = min(K, n);
            unsigned d = reg_d;
            int id = reg_id;
            unsigned cur_max = __reduce_max_sync(0xffffffffu, lane < M ? d : 0u);
            for (int i = M; i < n; ++i) {
                const unsigned di = __shfl_sync(0xffffffffu, d, i);
                const int ii = __shfl_sync(0xffffffffu, id, i);
                if (di < cur_max) {
                    const int o = __ffs(__ballot_sync(0xffffffffu, lane < M && d == cur_max)) - 1;
                    const int oi = __shfl_sync(0xffffffffu, id, o);
                    if (lane == o) {
                        d = di;
                        id = ii;
                    }
                    if (lane == i) {
                        d = cur_max;
                        id = oi;
                    }
                    cur_max = __reduce_max_sync(0xffffffffu, lane < M ? d : 0u);
                }
            }
            // the kept M ascending (distinct: rank = number of smaller ones),
            // then the tail slots within the threshold, in slot order
            const float threshold = std_max(L.tau, __uint_as_float(cur_max));
            int rank = 0;
            for (int j = 0; j < M; ++j) rank += __shfl_sync(0xffffffffu, d, j) < d ? 1 : 0;
            const bool keep_tail = lane >= M && lane < n && __uint_as_float(d) <= threshold;
            const unsigned tail_mask = __ballot_sync(0xffffffffu, keep_tail);
            if (lane < M) {
                buf_d[rank] = __uint_as_float(d);
                buf_i[rank] = id;
            } else if (keep_tail) {
                const int pos = M + __popc(tail_mask & ((1u << lane) - 1u));
                buf_d[pos] = __uint_as_float(d);
                buf_i[pos] = id;
            }
            S = M + __popc(tail_mask);
            selected_in_warp = true;
        } else if (lane < n) {
            buf_d[lane] = __uint_as_float(reg_d);
            buf_i[lane] = reg_id;
        }
        __syncwarp();
    }

    // select_similar_patches (core.cpp:1200-1243): single lane.
    if (!selected_in_warp && lane == 0) {
        const int n = s.count;
        if (K <= 1) {
            // similar <= 1: the anchor itself (core.cpp:1253-1257)
            buf_d[0] = 0.0f;
            buf_i[0] = -1;
            S = 1;
        } else {
            const int selected = min(K, n);
            partial_sort_pairs(buf_d, buf_i, selected, n);
            const float threshold = std_max(L.tau, buf_d[selected - 1]);
            int out = 0;
            for (int i = 0; i < n; ++i)
                if (buf_d[i] <= threshold) {
                    buf_d[out] = buf_d[i];
                    buf_i[out] = buf_i[i];
                    ++out;
                }
            const int output_cap = min(L.soft_cap, n);
            if (out > output_cap) {
                partial_sort_pairs(buf_d, buf_i, output_cap, out);
                out = output_cap;
            }
            S = out;
        }
    }
    if (!selected_in_warp) S = __shfl_sync(0xffffffffu, S, 0);
    __syncwarp();
    MatchRow* rows_out = L.rows + static_cast<size_t>(g) * L.max_rows;
    int nvict = 0;
    for (int i = lane; i < S; i += 32) {
        const int id = buf_i[i];
        MatchRow m;
        m.distance = buf_d[i];
        if (id < 0) {
            m.x = ax;
            m.y = ay;
            m.frame = L.anchor_frame;
        } else {
            const int kk = id >> 20;
            const int cell = id & 0xfffff;
            const int cy = cell / Wx;
            int fxl = xl, fyl = yl;
            if constexpr (kFlow) {  // frame kk's window
                const int2 c = L.centers[static_cast<size_t>(g) * L.schedule_len + kk];
                int hi;
                spatial_range(c.x, L.width, Pd, L.search_window, fxl, hi);
                spatial_range(c.y, L.height, Pd, L.search_window, fyl, hi);
            }
            m.x = fxl + (cell - cy * Wx);
            m.y = fyl + cy;
            m.frame = L.schedule[kk];
        }
        rows_out[i] = m;
    }
    if (lane == 0) L.row_counts[g] = S;
    // Paste-mask victims (apply_frame_paste_mask, core.cpp:980-1008): later
    // grid anchors whose position an anchor-frame match clears.
    int* vict = L.victims + static_cast<size_t>(g) * L.victim_stride;
    for (int i0 = 0; i0 < S; i0 += 32) {
        const int i = i0 + lane;
        int found[5];
        int nf = 0;
        if (i < S) {
            const MatchRow m = rows_out[i];
            if (m.frame == L.anchor_frame) {
                const int px[5] = {m.x, m.x, m.x, m.x - 1, m.x + 1};
                const int py[5] = {m.y, m.y - 1, m.y + 1, m.y, m.y};
                const bool use[5] = {true, m.y > 2 * Pd, m.y < L.height - 2 * Pd, m.x > 2 * Pd,
                                     m.x < L.width - 2 * Pd};
#pragma unroll
                for (int e = 0; e < 5; ++e) {
                    if (!use[e] || px[e] < 0 || px[e] >= L.width || py[e] < 0 || py[e] >= L.height) continue;
                    const int j = L.anchor_map[static_cast<size_t>(py[e]) * L.width + px[e]];
                    if (j > g) found[nf++] = j;
                }
            }
        }
        // warp-ordered append
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
    if (lane == 0) L.victim_counts[g] = min(nvict, L.victim_stride);
}

// Flow-guided search centres: MVToolsVectorGrid::nearest_vector
// (src/flow/flow.hpp:72-120), round_subpixel_to_pixel (flow.hpp:183-191) and
// MVToolsFlowProvider::center_for (flow.hpp:341-389).  The centre starts at
// the anchor and walks frame by frame toward the candidate frame (mvfw grids
// toward earlier frames, mvbw toward later ones): each usable grid moves it
// by the vector of the block nearest to the patch centre, rounded to whole
// pixels, then it is clamped to the frame.
__device__ __forceinline__ int nearest_block_index(int coordinate, int first_center, int step, int count) {
    if (count <= 1) return 0;
    const int shifted = coordinate - first_center;
    const int index = shifted >= 0 ? (shifted + step / 2) / step : -((-shifted + step / 2) / step);
    return min(max(index, 0), count - 1);
}

__device__ __forceinline__ int round_subpixel(int value, int pel) {
    if (pel <= 1) return value;
    return value >= 0 ? (value + pel / 2) / pel : -((-value + pel / 2) / pel);
}

__device__ __forceinline__ void flow_step(const FlowGridsDevice& g, int frame, int patch_center, int width,
                                          int height, int& cx, int& cy) {
    if (!g.present || !g.usable[frame] || g.pel <= 0 || g.block_size_x <= 0 || g.block_size_y <= 0 ||
        g.block_count_x <= 0 || g.block_count_y <= 0)
        return;
    const int step_x = max(1, g.block_size_x - max(0, g.overlap_x));
    const int step_y = max(1, g.block_size_y - max(0, g.overlap_y));
    const int bx = nearest_block_index(cx + patch_center, g.block_size_x / 2, step_x, g.block_count_x);
    const int by = nearest_block_index(cy + patch_center, g.block_size_y / 2, step_y, g.block_count_y);
    const int2 v = g.vectors[(static_cast<size_t>(frame) * g.block_count_y + by) * g.block_count_x + bx];
    cx += round_subpixel(v.x, g.pel);
    cy += round_subpixel(v.y, g.pel);
    if (width > 0) cx = min(max(cx, 0), width - 1);
    if (height > 0) cy = min(max(cy, 0), height - 1);
}

__global__ void centers_kernel(CentersLaunch L) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.anchor_count * L.schedule_len) return;
    const int g = i / L.schedule_len;
    const int k = i - g * L.schedule_len;
    const int af = L.anchor_frame;
    const int cf = L.schedule[k];
    int cx = L.anchors[g].x, cy = L.anchors[g].y;
    const int patch_center = max(0, L.P / 2);
    if (cf < af) {
        for (int f = af; f > cf; --f) flow_step(L.fw, f, patch_center, L.width, L.height, cx, cy);
    } else {
        for (int f = af; f < cf; ++f) flow_step(L.bw, f, patch_center, L.width, L.height, cx, cy);
    }
    L.centers[i] = make_int2(cx, cy);
}

}  // namespace

cudaError_t launch_centers(const CentersLaunch& L, cudaStream_t stream) {
    const int n = L.anchor_count * L.schedule_len;
    if (n <= 0) return cudaSuccess;
    centers_kernel<<<(n + 255) / 256, 256, 0, stream>>>(L);
    return cudaGetLastError();
}

size_t match_shared_bytes(const MatchLaunch& L, int warps) {
    const size_t plane = static_cast<size_t>(L.plane_floats);
    const size_t planes = static_cast<size_t>(L.search_channels) * L.Pt * plane + (L.approx ? 2 * plane : 0);
    return (planes + static_cast<size_t>(warps) * L.warp_floats) * sizeof(float);
}

int match_warp_floats(int window_cells, int planes_n, int P, int buffer_cap) {
    int f = window_cells + planes_n * P * P + 2 * buffer_cap;
    return (f + 3) & ~3;
}

bool encode_store_map(CUtensorMap* map, const float* base, int width, long long rows, int box_w, int box_h) {
    const uintptr_t addr = reinterpret_cast<uintptr_t>(base);
    if (!base || addr % 16 != 0 || (static_cast<size_t>(width) * sizeof(float)) % 16 != 0 || box_w <= 0 ||
        box_w > 256 || box_h <= 0 || box_h > 256 || (box_w * sizeof(float)) % 16 != 0 || rows <= 0)
        return false;
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult found{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &found) != cudaSuccess ||
            found != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<Encode>(fn);
    }();
    if (!encode) return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(width), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(width) * sizeof(float)};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_w), static_cast<cuuint32_t>(box_h)};
    const cuuint32_t elem[2] = {1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, elem,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_match(const MatchLaunch& L, int strips, int warps, const CUtensorMap* tmap, cudaStream_t stream) {
    if (strips <= 0) return cudaSuccess;
    if (L.tma && (!tmap || L.centers || L.region_stride % 4 != 0 || L.plane_floats % 32 != 0))
        return cudaErrorInvalidValue;
    const size_t smem = match_shared_bytes(L, warps);
    const dim3 block(32 * warps);
    CUtensorMap map{};
    if (tmap) map = *tmap;
    cudaError_t err = cudaSuccess;
    auto launch = [&](auto kernel) {
        err = raise_smem_limit(reinterpret_cast<const void*>(kernel), static_cast<int>(smem));
        if (err != cudaSuccess) return;
        kernel<<<strips, block, smem, stream>>>(L, map);
        err = cudaGetLastError();
    };
    if (L.centers) {  // flow-guided search: windows around per-frame search centres
        if (L.approx || warps > 8) return cudaErrorInvalidValue;
        switch (L.P) {
            case 4: launch(match_kernel<4, false, true>); break;
            case 5: launch(match_kernel<5, false, true>); break;
            case 6: launch(match_kernel<6, false, true>); break;
            case 7: launch(match_kernel<7, false, true>); break;
            case 8: launch(match_kernel<8, false, true>); break;
            default: launch(match_kernel<0, false, true>); break;
        }
        return err;
    }
    if (L.approx) {
        if (L.P != kLanes) return cudaErrorInvalidValue;
        launch(match_kernel<8, true, false>);
        return err;
    }
    switch (L.P) {
        case 4: launch(match_kernel<4, false, false>); break;
        case 5: launch(match_kernel<5, false, false>); break;
        case 6: launch(match_kernel<6, false, false>); break;
        case 7: launch(match_kernel<7, false, false>); break;
        case 8: launch(match_kernel<8, false, false>); break;
        default: launch(match_kernel<0, false, false>); break;
    }
    return err;
}

}  // namespace vnlbgpu
