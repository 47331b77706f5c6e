// Block matching for one anchor frame, chosen_tc form: candidate dot products
// on the 5th-generation tensor cores (tcgen05.mma with BF16 operands in shared
// memory and FP32 accumulators in tensor memory), exact FP32 re-rank.
//
// The selected rows feed the same filter and aggregation as the plain form.
// What changes is how the candidates are scored:
//
//   1. approximate distance ||a||^2 + ||b||^2 - 2 a.b for every candidate:
//      the dot products on the tensor cores (BF16 samples, FP32
//      accumulation), the norms in FP32 from the FP32 samples;
//   2. the CPU's sequential selection (find_similar_patches,
//      core.cpp:1277-1359: the K-smallest front and the capped buffer) run on
//      the approximate distances, frame by frame in the CPU's candidate order;
//   3. the exact FP32 SSD, in the CPU's arithmetic order (the bits the plain
//      form computes), of every buffer entry a frame brings in;
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
// Two kernels.  The distance kernel computes step 1 for every anchor and
// candidate and writes the approximate distances to global memory
// ([anchor][scheduled frame][window row][window column], 4 bytes each: the
// 142 MB of a 1080p anchor frame cross HBM in tens of microseconds); the
// selection kernel runs steps 2-4 with one warp per anchor at full occupancy.
//
// Distance kernel.  One CTA takes a strip of up to 8 consecutive anchors of
// one grid row whose search windows lie within 64 consecutive candidate
// columns.  Per scheduled frame:
//
//   a. The strip's search region is read from global memory once and written
//      to shared memory as BF16 core matrices of the tcgen05 no-swizzle
//      K-major layout (8 rows of 16 bytes each): for region row r and column
//      block b the 8x8 block H[i][j] = region[r][8b + i + j], so its row i is
//      the 8-sample patch row of candidate column 8b + i.  Blocks are stored
//      row-major (r, b), 128 bytes each.  The A operand of candidate rows
//      (y, y + 1) x 64 columns against patch rows (py, py + 1) is then one
//      descriptor: 8-row groups 128 bytes apart (blocks b = 0..7 of row y + py,
//      then of row y + py + 1, which is candidate row y + 1), the second K
//      chunk 1024 bytes further (row y + py + 1 = patch row py + 1).  A warp
//      builds one region row: each lane loads 3 samples, the 8-sample rows of
//      candidate columns lane and lane + 32 come from the other lanes by
//      shuffles, and the 64 block rows go out as consecutive 16-byte stores
//      (no bank conflicts).  The same pass sums the squares of the 8-sample
//      row segments (candidate norms).
//   b. One thread issues, per pair of candidate rows p, the M = 128 x N = 16 x
//      K = 16 MMAs over the patch rows and planes into tensor-memory columns
//      16 p .. 16 p + 15 (column n = anchor n; reference rows of missing
//      anchors are zero) and commits them to an mbarrier.
//   c. The 8 warps read the accumulators back (tcgen05.ld; warp w reads TMEM
//      lanes 32 (w % 4) .. + 31, i.e. candidate row 2p + (w % 4) / 2, columns
//      32 (w % 2) .. + 31) and store each anchor's window distances.
//
// Tensor memory: each CTA allocates kChosenTmemCols columns and holds at most
// two CTAs per SM (launch bounds and shared memory), so allocations never
// wait on each other.  The MMA completion wait is bounded: when it runs out
// the kernel records kStatusTensorTimeout in the session status word, which
// the host turns into an error, and carries on without spinning further.
#include <cuda_bf16.h>

#include <cstdint>

#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr int kTcThreads = 32 * kChosenWarps;
constexpr int kPatch = 8;  // the tensor-core matcher is built for 8 x 8 patches
constexpr int kTcN = 16;   // MMA N: anchor slots per strip (kChosenAnchors used)
// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits
// 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 =
// 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(kTcN >> 3) << 17) |
                            (static_cast<uint32_t>(128 >> 4) << 24);
constexpr int kSpinLimit = 1 << 22;  // mbarrier polls before a wait gives up
// distance kernel roles and pipeline
constexpr int kProducerWarps = 8;
constexpr int kConsumerWarps = 4;  // warps 8-11: tensor-memory lane quarters 0-3
constexpr int kMmaWarp = kProducerWarps + kConsumerWarps;
constexpr int kPipeThreads = 32 * (kMmaWarp + 1);
constexpr int kStages = 2;
constexpr int kPipeTmemCols = kStages * kChosenTmemCols;
// shared memory of at least this size keeps a second distance CTA (and its
// tensor-memory allocation) off the SM
constexpr int kMinSharedBytes = 116 * 1024;

// Per-stage window metadata (producers -> consumers).
struct StageMeta {
    int first, count, k, pad;
    int win_lo[kChosenAnchors];  // window columns relative to the strip origin
    int win_wx[kChosenAnchors];
    float na[kChosenAnchors];    // reference norms
};

// Shared-memory layout of the distance kernel in bytes (128-byte aligned
// parts): two stages of [BF16 blocks | reference block | norms | metadata],
// then the producers' row sums, the mbarriers and the tensor-memory address.
struct PipeLayout {
    int hank, bop, nb, meta, stage_bytes, rowsq, bars, tmem, bytes;
};

__host__ __device__ inline int align128(int v) { return (v + 127) & ~127; }

__host__ __device__ inline PipeLayout pipe_layout(int planes_n, int pairs) {
    const int R = 2 * pairs + kPatch - 1;  // region rows
    PipeLayout l{};
    int off = 0;
    l.hank = off;  off = align128(off + planes_n * R * 8 * 128);       // [q][r][b] 8x8 BF16 blocks
    l.bop = off;   off = align128(off + planes_n * kPatch * 2 * 128);   // [q][py][n/8] 8x8 BF16 blocks
    l.nb = off;    off = align128(off + 2 * pairs * kChosenCols * 4);   // candidate norms
    l.meta = off;  off = align128(off + static_cast<int>(sizeof(StageMeta)));
    l.stage_bytes = off;
    off = kStages * l.stage_bytes;
    l.rowsq = off; off = align128(off + R * kChosenCols * 4);           // row sums of squares
    l.bars = off;  off += 3 * kStages * 8;
    l.tmem = off;  off += 8;
    l.bytes = align128(off);
    return l;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between the two K chunks), stride byte offset (between 8-row
// groups), all in 16-byte units; bits 46-47 = 1 (the sm_100 descriptor).
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Issued by a whole converged warp with warp-uniform operands; only the lane
// with `leader` set executes the instruction (the same lane for the MMAs and
// their commit, which tracks the MMAs of the issuing thread).
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate, uint32_t leader) {
    asm volatile(
        "{\n\t.reg .pred p, e;\n\tsetp.ne.b32 p, %4, 0;\n\tsetp.ne.b32 e, %5, 0;\n\t"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(leader)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar, uint32_t leader) {
    asm volatile(
        "{\n\t.reg .pred e;\n\tsetp.ne.b32 e, %1, 0;\n\t"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}\n" ::"r"(bar),
        "r"(leader)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// generic-proxy shared-memory writes made visible to the tensor cores
__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ uint32_t full_bar(uint32_t bars, int s) { return bars + 8 * s; }
__device__ __forceinline__ uint32_t tfull_bar(uint32_t bars, int s) { return bars + 8 * (kStages + s); }
__device__ __forceinline__ uint32_t free_bar(uint32_t bars, int s) { return bars + 8 * (2 * kStages + s); }

// named barrier of the producer warps
__device__ __forceinline__ void producer_sync() {
    asm volatile("bar.sync 1, %0;" ::"n"(kProducerWarps * 32) : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns (two row pairs), then the wait.
__device__ __forceinline__ void tmem_load32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Persistent, warp-specialised distance kernel.  Each CTA walks the items
// (strip, scheduled frame) of strips blockIdx.x, blockIdx.x + gridDim.x, ...
// through two shared-memory stages and two halves of its tensor memory:
//   warps 0-7   producers: build stage i % 2 (BF16 blocks, reference block,
//               norms, window metadata), then arrive on full[i % 2];
//   warp 12     issuer: waits full, issues the item's MMAs into tensor-memory
//               columns 256 (i % 2) .., commits them to tfull[i % 2];
//   warps 8-11  consumers (TMEM lane quarters 0-3): wait tfull, read the
//               accumulators back, store the distances, arrive on free[i % 2],
//               which the producers wait for before refilling the stage.
template <int PLANES>  // planes compared: search channels x patch_time
__global__ void __launch_bounds__(kPipeThreads, 1) tc_distance_kernel(MatchLaunch L) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    constexpr int P = kPatch;
    const int Wy = L.window_rows;
    const int pairs = (Wy + 1) >> 1;
    const int R = 2 * pairs + P - 1;
    const PipeLayout lay = pipe_layout(PLANES, pairs);
    const uint32_t bars = smem_addr(smem + lay.bars);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + lay.tmem);
    float* rowsq = reinterpret_cast<float*>(smem + lay.rowsq);
    const size_t plane_values = static_cast<size_t>(L.height) * L.width;
    const int T = L.schedule_len;

    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(kPipeTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // completion of every MMA this CTA issued, committed once before the
    // tensor memory is released
    __shared__ __align__(8) unsigned long long drain_bar;
    const uint32_t drain = smem_addr(reinterpret_cast<unsigned char*>(&drain_bar));
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(full_bar(bars, s), 1);
            mbar_init(tfull_bar(bars, s), 1);
            mbar_init(free_bar(bars, s), kConsumerWarps);
        }
        mbar_init(drain, 1);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    bool timed_out = false;
    auto wait = [&](uint32_t bar, uint32_t parity) {
        if (timed_out) return;
        int polls = 0;
        while (!mbar_try_wait(bar, parity)) {
            if (++polls >= kSpinLimit) {
                timed_out = true;
                atomicCAS(L.status, 0, kStatusTensorTimeout);
                return;
            }
        }
    };

    if (warp < kProducerWarps) {
        int i = 0;
        for (int si = blockIdx.x; si < L.strip_count; si += gridDim.x) {
            const Strip strip = L.strips[si];
            int yl, yh;
            spatial_range(strip.y, L.height, P, L.search_window, yl, yh);
            const int rx0 = strip.region_x;
            const int count = strip.count;
            for (int k = 0; k < T; ++k, ++i) {
                const int b = i & 1;
                const int frame = L.schedule[k];
                // global loads that need no stage: the reference samples of
                // anchor `warp` (pairs of columns) and the first region row
                const int n = warp;
                float refv[PLANES][2];
                {
                    int2 a = make_int2(0, 0);
                    if (n < count) a = L.anchors[strip.first + n];
                    const float* anchor_frame =
                        L.video + static_cast<size_t>(L.schedule[0] % L.ring) * L.channels * plane_values;
#pragma unroll
                    for (int j = 0; j < PLANES; ++j) {
                        const int e = 2 * (lane + 32 * j);
                        const int q = e >> 6, py = (e >> 3) & 7, px = e & 7;
                        const int c = q / L.Pt, tt = q % L.Pt;
                        const float* src = anchor_frame + (static_cast<size_t>(tt) * L.channels + c) * plane_values +
                                           static_cast<size_t>(a.y + py) * L.width + a.x + px;
                        refv[j][0] = n < count ? __ldg(src) : 0.0f;
                        refv[j][1] = n < count ? __ldg(src + 1) : 0.0f;
                    }
                }
                float cur[PLANES][3], nxt[PLANES][3];
                auto load_row = [&](int r, float (&s)[PLANES][3]) {
                    const int gy = yl + r;
                    const bool row_in = gy < L.height;
                    const int x0 = rx0 + lane;
#pragma unroll
                    for (int q = 0; q < PLANES; ++q) {
                        const int c = q / L.Pt, tt = q % L.Pt;
                        const float* src = L.video + (static_cast<size_t>(frame % L.ring + tt) * L.channels + c) * plane_values +
                                           static_cast<size_t>(row_in ? gy : 0) * L.width;
                        s[q][0] = row_in && x0 < L.width ? __ldg(src + x0) : 0.0f;
                        s[q][1] = row_in && x0 + 32 < L.width ? __ldg(src + x0 + 32) : 0.0f;
                        s[q][2] = row_in && lane < P - 1 && x0 + 64 < L.width ? __ldg(src + x0 + 64) : 0.0f;
                    }
                };
                if (warp < R) load_row(warp, cur);
                wait(free_bar(bars, b), ((i >> 1) & 1) ^ 1);
                unsigned char* st = smem + b * lay.stage_bytes;
                unsigned char* hank = st + lay.hank;
                uint32_t* b32 = reinterpret_cast<uint32_t*>(st + lay.bop);
                float* nb = reinterpret_cast<float*>(st + lay.nb);
                StageMeta* meta = reinterpret_cast<StageMeta*>(st + lay.meta);
                if (threadIdx.x < kChosenAnchors) {
                    const int m = threadIdx.x;
                    int xl = 0, xh = -1;
                    if (m < count) spatial_range(L.anchors[strip.first + m].x, L.width, P, L.search_window, xl, xh);
                    meta->win_lo[m] = xl - rx0;
                    meta->win_wx[m] = xh - xl + 1;
                }
                if (threadIdx.x == 0) {
                    meta->first = strip.first;
                    meta->count = count;
                    meta->k = k;
                }
                {
                    // B operand and reference norm: warp n takes anchor n (row
                    // n of block (q * 8 + py, 0)) and zeroes row n of block
                    // (q * 8 + py, 1); absent anchors are zero
                    float acc = 0.0f;
#pragma unroll
                    for (int j = 0; j < PLANES; ++j) {
                        const int e = 2 * (lane + 32 * j);
                        const int qpy = e >> 3, px = e & 7;
                        acc = fmaf(refv[j][0], refv[j][0], acc);
                        acc = fmaf(refv[j][1], refv[j][1], acc);
                        b32[(((qpy * 2) * 8 + n) * 8 + px) >> 1] = pack_bf16(refv[j][0], refv[j][1]);
                        b32[(((qpy * 2 + 1) * 8 + n) * 8 + px) >> 1] = 0u;
                    }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
                    if (lane == 0) meta->na[n] = acc;
                }
                // BF16 blocks and row sums of squares, one region row per warp:
                // lane l holds samples l, l + 32 and l + 64 (l < 7) of the row;
                // block row c (= 8 b + i) is samples c .. c + 7, for c = l and
                // c = l + 32.  The next row's samples are loaded ahead.
                for (int r = warp; r < R; r += kProducerWarps) {
                    if (r + kProducerWarps < R) load_row(r + kProducerWarps, nxt);
                    float sq0 = 0.0f, sq1 = 0.0f;
#pragma unroll
                    for (int q = 0; q < PLANES; ++q) {
                        float av[8], bv[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            // source lane m = (lane + j) % 32 serves lane m - j
                            // (no wrap: wants its sample m) when m >= j, else
                            // lane m - j + 32 (wrap: wants its sample m + 64)
                            const int from = (lane + j) & 31;
                            const float f1 = __shfl_sync(0xffffffffu, cur[q][1], from);
                            const float f02 = __shfl_sync(0xffffffffu, lane >= j ? cur[q][0] : cur[q][2], from);
                            const bool wrap = lane + j >= 32;
                            av[j] = wrap ? f1 : f02;  // sample lane + j
                            bv[j] = wrap ? f02 : f1;  // sample lane + 32 + j
                        }
                        uint4* dst = reinterpret_cast<uint4*>(hank + (q * R + r) * 1024);
                        dst[lane] = make_uint4(pack_bf16(av[0], av[1]), pack_bf16(av[2], av[3]),
                                               pack_bf16(av[4], av[5]), pack_bf16(av[6], av[7]));
                        dst[lane + 32] = make_uint4(pack_bf16(bv[0], bv[1]), pack_bf16(bv[2], bv[3]),
                                                    pack_bf16(bv[4], bv[5]), pack_bf16(bv[6], bv[7]));
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            sq0 = fmaf(av[j], av[j], sq0);
                            sq1 = fmaf(bv[j], bv[j], sq1);
                        }
                    }
                    rowsq[r * kChosenCols + lane] = sq0;
                    rowsq[r * kChosenCols + lane + 32] = sq1;
#pragma unroll
                    for (int q = 0; q < PLANES; ++q)
#pragma unroll
                        for (int e = 0; e < 3; ++e) cur[q][e] = nxt[q][e];
                }
                producer_sync();  // row sums complete
                for (int it = threadIdx.x; it < 2 * pairs * kChosenCols; it += kProducerWarps * 32) {
                    const int y = it / kChosenCols, c = it - y * kChosenCols;
                    float acc = 0.0f;
#pragma unroll
                    for (int r = 0; r < P; ++r) acc += rowsq[(y + r) * kChosenCols + c];
                    nb[it] = acc;
                }
                fence_async_shared();
                producer_sync();  // stage complete; the row sums free for the next item
                if (threadIdx.x == 0) mbar_arrive(full_bar(bars, b));
            }
        }
    } else if (warp == kMmaWarp) {
        int i = 0;
        for (int si = blockIdx.x; si < L.strip_count; si += gridDim.x) {
            for (int k = 0; k < T; ++k, ++i) {
                const int b = i & 1;
                wait(full_bar(bars, b), (i >> 1) & 1);
                // after a wait ran out no further MMA is issued (the whole
                // warp agrees); L.stall_mma, a test switch, issues none at
                // all so that the consumers' waits run out
                timed_out = __any_sync(0xffffffffu, timed_out);
                if (timed_out || L.stall_mma) continue;
                tc_fence_after();
                {
                    const unsigned char* st = smem + b * lay.stage_bytes;
                    const uint32_t ha = smem_addr(st + lay.hank), ba = smem_addr(st + lay.bop);
                    const uint32_t td = tmem + static_cast<uint32_t>(b * kChosenTmemCols);
                    const uint32_t leader = lane == 0 ? 1u : 0u;
                    for (int p = 0; p < pairs; ++p) {
#pragma unroll
                        for (int s = 0; s < PLANES * 4; ++s) {
                            const int q = s >> 2, py = 2 * (s & 3);
                            const uint64_t ad = tc_desc(ha + (q * R + 2 * p + py) * 1024, 1024, 128);
                            const uint64_t bd = tc_desc(ba + (q * P + py) * 256, 256, 128);
                            tc_mma(td + p * kTcN, ad, bd, s > 0 ? 1u : 0u, leader);
                        }
                    }
                    tc_commit(tfull_bar(bars, b), leader);
                }
                __syncwarp();
            }
        }
    } else if (warp < kProducerWarps + kConsumerWarps) {
        const int quarter = warp & 3;
        const int m = 32 * quarter + lane;  // accumulator row: candidate row 2p + m / 64, column m % 64
        const int dy = m >> 6, x = m & 63;
        int i = 0;
        for (int si = blockIdx.x; si < L.strip_count; si += gridDim.x) {
            for (int k = 0; k < T; ++k, ++i) {
                const int b = i & 1;
                const uint32_t parity = (i >> 1) & 1;
                wait(full_bar(bars, b), parity);  // the stage's metadata (producers' writes)
                wait(tfull_bar(bars, b), parity);
                tc_fence_after();
                const unsigned char* st = smem + b * lay.stage_bytes;
                const float* nb = reinterpret_cast<const float*>(st + lay.nb);
                const StageMeta* meta = reinterpret_cast<const StageMeta*>(st + lay.meta);
                const int count = meta->count;
                // per anchor: this lane's window column (or -1), row stride,
                // reference norm and output base
                int rel[kChosenAnchors], wx[kChosenAnchors];
                float na[kChosenAnchors];
                float* out[kChosenAnchors];
#pragma unroll
                for (int n = 0; n < kChosenAnchors; ++n) {
                    const int r0 = x - meta->win_lo[n];
                    wx[n] = meta->win_wx[n];
                    rel[n] = n < count && r0 >= 0 && r0 < wx[n] ? r0 : -1;
                    na[n] = meta->na[n];
                    out[n] = L.approx_dist + static_cast<size_t>(meta->first + n) * L.approx_stride +
                             static_cast<size_t>(meta->k) * L.window_cells;
                }
                const uint32_t ta = tmem + (static_cast<uint32_t>(32 * quarter) << 16) +
                                    static_cast<uint32_t>(b * kChosenTmemCols);
                for (int p0 = 0; p0 < pairs; p0 += 2) {
                    uint32_t v[32];
                    tmem_load32(ta + static_cast<uint32_t>(p0 * kTcN), v);
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int cy = 2 * (p0 + h) + dy;
                        if (cy >= Wy) continue;
                        const float bn = nb[cy * kChosenCols + x];
#pragma unroll
                        for (int n = 0; n < kChosenAnchors; ++n)
                            if (rel[n] >= 0)
                                out[n][cy * wx[n] + rel[n]] = fmaxf(na[n] + bn - 2.0f * __uint_as_float(v[16 * h + n]), 0.0f);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(free_bar(bars, b));
            }
        }
    }
    // release the tensor memory once every MMA issued has completed: a
    // commit of all of them to the drain barrier, waited for with a bound,
    // also after a timeout left MMAs unread
    tc_fence_before();
    __syncthreads();
    if (warp == kMmaWarp) {
        tc_fence_after();
        tc_commit(drain, lane == 0 ? 1u : 0u);
        int polls = 0;
        while (!mbar_try_wait(drain, 0) && ++polls < kSpinLimit) {
        }
        if (polls >= kSpinLimit) atomicCAS(L.status, 0, kStatusTensorTimeout);
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kPipeTmemCols)
                     : "memory");
    }
}

// Steps 2-4 for one anchor per warp, from the approximate distances.
template <int PLANES>
__global__ void __launch_bounds__(kTcThreads) tc_select_kernel(MatchLaunch L) {
    __shared__ float sorted_d[kChosenWarps][32];
    __shared__ int sorted_i[kChosenWarps][32];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    constexpr int P = kPatch;
    const int gi = blockIdx.x * kChosenWarps + warp;
    if (gi >= L.anchor_count) return;  // no block-wide synchronisation below
    const int2 anchor = L.anchors[gi];
    int xl, xh, yl, yh;
    spatial_range(anchor.x, L.width, P, L.search_window, xl, xh);
    spatial_range(anchor.y, L.height, P, L.search_window, yl, yh);
    const int Wx = xh - xl + 1;
    const int cells = Wx * (yh - yl + 1);
    const size_t plane_values = static_cast<size_t>(L.height) * L.width;
    const float* approx = L.approx_dist + static_cast<size_t>(gi) * L.approx_stride;
    const float* anchor_frame = L.video + static_cast<size_t>(L.schedule[0] % L.ring) * L.channels * plane_values;

    // selection state (the plain matcher's WarpSelect)
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
        // the CPU's sequential selection over frame k (raster order) on the
        // approximate distances: the K-smallest front and the capped buffer,
        // buffer slot i in lane i (the plain matcher's register replay)
        const float* dk = approx + k * L.window_cells;
        float next = lane < cells ? __ldg(dk + lane) : kInf;
        for (int base = 0; base < cells; base += 32) {
            const int idx = base + lane;
            const float mine = next;
            next = idx + 32 < cells ? __ldg(dk + idx + 32) : kInf;  // the next chunk in flight
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
    }
    // exact FP32 distance of every entry left in the buffer (slot i in lane
    // i), in the plain form's arithmetic order: once, after the last frame
    if (lane < s.count) {
        const int i = reg_id & 0xfffff;
        const int cy = i / Wx;
        const int col = xl + (i - cy * Wx);
        const int frame = L.schedule[reg_id >> 20];
        float d = 0.0f;
#pragma unroll 1
        for (int q = 0; q < PLANES; ++q) {
            const int c = q / L.Pt, t = q % L.Pt;
            const float* rp = anchor_frame + (static_cast<size_t>(t) * L.channels + c) * plane_values +
                              static_cast<size_t>(anchor.y) * L.width + anchor.x;
            const float* cp = L.video + (static_cast<size_t>(frame % L.ring + t) * L.channels + c) * plane_values +
                              static_cast<size_t>(yl + cy) * L.width + col;
            // the candidate's samples first (all loads in flight), the
            // reference rows (one address for the whole warp) as they are used
            float cv[P][P];
#pragma unroll
            for (int r = 0; r < P; ++r)
#pragma unroll
                for (int ii = 0; ii < P; ++ii) cv[r][ii] = __ldg(cp + static_cast<size_t>(r) * L.width + ii);
#pragma unroll
            for (int r = 0; r < P; ++r) {
                const float* rr = rp + static_cast<size_t>(r) * L.width;
                float2 a2[4], b2[4];
#pragma unroll
                for (int ii = 0; ii < 4; ++ii) {
                    a2[ii] = make_float2(__ldg(rr + 2 * ii), __ldg(rr + 2 * ii + 1));
                    b2[ii] = make_float2(cv[r][2 * ii], cv[r][2 * ii + 1]);
                }
                d = row_ssd8_x2(d, a2, b2);
            }
        }
        reg_exact = d;
    }

    // select_similar_patches on the exact distances of the buffer: the K
    // smallest, the threshold max(tau, d_K), the entries within it, closest
    // first (ties by candidate order), at most the cap
    float* sd = sorted_d[warp];
    int* si = sorted_i[warp];
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

bool chosen_match_supported(int P, int planes_n, int window_w, int window_h) {
    return P == kPatch && planes_n >= 1 && planes_n <= 3 && window_w <= kChosenCols && window_h <= kChosenMaxRows;
}

size_t chosen_match_shared_bytes(const MatchLaunch& L) {
    const int planes_n = L.search_channels * L.Pt;
    const PipeLayout lay = pipe_layout(planes_n, (L.window_rows + 1) / 2);
    return static_cast<size_t>(lay.bytes > kMinSharedBytes ? lay.bytes : kMinSharedBytes);
}

cudaError_t launch_match_chosen(const MatchLaunch& L, int strips, cudaStream_t stream) {
    if (strips <= 0) return cudaSuccess;
    const int planes_n = L.search_channels * L.Pt;
    if (L.P != kPatch || planes_n < 1 || planes_n > 3 || L.window_rows > kChosenMaxRows || !L.status ||
        !L.approx_dist || L.approx_stride < L.schedule_len * L.window_cells || L.strip_count != strips)
        return cudaErrorInvalidValue;
    int device = 0, sms = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return err;
    err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err != cudaSuccess) return err;
    const size_t smem = chosen_match_shared_bytes(L);
    // a quarter of the SMs stays free for the other pipeline lane's kernels
    // (measured: +1.5% frames/s at 1080p over a grid of every SM)
    const int persistent = sms - sms / 4;
    const int grid = strips < persistent ? strips : persistent;
    const int select_blocks = (L.anchor_count + kChosenWarps - 1) / kChosenWarps;
    auto launch = [&](auto distance, auto select) {
        err = cudaFuncSetAttribute(distance, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (err != cudaSuccess) return;
        distance<<<grid, kPipeThreads, smem, stream>>>(L);
        err = cudaGetLastError();
        if (err != cudaSuccess || select_blocks <= 0) return;
        select<<<select_blocks, kTcThreads, 0, stream>>>(L);
        err = cudaGetLastError();
    };
    switch (planes_n) {
        case 1: launch(tc_distance_kernel<1>, tc_select_kernel<1>); break;
        case 2: launch(tc_distance_kernel<2>, tc_select_kernel<2>); break;
        default: launch(tc_distance_kernel<3>, tc_select_kernel<3>); break;
    }
    return err;
}

}  // namespace vnlbgpu
