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
// Three kernels.  A small one computes each strip's plane offsets (below);
// the distance kernel computes step 1 for every anchor and candidate and
// writes the approximate distances to global memory ([anchor][scheduled
// frame][window row][window column], 4 bytes each: the 82-87 MB of a 1080p
// anchor frame cross HBM in tens of microseconds); the selection kernel runs
// steps 2-4 with one warp per anchor at full occupancy.
//
// Samples are staged minus a per-strip, per-plane offset (the mean of the
// strip's first anchor's reference patch).  A distance does not change, but
// the BF16 roundings then scale with the samples' spread around the local
// level rather than with the level: at low noise the approximate distance
// is a small difference of large norms, and without the offset sigma-5
// clips lost 0.05 dB against the plain form.
//
// Distance kernel.  One CTA takes a strip of up to 8 consecutive anchors of
// each of one or two consecutive grid rows (anchor slots 0-7 and 8-15),
// whose search windows lie within 64 consecutive candidate columns and span
// at most 32 rows.  Pairing two grid rows fills the MMA's 16 anchor columns
// (a strip of one row fills about 6 at step 8), so each staged region row
// serves twice the anchors.  Per scheduled frame, and per group of up to
// three planes of it:
//
//   a. The strip's search region is read from global memory once (each
//      producer warp loads its rows of the plane group ahead of the stage
//      wait) and written to shared memory as BF16 core matrices of the
//      tcgen05 no-swizzle
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
//      (no bank conflicts).  The same pass sums the squares of the P-sample
//      row segments (candidate norms).  7 x 7 patches use the same 8 x 8
//      blocks: the reference operand's eighth column and eighth row are zero,
//      so the eighth sample of every block row adds nothing.
//   b. One thread issues, per pair of candidate rows p, the M = 128 x N = 16 x
//      K = 16 MMAs over the patch rows and the group's planes into
//      tensor-memory columns 16 p .. 16 p + 15 (column n = anchor slot n;
//      reference rows of empty slots are zero), accumulating over the
//      plane groups of the frame, and commits them to mbarriers: one that
//      frees the group's shared-memory stage, and after the last group one
//      that hands the accumulators to the readers.
//   c. The 4 reader warps read the accumulators back (tcgen05.ld; warp w
//      reads TMEM lanes 32 (w % 4) .. + 31, i.e. candidate row
//      2p + (w % 4) / 2, columns 32 (w % 2) .. + 31) and store each anchor's
//      window distances (rows relative to that anchor's own window).
//
// A frame of more planes than one shared-memory stage holds (vnlbcu's
// defaults: 3 channels x patch_time 2 = 6 planes of a 27-row window) takes
// several stages, so shared-memory stages and tensor-memory halves turn over
// separately: a stage is free once its MMAs completed, a tensor-memory half
// once its readers are done.
//
// Tensor memory: each CTA allocates 2 x kChosenTmemCols columns and holds
// one CTA per SM (launch bounds and shared memory), so allocations never
// wait on each other.  Every mbarrier wait is bounded: when one runs out the
// kernel records kStatusTensorTimeout in the session status word, which the
// host turns into an error, and carries on without spinning further.
#include <cuda_bf16.h>

#include <cstdint>

#include "vnlb_kernels.h"

#ifndef VNLB_TC_SPARE_SMS
#define VNLB_TC_SPARE_SMS 1
#endif

namespace vnlbgpu {
namespace {

constexpr int kTcThreads = 32 * kChosenWarps;
constexpr int kBlock = 8;  // core-matrix side: patch rows and columns are padded to 8
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
constexpr int kStages = 2;  // shared-memory stages, and tensor-memory halves
constexpr int kPipeTmemCols = kStages * kChosenTmemCols;
constexpr int kMaxPlaneGroup = 3;
// region rows per producer warp and plane group (at most 2 * 16 + 7 rows)
constexpr int kRowsPerWarp = (2 * kChosenMaxRows / 2 + kBlock - 1 + kProducerWarps - 1) / kProducerWarps;
// shared memory of at least this size keeps a second distance CTA (and its
// tensor-memory allocation) off the SM
constexpr int kMinSharedBytes = 116 * 1024;
constexpr int kSharedLimit = 227 * 1024;

// Per-item window metadata and reference norms (producers -> readers), one
// per tensor-memory half.  Anchor slot n is anchor n % 8 of grid row n / 8
// of the strip.
struct StageMeta {
    int k;        // scheduled frame
    int rows;     // window rows the strip's anchors span
    int off1;     // first window row of the second grid row's anchors
    int h[2];     // window rows of each grid row's anchors
    int pad[3];
    int win_lo[kTcN];  // window columns relative to the strip origin
    int win_wx[kTcN];  // 0: no anchor in the slot
    int gi[kTcN];      // anchor index
    float na[kTcN];    // reference norms
};

// The rows of a strip's windows: yl of the first grid row's anchors, and the
// rows spanned from there to the last row of the second grid row's.
__device__ __forceinline__ void strip_rows(const MatchLaunch& L, const TcStrip& st, int& yl0, int& yh0, int& yl1,
                                           int& yh1) {
    spatial_range(st.y[0], L.height, L.P, L.search_window, yl0, yh0);
    yl1 = yl0;
    yh1 = yh0;
    if (st.count[1] > 0) spatial_range(st.y[1], L.height, L.P, L.search_window, yl1, yh1);
}

// Shared-memory layout of the distance kernel in bytes (128-byte aligned
// parts): two stages of [BF16 blocks | reference blocks] for `group` planes,
// then per tensor-memory half the candidate norms and the metadata, the
// producers' row sums, the mbarriers and the tensor-memory address.
struct PipeLayout {
    int hank, bop, stage_bytes, nb, meta, rowsq, bars, tmem, bytes;
};

__host__ __device__ inline int align128(int v) { return (v + 127) & ~127; }

__host__ __device__ inline int region_rows(int pairs) { return 2 * pairs + kBlock - 1; }

__host__ __device__ inline PipeLayout pipe_layout(int group, int pairs) {
    const int R = region_rows(pairs);
    PipeLayout l{};
    int off = 0;
    l.hank = off;  off = align128(off + group * R * 8 * 128);           // [q][r][b] 8x8 BF16 blocks
    l.bop = off;   off = align128(off + group * kBlock * 2 * 128);      // [q][py][n/8] 8x8 BF16 blocks
    l.stage_bytes = off;
    off = kStages * l.stage_bytes;
    l.nb = off;    off = align128(off + kStages * 2 * pairs * kChosenCols * 4);  // candidate norms per half
    l.meta = off;  off = align128(off + kStages * static_cast<int>(sizeof(StageMeta)));
    l.rowsq = off; off = align128(off + R * kChosenCols * 4);           // row sums of squares
    l.bars = off;  off += 5 * kStages * 8;
    l.tmem = off;  off += 8;
    l.bytes = align128(off);
    return l;
}

// planes per shared-memory stage: the most (up to three) whose two stages
// fit in shared memory
inline int plane_group(int planes_n, int pairs) {
    for (int g = planes_n < kMaxPlaneGroup ? planes_n : kMaxPlaneGroup; g > 1; --g)
        if (pipe_layout(g, pairs).bytes <= kSharedLimit) return g;
    return 1;
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

// stage s filled (producers -> issuer); stage s consumed by its MMAs (MMA
// completion -> producers); half h accumulated (MMA completion -> readers);
// half h read (readers -> issuer, producers); half h's norms and metadata
// written (producers -> readers)
__device__ __forceinline__ uint32_t full_bar(uint32_t bars, int s) { return bars + 8 * s; }
__device__ __forceinline__ uint32_t sfree_bar(uint32_t bars, int s) { return bars + 8 * (kStages + s); }
__device__ __forceinline__ uint32_t tfull_bar(uint32_t bars, int h) { return bars + 8 * (2 * kStages + h); }
__device__ __forceinline__ uint32_t tfree_bar(uint32_t bars, int h) { return bars + 8 * (3 * kStages + h); }
__device__ __forceinline__ uint32_t mfull_bar(uint32_t bars, int h) { return bars + 8 * (4 * kStages + h); }

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

// The offset of each plane of each strip: the mean of the strip's first
// anchor's reference patch, one warp per strip.  The distance kernel stages
// candidates and references minus it (a distance does not change), so that
// the BF16 roundings scale with the samples' spread around the local level
// rather than with the level itself: at low noise the approximate distances
// are small differences of large norms.
template <int P>
__global__ void __launch_bounds__(256) strip_offsets_kernel(MatchLaunch L) {
    const int si = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (si >= L.strip_count) return;
    const TcStrip st = L.tc_strips[si];
    const int2 a = L.anchors[st.count[0] > 0 ? st.first[0] : st.first[1]];
    const size_t plane_values = static_cast<size_t>(L.height) * L.width;
    const float* frame = L.video + static_cast<size_t>(L.schedule[0] % L.ring) * L.channels * plane_values;
    const int planes_n = L.search_channels * L.Pt;
    for (int q = 0; q < planes_n; ++q) {
        const int c = q / L.Pt, t = q % L.Pt;
        const float* src = frame + (static_cast<size_t>(t) * L.channels + c) * plane_values +
                           static_cast<size_t>(a.y) * L.width + a.x;
        float sum = 0.0f;
        for (int e = lane; e < P * P; e += 32) sum += __ldg(src + static_cast<size_t>(e / P) * L.width + e % P);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) L.strip_mu[static_cast<size_t>(si) * kChosenMaxPlanes + q] = sum / static_cast<float>(P * P);
    }
}

// Persistent, warp-specialised distance kernel.  Each CTA walks the items
// (strip, scheduled frame) of strips blockIdx.x, blockIdx.x + gridDim.x, ...;
// item i takes tensor-memory half i % 2 and fills shared-memory stages with
// its plane groups, fill j in stage j % 2:
//   warps 0-7   producers: per plane group fill a stage (BF16 blocks and
//               reference blocks) and arrive on full; after the last group
//               write the half's norms and metadata and arrive on mfull;
//   warp 12     issuer: per plane group wait full, issue the MMAs into the
//               item's tensor-memory half, commit them to sfree (the
//               producers' wait before refilling the stage); after the last
//               group commit to tfull;
//   warps 8-11  readers (TMEM lane quarters 0-3): wait mfull and tfull, read
//               the accumulators back, store the distances, arrive on tfree,
//               which the issuer and the producers wait for before reusing
//               the half.
template <int P, int G>  // patch size (7 or 8), planes per shared-memory stage
// 128 registers per thread: the 13 warps spread over the SM's four
// 16,384-register partitions 4-3-3-3, and 4 warps x 32 x 128 fill one.
__global__ void __launch_bounds__(kPipeThreads, 1) tc_distance_kernel(MatchLaunch L) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int Wy = L.window_rows;
    const int pairs = (Wy + 1) >> 1;
    const int R = region_rows(pairs);
    const PipeLayout lay = pipe_layout(G, pairs);
    const uint32_t bars = smem_addr(smem + lay.bars);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + lay.tmem);
    float* rowsq = reinterpret_cast<float*>(smem + lay.rowsq);
    const size_t plane_values = static_cast<size_t>(L.height) * L.width;
    const int T = L.schedule_len;
    const int planes_n = L.search_channels * L.Pt;
    const int groups = (planes_n + G - 1) / G;
    const int nb_floats = 2 * pairs * kChosenCols;

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
            mbar_init(sfree_bar(bars, s), 1);
            mbar_init(tfull_bar(bars, s), 1);
            mbar_init(tfree_bar(bars, s), kConsumerWarps);
            mbar_init(mfull_bar(bars, s), 1);
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
        int i = 0, j = 0;
        const float* anchor_frame =
            L.video + static_cast<size_t>(L.schedule[0] % L.ring) * L.channels * plane_values;
        for (int si = blockIdx.x; si < L.strip_count; si += gridDim.x) {
            const TcStrip strip = L.tc_strips[si];
            int yl, yh0, yl1, yh1;
            strip_rows(L, strip, yl, yh0, yl1, yh1);
            const int wy = yh1 - yl + 1;
            const int Rs = region_rows((wy + 1) >> 1);  // region rows this strip uses
            const int nb_used = 2 * ((wy + 1) >> 1) * kChosenCols;
            const int rx0 = strip.region_x;
            // the anchors whose reference rows this warp stages: slot warp
            // (first grid row) and slot warp + 8 (second grid row)
            int2 anc[2];
            bool has[2];
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                has[half] = warp < strip.count[half];
                anc[half] = has[half] ? L.anchors[strip.first[half] + warp] : make_int2(0, 0);
            }
            // the strip's offset of each plane (strip_offsets_kernel):
            // candidates and references are staged minus it
            const float* mu = L.strip_mu + static_cast<size_t>(si) * kChosenMaxPlanes;
            for (int k = 0; k < T; ++k, ++i) {
                const int h = i & 1;
                const int frame = L.schedule[k];
                // the half's norms and metadata are rewritten below: its
                // readers must be done with item i - 2
                wait(tfree_bar(bars, h), ((i >> 1) & 1) ^ 1);
                StageMeta* meta = reinterpret_cast<StageMeta*>(smem + lay.meta) + h;
                float* nb = reinterpret_cast<float*>(smem + lay.nb) + h * nb_floats;
                if (threadIdx.x < kTcN) {
                    const int m = threadIdx.x, row = m >> 3, idx = m & 7;
                    int xl = 0, xh = -1, gi = 0;
                    if (idx < strip.count[row]) {
                        gi = strip.first[row] + idx;
                        spatial_range(L.anchors[gi].x, L.width, P, L.search_window, xl, xh);
                    }
                    meta->win_lo[m] = xl - rx0;
                    meta->win_wx[m] = xh - xl + 1;
                    meta->gi[m] = gi;
                }
                if (threadIdx.x == 0) {
                    meta->k = k;
                    meta->rows = wy;
                    meta->off1 = yl1 - yl;
                    meta->h[0] = yh0 - yl + 1;
                    meta->h[1] = yh1 - yl1 + 1;
                }
                float na[2] = {0.0f, 0.0f};
                for (int g = 0; g < groups; ++g, ++j) {
                    const int b = j & 1;
                    const int q0 = g * G;
                    // this warp's region rows r = warp + 8 rr of the group:
                    // the first kPre loaded before the stage wait (their
                    // latency overlaps the stage's previous MMAs), each later
                    // one as soon as a register slot is free
                    constexpr int kPre = G == 1 ? kRowsPerWarp : 3;
                    float rowv[kPre][G][3];
                    auto load_row = [&](int r, float (&v)[G][3]) {
                        const int gy = yl + r;
                        const bool row_in = gy < L.height;
                        const int x0 = rx0 + lane;
#pragma unroll
                        for (int ql = 0; ql < G; ++ql) {
                            const int q = q0 + ql;
                            const bool in = row_in && q < planes_n;
                            const int c = q / L.Pt, tt = q % L.Pt;
                            const float* src =
                                L.video + (static_cast<size_t>(frame % L.ring + tt) * L.channels + c) * plane_values +
                                static_cast<size_t>(row_in ? gy : 0) * L.width;
                            // the loads only: their results are used (and the
                            // offset taken off) when the row is staged
                            v[ql][0] = in && x0 < L.width ? __ldg(src + x0) : 0.0f;
                            v[ql][1] = in && x0 + 32 < L.width ? __ldg(src + x0 + 32) : 0.0f;
                            v[ql][2] = in && lane < kBlock - 1 && x0 + 64 < L.width ? __ldg(src + x0 + 64) : 0.0f;
                        }
                    };
#pragma unroll
                    for (int rr = 0; rr < kPre; ++rr)
                        if (warp + kProducerWarps * rr < Rs) load_row(warp + kProducerWarps * rr, rowv[rr]);
                    // the group's plane offsets (samples outside the frame, never
                    // part of a window's patches, become -offset: unused)
                    float mq[G];
#pragma unroll
                    for (int ql = 0; ql < G; ++ql) mq[ql] = q0 + ql < planes_n ? __ldg(mu + q0 + ql) : 0.0f;
                    // the stage's MMAs of fill j - 2 have completed
                    wait(sfree_bar(bars, b), ((j >> 1) & 1) ^ 1);
                    unsigned char* st = smem + b * lay.stage_bytes;
                    unsigned char* hank = st + lay.hank;
                    uint32_t* b32 = reinterpret_cast<uint32_t*>(st + lay.bop);
#pragma unroll
                    for (int half = 0; half < 2; ++half) {
                        // B operand: the warp writes the rows of anchor slot
                        // warp + 8 half (row `warp` of block (q * 8 + py,
                        // half)), in pairs of columns; absent anchors, planes
                        // past the last, and a 7 x 7 patch's eighth row and
                        // column are zero
#pragma unroll
                        for (int jj = 0; jj < G; ++jj) {
                            const int e = 2 * (lane + 32 * jj);
                            const int ql = e >> 6, py = (e >> 3) & 7, px = e & 7;
                            const int q = q0 + ql;
                            float r0 = 0.0f, r1 = 0.0f;
                            if (has[half] && q < planes_n && py < P && px < P) {
                                const int c = q / L.Pt, tt = q % L.Pt;
                                const float* src = anchor_frame +
                                                   (static_cast<size_t>(tt) * L.channels + c) * plane_values +
                                                   static_cast<size_t>(anc[half].y + py) * L.width + anc[half].x + px;
                                const float m = __ldg(mu + q);
                                r0 = __ldg(src) - m;
                                if (px + 1 < P) r1 = __ldg(src + 1) - m;
                            }
                            na[half] = fmaf(r0, r0, na[half]);
                            na[half] = fmaf(r1, r1, na[half]);
                            b32[((((e >> 3) * 2 + half) * 8 + warp) * 8 + px) >> 1] = pack_bf16(r0, r1);
                        }
                    }
                    // BF16 blocks and row sums of squares, one region row per
                    // warp: lane l holds samples l, l + 32 and l + 64 (l < 7)
                    // of the row; block row c (= 8 b + i) is samples c .. c + 7,
                    // for c = l and c = l + 32.  The row sums add up over plane
                    // groups.
#pragma unroll
                    for (int rr = 0; rr < kRowsPerWarp; ++rr) {
                        const int r = warp + kProducerWarps * rr;
                        if (r >= Rs) break;
                        float (&cur)[G][3] = rowv[rr % kPre];
#pragma unroll
                        for (int ql = 0; ql < G; ++ql)
#pragma unroll
                            for (int e = 0; e < 3; ++e) cur[ql][e] -= mq[ql];
                        float sq0 = 0.0f, sq1 = 0.0f;
#pragma unroll
                        for (int ql = 0; ql < G; ++ql) {
                            float av[8], bv[8];
#pragma unroll
                            for (int jj = 0; jj < 8; ++jj) {
                                // source lane m = (lane + jj) % 32 serves lane
                                // m - jj (no wrap: wants its sample m) when
                                // m >= jj, else lane m - jj + 32 (wrap: wants
                                // its sample m + 64)
                                const int from = (lane + jj) & 31;
                                const float f1 = __shfl_sync(0xffffffffu, cur[ql][1], from);
                                const float f02 = __shfl_sync(0xffffffffu, lane >= jj ? cur[ql][0] : cur[ql][2], from);
                                const bool wrap = lane + jj >= 32;
                                av[jj] = wrap ? f1 : f02;  // sample lane + jj
                                bv[jj] = wrap ? f02 : f1;  // sample lane + 32 + jj
                            }
                            uint4* dst = reinterpret_cast<uint4*>(hank + (ql * R + r) * 1024);
                            dst[lane] = make_uint4(pack_bf16(av[0], av[1]), pack_bf16(av[2], av[3]),
                                                   pack_bf16(av[4], av[5]), pack_bf16(av[6], av[7]));
                            dst[lane + 32] = make_uint4(pack_bf16(bv[0], bv[1]), pack_bf16(bv[2], bv[3]),
                                                        pack_bf16(bv[4], bv[5]), pack_bf16(bv[6], bv[7]));
#pragma unroll
                            for (int jj = 0; jj < P; ++jj) {
                                sq0 = fmaf(av[jj], av[jj], sq0);
                                sq1 = fmaf(bv[jj], bv[jj], sq1);
                            }
                        }
                        // the slot is read: the row kPre rows further takes it
                        if (rr + kPre < kRowsPerWarp && r + kProducerWarps * kPre < Rs)
                            load_row(r + kProducerWarps * kPre, rowv[rr % kPre]);
                        if (g == 0) {
                            rowsq[r * kChosenCols + lane] = sq0;
                            rowsq[r * kChosenCols + lane + 32] = sq1;
                        } else {
                            rowsq[r * kChosenCols + lane] += sq0;
                            rowsq[r * kChosenCols + lane + 32] += sq1;
                        }
                    }
                    fence_async_shared();
                    producer_sync();  // stage complete (and, after the last group, the row sums)
                    if (threadIdx.x == 0) mbar_arrive(full_bar(bars, b));
                }
                // reference norms and candidate norms of the half
#pragma unroll
                for (int half = 0; half < 2; ++half) {
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) na[half] += __shfl_xor_sync(0xffffffffu, na[half], o);
                    if (lane == 0) meta->na[warp + 8 * half] = na[half];
                }
                for (int it = threadIdx.x; it < nb_used; it += kProducerWarps * 32) {
                    const int y = it / kChosenCols, c = it - y * kChosenCols;
                    float acc = 0.0f;
#pragma unroll
                    for (int r = 0; r < P; ++r) acc += rowsq[(y + r) * kChosenCols + c];
                    nb[it] = acc;
                }
                producer_sync();  // norms complete; the row sums free for the next item
                if (threadIdx.x == 0) mbar_arrive(mfull_bar(bars, h));
            }
        }
    } else if (warp == kMmaWarp) {
        int i = 0, j = 0;
        const uint32_t leader = lane == 0 ? 1u : 0u;
        for (int si = blockIdx.x; si < L.strip_count; si += gridDim.x) {
            const TcStrip strip = L.tc_strips[si];
            int yl, yh0, yl1, yh1;
            strip_rows(L, strip, yl, yh0, yl1, yh1);
            const int pairs_s = (yh1 - yl + 2) >> 1;  // row pairs this strip uses
            for (int k = 0; k < T; ++k, ++i) {
                const int h = i & 1;
                const uint32_t td = tmem + static_cast<uint32_t>(h * kChosenTmemCols);
                wait(tfree_bar(bars, h), ((i >> 1) & 1) ^ 1);
                for (int g = 0; g < groups; ++g, ++j) {
                    const int b = j & 1;
                    wait(full_bar(bars, b), (j >> 1) & 1);
                    // after a wait ran out no further MMA is issued (the whole
                    // warp agrees); L.stall_mma, a test switch, issues none at
                    // all so that the other roles' waits run out
                    timed_out = __any_sync(0xffffffffu, timed_out);
                    if (timed_out || L.stall_mma) continue;
                    tc_fence_after();
                    const unsigned char* st = smem + b * lay.stage_bytes;
                    const uint32_t ha = smem_addr(st + lay.hank), ba = smem_addr(st + lay.bop);
                    const int gq = planes_n - g * G < G ? planes_n - g * G : G;  // planes of this group
                    for (int p = 0; p < pairs_s; ++p) {
#pragma unroll
                        for (int s = 0; s < G * 4; ++s) {
                            const int ql = s >> 2, py = 2 * (s & 3);
                            if (ql >= gq) break;
                            const uint64_t ad = tc_desc(ha + (ql * R + 2 * p + py) * 1024, 1024, 128);
                            const uint64_t bd = tc_desc(ba + (ql * kBlock + py) * 256, 256, 128);
                            tc_mma(td + p * kTcN, ad, bd, (g > 0 || s > 0) ? 1u : 0u, leader);
                        }
                    }
                    tc_commit(sfree_bar(bars, b), leader);
                    if (g == groups - 1) tc_commit(tfull_bar(bars, h), leader);
                    __syncwarp();
                }
            }
        }
    } else if (warp < kProducerWarps + kConsumerWarps) {
        const int quarter = warp & 3;
        const int m = 32 * quarter + lane;  // accumulator row: candidate row 2p + m / 64, column m % 64
        const int dy = m >> 6, x = m & 63;
        int i = 0;
        for (int si = blockIdx.x; si < L.strip_count; si += gridDim.x) {
            for (int k = 0; k < T; ++k, ++i) {
                const int h = i & 1;
                const uint32_t parity = (i >> 1) & 1;
                wait(mfull_bar(bars, h), parity);  // the half's norms and metadata (producers' writes)
                wait(tfull_bar(bars, h), parity);
                // after a wait ran out the metadata may not be written yet:
                // the warp reads and stores nothing more (the status word
                // already reports the failure)
                timed_out = __any_sync(0xffffffffu, timed_out);
                if (timed_out) {
                    if (lane == 0) mbar_arrive(tfree_bar(bars, h));
                    continue;
                }
                tc_fence_after();
                const float* nb = reinterpret_cast<const float*>(smem + lay.nb) + h * nb_floats;
                const StageMeta* meta = reinterpret_cast<const StageMeta*>(smem + lay.meta) + h;
                const int wy = meta->rows, off1 = meta->off1, h0 = meta->h[0], h1 = meta->h[1];
                const unsigned kofs = static_cast<unsigned>(meta->k) * static_cast<unsigned>(L.window_cells);
                // per anchor slot: the offset o0 of this lane's column in
                // the anchor's frame-k distances at strip row 0 (so that
                // strip row cy is at o0 + cy * wx; 32-bit: the launch
                // checks the buffer's size), the row stride wx (0: the
                // column is outside the window), and the reference norm
                unsigned o0[kTcN];
                int wxs[kTcN];
                float na[kTcN];
#pragma unroll
                for (int n = 0; n < kTcN; ++n) {
                    const int r0 = x - meta->win_lo[n];
                    const int wxn = meta->win_wx[n];
                    const bool in = r0 >= 0 && r0 < wxn;
                    wxs[n] = in ? wxn : 0;
                    const int first_row = n < 8 ? 0 : off1;  // the anchor's window row 0 in strip rows
                    o0[n] = static_cast<unsigned>(meta->gi[n]) * static_cast<unsigned>(L.approx_stride) + kofs +
                            static_cast<unsigned>(r0 - first_row * wxn);
                    na[n] = meta->na[n];
                }
                const uint32_t ta = tmem + (static_cast<uint32_t>(32 * quarter) << 16) +
                                    static_cast<uint32_t>(h * kChosenTmemCols);
                const int pairs_s = (wy + 1) >> 1;
                for (int p0 = 0; p0 < pairs_s; p0 += 2) {
                    uint32_t v[32];
                    tmem_load32(ta + static_cast<uint32_t>(p0 * kTcN), v);
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {
                        const int cy = 2 * (p0 + hh) + dy;
                        if (cy >= wy) continue;
                        const float bn = nb[cy * kChosenCols + x];
                        // the strip rows of each grid row's windows
                        const bool in0 = cy < h0;
                        const bool in1 = static_cast<unsigned>(cy - off1) < static_cast<unsigned>(h1);
#pragma unroll
                        for (int n = 0; n < kTcN; ++n) {
                            if (wxs[n] == 0 || !(n < 8 ? in0 : in1)) continue;
                            L.approx_dist[o0[n] + static_cast<unsigned>(cy * wxs[n])] =
                                fmaxf(fmaf(-2.0f, __uint_as_float(v[16 * hh + n]), na[n] + bn), 0.0f);
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(tfree_bar(bars, h));
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

// Exact FP32 distance of candidate (frame, row y, column col) to the anchor,
// in the plain form's arithmetic order: planes (channel, t), patch rows, the
// row SSD of row_ssd (packed pairs for 8 samples).
template <int P>
__device__ __forceinline__ float exact_distance(const MatchLaunch& L, const float* anchor_frame, int2 anchor,
                                                int frame, int y, int col, int planes_n, size_t plane_values) {
    float d = 0.0f;
#pragma unroll 1
    for (int q = 0; q < planes_n; ++q) {
        const int c = q / L.Pt, t = q % L.Pt;
        const float* rp = anchor_frame + (static_cast<size_t>(t) * L.channels + c) * plane_values +
                          static_cast<size_t>(anchor.y) * L.width + anchor.x;
        const float* cp = L.video + (static_cast<size_t>(frame % L.ring + t) * L.channels + c) * plane_values +
                          static_cast<size_t>(y) * L.width + col;
        // the candidate's samples first (all loads in flight), the reference
        // rows (one address for the whole warp) as they are used
        float cv[P][P];
#pragma unroll
        for (int r = 0; r < P; ++r)
#pragma unroll
            for (int ii = 0; ii < P; ++ii) cv[r][ii] = __ldg(cp + static_cast<size_t>(r) * L.width + ii);
#pragma unroll
        for (int r = 0; r < P; ++r) {
            const float* rr = rp + static_cast<size_t>(r) * L.width;
            if constexpr (P == kLanes) {
                float2 a2[4], b2[4];
#pragma unroll
                for (int ii = 0; ii < 4; ++ii) {
                    a2[ii] = make_float2(__ldg(rr + 2 * ii), __ldg(rr + 2 * ii + 1));
                    b2[ii] = make_float2(cv[r][2 * ii], cv[r][2 * ii + 1]);
                }
                d = row_ssd8_x2(d, a2, b2);
            } else {
                d = row_ssd<P>(d, [&](int ii) { return __ldg(rr + ii); }, [&](int ii) { return cv[r][ii]; });
            }
        }
    }
    return d;
}

// Steps 2-4 for one anchor per warp, from the approximate distances.  The
// capped buffer's slot s lives in lane s % 32, register s / 32 (CW registers:
// buffers of up to 32 CW entries).
template <int P, int CW>
__global__ void __launch_bounds__(kTcThreads) tc_select_kernel(MatchLaunch L) {
    __shared__ float sorted_d[kChosenWarps][32 * CW];
    __shared__ int sorted_i[kChosenWarps][32 * CW];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int gi = blockIdx.x * kChosenWarps + warp;
    if (gi >= L.anchor_count) return;  // no block-wide synchronisation below
    const int2 anchor = L.anchors[gi];
    int xl, xh, yl, yh;
    spatial_range(anchor.x, L.width, P, L.search_window, xl, xh);
    spatial_range(anchor.y, L.height, P, L.search_window, yl, yh);
    const int Wx = xh - xl + 1;
    const int cells = Wx * (yh - yl + 1);
    const size_t plane_values = static_cast<size_t>(L.height) * L.width;
    const int planes_n = L.search_channels * L.Pt;
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
    unsigned reg_d[CW], reg_top = 0u;  // bits of non-negative distances
    int reg_id[CW];
    float reg_exact[CW];
#pragma unroll
    for (int w = 0; w < CW; ++w) {
        reg_d[w] = 0u;
        reg_id[w] = 0;
        reg_exact[w] = 0.0f;
    }
    // the buffer's largest distance and its lowest slot
    auto find_worst = [&]() {
        unsigned m = reg_d[0];
#pragma unroll
        for (int w = 1; w < CW; ++w) m = m > reg_d[w] ? m : reg_d[w];
        const unsigned wmax = __reduce_max_sync(0xffffffffu, m);
        s.worst = __uint_as_float(wmax);
#pragma unroll
        for (int w = CW - 1; w >= 0; --w) {
            const unsigned hit = __ballot_sync(0xffffffffu, reg_d[w] == wmax);
            if (hit) s.worst_idx = 32 * w + __ffs(hit) - 1;
        }
    };
    auto put = [&](int slot, float d, int id) {
#pragma unroll
        for (int w = 0; w < CW; ++w)
            if (slot >> 5 == w && lane == (slot & 31)) {
                reg_d[w] = __float_as_uint(d);
                reg_id[w] = id;
            }
    };

    for (int k = 0; k < L.schedule_len; ++k) {
        // the CPU's sequential selection over frame k (raster order) on the
        // approximate distances: the K-smallest front and the capped buffer;
        // kSelectBatch chunks of 32 candidates are loaded at once (the
        // replay of a chunk is short next to a load's latency; fewer for the
        // larger buffers, whose registers would spill)
        constexpr int kSelectBatch = CW == 1 ? 8 : 4;
        const float* dk = approx + k * L.window_cells;
        for (int base0 = 0; base0 < cells; base0 += 32 * kSelectBatch) {
          float vals[kSelectBatch];
#pragma unroll
          for (int b = 0; b < kSelectBatch; ++b) {
              const int idx = base0 + 32 * b + lane;
              vals[b] = idx < cells ? __ldg(dk + idx) : kInf;
          }
#pragma unroll
          for (int b = 0; b < kSelectBatch; ++b) {
            const int base = base0 + 32 * b;
            if (base >= cells) break;  // uniform
            const int idx = base + lane;
            const float mine = vals[b];
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
                    put(s.count, d, id);
                    s.count++;
                    if (s.count == s.cap) find_worst();
                } else if (d < s.worst) {
                    put(s.worst_idx, d, id);
                    find_worst();
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
    }
    // exact FP32 distance of every entry left in the buffer, in the plain
    // form's arithmetic order: once, after the last frame
#pragma unroll
    for (int w = 0; w < CW; ++w) {
        if (32 * w + lane < s.count) {
            const int i = reg_id[w] & 0xfffff;
            const int cy = i / Wx;
            reg_exact[w] = exact_distance<P>(L, anchor_frame, anchor, L.schedule[reg_id[w] >> 20], yl + cy,
                                             xl + (i - cy * Wx), planes_n, plane_values);
        }
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
        int rank[CW];
#pragma unroll
        for (int w = 0; w < CW; ++w) rank[w] = 0;
        for (int jj = 0; jj < n; ++jj) {
            float dsrc = reg_exact[0];
            int isrc = reg_id[0];
#pragma unroll
            for (int w = 1; w < CW; ++w)
                if (jj >> 5 == w) {
                    dsrc = reg_exact[w];
                    isrc = reg_id[w];
                }
            const float dj = __shfl_sync(0xffffffffu, dsrc, jj & 31);
            const int ij = __shfl_sync(0xffffffffu, isrc, jj & 31);
#pragma unroll
            for (int w = 0; w < CW; ++w)
                rank[w] += (dj < reg_exact[w] || (dj == reg_exact[w] && ij < reg_id[w])) ? 1 : 0;
        }
#pragma unroll
        for (int w = 0; w < CW; ++w)
            if (32 * w + lane < n) {
                sd[rank[w]] = reg_exact[w];
                si[rank[w]] = reg_id[w];
            }
        __syncwarp();
        const int selected = min(K, n);
        const float threshold = std_max(L.tau, sd[selected - 1]);
        int within = 0;
#pragma unroll
        for (int w = 0; w < CW; ++w)
            within += __popc(__ballot_sync(0xffffffffu, 32 * w + lane < n && sd[32 * w + lane] <= threshold));
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
    return (P == 7 || P == 8) && planes_n >= 1 && planes_n <= kChosenMaxPlanes && window_w <= kChosenCols &&
           window_h <= kChosenMaxRows;
}

int chosen_max_plane_group(int planes_n, int window_rows) { return plane_group(planes_n, (window_rows + 1) / 2); }

// planes per stage of a launch: the requested number when it fits, else the most that fit
static int launch_plane_group(const MatchLaunch& L) {
    const int most = chosen_max_plane_group(L.search_channels * L.Pt, L.window_rows);
    return L.plane_group > 0 && L.plane_group < most ? L.plane_group : most;
}

size_t chosen_match_shared_bytes(const MatchLaunch& L) {
    const int pairs = (L.window_rows + 1) / 2;
    const PipeLayout lay = pipe_layout(launch_plane_group(L), pairs);
    return static_cast<size_t>(lay.bytes > kMinSharedBytes ? lay.bytes : kMinSharedBytes);
}

cudaError_t launch_match_chosen(const MatchLaunch& L, int strips, cudaStream_t stream) {
    if (strips <= 0) return cudaSuccess;
    const int planes_n = L.search_channels * L.Pt;
    // entries the buffer can hold at once: the cap, or every candidate of
    // the window when there are fewer
    const long long candidates = static_cast<long long>(L.window_cells) * L.schedule_len;
    const int cap = L.soft_cap < candidates ? L.soft_cap : static_cast<int>(candidates);
    if (!chosen_match_supported(L.P, planes_n, kChosenCols, L.window_rows) || !L.status || !L.approx_dist ||
        !L.tc_strips || !L.strip_mu ||
        L.approx_stride < L.schedule_len * L.window_cells || L.strip_count != strips || L.K > 32 ||
        static_cast<unsigned long long>(L.anchor_count) * static_cast<unsigned long long>(L.approx_stride) >
            0xffffffffull ||
        cap > kChosenMaxBuffer || L.max_rows < cap)
        return cudaErrorInvalidValue;
    int device = 0, sms = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return err;
    err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (err != cudaSuccess) return err;
    const int group = launch_plane_group(L);
    const size_t smem = chosen_match_shared_bytes(L);
    if (smem > static_cast<size_t>(kSharedLimit)) return cudaErrorInvalidValue;
    // a quarter of the SMs stays free for the other pipeline lanes' kernels
    // (measured: +1.5% frames/s at 1080p over a grid of every SM; the build
    // parameter VNLB_TC_SPARE_SMS=0 takes every SM, for comparisons)
    const int persistent = VNLB_TC_SPARE_SMS ? sms - sms / 4 : sms;
    const int grid = strips < persistent ? strips : persistent;
    const int select_blocks = (L.anchor_count + kChosenWarps - 1) / kChosenWarps;
    auto launch = [&](auto distance, auto select) {
        err = raise_smem_limit(reinterpret_cast<const void*>(distance), static_cast<int>(smem));
        if (err != cudaSuccess) return;
        if (L.P == 8) strip_offsets_kernel<8><<<(strips + 7) / 8, 256, 0, stream>>>(L);
        else strip_offsets_kernel<7><<<(strips + 7) / 8, 256, 0, stream>>>(L);
        err = cudaGetLastError();
        if (err != cudaSuccess) return;
        distance<<<grid, kPipeThreads, smem, stream>>>(L);
        err = cudaGetLastError();
        if (err != cudaSuccess || select_blocks <= 0) return;
        select<<<select_blocks, kTcThreads, 0, stream>>>(L);
        err = cudaGetLastError();
    };
    auto with_select = [&](auto distance) {
        if (L.P == 8) {
            if (cap <= 32) launch(distance, tc_select_kernel<8, 1>);
            else if (cap <= 64) launch(distance, tc_select_kernel<8, 2>);
            else launch(distance, tc_select_kernel<8, 3>);
        } else {
            if (cap <= 32) launch(distance, tc_select_kernel<7, 1>);
            else if (cap <= 64) launch(distance, tc_select_kernel<7, 2>);
            else launch(distance, tc_select_kernel<7, 3>);
        }
    };
    if (L.P == 8) {
        switch (group) {
            case 1: with_select(tc_distance_kernel<8, 1>); break;
            case 2: with_select(tc_distance_kernel<8, 2>); break;
            default: with_select(tc_distance_kernel<8, 3>); break;
        }
    } else {
        switch (group) {
            case 1: with_select(tc_distance_kernel<7, 1>); break;
            case 2: with_select(tc_distance_kernel<7, 2>); break;
            default: with_select(tc_distance_kernel<7, 3>); break;
        }
    }
    return err;
}

}  // namespace vnlbgpu
