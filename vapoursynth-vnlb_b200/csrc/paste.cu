// Ordered paste mask and active-group compaction for one anchor frame.
//
// Reference semantics: process_anchor_impl visits the staggered grid in raster
// order and skips an anchor whose mask bit an earlier processed group cleared
// (src/core/core.cpp:1851-1903, apply_frame_paste_mask at :980-1008).  The
// match kernel has already turned every anchor's anchor-frame matches into the
// list of later grid anchors they clear (its "victims"), so the mask only
// needs one bit per grid anchor.
//
// One warp walks the anchors in batches of 32 (lane k = anchor 32b+k): the
// batch's alive word is resolved in order (an alive anchor clears its
// in-batch victims), then alive anchors clear their later victims in the
// shared bitmask, and the batch is compacted (ordered ballot) into the active
// list with the exclusive prefix of retained rows.  The serial chain is
// O(G/32) warp steps.  The other warps of the block stage the next chunk of
// anchors (counts, rows, positions, first victims and each anchor's in-batch
// victim mask) into shared memory while the walker resolves the current one,
// so the walker reads only shared memory; one block barrier per chunk.
#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr int kPrefetch = 8;                   // victims staged per anchor
constexpr int kPasteThreads = 512;
constexpr int kChunkBatches = 16;
constexpr int kChunk = kChunkBatches * 32;     // anchors per staged chunk
constexpr unsigned kLaterFlag = 1u << 30;      // in meta: a victim lies beyond the batch

struct __align__(16) Chunk {
    int meta[kChunk];           // victim count | kLaterFlag
    int rows[kChunk];           // retained rows
    unsigned mine[kChunk];      // in-batch victims, bit k = anchor 32b+k
    int2 xy[kChunk];
    int v[kPrefetch][kChunk];   // first victims, transposed
};

// Stages anchors [first, first + kChunk) with threads [t0, t0 + nt).
__device__ __forceinline__ void stage_chunk(const PasteLaunch& L, Chunk& c, int first, int t0, int nt) {
    for (int i = threadIdx.x - t0; i < kChunk; i += nt) {
        const int j = first + i;
        int n = 0, rows = 0;
        int2 xy = make_int2(0, 0);
        int v[kPrefetch];
        if (j < L.groups) {
            n = __ldg(L.victim_counts + j);
            rows = __ldg(L.row_counts + j);
            xy = __ldg(L.anchors + j);
            // in bounds: every anchor owns victim_stride >= kPrefetch slots, so
            // the first entries are loaded without waiting on the count
            const int* vlist = L.victims + static_cast<size_t>(j) * L.victim_stride;
#pragma unroll
            for (int e = 0; e < kPrefetch; ++e) v[e] = __ldg(vlist + e);
        }
        const int batch_start = j & ~31;
        unsigned mine = 0;
        bool later = false;
        if (j < L.groups) {
            const int* vlist = L.victims + static_cast<size_t>(j) * L.victim_stride;
            for (int e = 0; e < n; ++e) {
                const int x = e < kPrefetch ? v[e] : __ldg(vlist + e);
                if (x < batch_start + 32) mine |= 1u << (x - batch_start);
                else later = true;
            }
        }
        c.meta[i] = n | (later ? static_cast<int>(kLaterFlag) : 0);
        c.rows[i] = rows;
        c.mine[i] = mine;
        c.xy[i] = xy;
#pragma unroll
        for (int e = 0; e < kPrefetch; ++e) c.v[e][i] = j < L.groups ? v[e] : 0;
    }
}

__global__ void __launch_bounds__(kPasteThreads) paste_kernel(PasteLaunch L) {
    extern __shared__ __align__(16) unsigned char paste_smem[];
    Chunk* chunks = reinterpret_cast<Chunk*>(paste_smem);                 // two buffers
    unsigned* alive = reinterpret_cast<unsigned*>(paste_smem + 2 * sizeof(Chunk));
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int words = (L.groups + 31) / 32;
    const int nchunks = (L.groups + kChunk - 1) / kChunk;
    for (int w = tid; w < words; w += kPasteThreads) {
        const int rem = L.groups - w * 32;
        alive[w] = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
    }
    stage_chunk(L, chunks[0], 0, 0, kPasteThreads);
    __syncthreads();

    int running_active = 0;
    int running_rows = 0;
    for (int ci = 0; ci < nchunks; ++ci) {
        if (warp != 0) {
            if (ci + 1 < nchunks) stage_chunk(L, chunks[(ci + 1) & 1], (ci + 1) * kChunk, 32, kPasteThreads - 32);
        } else {
            const Chunk& c = chunks[ci & 1];
            const int b_end = min(words, (ci + 1) * kChunkBatches);
            for (int b = ci * kChunkBatches; b < b_end; ++b) {
                const int base = (b - ci * kChunkBatches) * 32;
                const int idx = base + lane;
                const int j = b * 32 + lane;
                const int batch_end = (b + 1) * 32;
                const unsigned mine = c.mine[idx];
                const int meta = c.meta[idx];
                const int my_rows = c.rows[idx];
                unsigned bits = alive[b];
                if (__any_sync(0xffffffffu, mine != 0)) {
                    // all 32 masks first (broadcast loads), then the ordered chain
                    unsigned mk[32];
                    const uint4* m4 = reinterpret_cast<const uint4*>(c.mine + base);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const uint4 t = m4[q];
                        mk[4 * q] = t.x;
                        mk[4 * q + 1] = t.y;
                        mk[4 * q + 2] = t.z;
                        mk[4 * q + 3] = t.w;
                    }
#pragma unroll
                    for (int k = 0; k < 32; ++k)
                        if ((bits >> k) & 1u) bits &= ~mk[k];
                }
                const bool me = j < L.groups && ((bits >> lane) & 1u);
                if (me && (meta & static_cast<int>(kLaterFlag))) {
                    const int n = meta & ~static_cast<int>(kLaterFlag);
                    const int* vlist = L.victims + static_cast<size_t>(j) * L.victim_stride;
                    for (int e = 0; e < n; ++e) {
                        const int v = e < kPrefetch ? c.v[e][idx] : __ldg(vlist + e);
                        if (v >= batch_end) atomicAnd(&alive[v >> 5], ~(1u << (v & 31)));
                    }
                }
                // ordered compaction
                const unsigned ballot = __ballot_sync(0xffffffffu, me);
                const int rank = __popc(ballot & ((1u << lane) - 1u));
                const int s = me ? my_rows : 0;
                int prefix = s;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, prefix, o);
                    if (lane >= o) prefix += v;
                }
                if (j < L.groups) L.active_prefix[j] = running_active + rank;
                if (me) {
                    const int a = running_active + rank;
                    L.active[a] = j;
                    L.active_xy[a] = c.xy[idx];
                    L.row_offset[a] = running_rows + prefix - s;
                }
                running_active += __popc(ballot);
                running_rows += __shfl_sync(0xffffffffu, prefix, 31);
                __syncwarp();
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        L.row_offset[running_active] = running_rows;
        L.active_prefix[L.groups] = running_active;
        L.counters->active = running_active;
        L.counters->rows = running_rows;
        atomicAdd(L.totals, static_cast<unsigned long long>(running_active));
        atomicAdd(L.totals + 1, static_cast<unsigned long long>(running_rows));
    }
}

__global__ void anchor_map_kernel(const int2* anchors, int count, int width, int* map) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int2 a = anchors[i];
        map[static_cast<size_t>(a.y) * width + a.x] = i;
    }
}

}  // namespace

cudaError_t launch_anchor_map(const int2* anchors, int count, int width, int* map, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    anchor_map_kernel<<<(count + 255) / 256, 256, 0, stream>>>(anchors, count, width, map);
    return cudaGetLastError();
}

cudaError_t launch_paste(const PasteLaunch& L, cudaStream_t stream) {
    const size_t smem = 2 * sizeof(Chunk) + static_cast<size_t>((L.groups + 31) / 32) * sizeof(unsigned);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;  // more grid anchors than the bitmask holds
    cudaError_t err = raise_smem_limit(reinterpret_cast<const void*>(paste_kernel),
                                           static_cast<int>(smem));
    if (err != cudaSuccess) return err;
    paste_kernel<<<1, kPasteThreads, smem, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace vnlbgpu
