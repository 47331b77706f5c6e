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
// batch's alive word is resolved in order with 32 shuffles (an alive anchor
// clears its in-batch victims), then alive anchors clear their later victims
// in the shared bitmask, and the batch is compacted (ordered ballot) into the
// active list with the exclusive prefix of retained rows.  The serial chain is
// O(G/32) warp steps; the victim lists of the next batch are prefetched while
// the current one resolves.
#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

constexpr int kPrefetch = 8;

// Everything the walk needs about one grid anchor, loaded a batch ahead.
struct AnchorInfo {
    int n;             // victims
    int v[kPrefetch];  // the first victims
    int rows;          // retained rows
    int2 xy;
};

__device__ __forceinline__ AnchorInfo fetch(const PasteLaunch& L, int j) {
    AnchorInfo c;
    c.n = 0;
    c.rows = 0;
    c.xy = make_int2(0, 0);
    if (j < L.groups) {
        c.n = __ldg(L.victim_counts + j);
        c.rows = __ldg(L.row_counts + j);
        c.xy = __ldg(L.anchors + j);
        // the first entries are loaded unconditionally (in bounds: every anchor
        // owns victim_stride >= kPrefetch slots), so no load waits on the count
        const int* v = L.victims + static_cast<size_t>(j) * L.victim_stride;
#pragma unroll
        for (int e = 0; e < kPrefetch; ++e) c.v[e] = __ldg(v + e);
    }
    return c;
}

__global__ void __launch_bounds__(32) paste_kernel(PasteLaunch L) {
    extern __shared__ unsigned alive[];
    __shared__ unsigned masks[32];
    const int lane = threadIdx.x;
    const int words = (L.groups + 31) / 32;
    for (int w = lane; w < words; w += 32) {
        const int rem = L.groups - w * 32;
        alive[w] = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
    }
    __syncwarp();
    int running_active = 0;
    int running_rows = 0;
    // two batches in flight ahead of the one being resolved
    AnchorInfo next = fetch(L, lane);
    AnchorInfo after = fetch(L, lane + 32);
    for (int b = 0; b < words; ++b) {
        const AnchorInfo cur = next;
        next = after;
        const int j = b * 32 + lane;
        const int batch_end = (b + 1) * 32;
        after = fetch(L, j + 64);
        const int* vlist = L.victims + static_cast<size_t>(j) * L.victim_stride;
        // in-batch victims of this lane's anchor
        unsigned mine = 0;
        bool later = false;
        for (int e = 0; e < cur.n; ++e) {
            const int v = e < kPrefetch ? cur.v[e] : __ldg(vlist + e);
            if (v < batch_end) mine |= 1u << (v - b * 32);
            else later = true;
        }
        unsigned bits = alive[b];
        if (__any_sync(0xffffffffu, mine != 0)) {
            masks[lane] = mine;
            __syncwarp();
            unsigned mk[32];
#pragma unroll
            for (int k = 0; k < 32; ++k) mk[k] = masks[k];
#pragma unroll
            for (int k = 0; k < 32; ++k)
                if ((bits >> k) & 1u) bits &= ~mk[k];
            __syncwarp();
        }
        const bool me = j < L.groups && ((bits >> lane) & 1u);
        if (me && later) {
            for (int e = 0; e < cur.n; ++e) {
                const int v = e < kPrefetch ? cur.v[e] : __ldg(vlist + e);
                if (v >= batch_end) atomicAnd(&alive[v >> 5], ~(1u << (v & 31)));
            }
        }
        // ordered compaction
        const unsigned ballot = __ballot_sync(0xffffffffu, me);
        const int rank = __popc(ballot & ((1u << lane) - 1u));
        const int s = me ? cur.rows : 0;
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
            L.active_xy[a] = cur.xy;
            L.row_offset[a] = running_rows + prefix - s;
        }
        running_active += __popc(ballot);
        running_rows += __shfl_sync(0xffffffffu, prefix, 31);
        __syncwarp();
    }
    if (lane == 0) {
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
    const size_t smem = static_cast<size_t>((L.groups + 31) / 32) * sizeof(unsigned);
    cudaError_t err = cudaFuncSetAttribute(paste_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(smem));
    if (err != cudaSuccess) return err;
    paste_kernel<<<1, 32, smem, stream>>>(L);
    return cudaGetLastError();
}

}  // namespace vnlbgpu
