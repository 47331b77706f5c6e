// Host side of the B200 VNLB path: parameter validation, anchor grids,
// device buffers, the per-anchor-frame launch sequence and the contribution
// stack cache behind the C ABI of include/vnlbgpu.h.
//
// Reference counterparts: parse/validate/derive (src/vs/cuda_plugin.cpp:
// 370-807), build_anchor_grid (:628-689) and reference_processing_mask_selected
// (src/core/core.cpp:934-950), compute_temporal_range / schedule_temporal_range
// (core.cpp:873-908), render_frame (cuda_plugin.cpp:1635-1864) and
// render_stage_frame / render_aggregate_frame (src/vs/plugin.cpp:616-1045).
#include <algorithm>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <functional>
#include <vector>

#include "../../include/vnlbgpu.h"
#include "../../include/vnlbgpu_diag.h"
#include "learned.h"
#include "mvtools.h"
#include "vnlb_kernels.h"

namespace vnlbgpu {
namespace {

thread_local std::string g_last_error;

}  // namespace

void set_last_error(const std::string& message) { g_last_error = message; }

namespace {

struct Failure : std::runtime_error {
    using std::runtime_error::runtime_error;
};

[[noreturn]] void fail(const std::string& message) { throw Failure(message); }

void check(cudaError_t status, const char* what) {
    if (status != cudaSuccess) {
        std::ostringstream m;
        m << "VNLB CUDA: " << what << " failed: " << cudaGetErrorString(status);
        throw Failure(m.str());
    }
}

template <typename T> struct DeviceArray {
    T* ptr = nullptr;
    size_t count = 0;
    DeviceArray() = default;
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    ~DeviceArray() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    void allocate(size_t n, const char* what) {
        release();
        if (n == 0) return;
        check(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)), what);
        count = n;
    }
};

// soft_similar_cap / model_similar_cap (core.cpp:139-172)
int cap_of(int similar, float factor) {
    if (factor == 0.0f) return INT_MAX;
    const float max_factor = static_cast<float>(INT_MAX) / static_cast<float>(similar);
    if (factor >= max_factor) return INT_MAX;
    const float cap = std::ceil(static_cast<float>(similar) * factor);
    return std::max(similar, static_cast<int>(cap));
}

void temporal_range(int source_frames, int patch_time, int bwd, int fwd, int anchor, int& low, int& high) {
    const int max_origin = source_frames - patch_time;
    const int start = anchor - bwd;
    const int end = anchor + fwd;
    const int shift = std::min(0, start) + std::max(0, end - max_origin);
    low = std::max(0, start - shift);
    high = std::min(max_origin, end - shift);
}

struct Grid {
    std::vector<int2> anchors;
    std::vector<Strip> strips;
    std::vector<TcStrip> strips_chosen;  // tensor-core matcher strips (one or two grid rows)
    DeviceArray<int2> d_anchors;
    DeviceArray<Strip> d_strips;
    DeviceArray<TcStrip> d_strips_chosen;
    DeviceArray<int> d_map;  // [H][W] anchor index or -1
    // stack-tile reach tables (TileLaunch)
    DeviceArray<int2> d_tile_grid_rows;  // [tiles_y]
    DeviceArray<int2> d_tile_anchors;    // [grid rows][tiles_x]
    // the same for the flow-guided search, built for flow_reach (x, y)
    DeviceArray<int2> d_flow_grid_rows, d_flow_anchors;
    int2 flow_reach = make_int2(-1, -1);
    // learned form: strips that do not cross a tile, each strip's tile, and
    // per tile the anchor the full search checks (its first), as a one-anchor
    // strip over a compact anchor list
    std::vector<Strip> tile_strips;
    DeviceArray<Strip> d_tile_strips, d_check_strips;
    DeviceArray<int> d_strip_tile, d_check_anchor;
    DeviceArray<int2> d_check_anchors;
    int tiles = 0;
};

}  // namespace

struct Session {
    std::mutex lock;
    vnlbgpu_params params{};
    StageConfig cfg{};
    int width = 0, height = 0, frames = 0, channels = 0;
    int stage = 0;
    int P = 0, Pt = 0, patch_dim = 0, dim = 0, search_channels = 1;
    int K = 0, soft_cap = 0, model_cap = 0, step = 0;
    int slots = 0, valid_anchor_frames = 0, max_rows = 0, buffer_cap = 0;
    int max_groups = 0, victim_stride = 0, warps = 8;
    int region_rows = 0, region_stride = 0, region_w_max = 0;
    // region reservation of the flow-guided search: the strip's plus room for
    // anchors of one strip that move apart
    int flow_region_rows = 0, flow_region_stride = 0, flow_region_w_max = 0;
    int sched_max = 0;    // most scheduled frames of an anchor frame
    // matcher forms: approx (VNLBGPU_FORM_CHOSEN: approximate distances in
    // the plain matcher's tiling, exact re-rank) and tensor
    // (VNLBGPU_FORM_CHOSEN_TC: BF16 tensor-core distances, match_chosen.cu)
    bool approx = false;
    bool chosen = false;
    int chosen_tiles_x = 0, chosen_wy = 0, approx_stride = 0;
    int tc_group = 0;  // tensor-core matcher: planes per shared-memory stage (0: the most that fit; autotuned)
    bool coupled = true;
    int models = 1;   // filter models per group
    bool covariance_possible = false;  // some group takes the dim x dim covariance model
    int nmax = 0;                      // largest eigen problem of a group
    int row_dim = 0;  // filtered row width (patch_dim * channels)
    int device = 0;
    cudaStream_t stream = nullptr;      // the stream all work is enqueued on
    cudaStream_t own_stream = nullptr;  // created by the session
    vnlbgpu_stats stats{};
    long long stats_uploads = 0;  // source frames copied to the device
    bool allow_scatter = true;    // off while a diagnostic reads the filtered rows back
    bool force_plain_match = false;  // the learned form's training pairs: the full search
    bool stall_mma = false;          // test switch: the tensor-core matcher issues no MMA
    // learned form (VNLBGPU_FORM_LEARNED): the attached network, shortlist
    // size, recall threshold of the per-tile check, tile edge; the network
    // sees slots_max scheduled frames of search_channels planes
    bool learned = false;
    vnlbgpu_mlp* mlp = nullptr;
    MlpDevice mlp_net{};
    int shortlist_len = 64, learned_tile = 64, slots_max = 1, learned_inputs = 0, learned_outputs = 0;
    int cells_w = 0, cells_h = 0, max_tiles = 0;
    float recall_threshold = 0.9f;
    static constexpr int kLearnedChunk = 4096;  // anchors per network pass
    static constexpr float kFeatureScale = 10.0f;

    // optional per-kernel timing: (category, start, stop) event triples
    bool timing = false;
    struct Timed {
        int category;
        cudaEvent_t start, stop;
    };
    std::vector<Timed> timed;
    std::vector<cudaEvent_t> event_pool;
    double kernel_ms[kTimedCategories] = {};
    long long kernel_count[kTimedCategories] = {};

    cudaEvent_t take_event() {
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        check(cudaEventCreate(&e), "cudaEventCreate");
        return e;
    }
    cudaEvent_t begin_timed(cudaStream_t on) {
        if (!timing) return nullptr;
        cudaEvent_t e = take_event();
        check(cudaEventRecord(e, on), "cudaEventRecord");
        return e;
    }
    void end_timed(int category, cudaEvent_t start, cudaStream_t on) {
        if (!timing) return;
        cudaEvent_t e = take_event();
        check(cudaEventRecord(e, on), "cudaEventRecord");
        timed.push_back(Timed{category, start, e});
    }
    void collect_timing() {
        if (timed.empty()) return;
        drain();
        for (const Timed& t : timed) {
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, t.start, t.stop), "cudaEventElapsedTime");
            kernel_ms[t.category] += ms;
            kernel_count[t.category] += 1;
            event_pool.push_back(t.start);
            event_pool.push_back(t.stop);
        }
        timed.clear();
    }

    // Events recording reads (of a source frame or a stack), shared by every
    // place that refers to the same read and recycled when the last goes.
    std::vector<cudaEvent_t> read_event_pool;
    using ReadEvent = std::shared_ptr<CUevent_st>;
    ReadEvent record_read(cudaStream_t on) {
        cudaEvent_t e;
        if (!read_event_pool.empty()) {
            e = read_event_pool.back();
            read_event_pool.pop_back();
        } else {
            check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        }
        check(cudaEventRecord(e, on), "cudaEventRecord(read)");
        return ReadEvent(e, [this](cudaEvent_t x) { read_event_pool.push_back(x); });
    }
    // `on` waits for every recorded read, which are then forgotten.
    void wait_reads(cudaStream_t on, std::vector<ReadEvent>& reads) {
        for (const ReadEvent& r : reads) check(cudaStreamWaitEvent(on, r.get(), 0), "cudaStreamWaitEvent(read)");
        reads.clear();
    }
    // Drops reads that have finished, so that the list of a long-lived frame
    // slot or stack stays short.
    static void prune_reads(std::vector<ReadEvent>& reads) {
        if (reads.size() < 16) return;
        reads.erase(std::remove_if(reads.begin(), reads.end(),
                                   [](const ReadEvent& r) { return cudaEventQuery(r.get()) == cudaSuccess; }),
                    reads.end());
        cudaGetLastError();  // cudaErrorNotReady is not sticky, but leaves nothing behind either
    }

    // Source frames on the device (the reference's noisy and basic
    // FrameCaches, src/cuda/frame_cache.cpp:120-537).  Frame f of a source
    // lives in slot f % ring of a store of ring + patch_time - 1 frame slots;
    // the last patch_time - 1 slots repeat the first ones, so that a patch's
    // patch_time consecutive frames are consecutive slots (MatchLaunch).  A
    // session starts with ring = min(frames, source window + num_streams - 1),
    // the source window being 2 (search_bwd + search_fwd + patch_time - 1) + 1
    // frames, the most one output frame reads (derive_geometry's
    // max_source_window, cuda_plugin.cpp:761-773).  A whole-clip source
    // (vnlbgpu_set_clip_host / vnlbgpu_set_clip_device) makes ring = frames.
    // Frames are immutable, like VapourSynth's: giving a frame that is already
    // on the device copies nothing.
    struct FrameSlot {
        int frame = -1;       // frame held (-1: none)
        int pins = 0;         // calls that hold the slot between claiming it and queueing their reads
        bool filling = false; // claimed, its copy not queued yet
        bool copied = false;  // `ready` marks the copy that filled it
        cudaEvent_t ready = nullptr;
        std::vector<ReadEvent> reads;  // queued work that reads the held frame
    };
    struct SourceStore {
        DeviceArray<float> own;          // ring (+ patch_time - 1) frame slots
        const float* base = nullptr;     // own.ptr, or a caller's whole device clip
        bool borrowed = false;           // base is the caller's: every frame resident, nothing tracked
        std::vector<FrameSlot> slots;    // [ring]
    };
    SourceStore store[2];
    int ring = 0;
    int source_window = 0;  // frames one output frame may read
    const float* clip = nullptr;  // store[0].base
    const float* ref = nullptr;   // store[1].base

    int sources() const { return stage == 1 ? 2 : 1; }

    // (Re)allocates a source's own store for `ring` slots, dropping its frames.
    void reset_store(int source) {
        SourceStore& st = store[source];
        const int mirror = ring < frames ? Pt - 1 : 0;
        if (!st.own.ptr || st.own.count != frame_values() * static_cast<size_t>(ring + mirror)) {
            st.own.release();
            st.own.allocate(frame_values() * static_cast<size_t>(ring + mirror), "cudaMalloc(source frames)");
        }
        st.base = st.own.ptr;
        st.borrowed = false;
        if (static_cast<int>(st.slots.size()) != ring) {
            for (FrameSlot& sl : st.slots)
                if (sl.ready) cudaEventDestroy(sl.ready);
            st.slots.clear();
            st.slots.resize(static_cast<size_t>(ring));
            for (FrameSlot& sl : st.slots)
                check(cudaEventCreateWithFlags(&sl.ready, cudaEventDisableTiming), "cudaEventCreate(frame slot)");
        }
        for (FrameSlot& sl : st.slots) {
            sl.frame = -1;
            sl.pins = 0;
            sl.filling = false;
            sl.copied = false;
            sl.reads.clear();
        }
        if (source == VNLBGPU_SOURCE_CLIP) clip = st.base; else ref = st.base;
    }

    // Whole clips: every frame gets its own slot.  Waits for all queued work.
    void make_whole() {
        if (ring == frames) return;
        drain();
        ring = frames;
        for (int src = 0; src < 2; ++src)
            if (store[src].own.ptr && !store[src].borrowed) reset_store(src);
        invalidate();
    }

    bool resident(int source, int f) const {
        const SourceStore& st = store[source];
        if (st.borrowed) return true;
        if (!st.base) return false;
        const FrameSlot& sl = st.slots[static_cast<size_t>(f % ring)];
        return sl.frame == f;
    }
    const float* frame_ptr(int source, int f) const {
        return store[source].base + static_cast<size_t>(f % ring) * frame_values();
    }

    // Queues the copy of frame f of a source from a contiguous host frame
    // [planes][H][W] into its slot on `on`, after every queued read of the
    // slot's previous frame.
    void queue_copy(int source, int f, const float* host_frame, cudaStream_t on);

    // `on` waits for the copies of frames [first, last] of every source the
    // stage reads; each must be on the device.
    void wait_frames(cudaStream_t on, int first, int last) {
        first = std::max(first, 0);
        last = std::min(last, frames - 1);
        for (int src = 0; src < sources(); ++src) {
            SourceStore& st = store[src];
            if (st.borrowed) continue;
            for (int f = first; f <= last; ++f) {
                FrameSlot& sl = st.slots[static_cast<size_t>(f % ring)];
                if (sl.frame != f || sl.filling) fail(missing_frame_message(src, f));
                if (sl.copied) check(cudaStreamWaitEvent(on, sl.ready, 0), "cudaStreamWaitEvent(frame copied)");
            }
        }
    }
    // Records that work queued on `on` reads frames [first, last] (sources
    // as wait_frames), so that no copy overwrites them before it is done.
    void read_frames(cudaStream_t on, int first, int last, int only_source = -1) {
        first = std::max(first, 0);
        last = std::min(last, frames - 1);
        ReadEvent r;
        for (int src = 0; src < sources(); ++src) {
            if (only_source >= 0 && src != only_source) continue;
            SourceStore& st = store[src];
            if (st.borrowed) continue;
            if (!r) r = record_read(on);
            for (int f = first; f <= last; ++f) {
                FrameSlot& sl = st.slots[static_cast<size_t>(f % ring)];
                prune_reads(sl.reads);
                sl.reads.push_back(r);
            }
        }
    }
    std::string missing_frame_message(int source, int f) const {
        return "VNLB CUDA: frame " + std::to_string(f) + " of " + (source == 0 ? "clip" : "ref") +
               " is not on the device (give it with vnlbgpu_set_frame or vnlbgpu_render_frame_window)";
    }

    // Pipeline lanes: consecutive anchor frames go round the lanes, each lane
    // with its own stream and scratch, so that one anchor frame's serial
    // paste-mask walk and latency-bound kernels overlap the others' kernels
    // (1080p YUV444 Basic+Final, plain / tensor-core matcher: 220 / 224 fps
    // with 2 lanes, 231 / 237 with 4, 232 / 239 with 8).  A session takes fewer
    // lanes when their group buffers would take more than half of the free
    // device memory, so that a Basic session leaves room for its Final.
    struct Lane {
        cudaStream_t stream = nullptr;
        DeviceArray<MatchRow> rows, row_info;
        DeviceArray<int2> centers;  // flow-guided search: [anchor][scheduled frame]
        DeviceArray<int> row_counts, victims, victim_counts, active, row_offset, row_group, active_prefix, gflags;
        DeviceArray<int2> active_xy;
        DeviceArray<FrameCounters> counters;
        DeviceArray<float> filtered, weights, gmeans, gram, eig, dual, logw;
        DeviceArray<float> approx;  // tensor-core form: approximate distances [G][approx_stride]
        DeviceArray<float> tc_mu;   // tensor-core matcher: per-strip plane offsets [strips][kChosenMaxPlanes]
        // learned form
        DeviceArray<float> features, cells, mlp_acts, mlp_logits;
        DeviceArray<int> shortlist, check_counts, check_vcounts, check_victims, tile_fail;
        DeviceArray<MatchRow> check_rows;
    };
#ifndef VNLB_MAX_LANES
#define VNLB_MAX_LANES 8  // a build parameter for comparisons
#endif
    static constexpr int kMaxLanes = VNLB_MAX_LANES;
    Lane lanes[kMaxLanes];
    int lane_count = kMaxLanes;        // lanes in use: 1..lanes_allocated
    int lanes_allocated = kMaxLanes;   // lanes with streams and buffers
    int next_lane = 0;
    cudaEvent_t ev_fork = nullptr;     // main-stream point the lanes start after
    cudaEvent_t ev_lane[kMaxLanes] = {};

    // Whole-clip host transfers run on their own streams so that they overlap
    // the kernels: an anchor frame's lane waits only for the copies of the
    // frames it reads; each output frame of a whole-clip host render is
    // downloaded as soon as it is normalised.
    cudaStream_t upload_stream = nullptr, download_stream = nullptr;
    cudaEvent_t ev_main = nullptr;      // main-stream point a copy stream starts after
    cudaEvent_t ev_out = nullptr;       // an output frame is normalised
    cudaEvent_t ev_download = nullptr;  // the downloads are done

    // Per-frame calls (vnlbgpu_render_frame, vnlbgpu_render_frame_window,
    // vnlbgpu_set_frame) each lease one of num_streams workers, like the
    // reference's WorkerPool (cuda_plugin.cpp:1117-1199): a stream, an output
    // frame on the device and pinned host staging.  A call queues its work
    // under the session lock and waits for it with the lock released, so
    // calls from several threads overlap on the GPU.
    struct Worker {
        cudaStream_t stream = nullptr;
        DeviceArray<float> out;           // one output frame
        float* host_out = nullptr;        // pinned, one frame
        int* host_status = nullptr;       // pinned
        std::vector<float*> staging;      // pinned frames for source copies
        std::vector<cudaEvent_t> staged;  // the device copy out of staging[i] is done
        std::vector<bool> staged_used;
        cudaEvent_t done = nullptr;
        bool busy = false;
    };
    std::vector<std::unique_ptr<Worker>> workers;
    std::condition_variable changed;  // a worker was released, a slot filled or unpinned
    int staging_slots = 2;

    DeviceArray<unsigned long long> d_totals;
    DeviceArray<int> d_status;
    DeviceArray<float> d_window, d_out_frame, d_pack;
    std::map<int, std::unique_ptr<Grid>> grids;

    // Contribution stack cache (anchor -> stack), the reference's contribution
    // FrameCache (cuda_plugin.cpp:1530-1605): slots + lanes + num_streams - 1
    // stacks.  `ready` is recorded on the producing lane; `reads` are the
    // queued normalisations and packs that read the stack.
    struct CachedStack {
        int anchor = -1;
        long long last_use = 0;
        DeviceArray<float> data;
        int packed = 0;  // layout of data: 0 planar, else pixel-interleaved (compute_anchor)
        cudaEvent_t ready = nullptr;
        std::vector<ReadEvent> reads;
    };
    std::vector<std::unique_ptr<CachedStack>> cache;
    long long use_clock = 0;
    std::vector<float> host_window;

    ~Session() {
        drain();
        for (const Timed& t : timed) {
            cudaEventDestroy(t.start);
            cudaEventDestroy(t.stop);
        }
        for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
        for (auto& c : cache) {
            c->reads.clear();
            if (c->ready) cudaEventDestroy(c->ready);
        }
        for (SourceStore& st : store)
            for (FrameSlot& sl : st.slots) {
                sl.reads.clear();
                if (sl.ready) cudaEventDestroy(sl.ready);
            }
        for (cudaEvent_t e : read_event_pool) cudaEventDestroy(e);
        for (auto& w : workers) {
            if (w->stream) cudaStreamDestroy(w->stream);
            if (w->host_out) cudaFreeHost(w->host_out);
            if (w->host_status) cudaFreeHost(w->host_status);
            for (float* p : w->staging) cudaFreeHost(p);
            for (cudaEvent_t e : w->staged) cudaEventDestroy(e);
            if (w->done) cudaEventDestroy(w->done);
        }
        for (cudaEvent_t e : {ev_main, ev_out, ev_download})
            if (e) cudaEventDestroy(e);
        if (upload_stream) cudaStreamDestroy(upload_stream);
        if (download_stream) cudaStreamDestroy(download_stream);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (cudaEvent_t e : ev_lane)
            if (e) cudaEventDestroy(e);
        for (Lane& l : lanes)
            if (l.stream) cudaStreamDestroy(l.stream);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    // Waits for everything the session queued on any of its streams.
    void drain() {
        if (stream) cudaStreamSynchronize(stream);
        if (own_stream && own_stream != stream) cudaStreamSynchronize(own_stream);
        for (Lane& l : lanes)
            if (l.stream) cudaStreamSynchronize(l.stream);
        for (auto& w : workers)
            if (w->stream) cudaStreamSynchronize(w->stream);
        if (upload_stream) cudaStreamSynchronize(upload_stream);
        if (download_stream) cudaStreamSynchronize(download_stream);
    }

    // Lanes start after everything enqueued so far on `from` ...
    void fork(cudaStream_t from) {
        check(cudaEventRecord(ev_fork, from), "cudaEventRecord(fork)");
        for (int i = 0; i < lane_count; ++i) check(cudaStreamWaitEvent(lanes[i].stream, ev_fork, 0), "cudaStreamWaitEvent(fork)");
    }
    void fork() { fork(stream); }
    // ... and the main stream continues after everything the lanes did.
    void join() {
        for (int i = 0; i < lane_count; ++i) {
            check(cudaEventRecord(ev_lane[i], lanes[i].stream), "cudaEventRecord(join)");
            check(cudaStreamWaitEvent(stream, ev_lane[i], 0), "cudaStreamWaitEvent(join)");
        }
    }

    // The plain matcher's strips: `w` anchors (warps) per CTA, whose search
    // regions fit a reservation of region_w_max columns; false when the
    // staged planes and the warps' scratch exceed the shared memory.
    int max_warps = 8;  // the widest strip that fits
    bool match_width_fits(int w) {
        const int cw0 = std::min(params.search_window, width - P + 1);
        const int ch0 = std::min(params.search_window, height - P + 1);
        region_w_max = ((w - 1) * step + cw0 + P - 1 + 3 + 3) & ~3;
        // stride = 4 (mod 8): the 4 candidate rows of one lane task start 16
        // banks apart, which keeps neighbouring lane tasks off each other's banks
        region_stride = region_w_max;
        while (region_stride % 8 != 4) ++region_stride;
        MatchLaunch probe{};
        probe.search_channels = search_channels;
        probe.Pt = Pt;
        probe.region_rows = region_rows;
        probe.region_stride = region_stride;
        probe.plane_floats = plane_floats_of(region_rows, region_stride);
        probe.approx = approx ? 1 : 0;
        probe.warp_floats = match_warp_floats(cw0 * ch0, search_channels * Pt, P, buffer_cap);
        return match_shared_bytes(probe, w) <= 200 * 1024;
    }
    // flow-guided search: the strips' reservation widened by up to 16 columns
    // and 8 rows while the shared memory allows
    void set_flow_region() {
        const int cw0 = std::min(params.search_window, width - P + 1);
        const int ch0 = std::min(params.search_window, height - P + 1);
        for (int slack = 16; slack >= 0; slack -= 4) {
            flow_region_w_max = region_w_max + slack;
            flow_region_rows = region_rows + slack / 2;
            flow_region_stride = flow_region_w_max;
            while (flow_region_stride % 8 != 4) ++flow_region_stride;
            MatchLaunch probe{};
            probe.search_channels = search_channels;
            probe.Pt = Pt;
            probe.region_rows = flow_region_rows;
            probe.region_stride = flow_region_stride;
            probe.plane_floats = plane_floats_of(flow_region_rows, flow_region_stride);
            probe.warp_floats = match_warp_floats(cw0 * ch0, search_channels * Pt, P, buffer_cap);
            if (match_shared_bytes(probe, warps) <= 200 * 1024) break;
        }
    }
    bool apply_general = false;  // autotuned: the row-tiled apply where the warp-per-group one also fits

    // Shared floats per staged plane of the plain matcher: whole 128-byte
    // units, so that every plane starts where a tensor-memory-accelerator
    // tile load may write.
    static int plane_floats_of(int rows, int stride) { return (rows * stride + 31) & ~31; }

    // The plain matcher stages its search regions with tile loads from a
    // tensor map over the search store (rows of `width` floats: every plane
    // of every slot), when the row pitch allows (width a multiple of 4).
#ifndef VNLB_MATCH_TMA
#define VNLB_MATCH_TMA 1  // a build parameter for comparisons
#endif
    CUtensorMap search_map{};
    const float* search_map_base = nullptr;
    long long search_map_rows = 0;
    int search_map_stride = 0;
    const CUtensorMap* search_tensor_map(const float* base) {
        if (!VNLB_MATCH_TMA) return nullptr;
        const int src = stage == 1 ? VNLBGPU_SOURCE_REF : VNLBGPU_SOURCE_CLIP;
        const long long slots = store[src].borrowed ? frames : ring + (ring < frames ? Pt - 1 : 0);
        const long long rows = slots * channels * static_cast<long long>(height);
        if (base == search_map_base && rows == search_map_rows && region_stride == search_map_stride)
            return &search_map;
        search_map_base = nullptr;
        if (!encode_store_map(&search_map, base, width, rows, region_stride, region_rows)) return nullptr;
        search_map_base = base;
        search_map_rows = rows;
        search_map_stride = region_stride;
        return &search_map;
    }

    size_t plane() const { return static_cast<size_t>(width) * height; }
    size_t frame_values() const { return plane() * channels; }
    size_t stack_values() const { return static_cast<size_t>(slots) * (channels + 1) * plane(); }

    void validate(const vnlbgpu_params& p) {
        // validate_stage_parameters (core.cpp:1948-1995) + vnlbcu checks
        auto require = [](bool ok, const char* message) {
            if (!ok) fail(std::string("VNLB CUDA: ") + message);
        };
        require(p.stage == 0 || p.stage == 1, "stage must be Basic (0) or Final (1)");
        require(std::isfinite(p.sigma) && p.sigma > 0.0f, "sigma must be finite and positive");
        require(p.patch_size > 0 && p.patch_size <= width && p.patch_size <= height,
                "block_size must fit inside the frame");
        require(p.patch_time > 0 && p.patch_time <= frames, "patch_time must fit inside the clip");
        require(p.search_window > 0 && (p.search_window & 1) == 1, "bm_range must describe a positive odd search window");
        require(p.search_bwd >= 0 && p.search_fwd >= 0, "search_bwd and search_fwd must be non-negative");
        require(p.similar > 0, "group_size must be positive");
        require(p.rank >= 0, "rank must be non-negative");
        require(std::isfinite(p.similar_cap_factor) && (p.similar_cap_factor == 0.0f || p.similar_cap_factor >= 1.0f),
                "cap_factor must be zero or at least 1.0");
        // vnlb.* semantics (plugin.cpp:409-412); vnlbcu's own check (model_cap_factor = 1) stays in its
        // argument parser, as in cuda_plugin.cpp
        require(std::isfinite(p.model_cap_factor) && (p.model_cap_factor == 0.0f || p.model_cap_factor >= 1.0f),
                "model_cap_factor must be zero or at least 1.0");
        require(std::isfinite(p.beta) && p.beta > 0.0f, "beta must be finite and positive");
        require(std::isfinite(p.tau) && p.tau >= 0.0f, "tau must be finite and non-negative");
        require(std::isfinite(p.variance_threshold), "variance_threshold must be finite");
        require(std::isfinite(p.sigma_basic) && p.sigma_basic >= 0.0f, "sigma_basic must be finite and non-negative");
        require(std::isfinite(p.gamma) && p.gamma > 0.0f, "gamma must be finite and positive");
        require(std::isfinite(p.weight_alpha) && p.weight_alpha >= 0.0f, "weight_alpha must be finite and non-negative");
        require(std::isfinite(p.weight_beta) && p.weight_beta >= 0.0f, "weight_beta must be finite and non-negative");
        require(std::isfinite(p.weight_gamma) && p.weight_gamma >= 0.0f, "weight_gamma must be finite and non-negative");
        require(std::isfinite(p.weight_epsilon) && p.weight_epsilon > 0.0f, "weight_epsilon must be finite and positive");
        require(std::isfinite(p.membership_noise_floor) && p.membership_noise_floor > 0.0f,
                "membership_noise_floor must be finite and positive");
        require(p.proc_step >= 0, "block_step must be non-negative; use 0 for auto");
        require(p.device_id >= 0, "device_id must be non-negative");
        require(p.num_streams >= 1 && p.num_streams <= 32, "num_streams must be in the range 1..32");
        require(p.chunk_size > 0, "chunk_size must be positive");
        require(p.form == VNLBGPU_FORM_PLAIN || p.form == VNLBGPU_FORM_CHOSEN || p.form == VNLBGPU_FORM_CHOSEN_TC ||
                    p.form == VNLBGPU_FORM_LEARNED,
                "form must be plain (0), chosen (1), chosen_tc (2) or learned (3)");
    }

    void configure(const vnlbgpu_params& p, int w, int h, int n, int c) {
        if (!(c == 1 || c == 3) || w <= 0 || h <= 0 || n <= 0)
            fail("VNLB CUDA: only constant GrayS and YUV444PS clips are supported");
        width = w;
        height = h;
        frames = n;
        channels = c;
        validate(p);
        params = p;
        stage = p.stage;
        cfg = StageConfig{p.sigma, p.patch_size, p.patch_time, p.search_window, p.search_bwd, p.search_fwd,
                          p.similar, p.rank, p.similar_cap_factor, p.model_cap_factor, p.beta, p.tau,
                          p.variance_threshold, p.sigma_basic, p.gamma, p.weight_alpha, p.weight_beta,
                          p.weight_gamma, p.weight_epsilon, p.membership_noise_floor, p.proc_step, p.flat_areas,
                          p.couple_channels};
        P = p.patch_size;
        Pt = p.patch_time;
        patch_dim = P * P * Pt;
        dim = patch_dim * (p.couple_channels ? channels : 1);
        coupled = p.couple_channels != 0 && channels > 1;
        // uncoupled planes: one model per plane (transform_vnlb_group, core.cpp:848-870)
        models = (!coupled && channels > 1) ? channels : 1;
        row_dim = patch_dim * channels;
        search_channels = stage == 1 ? channels : 1;
        K = p.similar;
        soft_cap = cap_of(K, p.similar_cap_factor);
        model_cap = cap_of(K, p.model_cap_factor);
        step = p.proc_step > 0 ? p.proc_step : (P <= 1 ? 1 : P);
        slots = p.search_bwd + p.search_fwd + p.patch_time;
        valid_anchor_frames = frames - Pt + 1;
        if (p.rank > dim) fail("VNLB CUDA: rank must not exceed the effective patch dimension");
        if (K < std::min(dim, p.rank)) fail("VNLB CUDA: group_size must cover the effective VNLB rank");
        // candidate count (derive_geometry, cuda_plugin.cpp:691-807)
        const int temporal = std::min(p.search_bwd + p.search_fwd + 1, valid_anchor_frames);
        const int cw = std::min(p.search_window, width - P + 1);
        const int ch = std::min(p.search_window, height - P + 1);
        const long long candidates = static_cast<long long>(cw) * ch * temporal;
        // model rows per group: B = min(S, model cap) with S <= min(soft cap,
        // candidates) (model_similar_cap, core.cpp:159-172); every group takes
        // the dual path when the largest B is below the dimension
        const long long retained_max = std::min<long long>(cap_of(K, p.similar_cap_factor), candidates);
        const int basis = static_cast<int>(
            std::min<long long>(std::max<long long>(std::min<long long>(K, candidates),
                                                    std::min<long long>(cap_of(K, p.model_cap_factor), retained_max)),
                                retained_max));
        if (basis > 128) fail("VNLB CUDA: the CUDA dual-PCA filter supports at most 128 model samples");
        if (p.rank > basis) fail("VNLB CUDA: rank must not exceed min(group_size, candidate_count)");
        // groups whose model rows reach the dimension, or below dimension 64,
        // take the covariance model (use_dual_pca, core.cpp:656-658)
        covariance_possible = !(dim >= 64 && basis < dim);
        if (slots > kMaxContributors || p.search_bwd + p.search_fwd + 1 > kMaxContributors)
            fail("VNLB CUDA: search_bwd + search_fwd + patch_time must be at most 32");
        if (channels > 4) fail("VNLB CUDA: at most four planes are supported");
        const long long raw = static_cast<long long>(p.search_window) * p.search_window *
                              (p.search_bwd + p.search_fwd + 1);
        buffer_cap = static_cast<int>(std::min<long long>(soft_cap, raw));
        if (buffer_cap > 4096) fail("VNLB CUDA: the B200 matcher keeps at most 4096 retained patches per group");
        max_rows = buffer_cap;
        if (K > 128) fail("VNLB CUDA: group_size must be at most 128");
        if (P > 32) fail("VNLB CUDA: block_size must be at most 32");

        check(cudaSetDevice(p.device_id), "cudaSetDevice");
        device = p.device_id;
        check(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking), "cudaStreamCreate");
        stream = own_stream;

        // largest grid over the anchor phases
        for (int key = 0; key < step; ++key) max_groups = std::max(max_groups, static_cast<int>(build_anchor_list(key).size()));
        victim_stride = std::max(8, max_rows * 5);
        // match region geometry
        const int KY = 4;
        region_rows = std::min(p.search_window, height - P + 1) + P - 1 + KY - 1;
        const int cw0 = std::min(p.search_window, width - P + 1);
        const int ch0 = std::min(p.search_window, height - P + 1);
        sched_max = std::min(frames, p.search_bwd + p.search_fwd + 1);
        const long long cap_eff = std::min<long long>(soft_cap, static_cast<long long>(cw0) * ch0 * sched_max);
        // approximate distances need 8x8 patches and the register replay
        // (buffer and K front within a warp)
        approx = p.form == VNLBGPU_FORM_CHOSEN && P == kLanes && cap_eff <= 32 && K <= 32;
        for (warps = 8; warps >= 1; warps /= 2)
            if (match_width_fits(warps)) break;
        if (warps < 1) fail("VNLB CUDA: the search region of one anchor does not fit in shared memory");
        max_warps = warps;
        set_flow_region();
        // tensor-core matcher: strips of up to kChosenAnchors anchors whose
        // windows lie within kChosenCols candidate columns
        if (p.form == VNLBGPU_FORM_CHOSEN_TC && chosen_match_supported(P, search_channels * Pt, cw0, ch0)) {
            MatchLaunch probe{};
            probe.P = P;
            probe.Pt = Pt;
            probe.search_channels = search_channels;
            probe.window_rows = chosen_wy = ch0;
            probe.tiles_x = chosen_tiles_x = kChosenCols / 8;
            probe.window_cells = cw0 * ch0;
            // the register replay: the K front fits in a warp, the buffer in
            // up to three registers per lane
            chosen = cap_eff <= kChosenMaxBuffer && K <= 32 && 64 <= cw0 * ch0 &&
                     chosen_match_shared_bytes(probe) <= 227 * 1024;
            // strips of two grid rows: their windows span up to the window
            // plus the grid step (consecutive grid rows are at most a step
            // apart); pairs whose span is larger stay single rows
            probe.window_rows = std::min(kChosenMaxRows, ch0 + std::max(1, step));
            if (chosen && chosen_match_shared_bytes(probe) <= 227 * 1024) chosen_wy = probe.window_rows;
            approx_stride = sched_max * cw0 * ch0;
        }

        const size_t G = static_cast<size_t>(max_groups);
        const size_t R = G * max_rows;
        const size_t Bmax = static_cast<size_t>(std::min(model_cap, max_rows));
        nmax = static_cast<int>(covariance_possible ? std::max<size_t>(Bmax, dim) : Bmax);
        if (nmax > 128) fail("VNLB CUDA: eigen problems above 128 x 128 (model rows or covariance dimension) are not supported");
        {
            FilterLaunch probe{};
            probe.dim = dim;
            probe.rank = p.rank;
            probe.nmax = nmax;
            probe.model_cap = model_cap;
            probe.max_rows = max_rows;
            probe.stage = stage;
            const size_t need = filter_shared_bytes(probe);
            if (need > filter_shared_limit())
                fail("VNLB CUDA: the group filter needs " + std::to_string(need / 1024) +
                     " KB of shared memory per block at this dimension, rank and model size (at most " +
                     std::to_string(filter_shared_limit() / 1024) + " KB)");
        }
        size_t free_bytes = 0, total_bytes = 0;
        check(cudaMemGetInfo(&free_bytes, &total_bytes), "cudaMemGetInfo");
        const size_t M = G * models;  // models: one per group, or one per plane when uncoupled
        const size_t N = static_cast<size_t>(nmax);
        const size_t rank1 = static_cast<size_t>(std::max(1, p.rank));
        // bytes of one lane's buffers, as allocated below
        const size_t lane_bytes =
            G * max_rows * sizeof(MatchRow) + G * (6 * sizeof(int) + sizeof(int2) + victim_stride * sizeof(int)) +
            (chosen ? G * (static_cast<size_t>(approx_stride) + kChosenMaxPlanes) * sizeof(float) : 0) +
            R * (static_cast<size_t>(row_dim) + 1 + (models > 1 ? models : 0)) * sizeof(float) +
            R * (sizeof(MatchRow) + sizeof(int)) +
            M * (2 * static_cast<size_t>(dim) + N * N + rank1 + rank1 * N) * sizeof(float) + M * sizeof(int);
        lane_count = static_cast<int>(std::min<size_t>(kMaxLanes, free_bytes / 2 / std::max<size_t>(lane_bytes, 1)));
        if (lane_count < 1) fail("VNLB CUDA: the group buffers of one anchor frame do not fit in device memory");
        lanes_allocated = lane_count;
        for (int li = 0; li < lane_count; ++li) {
            Lane& l = lanes[li];
            check(cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking), "cudaStreamCreate(lane)");
            l.rows.allocate(G * max_rows, "cudaMalloc(match rows)");
            l.row_counts.allocate(G, "cudaMalloc(row counts)");
            l.victims.allocate(G * victim_stride, "cudaMalloc(victims)");
            l.victim_counts.allocate(G, "cudaMalloc(victim counts)");
            l.active.allocate(G, "cudaMalloc(active groups)");
            l.active_xy.allocate(G, "cudaMalloc(active positions)");
            l.row_offset.allocate(G + 1, "cudaMalloc(row offsets)");
            l.active_prefix.allocate(G + 1, "cudaMalloc(active prefix)");
            l.counters.allocate(1, "cudaMalloc(counters)");
            if (chosen) {
                l.approx.allocate(G * approx_stride, "cudaMalloc(approximate distances)");
                l.tc_mu.allocate(G * kChosenMaxPlanes, "cudaMalloc(strip offsets)");  // a strip has an anchor
            }
            l.filtered.allocate(R * row_dim, "cudaMalloc(filtered rows)");
            l.gmeans.allocate(M * 2 * dim, "cudaMalloc(group means)");
            l.gram.allocate(M * N * N, "cudaMalloc(group Gram)");
            l.eig.allocate(M * std::max(1, p.rank), "cudaMalloc(group eigenvalues)");
            l.dual.allocate(M * std::max(1, p.rank) * N, "cudaMalloc(group eigenvectors)");
            l.gflags.allocate(M, "cudaMalloc(group flags)");
            if (models > 1) l.logw.allocate(R * models, "cudaMalloc(row log weights)");
            l.weights.allocate(R, "cudaMalloc(row weights)");
            l.row_info.allocate(R, "cudaMalloc(row info)");
            l.row_group.allocate(R, "cudaMalloc(row groups)");
        }
        // learned form: network shape and per-lane buffers (the network's own
        // activations follow once one is attached)
        learned = p.form == VNLBGPU_FORM_LEARNED;
        slots_max = p.search_bwd + p.search_fwd + 1;
        learned_inputs = slots_max * search_channels * 9;
        learned_outputs = slots_max * p.search_window * p.search_window;
        cells_w = (width + kFeatureCell - 1) / kFeatureCell;
        cells_h = (height + kFeatureCell - 1) / kFeatureCell;
        if (learned) {
            max_tiles = ((width + learned_tile - 1) / learned_tile) * ((height + learned_tile - 1) / learned_tile);
            for (int li = 0; li < lane_count; ++li) {
                Lane& l = lanes[li];
                l.features.allocate(G * learned_inputs, "cudaMalloc(learned features)");
                l.cells.allocate(static_cast<size_t>(slots_max) * search_channels * cells_w * cells_h,
                                 "cudaMalloc(learned cells)");
                l.shortlist.allocate(G * kShortlistMax, "cudaMalloc(learned shortlist)");
                l.check_rows.allocate(static_cast<size_t>(max_tiles) * max_rows, "cudaMalloc(check rows)");
                l.check_counts.allocate(max_tiles, "cudaMalloc(check counts)");
                l.check_vcounts.allocate(max_tiles, "cudaMalloc(check victims)");
                l.check_victims.allocate(static_cast<size_t>(max_tiles) * victim_stride, "cudaMalloc(check victims)");
                l.tile_fail.allocate(max_tiles, "cudaMalloc(tile flags)");
            }
        }
        d_totals.allocate(4, "cudaMalloc(totals)");
        check(cudaMemset(d_totals.ptr, 0, 4 * sizeof(unsigned long long)), "cudaMemset(totals)");
        d_status.allocate(1, "cudaMalloc(status)");
        check(cudaMemset(d_status.ptr, 0, sizeof(int)), "cudaMemset(status)");
        check(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming), "cudaEventCreate");
        for (cudaEvent_t& e : ev_lane) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        check(cudaStreamCreateWithFlags(&upload_stream, cudaStreamNonBlocking), "cudaStreamCreate(upload)");
        check(cudaStreamCreateWithFlags(&download_stream, cudaStreamNonBlocking), "cudaStreamCreate(download)");
        for (cudaEvent_t* e : {&ev_main, &ev_out, &ev_download})
            check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
        // source window and frame stores (derive_geometry, cuda_plugin.cpp:761-773;
        // initialize_cuda's source slots, :1878-1884)
        source_window = static_cast<int>(std::min<long long>(
            frames, 2LL * (p.search_bwd + p.search_fwd + p.patch_time - 1) + 1));
        ring = std::min(frames, source_window + p.num_streams - 1);
        workers.resize(static_cast<size_t>(p.num_streams));
        for (auto& w : workers) w = std::make_unique<Worker>();
        // pinned staging per worker: 64 MiB of frames, at least two
        staging_slots = static_cast<int>(std::clamp<size_t>((static_cast<size_t>(64) << 20) /
                                                                (frame_values() * sizeof(float)),
                                                            2, static_cast<size_t>(2 * source_window)));
        // aggregation window (prepare_aggregation_window, core.cpp:296-324)
        host_window.assign(static_cast<size_t>(P) * P, 1.0f);
        if (!(p.weight_gamma == 0.0f || P <= 1)) {
            const float center = 0.5f * static_cast<float>(P - 1);
            const float radius = std_max(center, 0.5f);
            float max_weight = 0.0f;
            for (int y = 0; y < P; ++y) {
                const float dy = (static_cast<float>(y) - center) / radius;
                for (int x = 0; x < P; ++x) {
                    const float dx = (static_cast<float>(x) - center) / radius;
                    const float raw_w = cr_expf(-0.5f * ((dx * dx) + (dy * dy)));
                    host_window[static_cast<size_t>(y) * P + x] = raw_w;
                    max_weight = std_max(max_weight, raw_w);
                }
            }
            const float inv_max = max_weight > 0.0f ? 1.0f / max_weight : 1.0f;
            for (float& v : host_window)
                v = static_cast<float>(std::pow(static_cast<double>(v * inv_max), static_cast<double>(p.weight_gamma)));
        }
        d_window.allocate(host_window.size(), "cudaMalloc(window)");
        check(cudaMemcpy(d_window.ptr, host_window.data(), host_window.size() * sizeof(float), cudaMemcpyHostToDevice),
              "cudaMemcpy(window)");
        // every contributor of a frame, the lanes' work in flight and the
        // frames of concurrent per-frame calls
        const int cache_size = std::min(valid_anchor_frames + lane_count, slots + lane_count + p.num_streams - 1);
        for (int i = 0; i < cache_size; ++i) {
            auto entry = std::make_unique<CachedStack>();
            entry->data.allocate(stack_values(), "cudaMalloc(contribution stack)");
            check(cudaEventCreateWithFlags(&entry->ready, cudaEventDisableTiming), "cudaEventCreate");
            cache.push_back(std::move(entry));
        }
    }

    // Stack-tile reach tables of an anchor grid: per tile row the grid rows,
    // and per (grid row, tile column) the anchors, whose matches can cover
    // the tile when every match lies within (reach_x, reach_y) of its anchor.
    void build_reach_tables(const std::vector<int2>& a, int reach_x, int reach_y, DeviceArray<int2>& d_rows,
                            DeviceArray<int2>& d_anchors) {
        std::vector<int> row_y, row_first;
        for (size_t j = 0; j < a.size(); ++j)
            if (j == 0 || a[j].y != a[j - 1].y) {
                row_y.push_back(a[j].y);
                row_first.push_back(static_cast<int>(j));
            }
        row_first.push_back(static_cast<int>(a.size()));
        const int rows_n = static_cast<int>(row_y.size());
        const int tiles_x = (width + kTile - 1) / kTile, tiles_y = (height + kTile - 1) / kTile;
        std::vector<int2> tgr(tiles_y), tan(static_cast<size_t>(rows_n) * tiles_x);
        for (int ty = 0; ty < tiles_y; ++ty) {
            const int lo = ty * kTile - (P - 1) - reach_y, hi = ty * kTile + kTile - 1 + reach_y;
            int k0 = 0;
            while (k0 < rows_n && row_y[k0] < lo) ++k0;
            int k1 = k0;
            while (k1 < rows_n && row_y[k1] <= hi) ++k1;
            tgr[ty] = make_int2(k0, k1);
        }
        for (int k = 0; k < rows_n; ++k)
            for (int tx = 0; tx < tiles_x; ++tx) {
                const int lo = tx * kTile - (P - 1) - reach_x, hi = tx * kTile + kTile - 1 + reach_x;
                int j0 = row_first[k];
                while (j0 < row_first[k + 1] && a[j0].x < lo) ++j0;
                int j1 = j0;
                while (j1 < row_first[k + 1] && a[j1].x <= hi) ++j1;
                tan[static_cast<size_t>(k) * tiles_x + tx] = make_int2(j0, j1);
            }
        d_rows.allocate(tgr.size(), "cudaMalloc(tile rows)");
        d_anchors.allocate(tan.size(), "cudaMalloc(tile anchors)");
        check(cudaMemcpy(d_rows.ptr, tgr.data(), tgr.size() * sizeof(int2), cudaMemcpyHostToDevice),
              "cudaMemcpy(tile rows)");
        check(cudaMemcpy(d_anchors.ptr, tan.data(), tan.size() * sizeof(int2), cudaMemcpyHostToDevice),
              "cudaMemcpy(tile anchors)");
    }

    // staggered anchor grid (reference_processing_mask_selected, core.cpp:934-950)
    std::vector<int2> build_anchor_list(int phase_key) const {
        std::vector<int2> out;
        const int max_x = width - P, max_y = height - P;
        auto row_selected = [&](int y) { return y == 0 || y == max_y || y % step == phase_key % step; };
        for (int y = 0; y <= max_y; ++y) {
            if (!row_selected(y)) {
                // jump to the next candidate row
                continue;
            }
            const int phase_x = y == max_y ? 0 : phase_key + (y / step);
            for (int x = 0; x <= max_x; ++x) {
                if (x == 0 || x == max_x || x % step == phase_x % step) out.push_back(make_int2(x, y));
            }
        }
        return out;
    }

    int grid_key(int anchor) const {
        const int max_frame = frames - Pt;
        const int phase_y = anchor == max_frame ? 0 : anchor;
        return phase_y % step;
    }

    Grid& grid_for(int anchor) {
        const int key = grid_key(anchor);
        auto it = grids.find(key);
        if (it != grids.end()) return *it->second;
        auto grid = std::make_unique<Grid>();
        grid->anchors = build_anchor_list(key);
        // strips: runs of consecutive anchors of one row within the region width
        const auto& a = grid->anchors;
        size_t i = 0;
        while (i < a.size()) {
            Strip s{};
            s.first = static_cast<int>(i);
            s.y = a[i].y;
            int yl, yh;
            spatial_range(s.y, height, P, params.search_window, yl, yh);
            s.region_y = yl;
            s.region_h = yh - yl + 1 + P - 1;
            int x0 = INT_MAX, x1 = INT_MIN, count = 0;
            while (i < a.size() && a[i].y == s.y && count < warps) {
                int xl, xh;
                spatial_range(a[i].x, width, P, params.search_window, xl, xh);
                const int nx0 = std::min(x0, xl & ~3);
                const int nx1 = std::max(x1, xh + P - 1);
                if (count > 0 && nx1 - nx0 + 1 > region_w_max) break;
                x0 = nx0;
                x1 = nx1;
                ++count;
                ++i;
            }
            s.count = count;
            s.region_x = x0;
            s.region_w = x1 - x0 + 1;
            if (s.region_w > region_w_max) fail("VNLB CUDA: internal error: search region exceeds its reservation");
            grid->strips.push_back(s);
        }
        if (chosen) {
            // the grid's rows [begin, end) in the anchor list
            std::vector<std::pair<size_t, size_t>> rows;
            for (size_t k = 0; k < a.size();) {
                size_t e = k;
                while (e < a.size() && a[e].y == a[k].y) ++e;
                rows.emplace_back(k, e);
                k = e;
            }
            auto window_x = [&](size_t k, int& xl, int& xh) {
                spatial_range(a[k].x, width, P, params.search_window, xl, xh);
            };
            for (size_t r = 0; r < rows.size();) {
                // pair row r with row r + 1 when their windows span at most
                // chosen_wy rows
                bool pair = false;
                if (r + 1 < rows.size()) {
                    int yl0, yh0, yl1, yh1;
                    spatial_range(a[rows[r].first].y, height, P, params.search_window, yl0, yh0);
                    spatial_range(a[rows[r + 1].first].y, height, P, params.search_window, yl1, yh1);
                    pair = yh1 - yl0 + 1 <= chosen_wy;
                }
                size_t k[2] = {rows[r].first, pair ? rows[r + 1].first : 0};
                const size_t end[2] = {rows[r].second, pair ? rows[r + 1].second : 0};
                while (k[0] < end[0] || k[1] < end[1]) {
                    TcStrip st{};
                    for (int h = 0; h < 2; ++h) {
                        st.first[h] = static_cast<int>(k[h]);
                        st.y[h] = k[h] < end[h] ? a[k[h]].y : a[rows[r].first].y;
                    }
                    int x0 = INT_MAX, x1 = INT_MIN;
                    // take the anchors of both rows in x order while their
                    // windows fit in kChosenCols columns
                    for (;;) {
                        int h = -1;
                        for (int c = 0; c < 2; ++c)
                            if (k[c] < end[c] && st.count[c] < kChosenAnchors && (h < 0 || a[k[c]].x < a[k[h]].x))
                                h = c;
                        if (h < 0) break;
                        int xl, xh;
                        window_x(k[h], xl, xh);
                        const int nx0 = std::min(x0, xl), nx1 = std::max(x1, xh);
                        if (st.count[0] + st.count[1] > 0 && nx1 - nx0 + 1 > kChosenCols) break;
                        x0 = nx0;
                        x1 = nx1;
                        ++st.count[h];
                        ++k[h];
                    }
                    if (st.count[1] == 0) st.y[1] = st.y[0];
                    st.region_x = x0;  // first candidate column
                    grid->strips_chosen.push_back(st);
                }
                r += pair ? 2 : 1;
            }
            grid->d_strips_chosen.allocate(grid->strips_chosen.size(), "cudaMalloc(strips)");
            check(cudaMemcpy(grid->d_strips_chosen.ptr, grid->strips_chosen.data(),
                             grid->strips_chosen.size() * sizeof(TcStrip), cudaMemcpyHostToDevice),
                  "cudaMemcpy(strips)");
        }
        grid->d_anchors.allocate(a.size(), "cudaMalloc(anchors)");
        grid->d_strips.allocate(grid->strips.size(), "cudaMalloc(strips)");
        check(cudaMemcpy(grid->d_anchors.ptr, a.data(), a.size() * sizeof(int2), cudaMemcpyHostToDevice),
              "cudaMemcpy(anchors)");
        check(cudaMemcpy(grid->d_strips.ptr, grid->strips.data(), grid->strips.size() * sizeof(Strip),
                         cudaMemcpyHostToDevice),
              "cudaMemcpy(strips)");
        // reach tables: a match lies within search_window - 1 of its anchor on
        // each axis, so a stack tile gathers from the anchors in that reach
        build_reach_tables(a, params.search_window - 1, params.search_window - 1, grid->d_tile_grid_rows,
                           grid->d_tile_anchors);
        grid->d_map.allocate(plane(), "cudaMalloc(anchor map)");
        check(cudaMemsetAsync(grid->d_map.ptr, 0xff, plane() * sizeof(int), stream), "cudaMemsetAsync(anchor map)");
        check(launch_anchor_map(grid->d_anchors.ptr, static_cast<int>(a.size()), width, grid->d_map.ptr, stream),
              "anchor map kernel launch");
        check(cudaStreamSynchronize(stream), "cudaStreamSynchronize(anchor grid)");  // once per grid phase
        stats.kernel_launches += 1;
        Grid& ref_grid = *grid;
        grids.emplace(key, std::move(grid));
        return ref_grid;
    }

    // Learned form: the grid's tiles (learned_tile pixels by anchor
    // position), strips that stay inside one tile, and each tile's checked
    // anchor (its first) as a one-anchor strip over a compact anchor list.
    void ensure_tiles(Grid& grid) {
        if (grid.tiles > 0 && grid.d_tile_strips.ptr) return;
        const auto& a = grid.anchors;
        const int tx_n = (width + learned_tile - 1) / learned_tile;
        auto tile_of = [&](int2 p) { return (p.y / learned_tile) * tx_n + p.x / learned_tile; };
        std::vector<int> compact(static_cast<size_t>(max_tiles), -1);
        std::vector<int> check_anchor;
        for (size_t i = 0; i < a.size(); ++i) {
            int& c = compact[static_cast<size_t>(tile_of(a[i]))];
            if (c < 0) {
                c = static_cast<int>(check_anchor.size());
                check_anchor.push_back(static_cast<int>(i));
            }
        }
        std::vector<Strip> strips;
        std::vector<int> strip_tile;
        size_t i = 0;
        while (i < a.size()) {
            Strip st{};
            st.first = static_cast<int>(i);
            st.y = a[i].y;
            int yl, yh;
            spatial_range(st.y, height, P, params.search_window, yl, yh);
            st.region_y = yl;
            st.region_h = yh - yl + 1 + P - 1;
            const int tile = tile_of(a[i]);
            int x0 = INT_MAX, x1 = INT_MIN, count = 0;
            while (i < a.size() && a[i].y == st.y && count < warps && tile_of(a[i]) == tile) {
                int xl, xh;
                spatial_range(a[i].x, width, P, params.search_window, xl, xh);
                const int nx0 = std::min(x0, xl & ~3), nx1 = std::max(x1, xh + P - 1);
                if (count > 0 && nx1 - nx0 + 1 > region_w_max) break;
                x0 = nx0;
                x1 = nx1;
                ++count;
                ++i;
            }
            st.count = count;
            st.region_x = x0;
            st.region_w = x1 - x0 + 1;
            strips.push_back(st);
            strip_tile.push_back(compact[static_cast<size_t>(tile)]);
        }
        std::vector<Strip> checks;
        std::vector<int2> check_xy;
        for (size_t t = 0; t < check_anchor.size(); ++t) {
            const int2 p = a[static_cast<size_t>(check_anchor[t])];
            Strip st{};
            st.first = static_cast<int>(t);
            st.count = 1;
            st.y = p.y;
            int lo, hi;
            spatial_range(p.y, height, P, params.search_window, lo, hi);
            st.region_y = lo;
            st.region_h = hi - lo + 1 + P - 1;
            spatial_range(p.x, width, P, params.search_window, lo, hi);
            st.region_x = lo & ~3;
            st.region_w = hi + P - 1 - st.region_x + 1;
            checks.push_back(st);
            check_xy.push_back(p);
        }
        grid.tiles = static_cast<int>(check_anchor.size());
        grid.tile_strips = strips;
        grid.d_tile_strips.allocate(strips.size(), "cudaMalloc(tile strips)");
        grid.d_strip_tile.allocate(strip_tile.size(), "cudaMalloc(strip tiles)");
        grid.d_check_strips.allocate(checks.size(), "cudaMalloc(check strips)");
        grid.d_check_anchor.allocate(check_anchor.size(), "cudaMalloc(check anchors)");
        grid.d_check_anchors.allocate(check_xy.size(), "cudaMalloc(check anchors)");
        check(cudaMemcpy(grid.d_tile_strips.ptr, strips.data(), strips.size() * sizeof(Strip), cudaMemcpyHostToDevice),
              "cudaMemcpy(tile strips)");
        check(cudaMemcpy(grid.d_strip_tile.ptr, strip_tile.data(), strip_tile.size() * sizeof(int),
                         cudaMemcpyHostToDevice),
              "cudaMemcpy(strip tiles)");
        check(cudaMemcpy(grid.d_check_strips.ptr, checks.data(), checks.size() * sizeof(Strip), cudaMemcpyHostToDevice),
              "cudaMemcpy(check strips)");
        check(cudaMemcpy(grid.d_check_anchor.ptr, check_anchor.data(), check_anchor.size() * sizeof(int),
                         cudaMemcpyHostToDevice),
              "cudaMemcpy(check anchors)");
        check(cudaMemcpy(grid.d_check_anchors.ptr, check_xy.data(), check_xy.size() * sizeof(int2),
                         cudaMemcpyHostToDevice),
              "cudaMemcpy(check anchors)");
    }

    void require_sources() {
        if (!clip) fail("VNLB CUDA: clip frames were not provided");
        if (stage == 1 && !ref) fail("VNLB CUDA: ref frames were not provided");
        sync_flow();
    }

    // Flow-guided search (vnlbgpu_set_mvtools_*): per direction, 0 = mvfw,
    // 1 = mvbw, the analysis data and every frame's finest vectors and usable
    // flag, copied to the device before the next render that reads them.
    struct Flow {
        bool present = false;
        bool dirty = false;
        vnlbgpu_mvtools_analysis analysis{};
        std::vector<unsigned char> usable;  // [frames]
        std::vector<int2> vectors;          // [frames][block_count_y][block_count_x]
        DeviceArray<unsigned char> d_usable;
        DeviceArray<int2> d_vectors;
    };
    Flow flow[2];

    bool flow_on() const { return flow[0].present || flow[1].present; }

    // A bound on how far a search centre moves from its anchor: a walk crosses
    // at most search_bwd + search_fwd frames (the temporal window shifts at
    // the clip's ends), each moving the centre by at most the largest rounded
    // vector of a usable grid of that frame; clamping only shortens it.  A
    // match then lies within search_window - 1 plus this bound of its anchor.
    int2 flow_reach = make_int2(0, 0);

    void update_flow_reach() {
        int walk = params.search_bwd + params.search_fwd;
        std::vector<int> mx, my;
        for (const Flow& f : flow) {
            if (!f.present) continue;
            const size_t count = static_cast<size_t>(f.analysis.block_count_x) * f.analysis.block_count_y;
            const int pel = f.analysis.pel;
            auto rounded = [pel](int v) {
                const int a = v < 0 ? -v : v;
                return pel <= 1 ? a : (a + pel / 2) / pel;
            };
            for (int fr = 0; fr < frames; ++fr) {
                int bx = 0, by = 0;
                if (f.usable[static_cast<size_t>(fr)])
                    for (size_t i = 0; i < count; ++i) {
                        const int2 v = f.vectors[static_cast<size_t>(fr) * count + i];
                        bx = std::max(bx, rounded(v.x));
                        by = std::max(by, rounded(v.y));
                    }
                mx.push_back(bx);
                my.push_back(by);
            }
        }
        auto bound = [walk](std::vector<int> m, int cap) {
            std::sort(m.begin(), m.end(), std::greater<int>());
            long long s = 0;
            for (int i = 0; i < walk && i < static_cast<int>(m.size()); ++i) s += m[static_cast<size_t>(i)];
            return static_cast<int>(std::min<long long>(s, cap));
        };
        flow_reach = make_int2(bound(mx, width - 1), bound(my, height - 1));
    }

    void sync_flow() {
        if (!flow[0].dirty && !flow[1].dirty) return;
        // earlier renders may still read the device copies
        drain();
        for (Flow& f : flow) {
            if (!f.dirty) continue;
            if (f.d_usable.count != f.usable.size()) f.d_usable.allocate(f.usable.size(), "cudaMalloc(flow flags)");
            if (f.d_vectors.count != f.vectors.size())
                f.d_vectors.allocate(f.vectors.size(), "cudaMalloc(flow vectors)");
            check(cudaMemcpy(f.d_usable.ptr, f.usable.data(), f.usable.size(), cudaMemcpyHostToDevice),
                  "cudaMemcpy(flow flags)");
            check(cudaMemcpy(f.d_vectors.ptr, f.vectors.data(), f.vectors.size() * sizeof(int2),
                             cudaMemcpyHostToDevice),
                  "cudaMemcpy(flow vectors)");
            f.dirty = false;
        }
        update_flow_reach();
    }

    FlowGridsDevice flow_device(int direction) const {
        FlowGridsDevice g{};
        const Flow& f = flow[direction];
        if (!f.present) return g;
        g.present = 1;
        g.block_size_x = f.analysis.block_size_x;
        g.block_size_y = f.analysis.block_size_y;
        g.pel = f.analysis.pel;
        g.overlap_x = f.analysis.overlap_x;
        g.overlap_y = f.analysis.overlap_y;
        g.block_count_x = f.analysis.block_count_x;
        g.block_count_y = f.analysis.block_count_y;
        g.usable = f.d_usable.ptr;
        g.vectors = f.d_vectors.ptr;
        return g;
    }

    // The store a source's frames go to, allocated on first use.
    SourceStore& store_for(int source) {
        if (source != VNLBGPU_SOURCE_CLIP && source != VNLBGPU_SOURCE_REF)
            fail("VNLB CUDA: source must be clip (0) or ref (1)");
        if (source == VNLBGPU_SOURCE_REF && stage != 1) fail("VNLB CUDA: only the Final stage takes a ref clip");
        SourceStore& st = store[source];
        if (st.borrowed) fail("VNLB CUDA: this source reads a caller-owned device clip; give frames there");
        if (!st.own.ptr) reset_store(source);
        return st;
    }

    void invalidate() {
        for (auto& c : cache) c->anchor = -1;
    }

    // The source frames anchor frame a reads: its shifted temporal window and
    // the patch_time - 1 frames after it (anchor_source_range,
    // cuda_plugin.cpp:825-844).
    void anchor_frames(int a, int& first, int& last) const {
        int low, high;
        temporal_range(frames, Pt, params.search_bwd, params.search_fwd, a, low, high);
        first = low;
        last = high + Pt - 1;
    }
    // contributing_anchors (cuda_plugin.cpp:809-823)
    void contributors(int n, int& first, int& last) const {
        first = std::max(0, n - (params.search_fwd + Pt - 1));
        last = std::min(valid_anchor_frames - 1, n + params.search_bwd);
    }
    // required_source_range (cuda_plugin.cpp:846-858): what output frame n may read
    void required_range(int n, int& first, int& last) const {
        first = last = n;
        int a0, a1;
        contributors(n, a0, a1);
        for (int a = a0; a <= a1; ++a) {
            int f0, f1;
            anchor_frames(a, f0, f1);
            first = std::min(first, f0);
            last = std::max(last, f1);
        }
    }
    CachedStack* cached(int anchor) {
        for (auto& c : cache)
            if (c->anchor == anchor) return c.get();
        return nullptr;
    }

    // Before queueing output frame n (or, with stack_only, anchor frame n's
    // stack): is a frame it reads still being copied by another call?  Throws
    // when one is not on the device at all.
    bool frames_pending(int n, bool stack_only = false) {
        auto check_range = [&](int f0, int f1, int only) {
            bool pending = false;
            for (int src = 0; src < sources(); ++src) {
                if (only >= 0 && src != only) continue;
                const SourceStore& st = store[src];
                if (st.borrowed) continue;
                if (!st.base) fail(src == 0 ? "VNLB CUDA: clip frames were not provided"
                                            : "VNLB CUDA: ref frames were not provided");
                for (int f = std::max(f0, 0); f <= std::min(f1, frames - 1); ++f) {
                    const FrameSlot& sl = st.slots[static_cast<size_t>(f % ring)];
                    if (sl.frame != f) fail(missing_frame_message(src, f));
                    pending |= sl.filling;
                }
            }
            return pending;
        };
        bool pending = false;
        if (stack_only) {
            if (!cached(n)) {
                int f0, f1;
                anchor_frames(n, f0, f1);
                pending |= check_range(f0, f1, -1);
            }
            return pending;
        }
        pending |= check_range(n, n, VNLBGPU_SOURCE_CLIP);  // the fallback samples
        int a0, a1;
        contributors(n, a0, a1);
        for (int a = a0; a <= a1; ++a) {
            if (cached(a)) continue;
            int f0, f1;
            anchor_frames(a, f0, f1);
            pending |= check_range(f0, f1, -1);
        }
        return pending;
    }

    // One anchor frame on one lane: match -> paste mask -> filter -> stack
    // tiles.  Everything is enqueued on the lane's stream.  Returns the
    // stack's layout: 0 planar, else the floats of a pixel-interleaved one
    // (FilterLaunch::scatter_pack).
    int compute_anchor(int anchor, float* stack, Lane& lane) {
        Grid& grid = grid_for(anchor);
        const int G = static_cast<int>(grid.anchors.size());
        cudaStream_t ls = lane.stream;
        // schedule (compute_temporal_range / schedule_temporal_range)
        int low, high;
        temporal_range(frames, Pt, params.search_bwd, params.search_fwd, anchor, low, high);
        wait_frames(ls, low, high + Pt - 1);  // every sample the anchor frame reads is on the device
        int schedule[kMaxContributors];
        int schedule_len = 0;
        schedule[schedule_len++] = anchor;
        for (int f = anchor + 1; f <= high; ++f) schedule[schedule_len++] = f;
        for (int f = anchor - 1; f >= low; --f) schedule[schedule_len++] = f;
        const float* search = stage == 1 ? ref : clip;
        MatchLaunch m{};
        m.video = search;
        m.width = width;
        m.height = height;
        m.channels = channels;
        m.frames = frames;
        m.ring = ring;
        m.search_channels = search_channels;
        m.P = P;
        m.Pt = Pt;
        m.search_window = params.search_window;
        m.K = K;
        m.soft_cap = soft_cap;
        m.max_rows = max_rows;
        m.tau = params.tau;
        m.anchor_frame = anchor;
        for (int i = 0; i < schedule_len; ++i) m.schedule[i] = schedule[i];
        m.schedule_len = schedule_len;
        m.anchors = grid.d_anchors.ptr;
        m.strips = grid.d_strips.ptr;
        m.anchor_map = grid.d_map.ptr;
        m.region_rows = region_rows;
        m.region_stride = region_stride;
        m.plane_floats = plane_floats_of(region_rows, region_stride);
        const int cw = std::min(params.search_window, width - P + 1);
        const int chh = std::min(params.search_window, height - P + 1);
        m.window_cells = cw * chh;
        m.buffer_cap = buffer_cap;
        m.approx = approx ? 1 : 0;
        m.warp_floats = match_warp_floats(m.window_cells, search_channels * Pt, P, buffer_cap);
        m.rows = lane.rows.ptr;
        m.row_counts = lane.row_counts.ptr;
        m.victims = lane.victims.ptr;
        m.victim_counts = lane.victim_counts.ptr;
        m.victim_stride = victim_stride;
        m.status = d_status.ptr;
        cudaEvent_t t0 = begin_timed(ls);
        if (flow_on()) {
            // flow-guided search (plain matcher, the strips' warps in passes):
            // the search centre of every anchor in every scheduled frame first
            if (!lane.centers.ptr)
                lane.centers.allocate(static_cast<size_t>(max_groups) * sched_max, "cudaMalloc(search centres)");
            CentersLaunch cl{};
            cl.fw = flow_device(0);
            cl.bw = flow_device(1);
            cl.anchors = grid.d_anchors.ptr;
            cl.anchor_count = G;
            for (int i = 0; i < schedule_len; ++i) cl.schedule[i] = schedule[i];
            cl.schedule_len = schedule_len;
            cl.anchor_frame = anchor;
            cl.width = width;
            cl.height = height;
            cl.P = P;
            cl.centers = lane.centers.ptr;
            check(launch_centers(cl, ls), "centers kernel launch");
            stats.kernel_launches += 1;
            m.centers = lane.centers.ptr;
            m.approx = 0;
            m.region_rows = flow_region_rows;
            m.region_stride = flow_region_stride;
            m.plane_floats = plane_floats_of(flow_region_rows, flow_region_stride);
            m.region_w_max = flow_region_w_max;
            check(launch_match(m, static_cast<int>(grid.strips.size()), warps, nullptr, ls), "match kernel launch");
        } else if (learned && !force_plain_match) {
            if (!mlp) fail("VNLB CUDA: the learned form needs a network (vnlbgpu_set_learned)");
            ensure_tiles(grid);
            LearnedLaunch ll{};
            ll.video = search;
            ll.ring = ring;
            ll.width = width;
            ll.height = height;
            ll.channels = channels;
            ll.search_channels = search_channels;
            ll.P = P;
            ll.Pt = Pt;
            ll.search_window = params.search_window;
            for (int i = 0; i < schedule_len; ++i) ll.schedule[i] = schedule[i];
            ll.schedule_len = schedule_len;
            ll.slots_max = slots_max;
            ll.anchor_frame = anchor;
            ll.anchors = grid.d_anchors.ptr;
            ll.anchor_count = G;
            ll.anchor_map = grid.d_map.ptr;
            ll.cells = lane.cells.ptr;
            ll.cells_w = cells_w;
            ll.cells_h = cells_h;
            ll.features = lane.features.ptr;
            ll.inputs = learned_inputs;
            ll.feature_scale = kFeatureScale;
            ll.shortlist = lane.shortlist.ptr;
            ll.shortlist_len = shortlist_len;
            ll.K = K;
            ll.soft_cap = soft_cap;
            ll.max_rows = max_rows;
            ll.tau = params.tau;
            ll.rows = lane.rows.ptr;
            ll.row_counts = lane.row_counts.ptr;
            ll.victims = lane.victims.ptr;
            ll.victim_counts = lane.victim_counts.ptr;
            ll.victim_stride = victim_stride;
            ll.tiles = grid.tiles;
            ll.check_anchor = grid.d_check_anchor.ptr;
            ll.check_rows = lane.check_rows.ptr;
            ll.check_counts = lane.check_counts.ptr;
            ll.recall_threshold = recall_threshold;
            ll.tile_fail = lane.tile_fail.ptr;
            ll.totals = d_totals.ptr + 2;
            // features, the network's shortlist in chunks, the shortlist matcher
            check(launch_learned_features(ll, ls), "learned features launch");
            float* acts[kMlpMaxLayers];
            for (int l = 0; l < mlp_net.layers; ++l)
                acts[l] = lane.mlp_acts.ptr + static_cast<size_t>(l) * kLearnedChunk * mlp_net.hidden;
            for (int g0 = 0; g0 < G; g0 += kLearnedChunk) {
                const int n = std::min(kLearnedChunk, G - g0);
                check(mlp_infer(mlp_net, lane.features.ptr + static_cast<size_t>(g0) * learned_inputs, n, acts,
                                lane.mlp_logits.ptr, d_status.ptr, ls),
                      "learned network launch");
                check(logits_topk(lane.mlp_logits.ptr, n, learned_outputs, shortlist_len,
                                  lane.shortlist.ptr + static_cast<size_t>(g0) * shortlist_len, ls),
                      "shortlist launch");
            }
            check(launch_learned_match(ll, ls), "learned match launch");
            // the check: the full search for each tile's checked anchor
            const CUtensorMap* map = search_tensor_map(search);
            MatchLaunch mc = m;
            mc.tma = map ? 1 : 0;
            mc.anchors = grid.d_check_anchors.ptr;
            mc.strips = grid.d_check_strips.ptr;
            mc.rows = lane.check_rows.ptr;
            mc.row_counts = lane.check_counts.ptr;
            mc.victims = lane.check_victims.ptr;
            mc.victim_counts = lane.check_vcounts.ptr;
            check(launch_match(mc, grid.tiles, warps, map, ls), "check match launch");
            check(launch_learned_recall(ll, ls), "recall launch");
            // the full search for the tiles that failed it
            MatchLaunch mf = m;
            mf.tma = map ? 1 : 0;
            mf.strips = grid.d_tile_strips.ptr;
            mf.strip_tile = grid.d_strip_tile.ptr;
            mf.tile_fail = lane.tile_fail.ptr;
            check(launch_match(mf, static_cast<int>(grid.tile_strips.size()), warps, map, ls), "fallback match launch");
            stats.kernel_launches += 6 + 2 * ((G + kLearnedChunk - 1) / kLearnedChunk) * (mlp_net.layers + 1);
        } else if (chosen) {
            m.tc_strips = grid.d_strips_chosen.ptr;
            m.strip_mu = lane.tc_mu.ptr;
            m.plane_group = tc_group;
            m.tiles_x = chosen_tiles_x;
            m.approx_dist = lane.approx.ptr;
            m.approx_stride = approx_stride;
            m.anchor_count = static_cast<int>(grid.anchors.size());
            m.strip_count = static_cast<int>(grid.strips_chosen.size());
            m.window_rows = chosen_wy;
            m.stall_mma = stall_mma ? 1 : 0;
            check(launch_match_chosen(m, static_cast<int>(grid.strips_chosen.size()), ls), "match kernel launch");
        } else {
            const CUtensorMap* map = search_tensor_map(search);
            m.tma = map ? 1 : 0;
            check(launch_match(m, static_cast<int>(grid.strips.size()), warps, map, ls), "match kernel launch");
        }
        end_timed(kTimedMatch, t0, ls);

        check(cudaMemsetAsync(lane.counters.ptr, 0, sizeof(FrameCounters), ls), "cudaMemsetAsync(counters)");
        PasteLaunch pl{};
        pl.groups = G;
        pl.row_counts = lane.row_counts.ptr;
        pl.victims = lane.victims.ptr;
        pl.victim_counts = lane.victim_counts.ptr;
        pl.victim_stride = victim_stride;
        pl.anchors = grid.d_anchors.ptr;
        pl.active = lane.active.ptr;
        pl.active_xy = lane.active_xy.ptr;
        pl.row_offset = lane.row_offset.ptr;
        pl.active_prefix = lane.active_prefix.ptr;
        pl.counters = lane.counters.ptr;
        pl.totals = d_totals.ptr;
        t0 = begin_timed(ls);
        check(launch_paste(pl, ls), "paste kernel launch");
        end_timed(kTimedPaste, t0, ls);

        FilterLaunch fl{};
        fl.noisy = clip;
        fl.basic = ref;
        fl.ring = ring;
        // the chosen forms' filter (TF32 Gram, FP64 angles) goes with their
        // matchers; configurations that run the plain matcher stay exact
        fl.mixed = (approx || chosen) && !flow_on() ? 1 : 0;
        fl.apply_general = apply_general ? 1 : 0;
        fl.width = width;
        fl.height = height;
        fl.channels = channels;
        fl.stage = stage;
        fl.P = P;
        fl.Pt = Pt;
        fl.patch_dim = patch_dim;
        fl.dim = dim;
        fl.K = K;
        fl.model_cap = model_cap;
        fl.rank = params.rank;
        fl.max_rows = max_rows;
        fl.coupled = coupled ? 1 : 0;
        fl.models = models;
        fl.nmax = nmax;
        fl.row_dim = row_dim;
        fl.logw = lane.logw.ptr;
        fl.cfg = cfg;
        fl.rows = lane.rows.ptr;
        fl.row_counts = lane.row_counts.ptr;
        fl.active = lane.active.ptr;
        fl.row_offset = lane.row_offset.ptr;
        fl.counters = lane.counters.ptr;
        fl.status = d_status.ptr;
        fl.filtered = lane.filtered.ptr;
        fl.weights = lane.weights.ptr;
        fl.row_info = lane.row_info.ptr;
        fl.row_group = lane.row_group.ptr;
        fl.means = lane.gmeans.ptr;
        fl.gram = lane.gram.ptr;
        fl.eig = lane.eig.ptr;
        fl.dual = lane.dual.ptr;
        fl.flags = lane.gflags.ptr;
        // chosen forms on the warp-per-group shapes: apply adds its rows
        // straight into the cleared stack, and no stack tiles run
        const bool scatter = fl.mixed && allow_scatter && filter_can_scatter(fl);
        if (scatter) {
            check(cudaMemsetAsync(stack, 0, stack_values() * sizeof(float), ls), "cudaMemsetAsync(stack)");
            fl.scatter = stack;
            fl.scatter_pack = filter_scatter_pack(fl);
            fl.window = d_window.ptr;
            fl.windowed = params.weight_gamma != 0.0f ? 1 : 0;
            fl.slots = slots;
            fl.search_bwd = params.search_bwd;
            fl.anchor_frame = anchor;
        }
        t0 = begin_timed(ls);
        check(launch_filter(fl, G, ls), "filter kernel launch");
        end_timed(kTimedFilter, t0, ls);

        TileLaunch tl{};
        tl.width = width;
        tl.height = height;
        tl.channels = channels;
        tl.P = P;
        tl.Pt = Pt;
        tl.patch_dim = patch_dim;
        tl.dim = row_dim;  // filtered row stride
        tl.slots = slots;
        tl.search_bwd = params.search_bwd;
        tl.anchor_frame = anchor;
        tl.coupled = coupled ? 1 : 0;
        tl.windowed = params.weight_gamma != 0.0f ? 1 : 0;
        tl.window = d_window.ptr;
        tl.row_offset = lane.row_offset.ptr;
        tl.active_prefix = lane.active_prefix.ptr;
        tl.filtered = lane.filtered.ptr;
        tl.weights = lane.weights.ptr;
        tl.row_info = lane.row_info.ptr;
        tl.stack = stack;
        tl.tiles_x = (width + kTile - 1) / kTile;
        tl.tiles_y = (height + kTile - 1) / kTile;
        tl.tile_grid_rows = grid.d_tile_grid_rows.ptr;
        tl.tile_anchors = grid.d_tile_anchors.ptr;
        if (flow_on()) {
            // matches of the flow-guided search lie further from their anchors
            const int2 reach = make_int2(params.search_window - 1 + flow_reach.x,
                                         params.search_window - 1 + flow_reach.y);
            if (grid.flow_reach.x != reach.x || grid.flow_reach.y != reach.y) {
                build_reach_tables(grid.anchors, reach.x, reach.y, grid.d_flow_grid_rows, grid.d_flow_anchors);
                grid.flow_reach = reach;
            }
            tl.tile_grid_rows = grid.d_flow_grid_rows.ptr;
            tl.tile_anchors = grid.d_flow_anchors.ptr;
        }
        if (!scatter) {
            t0 = begin_timed(ls);
            check(launch_tiles(tl, ls), "tile kernel launch");
            end_timed(kTimedTiles, t0, ls);
        }
        read_frames(ls, low, high + Pt - 1);
        stats.anchor_frames += 1;
        stats.groups += G;
        stats.kernel_launches += (params.rank > 0 ? 6 : 5) - (scatter ? 1 : 0);
        return scatter ? fl.scatter_pack : 0;
    }

    // The stack of `anchor`, computed on the next lane when not cached.  The
    // returned slot's `ready` event marks the end of its production.
    CachedStack* stack_for(int anchor, int* lane_used = nullptr) {
        if (CachedStack* c = cached(anchor)) {
            c->last_use = ++use_clock;
            return c;
        }
        CachedStack* victim = cache.front().get();
        for (auto& c : cache)
            if (c->last_use < victim->last_use) victim = c.get();
        const int li = next_lane;
        next_lane = (next_lane + 1) % lane_count;
        Lane& lane = lanes[li];
        wait_reads(lane.stream, victim->reads);  // its previous contents may still be read
        // and still be written: a stack computed on another lane and evicted
        // before anything read it (its reads then ordered nothing)
        check(cudaStreamWaitEvent(lane.stream, victim->ready, 0), "cudaStreamWaitEvent(stack written)");
        victim->anchor = -1;                     // until the work below is queued
        victim->packed = compute_anchor(anchor, victim->data.ptr, lane);
        check(cudaEventRecord(victim->ready, lane.stream), "cudaEventRecord(stack ready)");
        victim->anchor = anchor;
        victim->last_use = ++use_clock;
        if (lane_used) *lane_used = li;
        return victim;
    }

    // vnlbcu.Basic/Final frame n: normalise over the contributing anchors
    // (contributing_anchors, cuda_plugin.cpp:809-823; render_aggregate_frame
    // order: anchors first..last), on `on`.  The lanes' hazards are ordered by
    // events, so `on` can be the main stream or a worker's.
    void render_to_device(int n, float* out, cudaStream_t on) {
        const int first = std::max(0, n - (params.search_fwd + Pt - 1));
        const int last = std::min(frames - 1, n + params.search_bwd);
        NormalizeLaunch nl{};
        nl.width = width;
        nl.height = height;
        nl.channels = channels;
        nl.count = 0;
        CachedStack* used[kMaxContributors];
        for (int a = first; a <= last; ++a) {
            if (a > frames - Pt) continue;  // cleared stacks contribute nothing
            CachedStack* c = stack_for(a);
            used[nl.count] = c;
            nl.stacks[nl.count] = c->data.ptr;
            nl.slots[nl.count] = n - a + params.search_bwd;
            nl.packed[nl.count] = c->packed;
            ++nl.count;
        }
        for (int i = 0; i < nl.count; ++i)
            check(cudaStreamWaitEvent(on, used[i]->ready, 0), "cudaStreamWaitEvent(stack ready)");
        if (!store[0].borrowed) {
            const FrameSlot& sl = store[0].slots[static_cast<size_t>(n % ring)];
            if (sl.frame != n || sl.filling) fail(missing_frame_message(0, n));
            if (sl.copied) check(cudaStreamWaitEvent(on, sl.ready, 0), "cudaStreamWaitEvent(frame copied)");
        }
        nl.source = frame_ptr(VNLBGPU_SOURCE_CLIP, n);
        nl.out = out;
        cudaEvent_t t0 = begin_timed(on);
        check(launch_normalize(nl, on), "normalize kernel launch");
        end_timed(kTimedNormalize, t0, on);
        ReadEvent r = record_read(on);
        for (int i = 0; i < nl.count; ++i) {
            prune_reads(used[i]->reads);
            used[i]->reads.push_back(r);
        }
        read_frames(on, n, n, VNLBGPU_SOURCE_CLIP);
        stats.kernel_launches += 1;
    }
    void render_to_device(int n, float* out) { render_to_device(n, out, stream); }

    // Leases a worker, waiting while all num_streams are busy; its stream,
    // buffers and pinned staging are made on first use.
    Worker& acquire_worker(std::unique_lock<std::mutex>& lk) {
        for (;;) {
            for (auto& wp : workers) {
                Worker& w = *wp;
                if (w.busy) continue;
                w.busy = true;
                try {
                    if (!w.stream) {
                        check(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking), "cudaStreamCreate(worker)");
                        check(cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming), "cudaEventCreate");
                    }
                    if (!w.out.ptr) w.out.allocate(frame_values(), "cudaMalloc(output frame)");
                    if (!w.host_out)
                        check(cudaMallocHost(reinterpret_cast<void**>(&w.host_out), frame_values() * sizeof(float)),
                              "cudaMallocHost(output frame)");
                    if (!w.host_status)
                        check(cudaMallocHost(reinterpret_cast<void**>(&w.host_status), sizeof(int)),
                              "cudaMallocHost(status)");
                } catch (...) {
                    w.busy = false;
                    throw;
                }
                return w;
            }
            changed.wait(lk);
        }
    }
    // Makes a worker's first `count` pinned staging frames.
    void ensure_staging(Worker& w, int count) {
        while (static_cast<int>(w.staging.size()) < count) {
            float* p = nullptr;
            check(cudaMallocHost(reinterpret_cast<void**>(&p), frame_values() * sizeof(float)), "cudaMallocHost(staging)");
            w.staging.push_back(p);
            cudaEvent_t e;
            check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
            w.staged.push_back(e);
            w.staged_used.push_back(false);
        }
    }

    // Device time of one timed kernel class for anchor frame `anchor` on lane
    // 0: one untimed pass (grids, caches), then the least of three timed ones.
    double time_class(int anchor, int category) {
        DeviceArray<float> stack;
        stack.allocate(stack_values(), "cudaMalloc(tuning stack)");
        fork();
        compute_anchor(anchor, stack.ptr, lanes[0]);
        join();
        check_status();
        const bool was = timing;
        collect_timing();
        timing = true;
        double best = 1e30;
        for (int rep = 0; rep < 3; ++rep) {
            const double before = kernel_ms[category];
            fork();
            compute_anchor(anchor, stack.ptr, lanes[0]);
            join();
            collect_timing();
            best = std::min(best, kernel_ms[category] - before);
        }
        check_status();
        timing = was;
        invalidate();
        return best;
    }

    // The autotuner: the plain matcher's strip width (anchors per CTA) and
    // the apply kernel (warp per group or row tiles, where both fit) by
    // measured time on one anchor frame.  Every choice computes the same
    // bits; only the speed differs.
    void autotune(int anchor, std::vector<std::pair<std::string, double>>& log) {
        const bool plain_matcher = !chosen && !flow_on();
        if (plain_matcher) {
            int best_w = warps;
            double best_t = 1e30;
            for (int w = max_warps; w >= 2; w /= 2) {
                if (!match_width_fits(w)) continue;
                warps = w;
                set_flow_region();
                grids.clear();
                const double t = time_class(anchor, kTimedMatch);
                log.emplace_back("match strip " + std::to_string(w), t);
                if (t < best_t) {
                    best_t = t;
                    best_w = w;
                }
            }
            warps = best_w;
            match_width_fits(warps);
            set_flow_region();
            grids.clear();
        }
        if (chosen && !flow_on()) {
            // the tensor-core matcher's planes per shared-memory stage: fewer
            // planes take more stages per frame but fewer registers per row
            const int most = chosen_max_plane_group(search_channels * Pt, chosen_wy);
            int best_g = most;
            double best_t = 1e30;
            for (int g = most; g >= 1 && most > 1; --g) {
                tc_group = g;
                const double t = time_class(anchor, kTimedMatch);
                log.emplace_back("tensor-core planes per stage " + std::to_string(g), t);
                if (t < best_t) {
                    best_t = t;
                    best_g = g;
                }
            }
            tc_group = best_g;
        }
        FilterLaunch probe{};
        probe.dim = dim;
        probe.rank = params.rank;
        probe.nmax = nmax;
        probe.model_cap = model_cap;
        probe.max_rows = max_rows;
        probe.models = models;
        const bool scatter = (approx || chosen) && filter_can_scatter(probe);
        if (!scatter && filter_can_scatter(probe)) {  // both apply kernels fit this shape
            double t[2];
            for (int g = 0; g < 2; ++g) {
                apply_general = g == 1;
                t[g] = time_class(anchor, kTimedFilter);
                log.emplace_back(g ? "apply row tiles" : "apply warp per group", t[g]);
            }
            apply_general = t[1] < t[0];
        }
    }

    void check_status() {
        int status = 0;
        check(cudaMemcpyAsync(&status, d_status.ptr, sizeof(status), cudaMemcpyDeviceToHost, stream),
              "cudaMemcpyAsync(status)");
        check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        if (status != 0) {
            check(cudaMemsetAsync(d_status.ptr, 0, sizeof(int), stream), "cudaMemsetAsync(status)");
            // any stack computed since the last check may hold the failed
            // kernel's output: none is reused
            invalidate();
            if (status == kStatusRankNotCovered) fail("VNLB CUDA: group_size must cover the effective VNLB rank");
            if (status == kStatusTensorTimeout)
                fail("VNLB CUDA: the tensor-core matcher timed out waiting for its MMAs");
            if (status == kStatusTmaTimeout)
                fail("VNLB CUDA: the matcher timed out waiting for a tensor-memory-accelerator load");
            if (status == kStatusLogitsTimeout)
                fail("VNLB CUDA: the network's tensor-core output layer timed out waiting for its MMAs");
            fail("VNLB CUDA: device status " + std::to_string(status));
        }
    }
};

void Session::queue_copy(int source, int f, const float* host_frame, cudaStream_t on) {
    SourceStore& st = store[source];
    const int j = f % ring;
    FrameSlot& sl = st.slots[static_cast<size_t>(j)];
    wait_reads(on, sl.reads);  // the previous frame's readers
    // and the previous frame's copy, which may be queued on another stream
    // and not have been read at all (a window frame that no queued work
    // needed): two copies into one slot must not overlap
    check(cudaStreamWaitEvent(on, sl.ready, 0), "cudaStreamWaitEvent(slot written)");
    const size_t bytes = frame_values() * sizeof(float);
    float* dst = st.own.ptr + static_cast<size_t>(j) * frame_values();
    check(cudaMemcpyAsync(dst, host_frame, bytes, cudaMemcpyHostToDevice, on), "cudaMemcpyAsync(frame upload)");
    if (ring < frames && j < Pt - 1)  // the slots after the last repeat the first ones
        check(cudaMemcpyAsync(st.own.ptr + static_cast<size_t>(ring + j) * frame_values(), dst, bytes,
                              cudaMemcpyDeviceToDevice, on),
              "cudaMemcpyAsync(frame mirror)");
    check(cudaEventRecord(sl.ready, on), "cudaEventRecord(frame copied)");
    sl.frame = f;
    sl.copied = true;
    sl.filling = false;
    stats_uploads += 1;
}

namespace {

// A leased worker, given back (under the session lock) when it goes out of
// scope.  Declare it before the call's unique_lock, so that the lock is
// released first.
struct WorkerLease {
    Session& s;
    Session::Worker* w = nullptr;
    explicit WorkerLease(Session& session) : s(session) {}
    WorkerLease(const WorkerLease&) = delete;
    WorkerLease& operator=(const WorkerLease&) = delete;
    ~WorkerLease() {
        if (!w) return;
        std::lock_guard guard(s.lock);
        w->busy = false;
        s.changed.notify_all();
    }
};

// The source frames one call gives (vnlbgpu_render_frame_window,
// vnlbgpu_set_frame): claimed all at once (the reference's atomic window
// acquisition, FrameCache::acquire), copied through the worker's pinned
// staging, and held until the call's reads are queued.  Frames already on the
// device are only held.
struct FrameClaim {
    struct Given {
        int source, frame;
        const float* const* planes;
        const ptrdiff_t* strides;
    };
    Session& s;
    std::vector<Given> given;
    std::vector<size_t> fills;  // indices into `given` this call copies
    bool held = false;
    explicit FrameClaim(Session& session) : s(session) {}
    FrameClaim(const FrameClaim&) = delete;
    FrameClaim& operator=(const FrameClaim&) = delete;
    ~FrameClaim() {
        if (!held) return;
        std::lock_guard guard(s.lock);
        release_locked();
    }

    Session::FrameSlot& slot(const Given& g) {
        return s.store[g.source].slots[static_cast<size_t>(g.frame % s.ring)];
    }

    // Waits until no frame of `given` needs a slot that another call holds
    // for a different frame, then holds them all.
    void take(std::unique_lock<std::mutex>& lk) {
        for (const Given& g : given) s.store_for(g.source);
        for (;;) {
            bool conflict = false;
            for (const Given& g : given) {
                const Session::FrameSlot& sl = slot(g);
                if (sl.frame != g.frame && sl.pins > 0) conflict = true;
            }
            if (!conflict) break;
            s.changed.wait(lk);
        }
        for (size_t i = 0; i < given.size(); ++i) {
            Session::FrameSlot& sl = slot(given[i]);
            sl.pins += 1;
            if (sl.frame != given[i].frame) {
                sl.frame = given[i].frame;
                sl.copied = false;
                sl.filling = true;
                fills.push_back(i);
            }
        }
        held = true;
    }

    // Copies the claimed frames: host copies into pinned staging with the
    // lock released, device copies queued on the worker's stream under it.
    void copy(std::unique_lock<std::mutex>& lk, Session::Worker& w) {
        const int W = s.width, H = s.height, C = s.channels;
        const size_t plane = static_cast<size_t>(W) * H;
        for (size_t i0 = 0; i0 < fills.size(); i0 += static_cast<size_t>(s.staging_slots)) {
            const size_t i1 = std::min(fills.size(), i0 + static_cast<size_t>(s.staging_slots));
            s.ensure_staging(w, static_cast<int>(i1 - i0));
            lk.unlock();
            for (size_t i = i0; i < i1; ++i) {
                const size_t k = i - i0;
                // the device copy out of this staging frame's previous contents
                if (w.staged_used[k]) vnlbgpu::check(cudaEventSynchronize(w.staged[k]), "cudaEventSynchronize(staging)");
                const Given& g = given[fills[i]];
                float* dst = w.staging[k];
                for (int c = 0; c < C; ++c) {
                    const char* src = reinterpret_cast<const char*>(g.planes[c]);
                    float* d = dst + static_cast<size_t>(c) * plane;
                    if (g.strides[c] == static_cast<ptrdiff_t>(W * sizeof(float))) {
                        std::memcpy(d, src, plane * sizeof(float));
                    } else {
                        for (int y = 0; y < H; ++y)
                            std::memcpy(d + static_cast<size_t>(y) * W, src + static_cast<size_t>(y) * g.strides[c],
                                        static_cast<size_t>(W) * sizeof(float));
                    }
                }
            }
            lk.lock();
            for (size_t i = i0; i < i1; ++i) {
                const Given& g = given[fills[i]];
                s.queue_copy(g.source, g.frame, w.staging[i - i0], w.stream);
                const size_t k = i - i0;
                vnlbgpu::check(cudaEventRecord(w.staged[k], w.stream), "cudaEventRecord(staging)");
                w.staged_used[k] = true;
            }
            s.changed.notify_all();
        }
    }

    // Under the session lock: stop holding the frames; a claimed frame whose
    // copy was never queued leaves its slot empty.
    void release_locked() {
        if (!held) return;
        for (size_t i : fills) {
            Session::FrameSlot& sl = slot(given[i]);
            if (sl.filling && sl.frame == given[i].frame) {
                sl.filling = false;
                sl.frame = -1;
                sl.copied = false;
            }
        }
        for (const Given& g : given) slot(g).pins -= 1;
        held = false;
        s.changed.notify_all();
    }
};

}  // namespace

}  // namespace vnlbgpu

using vnlbgpu::Session;

struct vnlbgpu_session {
    Session impl;
};

namespace {

template <typename Fn> int guarded(Fn&& fn) {
    try {
        fn();
        return 0;
    } catch (const std::exception& error) {
        vnlbgpu::g_last_error = error.what();
        return -1;
    } catch (...) {
        vnlbgpu::g_last_error = "VNLB CUDA: unknown failure";
        return -1;
    }
}

}  // namespace

extern "C" {

const char* vnlbgpu_last_error(void) { return vnlbgpu::g_last_error.c_str(); }

int vnlbgpu_create(const vnlbgpu_params* params, int width, int height, int frames, int channels,
                   vnlbgpu_session** out) {
    return guarded([&]() {
        if (!params || !out) vnlbgpu::fail("VNLB CUDA: null argument");
        auto s = std::make_unique<vnlbgpu_session>();
        s->impl.configure(*params, width, height, frames, channels);
        *out = s.release();
    });
}

void vnlbgpu_destroy(vnlbgpu_session* session) {
    if (!session) return;
    cudaSetDevice(session->impl.device);
    if (session->impl.stream) cudaStreamSynchronize(session->impl.stream);
    delete session;
}

int vnlbgpu_set_frame(vnlbgpu_session* session, int source, int frame, const float* const* planes,
                      const ptrdiff_t* strides) {
    return guarded([&]() {
        if (!session || !planes || !strides) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        vnlbgpu::WorkerLease lease(s);
        vnlbgpu::FrameClaim claim(s);
        std::unique_lock lk(s.lock);
        if (frame < 0 || frame >= s.frames) vnlbgpu::fail("VNLB CUDA: frame index out of range");
        for (int c = 0; c < s.channels; ++c)
            if (strides[c] < static_cast<ptrdiff_t>(s.width * sizeof(float)))
                vnlbgpu::fail("VNLB CUDA: unsupported frame stride");
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.store_for(source);
        lease.w = &s.acquire_worker(lk);
        claim.given.push_back({source, frame, planes, strides});
        claim.take(lk);
        claim.copy(lk, *lease.w);
        claim.release_locked();
    });
}

int vnlbgpu_set_clip_host(vnlbgpu_session* session, int source, const float* clip) {
    return guarded([&]() {
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        if (source == VNLBGPU_SOURCE_CLIP || source == VNLBGPU_SOURCE_REF) {
            if (source == VNLBGPU_SOURCE_REF && s.stage != 1) vnlbgpu::fail("VNLB CUDA: only the Final stage takes a ref clip");
            for (const auto& sl : s.store[source].slots)
                if (sl.pins > 0) vnlbgpu::fail("VNLB CUDA: a whole clip cannot replace frames that calls in flight hold");
        }
        s.make_whole();
        if (s.store[source].borrowed) {  // was a caller's device clip: take an own store again
            s.store[source].borrowed = false;
            s.store[source].base = nullptr;
        }
        s.store_for(source);
        // one copy per frame, so that anchor frames start as their frames land
        const size_t fv = s.frame_values();
        for (int f = 0; f < s.frames; ++f) s.queue_copy(source, f, clip + fv * f, s.upload_stream);
        s.invalidate();
    });
}

int vnlbgpu_set_clip_device(vnlbgpu_session* session, int source, const float* device_clip) {
    return guarded([&]() {
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        if (source != VNLBGPU_SOURCE_CLIP && source != VNLBGPU_SOURCE_REF)
            vnlbgpu::fail("VNLB CUDA: source must be clip (0) or ref (1)");
        if (source == VNLBGPU_SOURCE_REF && s.stage != 1) vnlbgpu::fail("VNLB CUDA: only the Final stage takes a ref clip");
        for (const auto& sl : s.store[source].slots)
            if (sl.pins > 0) vnlbgpu::fail("VNLB CUDA: a whole clip cannot replace frames that calls in flight hold");
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.make_whole();
        s.drain();
        Session::SourceStore& st = s.store[source];
        st.own.release();
        st.slots.clear();
        st.borrowed = true;
        st.base = device_clip;
        if (source == VNLBGPU_SOURCE_CLIP) s.clip = device_clip; else s.ref = device_clip;
        s.invalidate();
    });
}

int vnlbgpu_required_source_range(vnlbgpu_session* session, int n, int* first, int* last) {
    return guarded([&]() {
        if (!session || !first || !last) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        if (n < 0 || n >= s.frames) vnlbgpu::fail("VNLB CUDA: frame index out of range");
        s.required_range(n, *first, *last);
    });
}

namespace {

// The per-frame render shared by vnlbgpu_render_frame and
// vnlbgpu_render_frame_window: queue under the lock on the worker's stream,
// wait with the lock released, copy out.
void render_one(Session& s, int n, int first, int count, const float* const* clip_planes,
                const ptrdiff_t* clip_strides, const float* const* ref_planes, const ptrdiff_t* ref_strides,
                float* const* planes, const ptrdiff_t* strides) {
    if (!planes || !strides) vnlbgpu::fail("VNLB CUDA: null argument");
    vnlbgpu::WorkerLease lease(s);
    vnlbgpu::FrameClaim claim(s);
    std::unique_lock lk(s.lock);
    if (n < 0 || n >= s.frames) vnlbgpu::fail("VNLB CUDA: frame index out of range");
    vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
    if (count > 0) {
        if (!clip_planes || !clip_strides || (s.stage == 1 && (!ref_planes || !ref_strides)))
            vnlbgpu::fail("VNLB CUDA: null argument");
        if (first < 0 || first + count > s.frames) vnlbgpu::fail("VNLB CUDA: source frame range outside the clip");
        if (count > s.ring)
            vnlbgpu::fail("VNLB CUDA: " + std::to_string(count) + " source frames exceed the " +
                          std::to_string(s.ring) + " frame slots of the session");
        for (int i = 0; i < count * s.channels; ++i)
            if (clip_strides[i] < static_cast<ptrdiff_t>(s.width * sizeof(float)) ||
                (s.stage == 1 && ref_strides[i] < static_cast<ptrdiff_t>(s.width * sizeof(float))))
                vnlbgpu::fail("VNLB CUDA: unsupported frame stride");
        for (int i = 0; i < count; ++i) {
            const size_t k = static_cast<size_t>(i) * s.channels;
            claim.given.push_back({VNLBGPU_SOURCE_CLIP, first + i, clip_planes + k, clip_strides + k});
            if (s.stage == 1) claim.given.push_back({VNLBGPU_SOURCE_REF, first + i, ref_planes + k, ref_strides + k});
        }
    }
    lease.w = &s.acquire_worker(lk);
    Session::Worker& w = *lease.w;
    if (count > 0) {
        claim.take(lk);
        claim.copy(lk, w);
    }
    s.require_sources();
    while (s.frames_pending(n)) s.changed.wait(lk);
    s.render_to_device(n, w.out.ptr, w.stream);
    vnlbgpu::check(cudaMemcpyAsync(w.host_out, w.out.ptr, s.frame_values() * sizeof(float), cudaMemcpyDeviceToHost,
                                   w.stream),
                   "cudaMemcpyAsync(frame download)");
    vnlbgpu::check(cudaMemcpyAsync(w.host_status, s.d_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, w.stream),
                   "cudaMemcpyAsync(status)");
    vnlbgpu::check(cudaEventRecord(w.done, w.stream), "cudaEventRecord(frame done)");
    claim.release_locked();
    lk.unlock();
    vnlbgpu::check(cudaEventSynchronize(w.done), "cudaEventSynchronize(frame done)");
    const size_t plane = s.plane();
    for (int c = 0; c < s.channels; ++c) {
        const float* src = w.host_out + static_cast<size_t>(c) * plane;
        char* dst = reinterpret_cast<char*>(planes[c]);
        if (strides[c] == static_cast<ptrdiff_t>(s.width * sizeof(float))) {
            std::memcpy(dst, src, plane * sizeof(float));
        } else {
            for (int y = 0; y < s.height; ++y)
                std::memcpy(dst + static_cast<size_t>(y) * strides[c], src + static_cast<size_t>(y) * s.width,
                            static_cast<size_t>(s.width) * sizeof(float));
        }
    }
    if (*w.host_status != 0) {
        lk.lock();
        s.check_status();  // resets the status word and raises its message
    }
}

}  // namespace

int vnlbgpu_render_frame(vnlbgpu_session* session, int n, float* const* planes, const ptrdiff_t* strides) {
    return guarded([&]() {
        if (!session) vnlbgpu::fail("VNLB CUDA: null argument");
        for (int c = 0; planes && strides && c < session->impl.channels; ++c)
            if (strides[c] < static_cast<ptrdiff_t>(session->impl.width * sizeof(float)))
                vnlbgpu::fail("VNLB CUDA: unsupported frame stride");
        render_one(session->impl, n, 0, 0, nullptr, nullptr, nullptr, nullptr, planes, strides);
    });
}

int vnlbgpu_render_frame_window(vnlbgpu_session* session, int n, int first, int count,
                                const float* const* clip_planes, const ptrdiff_t* clip_strides,
                                const float* const* ref_planes, const ptrdiff_t* ref_strides, float* const* planes,
                                const ptrdiff_t* strides) {
    return guarded([&]() {
        if (!session) vnlbgpu::fail("VNLB CUDA: null argument");
        for (int c = 0; planes && strides && c < session->impl.channels; ++c)
            if (strides[c] < static_cast<ptrdiff_t>(session->impl.width * sizeof(float)))
                vnlbgpu::fail("VNLB CUDA: unsupported frame stride");
        render_one(session->impl, n, first, count, clip_planes, clip_strides, ref_planes, ref_strides, planes,
                   strides);
    });
}

namespace {

// Whole-clip renders read every frame: wait while another call still copies
// one, and raise if one is missing.
void require_all_frames(Session& s, std::unique_lock<std::mutex>& lk) {
    for (;;) {
        bool pending = false;
        for (int n = 0; n < s.frames; ++n) pending |= s.frames_pending(n);
        if (!pending) return;
        s.changed.wait(lk);
    }
}

}  // namespace

int vnlbgpu_render_clip_device(vnlbgpu_session* session, float* device_out) {
    return guarded([&]() {
        Session& s = session->impl;
        std::unique_lock lk(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.require_sources();
        require_all_frames(s, lk);
        s.fork();
        for (int n = 0; n < s.frames; ++n) s.render_to_device(n, device_out + static_cast<size_t>(n) * s.frame_values());
        s.join();
    });
}

int vnlbgpu_render_clip_host(vnlbgpu_session* session, float* out) {
    return guarded([&]() {
        Session& s = session->impl;
        std::unique_lock lk(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.require_sources();
        require_all_frames(s, lk);
        if (!s.d_pack.ptr || s.d_pack.count < s.frame_values() * s.frames)
            s.d_pack.allocate(s.frame_values() * s.frames, "cudaMalloc(clip output)");
        // Pinned output: each frame goes down on the download stream as soon
        // as it is normalised.  Pageable output: a copy into pageable memory
        // holds the calling thread, so everything is enqueued first and the
        // clip goes down in one copy at the end.
        cudaPointerAttributes attr{};
        const bool pinned = cudaPointerGetAttributes(&attr, out) == cudaSuccess && attr.type == cudaMemoryTypeHost;
        cudaGetLastError();  // a failed query leaves no sticky error
        const size_t fv = s.frame_values();
        if (!pinned) {
            s.fork();
            for (int n = 0; n < s.frames; ++n) s.render_to_device(n, s.d_pack.ptr + fv * n);
            s.join();
            vnlbgpu::check(cudaMemcpyAsync(out, s.d_pack.ptr, fv * s.frames * sizeof(float), cudaMemcpyDeviceToHost,
                                           s.stream),
                           "cudaMemcpyAsync(clip download)");
            s.check_status();
            return;
        }
        s.fork();
        vnlbgpu::check(cudaEventRecord(s.ev_main, s.stream), "cudaEventRecord(download start)");
        vnlbgpu::check(cudaStreamWaitEvent(s.download_stream, s.ev_main, 0), "cudaStreamWaitEvent(download start)");
        for (int n = 0; n < s.frames; ++n) {
            s.render_to_device(n, s.d_pack.ptr + fv * n);
            vnlbgpu::check(cudaEventRecord(s.ev_out, s.stream), "cudaEventRecord(frame done)");
            vnlbgpu::check(cudaStreamWaitEvent(s.download_stream, s.ev_out, 0), "cudaStreamWaitEvent(frame done)");
            vnlbgpu::check(cudaMemcpyAsync(out + fv * n, s.d_pack.ptr + fv * n, fv * sizeof(float),
                                           cudaMemcpyDeviceToHost, s.download_stream),
                           "cudaMemcpyAsync(frame download)");
        }
        s.join();
        vnlbgpu::check(cudaEventRecord(s.ev_download, s.download_stream), "cudaEventRecord(downloads done)");
        vnlbgpu::check(cudaStreamWaitEvent(s.stream, s.ev_download, 0), "cudaStreamWaitEvent(downloads done)");
        s.check_status();
    });
}

int vnlbgpu_render_chain_device(vnlbgpu_session* basic_session, vnlbgpu_session* final_session, float* basic_out,
                                float* final_out) {
    return guarded([&]() {
        if (!basic_session || !final_session || !basic_out || !final_out) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& b = basic_session->impl;
        Session& f = final_session->impl;
        if (&b == &f || b.stage != 0 || f.stage != 1)
            vnlbgpu::fail("VNLB CUDA: a chain takes a Basic session and a Final session");
        if (b.width != f.width || b.height != f.height || b.frames != f.frames || b.channels != f.channels ||
            b.device != f.device)
            vnlbgpu::fail("VNLB CUDA: the Basic and Final sessions of a chain must share clip geometry and device");
        std::scoped_lock locks(b.lock, f.lock);
        if (!f.store[1].borrowed || f.ref != basic_out)
            vnlbgpu::fail("VNLB CUDA: the Final session's ref must be the chain's Basic output "
                          "(vnlbgpu_set_clip_device with that buffer)");
        vnlbgpu::check(cudaSetDevice(b.device), "cudaSetDevice");
        b.require_sources();
        f.require_sources();
        for (int n = 0; n < b.frames; ++n)
            if (b.frames_pending(n) || f.frames_pending(n))
                vnlbgpu::fail("VNLB CUDA: a chain render needs every source frame on the device, with no copy in flight");
        // Basic on its stream; Final's normalisations on a stream of its own
        // (its session stream, or its own stream when the two share one), so
        // that Final frames do not hold up later Basic frames; the caller's
        // Basic stream waits for everything at the end.
        cudaStream_t fs = f.stream == b.stream ? f.own_stream : f.stream;
        b.fork(b.stream);
        f.fork(b.stream);
        vnlbgpu::check(cudaEventRecord(f.ev_fork, b.stream), "cudaEventRecord(chain fork)");
        vnlbgpu::check(cudaStreamWaitEvent(fs, f.ev_fork, 0), "cudaStreamWaitEvent(chain fork)");
        const size_t fv = b.frame_values();
        int next_final = 0;
        for (int n = 0; n < b.frames; ++n) {
            b.render_to_device(n, basic_out + fv * n, b.stream);
            int lo, hi;
            if (next_final < f.frames) f.required_range(next_final, lo, hi);
            if (next_final < f.frames && (hi <= n || n == b.frames - 1)) {
                // Basic frames 0..n are normalised once this point of the
                // Basic stream is reached (in frame order): Final's lanes may
                // read them after it
                auto ready = b.record_read(b.stream);
                for (int i = 0; i < f.lane_count; ++i)
                    vnlbgpu::check(cudaStreamWaitEvent(f.lanes[i].stream, ready.get(), 0),
                                   "cudaStreamWaitEvent(chain Basic frames)");
                while (next_final < f.frames) {
                    f.required_range(next_final, lo, hi);
                    if (hi > n) break;
                    f.render_to_device(next_final, final_out + fv * next_final, fs);
                    ++next_final;
                }
            }
        }
        b.join();
        for (int i = 0; i < f.lane_count; ++i) {
            vnlbgpu::check(cudaEventRecord(f.ev_lane[i], f.lanes[i].stream), "cudaEventRecord(chain join)");
            vnlbgpu::check(cudaStreamWaitEvent(fs, f.ev_lane[i], 0), "cudaStreamWaitEvent(chain join)");
        }
        vnlbgpu::check(cudaEventRecord(f.ev_main, fs), "cudaEventRecord(chain end)");
        vnlbgpu::check(cudaStreamWaitEvent(b.stream, f.ev_main, 0), "cudaStreamWaitEvent(chain end)");
    });
}

int vnlbgpu_synchronize(vnlbgpu_session* session) {
    return guarded([&]() {
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.check_status();
    });
}

int vnlbgpu_render_stack(vnlbgpu_session* session, int n, float* const* planes, const ptrdiff_t* strides) {
    return guarded([&]() {
        Session& s = session->impl;
        std::unique_lock lk(s.lock);
        if (n < 0 || n >= s.frames) vnlbgpu::fail("VNLB CUDA: frame index out of range");
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.require_sources();
        const size_t packed = static_cast<size_t>(s.channels) * s.slots * 2 * s.plane();
        if (!s.d_pack.ptr || s.d_pack.count < packed) s.d_pack.allocate(packed, "cudaMalloc(stack pack)");
        if (n > s.frames - s.Pt) {
            vnlbgpu::check(cudaMemsetAsync(s.d_pack.ptr, 0, packed * sizeof(float), s.stream), "cudaMemsetAsync(stack)");
        } else {
            while (s.frames_pending(n, true)) s.changed.wait(lk);
            s.fork();
            Session::CachedStack* c = s.stack_for(n);
            vnlbgpu::check(cudaStreamWaitEvent(s.stream, c->ready, 0), "cudaStreamWaitEvent(stack ready)");
            vnlbgpu::check(vnlbgpu::launch_pack_stack(c->data.ptr, c->packed, s.width, s.height, s.channels, s.slots,
                                                      s.d_pack.ptr, s.stream),
                           "pack kernel launch");
            c->reads.push_back(s.record_read(s.stream));
            s.join();
        }
        const int rows = s.slots * 2 * s.height;
        for (int c = 0; c < s.channels; ++c) {
            vnlbgpu::check(cudaMemcpy2DAsync(planes[c], static_cast<size_t>(strides[c]),
                                             s.d_pack.ptr + static_cast<size_t>(c) * rows * s.width,
                                             static_cast<size_t>(s.width) * sizeof(float),
                                             static_cast<size_t>(s.width) * sizeof(float), rows,
                                             cudaMemcpyDeviceToHost, s.stream),
                           "cudaMemcpy2DAsync(stack download)");
        }
        s.check_status();
    });
}

int vnlbgpu_aggregate(const float* stacks, const float* source, int width, int height, int frames, int channels,
                      int search_bwd, int search_fwd, int patch_time, int device_id, float* out) {
    return guarded([&]() {
        if (!stacks || !source || !out) vnlbgpu::fail("VNLB: null argument");
        if (width <= 0 || height <= 0 || frames <= 0 || !(channels == 1 || channels == 3))
            vnlbgpu::fail("VNLB: Aggregate requires matching constant GrayS or YUV444PS clips");
        if (patch_time <= 0 || search_bwd < 0 || search_fwd < 0)
            vnlbgpu::fail("VNLB: patch_time must be positive and search_bwd/search_fwd must be non-negative");
        const int slots = search_bwd + search_fwd + patch_time;
        if (slots > vnlbgpu::kMaxContributors) vnlbgpu::fail("VNLB: at most 32 contribution slots are supported");
        vnlbgpu::check(cudaSetDevice(device_id), "cudaSetDevice");
        const size_t plane = static_cast<size_t>(width) * height;
        const size_t stack_values = plane * channels * slots * 2;
        vnlbgpu::DeviceArray<float> d_stacks, d_source, d_out;
        d_stacks.allocate(stack_values * frames, "cudaMalloc(stacks)");
        d_source.allocate(plane * channels * frames, "cudaMalloc(source)");
        d_out.allocate(plane * channels * frames, "cudaMalloc(output)");
        vnlbgpu::check(cudaMemcpy(d_stacks.ptr, stacks, stack_values * frames * sizeof(float), cudaMemcpyHostToDevice),
                       "cudaMemcpy(stacks)");
        vnlbgpu::check(cudaMemcpy(d_source.ptr, source, plane * channels * frames * sizeof(float),
                                  cudaMemcpyHostToDevice),
                       "cudaMemcpy(source)");
        // render_aggregate_frame (src/vs/plugin.cpp:966-1045)
        for (int n = 0; n < frames; ++n) {
            vnlbgpu::AggregateLaunch L{};
            L.width = width;
            L.height = height;
            L.channels = channels;
            L.slots = slots;
            const int first = std::max(0, n - (search_fwd + patch_time - 1));
            const int last = std::min(frames - 1, n + search_bwd);
            for (int a = first; a <= last; ++a) {
                L.stacks[L.count] = d_stacks.ptr + stack_values * a;
                L.slots_of[L.count] = n - a + search_bwd;
                ++L.count;
            }
            L.source = d_source.ptr + plane * channels * n;
            L.out = d_out.ptr + plane * channels * n;
            vnlbgpu::check(vnlbgpu::launch_aggregate_stacks(L, nullptr), "aggregate kernel launch");
        }
        vnlbgpu::check(cudaMemcpy(out, d_out.ptr, plane * channels * frames * sizeof(float), cudaMemcpyDeviceToHost),
                       "cudaMemcpy(output)");
    });
}

int vnlbgpu_aggregate_frame_noalloc(const float* stacks, const float* source, int width, int height, int frames,
                                    int channels, int search_bwd, int search_fwd, int patch_time, int device_id, int n,
                                    float* out) {
    // no exception and no host allocation on success: the failure text is
    // copied into the error string only when there is one
    const char* failure = vnlbgpu::aggregate_frame_noalloc(stacks, source, width, height, frames, channels,
                                                           search_bwd, search_fwd, patch_time, device_id, n, out);
    if (!failure) return 0;
    vnlbgpu::g_last_error = failure;
    return -1;
}

int vnlbgpu_set_mvtools_analysis(vnlbgpu_session* session, int direction, const void* data, size_t size) {
    return guarded([&]() {
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        if (direction != 0 && direction != 1) vnlbgpu::fail("VNLB: MVTools direction must be 0 (mvfw) or 1 (mvbw)");
        if (!data) vnlbgpu::fail("VNLB: null argument");
        const std::string name = direction == 0 ? "mvfw" : "mvbw";
        vnlbgpu_mvtools_analysis a{};
        try {
            a = vnlbgpu::mvtools::parse_analysis(data, size);
        } catch (const std::invalid_argument& e) {
            vnlbgpu::fail(std::string("VNLB: ") + e.what());
        }
        // validate_mvtools_clip (src/vs/plugin.cpp:452-474)
        if (a.width != s.width || a.height != s.height)
            vnlbgpu::fail("VNLB: " + name + " analysis dimensions must match clip");
        if (a.delta_frame != 1) vnlbgpu::fail("VNLB: " + name + " must use MVTools delta=1 vectors");
        if ((a.backwards != 0) != (direction == 1))
            vnlbgpu::fail(direction == 1 ? "VNLB: mvbw must be generated with isb=True"
                                         : "VNLB: mvfw must be generated with isb=False");
        Session::Flow& f = s.flow[direction];
        f.present = true;
        f.analysis = a;
        f.usable.assign(static_cast<size_t>(s.frames), 0);
        f.vectors.assign(static_cast<size_t>(s.frames) * a.block_count_x * a.block_count_y, make_int2(0, 0));
        f.dirty = true;
        s.invalidate();
    });
}

int vnlbgpu_set_mvtools_frame(vnlbgpu_session* session, int direction, int frame, const void* vectors, size_t size,
                              int scene_change) {
    return guarded([&]() {
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        if (direction != 0 && direction != 1) vnlbgpu::fail("VNLB: MVTools direction must be 0 (mvfw) or 1 (mvbw)");
        if (!vectors) vnlbgpu::fail("VNLB: null argument");
        Session::Flow& f = s.flow[direction];
        if (!f.present)
            vnlbgpu::fail(std::string("VNLB: the ") + (direction == 0 ? "mvfw" : "mvbw") +
                          " analysis data must be set before its frames");
        if (frame < 0 || frame >= s.frames) vnlbgpu::fail("VNLB CUDA: frame index out of range");
        std::vector<int> xy;
        bool valid = false;
        try {
            valid = vnlbgpu::mvtools::parse_vectors(vectors, size, f.analysis, xy);
        } catch (const std::invalid_argument& e) {
            vnlbgpu::fail(std::string("VNLB: ") + e.what());
        }
        // cache_mvtools_grid (plugin.cpp:507-525): a scene change in the source
        // clip makes the frame's grid invalid
        const size_t count = static_cast<size_t>(f.analysis.block_count_x) * f.analysis.block_count_y;
        f.usable[static_cast<size_t>(frame)] = valid && !scene_change ? 1 : 0;
        for (size_t i = 0; i < count; ++i)
            f.vectors[static_cast<size_t>(frame) * count + i] = valid ? make_int2(xy[2 * i], xy[2 * i + 1])
                                                                     : make_int2(0, 0);
        f.dirty = true;
        s.invalidate();
    });
}

int vnlbgpu_shard_plan(int frames, int world, int rank, int basic_search_bwd, int basic_search_fwd,
                       int basic_patch_time, int final_search_bwd, int final_search_fwd, int final_patch_time,
                       int out[2], int basic[2], int source[2]) {
    return guarded([&]() {
        if (!out || !basic || !source) vnlbgpu::fail("VNLB CUDA: null argument");
        if (frames <= 0 || world <= 0 || rank < 0 || rank >= world)
            vnlbgpu::fail("VNLB CUDA: shard plan needs frames > 0 and 0 <= rank < world");
        if (basic_patch_time <= 0 || final_patch_time <= 0 || basic_patch_time > frames || final_patch_time > frames ||
            basic_search_bwd < 0 || basic_search_fwd < 0 || final_search_bwd < 0 || final_search_fwd < 0)
            vnlbgpu::fail("VNLB CUDA: patch_time must fit inside the clip and the search radii must be non-negative");
        // required_source_range of one stage (cuda_plugin.cpp:809-858)
        auto required = [frames](int sb, int sf, int pt, int n, int& lo, int& hi) {
            const int valid = frames - pt + 1;
            lo = hi = n;
            const int a0 = std::max(0, n - (sf + pt - 1));
            const int a1 = std::min(valid - 1, n + sb);
            for (int a = a0; a <= a1; ++a) {
                int low, high;
                vnlbgpu::temporal_range(frames, pt, sb, sf, a, low, high);
                lo = std::min(lo, low);
                hi = std::max(hi, high + pt - 1);
            }
        };
        const long long o0 = static_cast<long long>(rank) * frames / world;
        const long long o1 = static_cast<long long>(rank + 1) * frames / world - 1;
        out[0] = out[1] = basic[0] = basic[1] = source[0] = source[1] = -1;
        if (o1 < o0) return;
        out[0] = static_cast<int>(o0);
        out[1] = static_cast<int>(o1);
        int b0 = out[0], b1 = out[1];
        for (int n = out[0]; n <= out[1]; ++n) {
            int lo, hi;
            required(final_search_bwd, final_search_fwd, final_patch_time, n, lo, hi);
            b0 = std::min(b0, lo);
            b1 = std::max(b1, hi);
        }
        basic[0] = b0;
        basic[1] = b1;
        int s0 = b0, s1 = b1;
        for (int m = b0; m <= b1; ++m) {
            int lo, hi;
            required(basic_search_bwd, basic_search_fwd, basic_patch_time, m, lo, hi);
            s0 = std::min(s0, lo);
            s1 = std::max(s1, hi);
        }
        source[0] = s0;
        source[1] = s1;
    });
}

int vnlbgpu_set_learned(vnlbgpu_session* session, vnlbgpu_mlp* mlp, int shortlist, float recall_threshold,
                        int tile) {
    return guarded([&]() {
        if (!session || !mlp) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        if (!s.learned) vnlbgpu::fail("VNLB CUDA: the session's form is not learned (3)");
        if (shortlist < 1 || shortlist > vnlbgpu::kShortlistMax)
            vnlbgpu::fail("VNLB CUDA: the shortlist must hold 1.." + std::to_string(vnlbgpu::kShortlistMax) +
                          " offsets");
        if (!(recall_threshold >= 0.0f) || !std::isfinite(recall_threshold))
            vnlbgpu::fail("VNLB CUDA: the recall threshold must be finite and non-negative");
        if (tile != s.learned_tile) vnlbgpu::fail("VNLB CUDA: the tile edge of this build is " +
                                                  std::to_string(s.learned_tile) + " pixels");
        const vnlbgpu::MlpDevice net = vnlbgpu::mlp_device(mlp);
        if (net.inputs != s.learned_inputs || net.outputs != s.learned_outputs)
            vnlbgpu::fail("VNLB CUDA: the network must have " + std::to_string(s.learned_inputs) + " inputs and " +
                          std::to_string(s.learned_outputs) + " outputs for this session");
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.drain();
        for (int li = 0; li < s.lanes_allocated; ++li) {
            Session::Lane& l = s.lanes[li];
            l.mlp_acts.allocate(static_cast<size_t>(net.layers) * Session::kLearnedChunk * net.hidden,
                                "cudaMalloc(network activations)");
            l.mlp_logits.allocate(static_cast<size_t>(Session::kLearnedChunk) * net.outputs,
                                  "cudaMalloc(network logits)");
        }
        s.mlp = mlp;
        s.mlp_net = net;
        s.shortlist_len = shortlist;
        s.recall_threshold = recall_threshold;
        s.invalidate();
    });
}

int vnlbgpu_learned_pairs(vnlbgpu_session* session, int anchor, float* features, int* targets, int capacity, int k,
                          int* count, int* inputs) {
    return guarded([&]() {
        if (!session || !count || !inputs || k <= 0) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.require_sources();
        if (anchor < 0 || anchor > s.frames - s.Pt) vnlbgpu::fail("VNLB CUDA: anchor frame out of range");
        vnlbgpu::DeviceArray<float> stack, cells, feats;
        stack.allocate(s.stack_values(), "cudaMalloc(diag stack)");
        vnlbgpu::Grid& grid = s.grid_for(anchor);
        const int G = static_cast<int>(grid.anchors.size());
        *count = G;
        *inputs = s.learned_inputs;
        // the full exact search (and the rest of the anchor frame) on lane 0
        s.fork();
        Session::Lane& lane = s.lanes[0];
        s.force_plain_match = true;
        s.allow_scatter = false;
        try {
            s.compute_anchor(anchor, stack.ptr, lane);
        } catch (...) {
            s.force_plain_match = false;
            s.allow_scatter = true;
            throw;
        }
        s.force_plain_match = false;
        s.allow_scatter = true;
        // features of the same anchors
        int low, high;
        vnlbgpu::temporal_range(s.frames, s.Pt, s.params.search_bwd, s.params.search_fwd, anchor, low, high);
        vnlbgpu::LearnedLaunch ll{};
        ll.video = s.stage == 1 ? s.ref : s.clip;
        ll.ring = s.ring;
        ll.width = s.width;
        ll.height = s.height;
        ll.channels = s.channels;
        ll.search_channels = s.search_channels;
        ll.P = s.P;
        ll.Pt = s.Pt;
        ll.search_window = s.params.search_window;
        int schedule[vnlbgpu::kMaxContributors];
        int len = 0;
        schedule[len++] = anchor;
        for (int f = anchor + 1; f <= high; ++f) schedule[len++] = f;
        for (int f = anchor - 1; f >= low; --f) schedule[len++] = f;
        for (int i = 0; i < len; ++i) ll.schedule[i] = schedule[i];
        ll.schedule_len = len;
        ll.slots_max = s.slots_max;
        ll.anchor_frame = anchor;
        ll.anchors = grid.d_anchors.ptr;
        ll.anchor_count = G;
        cells.allocate(static_cast<size_t>(s.slots_max) * s.search_channels * s.cells_w * s.cells_h, "cudaMalloc");
        feats.allocate(static_cast<size_t>(G) * s.learned_inputs, "cudaMalloc(features)");
        ll.cells = cells.ptr;
        ll.cells_w = s.cells_w;
        ll.cells_h = s.cells_h;
        ll.features = feats.ptr;
        ll.inputs = s.learned_inputs;
        ll.feature_scale = Session::kFeatureScale;
        vnlbgpu::check(vnlbgpu::launch_learned_features(ll, lane.stream), "learned features launch");
        s.join();
        s.check_status();
        const int n = std::min(G, capacity);
        if (features && n > 0)
            vnlbgpu::check(cudaMemcpy(features, feats.ptr, static_cast<size_t>(n) * s.learned_inputs * sizeof(float),
                                      cudaMemcpyDeviceToHost),
                           "copy");
        if (targets && n > 0) {
            std::vector<int> counts(G);
            std::vector<vnlbgpu::MatchRow> rows(static_cast<size_t>(G) * s.max_rows);
            vnlbgpu::check(cudaMemcpy(counts.data(), lane.row_counts.ptr, G * sizeof(int), cudaMemcpyDeviceToHost),
                           "copy");
            vnlbgpu::check(cudaMemcpy(rows.data(), lane.rows.ptr, rows.size() * sizeof(vnlbgpu::MatchRow),
                                      cudaMemcpyDeviceToHost),
                           "copy");
            const int W = s.params.search_window;
            for (int g = 0; g < n; ++g) {
                const int2 a = grid.anchors[static_cast<size_t>(g)];
                int xl, xh, yl, yh;
                vnlbgpu::spatial_range(a.x, s.width, s.P, W, xl, xh);
                vnlbgpu::spatial_range(a.y, s.height, s.P, W, yl, yh);
                for (int j = 0; j < k; ++j) {
                    int cls = -1;
                    if (j < counts[g]) {
                        const vnlbgpu::MatchRow m = rows[static_cast<size_t>(g) * s.max_rows + j];
                        int kk = 0;
                        while (kk < len && schedule[kk] != m.frame) ++kk;
                        if (kk < len) cls = (kk * W + (m.y - yl)) * W + (m.x - xl);
                    }
                    targets[static_cast<size_t>(g) * k + j] = cls;
                }
            }
        }
        s.invalidate();
    });
}

int vnlbgpu_get_stats(vnlbgpu_session* session, vnlbgpu_stats* stats) {
    return guarded([&]() {
        if (!session || !stats) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        unsigned long long totals[4] = {0, 0, 0, 0};
        s.drain();
        vnlbgpu::check(cudaMemcpyAsync(totals, s.d_totals.ptr, sizeof(totals), cudaMemcpyDeviceToHost, s.stream),
                       "cudaMemcpyAsync(totals)");
        vnlbgpu::check(cudaStreamSynchronize(s.stream), "cudaStreamSynchronize");
        s.stats.active_groups = static_cast<long long>(totals[0]);
        s.stats.rows = static_cast<long long>(totals[1]);
        s.stats.learned_tiles = static_cast<long long>(totals[2]);
        s.stats.learned_fallback_tiles = static_cast<long long>(totals[3]);
        s.stats.pipeline_lanes = s.lane_count;
        s.stats.source_slots = s.ring;
        s.stats.source_uploads = s.stats_uploads;
        *stats = s.stats;
    });
}

void* vnlbgpu_stream(vnlbgpu_session* session) { return session ? session->impl.stream : nullptr; }

int vnlbgpu_set_stream(vnlbgpu_session* session, void* stream) {
    return guarded([&]() {
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.collect_timing();
        vnlbgpu::check(cudaStreamSynchronize(s.stream), "cudaStreamSynchronize");
        for (int i = 0; i < s.lane_count; ++i)
            vnlbgpu::check(cudaStreamSynchronize(s.lanes[i].stream), "cudaStreamSynchronize");
        s.stream = stream ? static_cast<cudaStream_t>(stream) : s.own_stream;
    });
}

int vnlbgpu_diag_kernel_timing(vnlbgpu_session* session, int enable, double* ms, long long* launches) {
    return guarded([&]() {
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.collect_timing();
        for (int i = 0; i < vnlbgpu::kTimedCategories; ++i) {
            if (ms) ms[i] = s.kernel_ms[i];
            if (launches) launches[i] = s.kernel_count[i];
            s.kernel_ms[i] = 0.0;
            s.kernel_count[i] = 0;
        }
        s.timing = enable != 0;
    });
}

int vnlbgpu_autotune(vnlbgpu_session* session, int anchor, int* match_warps, int* apply_rows, char* log,
                     size_t log_size) {
    return guarded([&]() {
        if (!session) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.require_sources();
        if (anchor < 0 || anchor > s.frames - s.Pt) vnlbgpu::fail("VNLB CUDA: anchor frame out of range");
        if (s.learned) vnlbgpu::fail("VNLB CUDA: the learned form is not autotuned");
        s.drain();
        std::vector<std::pair<std::string, double>> entries;
        s.autotune(anchor, entries);
        if (match_warps) *match_warps = s.warps;
        if (apply_rows) *apply_rows = s.apply_general ? 1 : 0;
        if (log && log_size > 0) {
            std::ostringstream o;
            for (const auto& e : entries) o << e.first << ": " << e.second << " ms\n";
            const std::string text = o.str();
            const size_t n = std::min(log_size - 1, text.size());
            std::memcpy(log, text.data(), n);
            log[n] = '\0';
        }
    });
}

int vnlbgpu_diag_stall_tensor_waits(vnlbgpu_session* session, int on) {
    return guarded([&]() {
        if (!session) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        s.stall_mma = on != 0;
        s.invalidate();
    });
}

int vnlbgpu_diag_set_lanes(vnlbgpu_session* session, int lanes) {
    return guarded([&]() {
        if (!session) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.drain();
        s.lane_count = lanes <= 0 ? s.lanes_allocated : std::min(lanes, s.lanes_allocated);
        s.next_lane = 0;
    });
}

int vnlbgpu_diag_filtered(vnlbgpu_session* session, int anchor, float* out, int capacity, int* rows, int* row_dim) {
    return guarded([&]() {
        if (!session || !rows || !row_dim) vnlbgpu::fail("VNLB CUDA: null argument");
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.require_sources();
        if (anchor < 0 || anchor > s.frames - s.Pt) vnlbgpu::fail("VNLB CUDA: anchor frame out of range");
        vnlbgpu::DeviceArray<float> stack;
        stack.allocate(s.stack_values(), "cudaMalloc(diag stack)");
        s.fork();
        Session::Lane& lane = s.lanes[0];
        s.allow_scatter = false;  // the rows are written out, for the read-back
        try {
            s.compute_anchor(anchor, stack.ptr, lane);
        } catch (...) {
            s.allow_scatter = true;
            throw;
        }
        s.allow_scatter = true;
        s.join();
        s.check_status();
        vnlbgpu::FrameCounters c{};
        vnlbgpu::check(cudaMemcpy(&c, lane.counters.ptr, sizeof(c), cudaMemcpyDeviceToHost), "copy");
        *rows = c.rows;
        *row_dim = s.row_dim;
        const int n = std::min(c.rows, capacity);
        if (out && n > 0)
            vnlbgpu::check(cudaMemcpy(out, lane.filtered.ptr, static_cast<size_t>(n) * s.row_dim * sizeof(float),
                                      cudaMemcpyDeviceToHost),
                           "copy");
        s.invalidate();
    });
}

int vnlbgpu_diag_anchor(vnlbgpu_session* session, int anchor, int* grid_xy, int* grid_counts,
                        vnlbgpu_diag_row* grid_rows, int grid_capacity, int grid_row_capacity, int* active,
                        vnlbgpu_diag_row* active_rows, int active_capacity, int active_row_capacity, int* groups,
                        int* active_groups, int* rows, int* max_rows) {
    return guarded([&]() {
        Session& s = session->impl;
        std::lock_guard guard(s.lock);
        vnlbgpu::check(cudaSetDevice(s.device), "cudaSetDevice");
        s.require_sources();
        if (anchor < 0 || anchor > s.frames - s.Pt) vnlbgpu::fail("VNLB CUDA: anchor frame out of range");
        vnlbgpu::DeviceArray<float> stack;
        stack.allocate(s.stack_values(), "cudaMalloc(diag stack)");
        s.fork();
        Session::Lane& lane = s.lanes[0];
        s.compute_anchor(anchor, stack.ptr, lane);
        s.join();
        s.check_status();
        vnlbgpu::Grid& grid = s.grid_for(anchor);
        const int G = static_cast<int>(grid.anchors.size());
        *groups = G;
        *max_rows = s.max_rows;
        std::vector<int> counts(G);
        vnlbgpu::check(cudaMemcpy(counts.data(), lane.row_counts.ptr, G * sizeof(int), cudaMemcpyDeviceToHost), "copy");
        std::vector<vnlbgpu::MatchRow> mrows(static_cast<size_t>(G) * s.max_rows);
        vnlbgpu::check(cudaMemcpy(mrows.data(), lane.rows.ptr, mrows.size() * sizeof(vnlbgpu::MatchRow),
                                  cudaMemcpyDeviceToHost),
                       "copy");
        for (int g = 0; g < G && g < grid_capacity; ++g) {
            grid_xy[2 * g] = grid.anchors[g].x;
            grid_xy[2 * g + 1] = grid.anchors[g].y;
            grid_counts[g] = counts[g];
            for (int j = 0; j < counts[g] && static_cast<long long>(g) * s.max_rows + j < grid_row_capacity; ++j) {
                const auto& m = mrows[static_cast<size_t>(g) * s.max_rows + j];
                grid_rows[static_cast<size_t>(g) * s.max_rows + j] = vnlbgpu_diag_row{m.distance, m.x, m.y, m.frame, 0.0f};
            }
        }
        vnlbgpu::FrameCounters c{};
        vnlbgpu::check(cudaMemcpy(&c, lane.counters.ptr, sizeof(c), cudaMemcpyDeviceToHost), "copy");
        *active_groups = c.active;
        *rows = c.rows;
        std::vector<int> act(c.active);
        if (c.active > 0)
            vnlbgpu::check(cudaMemcpy(act.data(), lane.active.ptr, c.active * sizeof(int), cudaMemcpyDeviceToHost), "copy");
        for (int i = 0; i < c.active && i < active_capacity; ++i) active[i] = act[i];
        std::vector<vnlbgpu::MatchRow> info(c.rows);
        std::vector<float> w(c.rows);
        if (c.rows > 0) {
            vnlbgpu::check(cudaMemcpy(info.data(), lane.row_info.ptr, c.rows * sizeof(vnlbgpu::MatchRow),
                                      cudaMemcpyDeviceToHost),
                           "copy");
            vnlbgpu::check(cudaMemcpy(w.data(), lane.weights.ptr, c.rows * sizeof(float), cudaMemcpyDeviceToHost), "copy");
        }
        for (int r = 0; r < c.rows && r < active_row_capacity; ++r)
            active_rows[r] = vnlbgpu_diag_row{info[r].distance, info[r].x, info[r].y, info[r].frame, w[r]};
        s.invalidate();
    });
}

}  // extern "C"
