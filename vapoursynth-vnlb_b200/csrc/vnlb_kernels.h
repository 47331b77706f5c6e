// Launch descriptors shared by the host pipeline (session.cpp) and the
// kernels (match.cu, paste.cu, filter.cu, aggregate.cu).  Plain structs of
// device pointers and sizes; one descriptor per launch.
#pragma once

#include <cstddef>
#include <cuda.h>  // CUtensorMap (the type only; the encoder is fetched at run time)
#include <cuda_runtime.h>

#include "vnlb_common.cuh"

namespace vnlbgpu {

// Kernel classes timed by the session (vnlbgpu_diag_kernel_timing).
enum TimedCategory { kTimedMatch = 0, kTimedPaste, kTimedFilter, kTimedTiles, kTimedNormalize, kTimedCategories };

// Most temporal slots (search_bwd + search_fwd + patch_time) and scheduled
// candidate frames the GPU path handles.
constexpr int kMaxContributors = 32;

// A run of consecutive grid anchors of one grid row handled by one CTA of the
// match kernel, with the shared-memory region that covers all their windows.
struct Strip {
    int first;     // index of the first anchor in the anchor list
    int count;     // anchors in the strip (<= warps per CTA)
    int y;         // their common row
    int region_x;  // region origin (x multiple of 4), in pixels
    int region_y;
    int region_w;  // region extent in pixels
    int region_h;
};

// A strip of the tensor-core matcher: up to kChosenAnchors consecutive
// anchors of each of one or two consecutive grid rows, all of whose search
// windows lie within kChosenCols candidate columns from region_x.
struct TcStrip {
    int first[2];  // index of each row's first anchor in the anchor list
    int count[2];  // anchors of each row (the second row's may be 0)
    int y[2];      // the rows' anchor y
    int region_x;  // first candidate column
    int pad;
};

// Source frames on the device: frame f of a source lives in slot f % ring of
// a store of ring + patch_time - 1 frame slots [slot][channels][H][W], whose
// last patch_time - 1 slots repeat the first ones, so that the patch_time
// consecutive frames of a patch are consecutive slots.  ring = frames for a
// whole resident clip.
struct MatchLaunch {
    const float* video;   // search source, frame slots as above
    int width, height, channels, frames;
    int ring;             // frame slots of the source store (f -> f % ring)
    int search_channels;  // channels compared (1 = first plane only)
    int P, Pt, search_window;
    int K, soft_cap, max_rows;
    float tau;
    int anchor_frame;
    int schedule[kMaxContributors];  // scheduled candidate frames (CPU order)
    int schedule_len;
    const int2* anchors;  // grid anchors in raster order
    const Strip* strips;
    const TcStrip* tc_strips;  // tensor-core matcher strips
    float* strip_mu;           // [strips][kChosenMaxPlanes] their per-plane offsets (tensor-core matcher)
    int plane_group;           // tensor-core matcher: planes per shared-memory stage (0: the most that fit)
    const int* anchor_map;  // [H][W] anchor index or -1
    int region_rows;      // shared rows per plane (incl. padding)
    int region_stride;    // shared row stride in floats
    int plane_floats;     // shared floats per plane (region_rows * region_stride, or rounded up to 32
                          // floats when the planes are loaded by the tensor memory accelerator)
    int tma;              // stage each frame's planes with cp.async.bulk.tensor (the tensor map
                          // covers the source store as rows of width `width`)
    int region_w_max;     // widest region a pass may stage (flow-guided search)
    int window_cells;     // max Wx*Wy
    int buffer_cap;       // match buffer capacity per warp
    int warp_floats;      // shared floats per warp
    int approx;           // chosen form in this matcher: approximate distances, exact re-rank
    // tensor-core form (match_chosen.cu)
    int tiles_x;          // 8-column candidate blocks per strip
    int window_rows;      // max Wy
    int* status;          // session status word (kStatus* codes, first error wins)
    // flow-guided search (plain matcher): the search centre of every anchor in
    // every scheduled frame, [anchor][schedule_len]; null = the anchor itself.
    // With centres, each frame's region is the bounding box of the strip's
    // windows around their centres, staged in passes when it does not fit.
    const int2* centers;
    float* approx_dist;   // [anchor][approx_stride] approximate distances (tensor-core form)
    int approx_stride;    // >= schedule_len * window_cells
    int anchor_count;     // grid anchors of this anchor frame
    int strip_count;      // strips of the launch (tensor-core form)
    // learned form's fallback: strip s belongs to tile strip_tile[s] and runs
    // only when tile_fail of that tile is set (null: every strip runs)
    const int* strip_tile;
    const int* tile_fail;
    // tensor-core matcher, for tests of its bounded waits: the MMA warp issues
    // no MMA, so the waits for their completion run out (no MMA in flight)
    int stall_mma;
    // outputs
    MatchRow* rows;       // [G][max_rows]
    int* row_counts;      // [G]
    int* victims;         // [G][victim_stride]
    int* victim_counts;   // [G]
    int victim_stride;
};

// Chosen form on tensor cores (match_chosen.cu): a CTA matches a strip of up
// to kChosenAnchors consecutive anchors of each of one or two consecutive
// grid rows whose search windows lie within kChosenCols consecutive
// candidate columns.  One tcgen05 MMA (M = 128, N = 16, K = 16) covers two
// candidate rows of those columns against the strip's 16 anchor slots, so
// the strip's windows may span at most 2 * 16 rows (16 row pairs of 16
// accumulator columns fill kChosenTmemCols).
// Patches are 7 x 7 or 8 x 8, compared over up to kChosenMaxPlanes planes
// (search channels x patch_time), and the capped buffer holds up to
// kChosenMaxBuffer entries.
constexpr int kChosenAnchors = 8;
constexpr int kChosenWarps = 8;
constexpr int kChosenCols = 64;
constexpr int kChosenMaxRows = 32;
constexpr int kChosenTmemCols = 256;
constexpr int kChosenMaxPlanes = 6;
constexpr int kChosenMaxBuffer = 96;

bool chosen_match_supported(int P, int planes_n, int window_w, int window_h);
size_t chosen_match_shared_bytes(const MatchLaunch& L);
// the most planes per shared-memory stage of the tensor-core matcher
int chosen_max_plane_group(int planes_n, int window_rows);
cudaError_t launch_match_chosen(const MatchLaunch& L, int strips, cudaStream_t stream);

// One direction of MVTools motion vectors on the device (mvfw or mvbw).
struct FlowGridsDevice {
    int present;
    int block_size_x, block_size_y, pel, overlap_x, overlap_y, block_count_x, block_count_y;
    const unsigned char* usable;  // [frames]
    const int2* vectors;          // [frames][block_count_y][block_count_x], sub-pel units
};

// Search centres of one anchor frame (MVToolsFlowProvider::center_for,
// src/flow/flow.hpp:341-389), one thread per anchor and scheduled frame.
struct CentersLaunch {
    FlowGridsDevice fw, bw;
    const int2* anchors;
    int anchor_count;
    int schedule[kMaxContributors];
    int schedule_len;
    int anchor_frame;
    int width, height, P;
    int2* centers;  // [anchor][schedule_len]
};

cudaError_t launch_centers(const CentersLaunch& L, cudaStream_t stream);

size_t match_shared_bytes(const MatchLaunch& L, int warps);
int match_warp_floats(int window_cells, int planes_n, int P, int buffer_cap);
// tmap: the search source store as a 2-D float tensor (width x rows of every
// plane of every slot), box (region_stride, region_rows); used when L.tma.
cudaError_t launch_match(const MatchLaunch& L, int strips, int warps, const CUtensorMap* tmap,
                         cudaStream_t stream);
// Encodes the tensor map of a source store for the plain matcher's staging:
// rows of `width` floats, `rows` of them, box (box_w, box_h).  False when the
// layout cannot be loaded by TMA (row pitch or base not 16-byte aligned).
bool encode_store_map(CUtensorMap* map, const float* base, int width, long long rows, int box_w, int box_h);

// Device-side counters of one anchor frame.
struct FrameCounters {
    int active;      // active (processed) groups
    int rows;        // total retained rows of the active groups
    int status;      // 0 or an error code (see kStatus*)
    int detail;
};

constexpr int kStatusRankNotCovered = 1;  // fewer model rows than the rank
constexpr int kStatusPasteCapacity = 2;   // too many anchors for the paste kernel
constexpr int kStatusTensorTimeout = 3;   // an MMA completion wait ran out (tensor-core matcher)
constexpr int kStatusTmaTimeout = 4;      // a tensor-memory-accelerator load wait ran out (plain matcher)

struct PasteLaunch {
    int groups;
    const int* row_counts;
    const int* victims;
    const int* victim_counts;
    int victim_stride;
    const int2* anchors;
    // outputs
    int* active;          // [G] active anchor indices in raster order
    int2* active_xy;      // [G] their positions
    int* row_offset;      // [G + 1] exclusive prefix of retained rows
    int* active_prefix;   // [G + 1] active groups before grid anchor j
    FrameCounters* counters;
    unsigned long long* totals;  // session totals: active groups, rows
};

cudaError_t launch_paste(const PasteLaunch& L, cudaStream_t stream);

// Fills map[y*width + x] with the index of each grid anchor (the map must be
// preset to -1).
cudaError_t launch_anchor_map(const int2* anchors, int count, int width, int* map, cudaStream_t stream);

struct FilterLaunch {
    const float* noisy;     // frame slots [slot][C][H][W] (MatchLaunch)
    const float* basic;     // Final only, the same slots
    int ring;               // frame slots of both stores (f -> f % ring)
    int width, height, channels;
    int stage;
    int P, Pt, patch_dim, dim;
    int K, model_cap, rank, max_rows;
    int coupled;            // sample-major (coupled, C > 1) vs group path
    int models;             // models per group: 1, or the planes of an uncoupled clip
    int nmax;               // largest eigen problem: model rows, or dim where a covariance model occurs
    int row_dim;            // filtered row width: patch_dim * planes (dim when coupled)
    int mixed;              // chosen forms: dual Gram on TF32 tensor cores (FP32 accumulation) and
                            // FP64 Jacobi rotation angles; 0 = the CPU core's FP32 arithmetic
    // chosen forms, warp-per-group shapes: the apply kernel adds each filtered
    // row straight into the anchor frame's stack (atomics, any order) instead
    // of writing it out for the stack tiles; null = write the rows
    int apply_general;      // the row-tiled apply even where the warp-per-group one fits (autotuner)
    float* scatter;         // the stack, cleared before the launch: [slots][C+1][H][W], or
                            // [slots][H][W][C+1] where scatter_pack = C+1 (see filter_scatter_pack)
    int scatter_pack;       // 0: planar stack; C+1: pixel-interleaved (one vector addition per pixel)
    const float* window;    // [P*P] aggregation window
    int windowed, slots, search_bwd, anchor_frame;
    StageConfig cfg;
    const MatchRow* rows;   // [G][max_rows]
    const int* row_counts;
    const int* active;
    const int* row_offset;
    FrameCounters* counters;
    int* status;            // session status word (first error wins), not reset per anchor frame
    // per model v = active group a * models + plane (intermediates between the
    // three filter kernels)
    float* means;           // [G][2][dim]: model (membership) mean, reconstruction centre
    float* gram;            // [G][nmax*nmax]: dual Gram (B x B) or covariance (dim x dim)
    float* eig;             // [G][rank]
    float* dual;            // [G][rank][nmax]: dual vectors (B long) or covariance eigenvectors (dim long)
    int* flags;             // [G]: kGroupDone / kGroupSkip
    // outputs, indexed by global row r = row_offset[a] + i
    float* filtered;        // [R][row_dim]
    float* logw;            // [R][models], uncoupled only: each plane model's log-weight term
    float* weights;         // [R]
    MatchRow* row_info;     // [R]
    int* row_group;         // [R] active index of the row's group
};

constexpr int kGroupDone = 1;  // equal group: passed through, weights written
constexpr int kGroupSkip = 2;  // rank not covered: reported through the status word

// Three launches: prepare (equality, flat flag, means, Gram), batched Jacobi,
// and apply (basis, coefficients, weights, reconstruction).
cudaError_t launch_filter(const FilterLaunch& L, int max_groups, cudaStream_t stream);

// The most dynamic shared memory one CTA of the three filter kernels asks for
// at this shape (dim, rank, nmax, model rows, stage), and the most a CTA may
// have; a shape above the limit cannot be filtered.
size_t filter_shared_bytes(const FilterLaunch& L);
size_t filter_shared_limit();
// The shapes whose apply kernel can add rows straight into the stack
// (FilterLaunch::scatter): warp-per-group, one model per group.
bool filter_can_scatter(const FilterLaunch& L);
// The stack layout such a launch adds into: C+1 when every pixel's C values
// and weight can go in one 8- or 16-byte vector addition (C = 1, or C = 3
// with 64 columns per plane, which puts a lane's columns of the three planes
// on the same pixels), else 0 (planar).
int filter_scatter_pack(const FilterLaunch& L);

struct TileLaunch {
    int width, height, channels;
    int P, Pt, patch_dim, dim;
    int slots, search_bwd, anchor_frame;
    int coupled;            // sample-major contribution writer (coupled, C > 1)
    int windowed;           // weight_gamma != 0
    const float* window;    // [P*P]
    const int* row_offset;  // [active + 1]
    const int* active_prefix;  // [G + 1]
    const float* filtered;
    const float* weights;
    const MatchRow* row_info;
    float* stack;           // [slots][C+1][H][W]
    int tiles_x, tiles_y;
    // reach tables of the anchor grid (host-built per grid)
    const int2* tile_grid_rows;  // [tiles_y]: grid rows whose anchors can reach tile row
    const int2* tile_anchors;    // [grid rows][tiles_x]: anchor index range reaching tile column
};

constexpr int kTile = 16;  // stack tile edge, one pixel per thread

cudaError_t launch_tiles(const TileLaunch& L, cudaStream_t stream);

struct NormalizeLaunch {
    int width, height, channels;
    const float* stacks[kMaxContributors];  // contributing anchor stacks, in anchor order
    int slots[kMaxContributors];            // slot of the output frame in each stack
    int packed[kMaxContributors];           // 0: planar stack; C+1: pixel-interleaved [slots][H][W][C+1]
    int count;
    const float* source;         // fallback plane set of the output frame [C][H][W]
    float* out;                  // [C][H][W]
};

cudaError_t launch_normalize(const NormalizeLaunch& L, cudaStream_t stream);

// Packs one anchor stack into the vnlb.Basic/Final frame layout: per channel
// a plane of slots*2*H rows (numerators, then weights duplicated per channel).
// vnlb.Aggregate on stacks already in the plugin frame layout.
struct AggregateLaunch {
    int width, height, channels, slots;
    const float* stacks[kMaxContributors];  // [C][slots*2*H][W] per anchor
    int slots_of[kMaxContributors];
    int count;
    const float* source;  // [C][H][W]
    float* out;           // [C][H][W]
};

cudaError_t launch_aggregate_stacks(const AggregateLaunch& L, cudaStream_t stream);

cudaError_t launch_pack_stack(const float* stack, int packed, int width, int height, int channels, int slots,
                              float* out, cudaStream_t stream);

// vnlb.Aggregate of output frame n through a fixed device scratch of
// kNoAllocScratchBytes per device, with no allocation (aggregate_noalloc.cu).
// Returns null on success, else the failure text.
constexpr size_t kNoAllocScratchBytes = static_cast<size_t>(32) << 20;
const char* aggregate_frame_noalloc(const float* stacks, const float* source, int width, int height, int frames,
                                    int channels, int search_bwd, int search_fwd, int patch_time, int device_id,
                                    int n, float* out);

}  // namespace vnlbgpu
