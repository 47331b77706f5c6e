/*
 * vnlbgpu: C ABI of the B200-native VNLB denoising hot path.
 *
 * This is the boundary a VapourSynth plugin (or any other host) binds to.  It
 * replaces the CUDA stage pipeline and frame scheduler that the reference's
 * vnlbcu plugin drives from its getFrame callback, and adds GPU-backed
 * contribution stacks for the reference's vnlb plugin:
 *
 *   reference interface                              entry point here
 *   ---------------------------------------------    ----------------------------
 *   create_filter / parse_parameters /               vnlbgpu_create
 *     validate_parameters / derive_geometry /
 *     initialize_cuda  (src/vs/cuda_plugin.cpp:
 *     2066-2131, 370-807, 1866-2020)
 *   CudaFilterFree (cuda_plugin.cpp:2022-2036)       vnlbgpu_destroy
 *   upload_source_misses (cuda_plugin.cpp:           vnlbgpu_set_frame,
 *     1291-1361), noisy/basic FrameCache               vnlbgpu_set_clip_host,
 *     (src/cuda/frame_cache.cpp:120-537)               vnlbgpu_set_clip_device
 *   required_source_range (cuda_plugin.cpp:846-858)  vnlbgpu_required_source_range
 *   render_frame (cuda_plugin.cpp:1635-1864) =       vnlbgpu_render_frame_window,
 *     vnlbcu.Basic / vnlbcu.Final getFrame,            vnlbgpu_render_frame
 *     with fetch_frames + upload_source_misses
 *   render_stage_frame (src/vs/plugin.cpp:616-758)   vnlbgpu_render_stack
 *     = vnlb.Basic / vnlb.Final getFrame
 *   render_aggregate_frame (plugin.cpp:966-1045)     vnlbgpu_aggregate
 *     = vnlb.Aggregate getFrame
 *   setFilterError / mapSetError text                vnlbgpu_last_error
 *     ("VNLB CUDA: ..." / "VNLB: ...")
 *
 * Conventions: every call returns 0 on success and -1 on failure; the failure
 * text (prefixed like the reference's messages) is then available from
 * vnlbgpu_last_error() on the calling thread.  No C++ exception crosses this
 * boundary.  Sizes are in samples (float32); strides are in bytes, as
 * VapourSynth's getStride reports them.  A session is safe to call from
 * several threads.  Per-frame calls (set_frame, render_frame,
 * render_frame_window) each lease one of num_streams workers and queue their
 * GPU work under the session's lock, then wait for it with the lock released,
 * so up to num_streams of them overlap on the GPU; the other calls hold the
 * lock until they return.  Results match the reference CPU core bit for bit
 * for the plain form (see the parity tests).
 */
#ifndef VNLBGPU_H
#define VNLBGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VNLBGPU_STAGE_BASIC 0
#define VNLBGPU_STAGE_FINAL 1

#define VNLBGPU_SOURCE_CLIP 0 /* the noisy clip ("clip") */
#define VNLBGPU_SOURCE_REF 1  /* the basic estimate ("ref"), Final only */

/* Parameters in the core's units: sigma and sigma_basic already divided by
 * 255, tau by 255^2 (the plugin argument rules of parse_parameters,
 * cuda_plugin.cpp:370-536, and parse_stage_parameters, plugin.cpp:372-449,
 * are applied by the host-side plugin layer before this call). */
typedef struct vnlbgpu_params {
    int stage;
    float sigma;
    int patch_size;        /* block_size */
    int patch_time;
    int search_window;     /* 2 * bm_range + 1 */
    int search_bwd;
    int search_fwd;
    int similar;           /* group_size */
    int rank;
    float similar_cap_factor; /* cap_factor */
    float model_cap_factor;
    float beta;
    float tau;
    float variance_threshold;
    float sigma_basic;
    float gamma;           /* flat-area gamma */
    float weight_alpha;
    float weight_beta;
    float weight_gamma;
    float weight_epsilon;
    float membership_noise_floor;
    int proc_step;         /* block_step; 0 = automatic (patch_size) */
    int flat_areas;
    int couple_channels;   /* chroma */
    int device_id;
    int num_streams;       /* accepted like vnlbcu (1..32) */
    int chunk_size;        /* accepted like vnlbcu (> 0) */
    int form;              /* VNLBGPU_FORM_*; no reference counterpart */
} vnlbgpu_params;

/* Forms of the matcher (no reference counterpart).  PLAIN reproduces the
 * reference CPU core bit for bit.  CHOSEN ranks candidates by the
 * approximate distance ||a||^2 + ||b||^2 - 2 a.b (FP32 dot products, FP32
 * norms), runs the CPU's selection on those values, re-computes the exact
 * FP32 distance of every retained candidate and selects on the exact values:
 * within a PSNR tolerance of PLAIN rather than bit-identical.  CHOSEN_TC does
 * the same with the dot products on BF16 tensor cores (tcgen05, FP32
 * accumulation in tensor memory).  CHOSEN applies to 8x8 patches with a
 * buffer of at most 32 patches (group_size * cap_factor) and group_size <= 32.
 * CHOSEN_TC applies to 7x7 and 8x8 patches compared over at most 6 planes
 * (search channels x patch_time), a search window of at most 64 columns by
 * 32 rows, a buffer of at most 96 patches and group_size <= 32: vnlbcu's own
 * defaults included.  Other configurations run PLAIN.  With either chosen
 * matcher the group filter runs
 * in mixed precision too: the dual Gram on TF32 tensor cores with FP32
 * accumulation, the Jacobi rotation angles in FP64. */
#define VNLBGPU_FORM_PLAIN 0
#define VNLBGPU_FORM_CHOSEN 1
#define VNLBGPU_FORM_CHOSEN_TC 2
/* LEARNED: learned block-match proposals (vnlbgpu_set_learned).  An MLP
 * scores every offset of each anchor's search window from coarse features
 * of its neighbourhood; exact SSD runs on the best-scored offsets (and the
 * anchor itself) only, and the plain selection rule picks the rows among
 * them.  In every tile of anchors the full search runs for one anchor as the
 * check; where the learned rows' recall of its K nearest is below the
 * threshold, the whole tile is searched in full instead. */
#define VNLBGPU_FORM_LEARNED 3

typedef struct vnlbgpu_session vnlbgpu_session;

typedef struct vnlbgpu_stats {
    long long anchor_frames;   /* anchor frames computed */
    long long groups;          /* grid anchors matched */
    long long active_groups;   /* groups filtered (after the paste mask) */
    long long rows;            /* retained rows filtered and aggregated */
    long long kernel_launches; /* kernels this session launched */
    long long pipeline_lanes;  /* anchor frames the session keeps in flight (1-8, fewer
                                  when their group buffers would exceed half of the free
                                  device memory at create time) */
    long long source_slots;    /* frames each source store holds on the device */
    long long source_uploads;  /* source frames copied to the device */
    long long learned_tiles;   /* learned form: tiles checked against the full search */
    long long learned_fallback_tiles; /* ... and searched in full after the check */
} vnlbgpu_stats;

const char* vnlbgpu_last_error(void);

/* Validates the parameters for a clip of `frames` frames of width x height
 * with 1 (GrayS) or 3 (YUV444PS) planes and reserves device memory.  No
 * device memory is sized by `frames`: the group buffers follow the frame
 * size, the contribution stacks number slots + lanes + num_streams - 1, and
 * each source store holds min(frames, source window + num_streams - 1)
 * frames, the source window being 2 * (search_bwd + search_fwd + patch_time
 * - 1) + 1 frames (derive_geometry's max_source_window,
 * cuda_plugin.cpp:761-773), until a whole clip is given. */
int vnlbgpu_create(const vnlbgpu_params* params, int width, int height, int frames, int channels,
                   vnlbgpu_session** out);
void vnlbgpu_destroy(vnlbgpu_session* session);

/* Sources.  Frames are immutable, as VapourSynth's are: a frame index names
 * the same samples for the session's life.
 *
 * set_frame copies one frame from per-plane host pointers with byte strides
 * into the source's store on the device, unless that frame is there already;
 * the store is a ring, so a frame can push out the frame a store's capacity
 * before or after it.  set_clip_host copies a whole clip laid out
 * [frames][planes][H][W] and makes the stores hold every frame;
 * set_clip_device makes the session read a caller-owned device buffer of that
 * layout (no copy; it must stay valid while the session uses it).  The two
 * whole-clip calls drop the cached contribution stacks. */
int vnlbgpu_set_frame(vnlbgpu_session* session, int source, int frame, const float* const* planes,
                      const ptrdiff_t* strides);
int vnlbgpu_set_clip_host(vnlbgpu_session* session, int source, const float* clip);
int vnlbgpu_set_clip_device(vnlbgpu_session* session, int source, const float* device_clip);

/* The source frames [*first, *last] that output frame n may read: the union
 * of its contributing anchor frames' shifted temporal windows plus
 * patch_time - 1 (required_source_range, cuda_plugin.cpp:846-858).  A plugin
 * requests these frames in its arInitial step. */
int vnlbgpu_required_source_range(vnlbgpu_session* session, int n, int* first, int* last);

/* vnlbcu.Basic / vnlbcu.Final getFrame (render_frame, cuda_plugin.cpp:
 * 1635-1864): the denoised output frame n (aggregated), into per-plane host
 * pointers with byte strides.  The call gives the source frames first ..
 * first + count - 1, normally the required source range: clip_planes and
 * clip_strides hold count * planes entries, frame-major (frame first + i,
 * plane c at i * planes + c), and ref_planes / ref_strides the same for the
 * Final stage's ref clip (NULL for Basic).  Frames not on the device yet are
 * copied through pinned staging; the frames are held until the call's reads
 * are queued, so concurrent calls cannot push out one another's frames.
 * count must not exceed the store's frames (vnlbgpu_stats.source_slots).
 * Anchor frames whose contribution stacks are cached are not recomputed. */
int vnlbgpu_render_frame_window(vnlbgpu_session* session, int n, int first, int count,
                                const float* const* clip_planes, const ptrdiff_t* clip_strides,
                                const float* const* ref_planes, const ptrdiff_t* ref_strides, float* const* planes,
                                const ptrdiff_t* strides);

/* The same output frame from the frames already on the device (given by
 * set_frame or a whole-clip call); raises naming the first frame it needs
 * that is not. */
int vnlbgpu_render_frame(vnlbgpu_session* session, int n, float* const* planes, const ptrdiff_t* strides);

/* Whole clip in one call, [frames][planes][H][W], into host or device memory;
 * every frame of the sources must be on the device (a whole-clip source, or
 * a clip no longer than the stores).  The device form enqueues on the
 * session's stream and returns without waiting; vnlbgpu_synchronize waits and
 * reports device-side errors.  The host form allocates a device buffer of the
 * whole output clip. */
int vnlbgpu_render_clip_host(vnlbgpu_session* session, float* out);
int vnlbgpu_render_clip_device(vnlbgpu_session* session, float* device_out);
int vnlbgpu_synchronize(vnlbgpu_session* session);

/* vnlbcu.Basic into vnlbcu.Final over a whole clip on the device, the two
 * stages overlapped: Basic frame n is normalised on the Basic session's
 * stream, and the Final session's anchor frames start as soon as the Basic
 * frames of their windows are out, instead of after the whole Basic clip.
 * The Final session's ref must be basic_out (vnlbgpu_set_clip_device); every
 * source frame must be on the device.  Enqueues and returns; the Basic
 * session's stream ends after all of the chain's work (vnlbgpu_synchronize on
 * either session waits and reports device-side errors).  The reference runs
 * the two filters as separate VapourSynth nodes; this is their frame-level
 * dependency, scheduled on the device. */
int vnlbgpu_render_chain_device(vnlbgpu_session* basic_session, vnlbgpu_session* final_session, float* basic_out,
                                float* final_out);

/* vnlb.Basic / vnlb.Final: the contribution stack of anchor frame n in the
 * plugin's frame layout (per plane, slots*2*H rows: numerators then weights,
 * weights repeated in every plane). */
int vnlbgpu_render_stack(vnlbgpu_session* session, int n, float* const* planes, const ptrdiff_t* strides);

/* vnlb.Aggregate over host stacks [frames][planes][slots*2*H][W] and the
 * source clip [frames][planes][H][W], all frames. */
int vnlbgpu_aggregate(const float* stacks, const float* source, int width, int height, int frames, int channels,
                      int search_bwd, int search_fwd, int patch_time, int device_id, float* out);

/* vnlb.Aggregate of the single output frame n (0 <= n < frames), from the
 * same host stacks and source clip as vnlbgpu_aggregate, into host memory
 * [planes][H][W].  It has no counterpart in the reference.  It allocates
 * nothing: no cudaMalloc, no cudaFree, no allocating library routine.  It is
 * for hosts that cannot allocate device memory while serving frames, such as
 * a frame server that reserves its device memory budget at start-up and
 * shares the GPU with other filters; there an allocation in the middle of a
 * clip can fail under memory pressure, and a free waits for the whole device.
 * The rows pass through a fixed 32 MiB device scratch per device, in bands of
 * whole rows.  One row of the frame's contributing stacks, source and output
 * must fit: (contributing stacks * 2 + 2) * planes * width * 4 bytes
 * <= 32 MiB.  A larger frame is rejected with an error.  The first call on a
 * device sets up that device's scratch address; make it before any stream
 * capture begins.  Calls on one device are serialised inside, because calls
 * whose GPU work overlapped would race on the one scratch; an error return
 * comes only after the call's queued work has drained.  Every call queues its
 * copies and kernel on the legacy default stream, so it waits for the
 * caller's blocking streams on that device and must not run while one of them
 * is being captured.  device_id is current during the call; the caller's
 * current device is put back before it returns.  Returns when the output is
 * on the host.  Results equal vnlbgpu_aggregate's bit for bit. */
int vnlbgpu_aggregate_frame_noalloc(const float* stacks, const float* source, int width, int height, int frames,
                                    int channels, int search_bwd, int search_fwd, int patch_time, int device_id, int n,
                                    float* out);

/* One clip over several GPUs, one process per GPU, no exchange between them
 * (the reference has one device per filter, cuda_plugin.cpp:476; this is the
 * partition of its per-frame dependencies).  Output frames [0, frames) are
 * split into `world` contiguous blocks; rank `rank` renders Final frames
 * [out[0], out[1]] (-1, -1 when its block is empty).  Final frame n reads the
 * Basic frames and source frames of its required source range, and Basic
 * frame m reads the source frames of its own: so the rank also renders Basic
 * frames [basic[0], basic[1]], the union of its Final frames' ranges, and
 * needs source frames [source[0], source[1]], the union of those Basic
 * frames' ranges.  Each rank runs its own sessions over the whole clip's
 * frame count through the per-frame calls, so the temporal windows are the
 * whole clip's and the blocks joined equal the one-GPU output bit for bit.
 * Host only: needs no device. */
int vnlbgpu_shard_plan(int frames, int world, int rank, int basic_search_bwd, int basic_search_fwd,
                       int basic_patch_time, int final_search_bwd, int final_search_fwd, int final_patch_time,
                       int out[2], int basic[2], int source[2]);

int vnlbgpu_get_stats(vnlbgpu_session* session, vnlbgpu_stats* stats);

/* Tile-shape autotuner (no reference counterpart).  On anchor frame `anchor`
 * (its sources given), times the session's own kernels for each shape that
 * fits and keeps the fastest for the session's later calls: the plain
 * matcher's strip width (8, 4 or 2 anchors per CTA), the tensor-core
 * matcher's planes per shared-memory stage (the chosen_tc form), and the
 * warp-per-group against the row-tiled apply kernel where both fit.  The
 * plain form's choices compute the same bits; the tensor-core plane grouping
 * can move the approximate distances' last bits.  match_warps and
 * apply_rows (either may be NULL) receive the plain matcher's and the
 * apply's choices; log (log_size bytes, may be NULL) one "shape: ms" line per
 * timing.  The learned form is not autotuned. */
int vnlbgpu_autotune(vnlbgpu_session* session, int anchor, int* match_warps, int* apply_rows, char* log,
                     size_t log_size);

/* Learned block-match proposals (no reference counterpart): a multilayer
 * perceptron trained and run by this library's own CUDA kernels.
 *
 * The network maps `inputs` features through `layers` hidden ReLU layers of
 * `hidden` units to `outputs` logits.  Weights are FP32 for the optimiser and
 * BF16 for the products, which accumulate in FP32.  Training minimises the
 * softmax cross-entropy against up to tk target classes per row (class ids,
 * -1 = none, each weighted equally) with Adam.  x, targets, logits and
 * shortlist buffers are device pointers; weights and gradients are host
 * arrays laid out layer by layer as [W_l (fan_out x fan_in)][b_l]. */
typedef struct vnlbgpu_mlp vnlbgpu_mlp;
int vnlbgpu_mlp_create(int inputs, int hidden, int layers, int outputs, int max_batch, unsigned seed, int device_id,
                       vnlbgpu_mlp** out);
void vnlbgpu_mlp_destroy(vnlbgpu_mlp* mlp);
long long vnlbgpu_mlp_parameters(const vnlbgpu_mlp* mlp);
int vnlbgpu_mlp_get_weights(vnlbgpu_mlp* mlp, float* host);
int vnlbgpu_mlp_set_weights(vnlbgpu_mlp* mlp, const float* host);
/* gradients of the mean loss over the batch (no update) */
int vnlbgpu_mlp_gradients(vnlbgpu_mlp* mlp, const float* x, const int* targets, int batch, int tk, float* host_grads,
                          float* mean_loss);
int vnlbgpu_mlp_train_step(vnlbgpu_mlp* mlp, const float* x, const int* targets, int batch, int tk, float lr,
                           float* mean_loss);
int vnlbgpu_mlp_logits(vnlbgpu_mlp* mlp, const float* x, int batch, float* logits);
/* the k best-scored classes of each row, [batch][k] */
int vnlbgpu_mlp_shortlist(vnlbgpu_mlp* mlp, const float* x, int batch, int k, int* out);

/* Attaches a network to a session of form VNLBGPU_FORM_LEARNED (not owned;
 * it must outlive the session's renders).  Its inputs must be
 * (search_bwd + search_fwd + 1) * (1 for Basic, planes for Final) * 9 and its
 * outputs (search_bwd + search_fwd + 1) * search_window^2; shortlist offsets
 * (1..128) per anchor, the recall threshold of the per-tile check (0: the
 * learned rows always stand; above 1: every tile is searched in full), and
 * the tile edge in pixels (64 in this build). */
int vnlbgpu_set_learned(vnlbgpu_session* session, vnlbgpu_mlp* mlp, int shortlist, float recall_threshold,
                        int tile);

/* Training pairs of anchor frame `anchor`: for each grid anchor (raster
 * order) its features ([count][inputs], the learned form's) and the classes
 * of its k nearest rows under the full exact search ([count][k], -1 past the
 * retained rows), into host arrays of `capacity` anchors.  Any form. */
int vnlbgpu_learned_pairs(vnlbgpu_session* session, int anchor, float* features, int* targets, int capacity, int k,
                          int* count, int* inputs);

/* The CUDA stream the session enqueues on (a cudaStream_t), for callers that
 * time or order device work around it. */
void* vnlbgpu_stream(vnlbgpu_session* session);

/* Makes the session enqueue on a caller-owned stream (NULL: its own stream),
 * e.g. one stream shared by a Basic and a Final session so that Final is
 * ordered after the Basic frames it reads. */
int vnlbgpu_set_stream(vnlbgpu_session* session, void* stream);

/* Flow-guided search: the vnlb plugin's optional mvfw / mvbw clips (MVTools
 * delta-1 vectors; the reference's vnlbcu has no such search).
 *
 *   parse_mvtools_analysis (src/flow/flow.hpp:193-250)  vnlbgpu_parse_mvtools_analysis
 *   parse_mvtools_vectors  (flow.hpp:252-318)           vnlbgpu_parse_mvtools_vectors
 *   read_mvtools_analysis_from_node + validate_mvtools_clip
 *     (src/vs/plugin.cpp:429-474, 881-899)              vnlbgpu_set_mvtools_analysis
 *   cache_mvtools_grid (plugin.cpp:507-525)             vnlbgpu_set_mvtools_frame
 *   MVToolsFlowProvider::center_for (flow.hpp:341-389)  the search centres of
 *                                                       every render that follows
 *
 * direction 0 is mvfw (MVTools isb=False), walked toward earlier candidate
 * frames; 1 is mvbw (isb=True), walked toward later ones.  The two parsers
 * need no device and no session: parse_analysis reads the 21 32-bit fields of
 * an MVTools_MVAnalysisData frame property; parse_vectors the finest level of
 * an MVTools_vectors property, *valid its valid flag, xy up to capacity
 * (x, y) pairs, *count their number.  set_mvtools_analysis takes the
 * direction's analysis data (the property of the vector clip's frame 0) and
 * checks it against the clip; set_mvtools_frame then takes frame n's
 * MVTools_vectors property and whether the source clip's frame n marks a scene
 * change (_SceneChangePrev or Scenechange for mvfw, _SceneChangeNext for mvbw),
 * which makes the frame's vectors unusable.  Frames never given are unusable.
 * With any flow set, the session runs the plain matcher (the chosen forms
 * need windows centred on the anchor). */
typedef struct vnlbgpu_mvtools_analysis {
    int block_size_x, block_size_y, pel, level_count, delta_frame, backwards, width, height;
    int overlap_x, overlap_y, block_count_x, block_count_y, bits_per_sample;
    int chroma_ratio_x, chroma_ratio_y, padding_x, padding_y;
} vnlbgpu_mvtools_analysis;

int vnlbgpu_parse_mvtools_analysis(const void* data, size_t size, vnlbgpu_mvtools_analysis* out);
int vnlbgpu_parse_mvtools_vectors(const void* data, size_t size, const vnlbgpu_mvtools_analysis* analysis,
                                  int* valid, int* xy, size_t capacity, size_t* count);
int vnlbgpu_set_mvtools_analysis(vnlbgpu_session* session, int direction, const void* data, size_t size);
int vnlbgpu_set_mvtools_frame(vnlbgpu_session* session, int direction, int frame, const void* vectors,
                              size_t size, int scene_change);

#ifdef __cplusplus
}
#endif

#endif
