// Device side of the learned block-match proposals (learned.cu): the MLP's
// weights as the kernels read them, and its launchers.
#pragma once

#include <cstddef>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace vnlbgpu {

constexpr int kMlpMaxLayers = 4;  // hidden layers at most

struct MlpDevice {
    int inputs, hidden, layers, outputs;
    __nv_bfloat16* w16[kMlpMaxLayers + 1];  // layer l: [fan_out][fan_in], BF16 copy of the FP32 weights
    float* b[kMlpMaxLayers + 1];            // layer l: [fan_out]
};

// acts[l]: [batch][hidden] outputs of hidden layer l (after the ReLU);
// logits: [batch][outputs].
cudaError_t mlp_forward(const MlpDevice& net, const float* x, int batch, float* const* acts, float* logits,
                        cudaStream_t stream);

// Turns `dlogits` (the forward's logits) into their gradient and
// back-propagates: gw[l] [fan_out][fan_in], gb[l] [fan_out] receive the
// gradients of the mean softmax cross-entropy over the batch against
// `targets` [batch][tk] (class ids, -1 = none); loss[row] each row's loss.
// dacts[l] is scratch shaped like acts[l].
cudaError_t mlp_backward(const MlpDevice& net, const float* x, int batch, float* const* acts, float* dlogits,
                         const int* targets, int tk, float* loss, float* const* dacts, float* const* gw,
                         float* const* gb, cudaStream_t stream);

// One Adam step (step counts from 1) on the FP32 weights wmaster / net.b,
// refreshing the BF16 copies.
cudaError_t mlp_adam(const MlpDevice& net, float* const* gw, float* const* gb, float* const* mw, float* const* vw,
                     float* const* mb, float* const* vb, float* const* wmaster, float lr, int step,
                     cudaStream_t stream);

cudaError_t weights_to_bf16(const float* w, __nv_bfloat16* w16, size_t n, cudaStream_t stream);

// Inference for the shortlist: the hidden layers as mlp_forward, the output
// layer on the tensor cores (activations rounded to BF16, BF16 weights, FP32
// accumulation in tensor memory) when the last hidden width is a multiple of
// 16 up to 128, else as mlp_forward.  A tensor-core wait that runs out sets
// *status (when given) to kStatusLogitsTimeout.
constexpr int kStatusLogitsTimeout = 5;
cudaError_t mlp_infer(const MlpDevice& net, const float* x, int batch, float* const* acts, float* logits, int* status,
                      cudaStream_t stream);

// out[row][k]: the ids of the k largest logits of each row (ties: lower id).
cudaError_t logits_topk(const float* logits, int rows, int classes, int k, int* out, cudaStream_t stream);

}  // namespace vnlbgpu

struct vnlbgpu_mlp;  // the C ABI's network object (mlp.cpp)

namespace vnlbgpu {
// The network's weights as the kernels read them.
MlpDevice mlp_device(const vnlbgpu_mlp* mlp);
}  // namespace vnlbgpu

#include "vnlb_common.cuh"

namespace vnlbgpu {

constexpr int kFeatureCell = 16;   // box size of the coarse frames the features read
constexpr int kShortlistMax = 128; // most shortlisted offsets per anchor

// One anchor frame of the learned matcher.  Offsets are the classes of the
// MLP: class = k * W * W + wy * W + wx for scheduled frame k (the matcher's
// schedule: anchor, future, past) and window cell (wx, wy), W the search
// window; the network always has `slots_max` scheduled frames.
struct LearnedLaunch {
    const float* video;  // search source, frame slots (MatchLaunch)
    int ring, width, height, channels, search_channels, P, Pt, search_window;
    int schedule[32];
    int schedule_len, slots_max, anchor_frame;
    const int2* anchors;
    int anchor_count;
    const int* anchor_map;
    float* cells;        // [slots_max][search_channels][cells_h][cells_w]
    int cells_w, cells_h;
    float* features;     // [anchors][inputs]
    int inputs;
    float feature_scale;
    const int* shortlist;  // [anchors][shortlist_len] classes (-1 = none)
    int shortlist_len;
    // selection (the plain matcher's rule on the shortlisted candidates)
    int K, soft_cap, max_rows;
    float tau;
    MatchRow* rows;
    int* row_counts;
    int* victims;
    int* victim_counts;
    int victim_stride;
    // per-tile recall check
    int tiles;
    const int* check_anchor;     // [tiles] grid anchor checked in each tile
    const MatchRow* check_rows;  // [tiles][max_rows] the full search's rows of those anchors
    const int* check_counts;
    float recall_threshold;
    int* tile_fail;              // [tiles] 1 = the full search runs for the tile
    unsigned long long* totals;  // [2]: tiles checked, tiles that fell back
};

cudaError_t launch_learned_features(const LearnedLaunch& L, cudaStream_t stream);
cudaError_t launch_learned_match(const LearnedLaunch& L, cudaStream_t stream);
cudaError_t launch_learned_recall(const LearnedLaunch& L, cudaStream_t stream);

}  // namespace vnlbgpu
