/*
 * vnlbgpu diagnostics: read-back of the intermediate results of one anchor
 * frame, for parity tests against the CPU oracle.  Not part of the plugin
 * boundary (the reference exposes no such call; its own CUDA unit tests read
 * the same intermediates through C++ classes, tests/cpp/test_cuda_*.cpp).
 */
#ifndef VNLBGPU_DIAG_H
#define VNLBGPU_DIAG_H

#include "vnlbgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vnlbgpu_diag_row {
    float distance;
    int x;
    int y;
    int frame;
    float weight; /* aggregation weight (active groups only) */
} vnlbgpu_diag_row;

/* Runs anchor frame `anchor` and returns:
 *   grid:        every grid anchor (x, y) in raster order, grid_counts[i] its
 *                retained row count, grid_rows[i * max_rows + j] its rows;
 *   active:      indices (into the grid) of the processed groups, in order,
 *                active_rows their rows with weights, concatenated.
 * Capacities are in elements; *groups / *active_groups / *rows / *max_rows
 * receive the true sizes (copies are truncated to the capacities). */
int vnlbgpu_diag_anchor(vnlbgpu_session* session, int anchor, int* grid_xy, int* grid_counts,
                        vnlbgpu_diag_row* grid_rows, int grid_capacity, int grid_row_capacity, int* active,
                        vnlbgpu_diag_row* active_rows, int active_capacity, int active_row_capacity, int* groups,
                        int* active_groups, int* rows, int* max_rows);

/* Per-kernel device time.  Returns the milliseconds and launch counts
 * accumulated since the previous call for the kernel classes
 *   0 match, 1 paste mask, 2 group filter, 3 stack tiles, 4 normalise
 * (arrays of 5), resets them, and turns event timing on (enable != 0) or off.
 * Timing brackets each launch with CUDA events on the session's stream. */
int vnlbgpu_diag_kernel_timing(vnlbgpu_session* session, int enable, double* ms, long long* launches);

/* Runs anchor frame `anchor` and copies the filtered rows of its processed
 * groups, [*rows][*row_dim] floats in the order of vnlbgpu_diag_anchor's
 * active rows, up to `capacity` rows (*rows receives the true count). */
int vnlbgpu_diag_filtered(vnlbgpu_session* session, int anchor, float* out, int capacity, int* rows, int* row_dim);

/* Test switch of the tensor-core matcher's bounded waits: with on != 0 its
 * MMA warp issues no MMA, so every wait for MMA completion runs out after
 * its iteration limit, the kernel returns with nothing in flight, and the
 * render raises "timed out".  0 restores normal matching. */
int vnlbgpu_diag_stall_tensor_waits(vnlbgpu_session* session, int on);

/* Limits the pipeline lanes the session uses to min(lanes, the lanes it
 * allocated) after waiting for its queued work; lanes <= 0 restores them all.
 * With one lane the anchor frames' kernels run one after another, so the
 * per-kernel times above are those of each kernel alone. */
int vnlbgpu_diag_set_lanes(vnlbgpu_session* session, int lanes);

#ifdef __cplusplus
}
#endif

#endif
