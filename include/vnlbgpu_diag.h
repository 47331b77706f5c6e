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

#ifdef __cplusplus
}
#endif

#endif
