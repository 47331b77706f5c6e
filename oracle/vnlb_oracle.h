/*
 * C interface shared by the two CPU oracles of the VNLB hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load these libraries, and only as the checker.
 *
 *   oracle/_ref/libvnlb_ref.so   the reference's own CPU sources
 *                                (src/core, src/linalg, src/aggregate) compiled
 *                                out of tree by oracle/Makefile, driven by
 *                                oracle/ref_driver.cpp;
 *   oracle/libvnlb_oracle.so     oracle/vnlb_oracle.c, a plain-C restatement of
 *                                the same algorithm, validated bit-for-bit
 *                                against the former.
 *
 * Both export the same entry points with the prefixes vnlbref_ and
 * vnlboracle_ respectively.
 *
 * Video layout: frame-major planar float32, index
 *   ((frame * channels + channel) * height + y) * width + x.
 * Contribution stack layout (one anchor frame), the vnlb.Basic/Final frame
 * layout of src/vs/plugin.cpp:622-642: per channel a plane of height
 * slots*2*height; row slot*2*H + y holds numerators, row slot*2*H + H + y the
 * weights (duplicated in every channel), index
 *   ((channel * slots * 2 + slot * 2 + is_weight) * height + y) * width + x.
 */
#ifndef VNLB_ORACLE_H
#define VNLB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors vnlb::core::StageParameters (src/core/core.hpp:17-41), in the units
 * the core uses (sigma already divided by 255, tau by 255^2). */
typedef struct vnlb_stage_params {
    float sigma;
    int patch_size;
    int patch_time;
    int search_window;
    int search_bwd;
    int search_fwd;
    int similar;
    int rank;
    float similar_cap_factor;
    float model_cap_factor;
    float beta;
    float tau;
    float variance_threshold;
    float sigma_basic;
    float gamma;
    float weight_alpha;
    float weight_beta;
    float weight_gamma;
    float weight_epsilon;
    float membership_noise_floor;
    int proc_step;
    int flat_areas;
    int couple_channels;
} vnlb_stage_params;

enum { VNLB_STAGE_BASIC = 0, VNLB_STAGE_FINAL = 1 };

/* Per-anchor record of one processed group (restatement only). */
typedef struct vnlb_group_record {
    int anchor_x;
    int anchor_y;
    int similar;      /* retained rows S */
    int first_match;  /* index into the match array */
} vnlb_group_record;

typedef struct vnlb_match_record {
    float distance;
    int x;
    int y;
    int frame;
    float weight;     /* final aggregation weight of the row */
} vnlb_match_record;

/* Motion vectors of the flow-guided search: the vnlb plugin's optional
 * mvfw / mvbw clips (MVTools delta-1 vectors, finest level), as
 * MVToolsVectorGrid holds them (src/flow/flow.hpp:37-120).  One block
 * geometry per direction; per frame a usable flag (the vectors parsed valid
 * and the source frame is not a scene change, src/vs/plugin.cpp:476-485,
 * 507-525) and block_count_y x block_count_x vectors (x, y) in sub-pel
 * units.  MVToolsFlowProvider (flow.hpp:321-429) walks the mvfw grids toward
 * earlier candidate frames and the mvbw grids toward later ones. */
typedef struct vnlb_flow_grids {
    int present;  /* the clip was given */
    int block_size_x, block_size_y, pel, overlap_x, overlap_y, block_count_x, block_count_y;
    const unsigned char* usable; /* [frames] */
    const int* vectors;          /* [frames][block_count_y][block_count_x][2] */
} vnlb_flow_grids;

typedef struct vnlb_flow {
    vnlb_flow_grids fw; /* mvfw */
    vnlb_flow_grids bw; /* mvbw */
} vnlb_flow;

#ifdef __cplusplus
}
#endif

#endif
