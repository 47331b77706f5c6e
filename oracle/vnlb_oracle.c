/*
 * Plain-C restatement of the VNLB CPU hot path (block matching -> Bayesian
 * PCA group filter -> weighted contribution stacks -> aggregation).
 *
 * TEST INFRASTRUCTURE ONLY (see vnlb_oracle.h): the checker for the GPU path,
 * never the thing measured or shipped.  It follows the reference sources
 * operation by operation so that, compiled with -ffp-contract=off, it is
 * bit-identical to oracle/_ref/libvnlb_ref.so (the reference compiled with the
 * pinned Highway header hwy_pin/hwy/highway.h and the pinned libm_pin.c).
 * Each function cites the reference file:line it restates.
 */
#include "vnlb_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static _Thread_local char g_error[512];

static int fail(const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, args);
    va_end(args);
    return -1;
}

const char* vnlboracle_last_error(void) { return g_error; }

/* ------------------------------------------------------------------------ */
/* Elementary functions pinned like oracle/libm_pin.c.                       */
static float pin_expf(float x) { return (float)exp((double)x); }
static float pin_logf(float x) { return (float)log((double)x); }
static float pin_log1pf(float x) { return (float)log1p((double)x); }
static float pin_powf(float x, float y) { return (float)pow((double)x, (double)y); }

static float fmax_std(float a, float b) { return (a < b) ? b : a; } /* std::max */
static float fmin_std(float a, float b) { return (b < a) ? b : a; } /* std::min */
static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* ------------------------------------------------------------------------ */
/* Lane-structured kernels: the pinned 8-lane Highway semantics of
 * src/core/distance_highway.hpp:11-58 and src/linalg/kernels_highway.hpp.    */
#define LANES 8

static float reduce8(const float v[LANES]) {
    const float a0 = v[0] + v[4], a1 = v[1] + v[5];
    const float a2 = v[2] + v[6], a3 = v[3] + v[7];
    const float b0 = a0 + a2, b1 = a1 + a3;
    return b0 + b1;
}

/* add_squared_row_distance_highway (src/core/distance_highway.hpp:11-58) */
static float row_ssd(float distance, const float* l, const float* r, int count) {
    float v[LANES];
    int i;
    if (count <= 0) return distance;
    if (count == LANES) {
        for (i = 0; i < LANES; ++i) { const float d = l[i] - r[i]; v[i] = d * d; }
        return distance + reduce8(v);
    }
    if (count == 2 * LANES) {
        for (i = 0; i < LANES; ++i) { const float d = l[i] - r[i]; v[i] = d * d; }
        for (i = 0; i < LANES; ++i) { const float d = l[i + LANES] - r[i + LANES]; v[i] = fmaf(d, d, v[i]); }
        return distance + reduce8(v);
    }
    for (i = 0; i < LANES; ++i) v[i] = 0.0f;
    int index = 0;
    for (; index + LANES <= count; index += LANES) {
        for (i = 0; i < LANES; ++i) { const float d = l[index + i] - r[index + i]; v[i] = fmaf(d, d, v[i]); }
    }
    distance += reduce8(v);
    for (; index < count; ++index) { const float d = l[index] - r[index]; distance += d * d; }
    return distance;
}

/* dot_contiguous_highway (src/linalg/kernels_highway.hpp:10-41) */
static float dot8(const float* l, const float* r, int count) {
    float v[LANES];
    int i;
    if (count == LANES) {
        for (i = 0; i < LANES; ++i) v[i] = l[i] * r[i];
        return reduce8(v);
    }
    if (count == 2 * LANES) {
        for (i = 0; i < LANES; ++i) v[i] = l[i] * r[i];
        for (i = 0; i < LANES; ++i) v[i] = fmaf(l[i + LANES], r[i + LANES], v[i]);
        return reduce8(v);
    }
    for (i = 0; i < LANES; ++i) v[i] = 0.0f;
    int index = 0;
    for (; index + LANES <= count; index += LANES)
        for (i = 0; i < LANES; ++i) v[i] = fmaf(l[index + i], r[index + i], v[i]);
    float total = reduce8(v);
    for (; index < count; ++index) total += l[index] * r[index];
    return total;
}

/* add_scaled_contiguous_highway (kernels_highway.hpp:154-181): fused on full
 * 8-lane chunks (and on the count==8/16 shortcuts), unfused on the tail. */
static void add_scaled(float* out, const float* in, float scale, int count) {
    int index = 0;
    if (count == LANES || count == 2 * LANES) {
        for (; index < count; ++index) out[index] = fmaf(scale, in[index], out[index]);
        return;
    }
    for (; index + LANES <= count; index += LANES)
        for (int i = 0; i < LANES; ++i) out[index + i] = fmaf(scale, in[index + i], out[index + i]);
    for (; index < count; ++index) out[index] += scale * in[index];
}

/* ------------------------------------------------------------------------ */
/* Parameters (src/core/core.cpp:40-178, 1948-2024).                         */
static int proc_step_of(const vnlb_stage_params* p) {
    if (p->proc_step > 0) return p->proc_step;
    if (p->patch_size <= 1) return 1;
    return p->patch_size;
}

/* soft_similar_cap / model_similar_cap (core.cpp:139-172) */
static int cap_of(int similar, float factor) {
    if (factor == 0.0f) return 0x7fffffff;
    const float max_factor = (float)0x7fffffff / (float)similar;
    if (factor >= max_factor) return 0x7fffffff;
    const float cap = ceilf((float)similar * factor);
    return imax(similar, (int)cap);
}

static int validate(const vnlb_stage_params* p, int width, int height, int frames, int channels) {
#define REQUIRE(cond, msg) do { if (!(cond)) return fail("VNLB: %s", msg); } while (0)
    REQUIRE(isfinite(p->sigma) && p->sigma > 0.0f, "sigma must be finite and positive");
    REQUIRE(p->patch_size > 0, "block_size must be positive");
    REQUIRE(p->patch_time > 0, "patch_time must be positive");
    REQUIRE(p->search_window > 0 && p->search_window % 2 == 1, "bm_range must describe a positive odd search window");
    REQUIRE(p->search_bwd >= 0 && p->search_fwd >= 0, "search_bwd and search_fwd must be non-negative");
    REQUIRE(p->similar > 0, "group_size must be positive");
    REQUIRE(p->rank >= 0, "rank must be non-negative");
    REQUIRE(isfinite(p->similar_cap_factor) && (p->similar_cap_factor == 0.0f || p->similar_cap_factor >= 1.0f),
            "cap_factor must be zero or at least 1.0");
    REQUIRE(isfinite(p->model_cap_factor) && (p->model_cap_factor == 0.0f || p->model_cap_factor >= 1.0f),
            "model_cap_factor must be zero or at least 1.0");
    REQUIRE(isfinite(p->beta) && p->beta > 0.0f, "beta must be finite and positive");
    REQUIRE(isfinite(p->tau) && p->tau >= 0.0f, "tau must be finite and non-negative");
    REQUIRE(isfinite(p->variance_threshold), "variance_threshold must be finite");
    REQUIRE(isfinite(p->sigma_basic) && p->sigma_basic >= 0.0f, "sigma_basic must be finite and non-negative");
    REQUIRE(isfinite(p->gamma) && p->gamma > 0.0f, "gamma must be finite and positive");
    REQUIRE(isfinite(p->weight_alpha) && p->weight_alpha >= 0.0f, "weight_alpha must be finite and non-negative");
    REQUIRE(isfinite(p->weight_beta) && p->weight_beta >= 0.0f, "weight_beta must be finite and non-negative");
    REQUIRE(isfinite(p->weight_gamma) && p->weight_gamma >= 0.0f, "weight_gamma must be finite and non-negative");
    REQUIRE(isfinite(p->weight_epsilon) && p->weight_epsilon > 0.0f, "weight_epsilon must be finite and positive");
    REQUIRE(isfinite(p->membership_noise_floor) && p->membership_noise_floor > 0.0f,
            "membership_noise_floor must be finite and positive");
    REQUIRE(p->proc_step >= 0, "block_step must be non-negative; use 0 for auto");
    REQUIRE(p->search_bwd + p->search_fwd < 4096, "temporal search span is too large");
    REQUIRE(width > 0 && height > 0 && frames > 0 && channels > 0, "video geometry must be non-empty");
    REQUIRE(p->patch_size <= width && p->patch_size <= height, "block_size must fit inside the frame");
    REQUIRE(p->patch_time <= frames, "patch_time must fit inside the clip");
    {
        const int estimator_dim = p->patch_size * p->patch_size * p->patch_time * (p->couple_channels ? channels : 1);
        REQUIRE(p->rank <= estimator_dim, "rank must not exceed the effective patch dimension");
        REQUIRE(p->similar >= imin(estimator_dim, p->rank), "group_size must cover the effective VNLB rank");
    }
    return 0;
#undef REQUIRE
}

/* ------------------------------------------------------------------------ */
/* Video and stack access.                                                    */
typedef struct video {
    const float* data;
    int width, height, frames, channels;
} video;

static const float* plane_ptr(const video* v, int frame, int channel) {
    return v->data + ((size_t)frame * v->channels + channel) * (size_t)v->width * v->height;
}

typedef struct stack_view {
    float* data;
    int width, height, channels, slots, search_bwd;
} stack_view;

static float* stack_row(const stack_view* s, int channel, int slot, int is_weight, int y) {
    const size_t row = ((size_t)channel * s->slots * 2 + (size_t)slot * 2 + is_weight) * s->height + y;
    return s->data + row * s->width;
}

/* ------------------------------------------------------------------------ */
/* Search windows (core.cpp:873-932) and the staggered anchor grid
 * (core.cpp:934-967).                                                        */
static void temporal_range(const vnlb_stage_params* p, int source_frames, int anchor, int* low, int* high) {
    const int max_origin = source_frames - p->patch_time;
    const int start = anchor - p->search_bwd;
    const int end = anchor + p->search_fwd;
    const int shift = imin(0, start) + imax(0, end - max_origin);
    *low = imax(0, start - shift);
    *high = imin(max_origin, end - shift);
}

static void spatial_range(const vnlb_stage_params* p, int center, int axis, int* low, int* high) {
    const int max_origin = axis - p->patch_size;
    const int half = (p->search_window - 1) / 2;
    const int start = center - half;
    const int end = center + half;
    const int shift = imin(0, start) + imax(0, end - max_origin);
    *low = imax(0, start - shift);
    *high = imin(max_origin, end - shift);
}

static int grid_selected(const vnlb_stage_params* p, int width, int height, int source_frames,
                         int anchor, int x, int y) {
    const int step = proc_step_of(p);
    const int max_x = width - p->patch_size;
    const int max_y = height - p->patch_size;
    const int max_frame = source_frames - p->patch_time;
    const int phase_y = anchor == max_frame ? 0 : anchor;
    if (y != 0 && y != max_y && y % step != phase_y % step) return 0;
    const int phase_x = y == max_y ? 0 : phase_y + (y / step);
    return x == 0 || x == max_x || x % step == phase_x % step;
}

/* ------------------------------------------------------------------------ */
/* The selection heap of std::partial_sort as the oracle toolchain's C++
 * library implements it: Floyd heap construction, replacement of the heap top
 * by each later element that compares less, then heap sort of the head.  It
 * only decides the order of rows beyond the first K, which reaches the output
 * through the order of floating-point accumulation.                          */
typedef struct match {
    float distance;
    int x, y, frame;
} match;

static void heap_adjust(match* a, int hole, int len, match value) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (a[child].distance < a[child - 1].distance) child--;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    int parent = (hole - 1) / 2;
    while (hole > top && a[parent].distance < value.distance) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = value;
}

static void heap_make(match* a, int len) {
    if (len < 2) return;
    for (int parent = (len - 2) / 2;; --parent) {
        heap_adjust(a, parent, len, a[parent]);
        if (parent == 0) return;
    }
}

static void heap_pop_into(match* a, int len, int result) {
    const match value = a[result];
    a[result] = a[0];
    heap_adjust(a, 0, len, value);
}

static void partial_sort_matches(match* a, int middle, int last) {
    heap_make(a, middle);
    for (int i = middle; i < last; ++i)
        if (a[i].distance < a[0].distance) heap_pop_into(a, middle, i);
    for (int len = middle; len > 1; --len) heap_pop_into(a, len - 1, len - 1);
}

/* ------------------------------------------------------------------------ */
/* Workspace.                                                                 */
typedef struct workspace {
    vnlb_stage_params p;
    const vnlb_flow* flow;    /* flow-guided search centres, or NULL */
    int stage;
    int width, height, source_frames, channels;
    int patch_area, patch_dim, estimator_dim, max_similar;
    float* reference_patch;
    match* matches;
    int match_count, match_capacity;
    float* top;               /* K smallest distances so far */
    int top_count;
    float* group_noisy;       /* group layout [c][position][patch] */
    float* group_basic;
    float* samples_noisy;     /* sample layout [patch][dim] */
    float* samples_basic;
    float* centered_noisy;
    float* centered_basic;
    float* filtered;
    float* mean_noisy;
    float* mean_basic;
    float* eigenvalues;
    float* coefficients;
    float* eigenvectors;      /* rank x dim */
    float* dual;              /* rank x B */
    float* sym;               /* eigen input, n x n */
    float* jac_m;             /* Jacobi work matrix */
    float* jac_v;
    int* order;
    float* log_w;
    float* w;
    float* scores;
    int model_count;
    float* window;
    unsigned char* mask;
    int sample_major;
} workspace;

static void ws_free(workspace* w) {
    free(w->reference_patch); free(w->matches); free(w->top);
    free(w->group_noisy); free(w->group_basic); free(w->samples_noisy); free(w->samples_basic);
    free(w->centered_noisy); free(w->centered_basic); free(w->filtered);
    free(w->mean_noisy); free(w->mean_basic); free(w->eigenvalues); free(w->coefficients);
    free(w->eigenvectors); free(w->dual); free(w->sym); free(w->jac_m); free(w->jac_v); free(w->order);
    free(w->log_w); free(w->w); free(w->scores); free(w->window); free(w->mask);
    memset(w, 0, sizeof(*w));
}

/* prepare_aggregation_window (core.cpp:296-324) */
static void prepare_window(workspace* w) {
    const int P = w->p.patch_size;
    const float gamma = w->p.weight_gamma;
    for (int i = 0; i < P * P; ++i) w->window[i] = 1.0f;
    if (gamma == 0.0f || P <= 1) return;
    const float center = 0.5f * (float)(P - 1);
    const float radius = fmax_std(center, 0.5f);
    float max_weight = 0.0f;
    for (int y = 0; y < P; ++y) {
        const float dy = ((float)y - center) / radius;
        for (int x = 0; x < P; ++x) {
            const float dx = ((float)x - center) / radius;
            const float raw = pin_expf(-0.5f * ((dx * dx) + (dy * dy)));
            w->window[y * P + x] = raw;
            max_weight = fmax_std(max_weight, raw);
        }
    }
    const float inv_max = max_weight > 0.0f ? 1.0f / max_weight : 1.0f;
    for (int i = 0; i < P * P; ++i) w->window[i] = pin_powf(w->window[i] * inv_max, gamma);
}

static int ws_prepare(workspace* w, int stage, const vnlb_stage_params* p, int width, int height,
                      int source_frames, int channels) {
    ws_free(w);
    w->p = *p;
    w->stage = stage;
    w->width = width; w->height = height; w->source_frames = source_frames; w->channels = channels;
    w->patch_area = p->patch_size * p->patch_size;
    w->patch_dim = w->patch_area * p->patch_time;
    w->estimator_dim = w->patch_dim * (p->couple_channels ? channels : 1);
    {
        const int raw = p->search_window * p->search_window * (p->search_bwd + p->search_fwd + 1);
        w->max_similar = imin(cap_of(p->similar, p->similar_cap_factor), raw);
    }
    const size_t D = (size_t)channels * w->patch_dim;
    const size_t S = (size_t)w->max_similar;
    const size_t n = D; /* eigen inputs are at most D x D */
    w->match_capacity = w->max_similar + 1;
    w->reference_patch = calloc(D, sizeof(float));
    w->matches = calloc((size_t)w->match_capacity, sizeof(match));
    w->top = calloc((size_t)p->similar + 1, sizeof(float));
    w->group_noisy = calloc(D * S, sizeof(float));
    w->group_basic = calloc(D * S, sizeof(float));
    w->samples_noisy = calloc(D * S, sizeof(float));
    w->samples_basic = calloc(D * S, sizeof(float));
    w->centered_noisy = calloc(D * S, sizeof(float));
    w->centered_basic = calloc(D * S, sizeof(float));
    w->filtered = calloc(D * S, sizeof(float));
    w->mean_noisy = calloc(D, sizeof(float));
    w->mean_basic = calloc(D, sizeof(float));
    w->eigenvalues = calloc(D + 1, sizeof(float));
    w->coefficients = calloc(D + 1, sizeof(float));
    w->eigenvectors = calloc(D * D + 1, sizeof(float));
    w->dual = calloc(D * S + 1, sizeof(float));
    w->sym = calloc(n * n + S * S, sizeof(float));
    w->jac_m = calloc(n * n + S * S, sizeof(float));
    w->jac_v = calloc(n * n + S * S, sizeof(float));
    w->order = calloc(n + S, sizeof(int));
    w->log_w = calloc(S, sizeof(float));
    w->w = calloc(S, sizeof(float));
    w->scores = calloc(S, sizeof(float));
    w->window = calloc((size_t)w->patch_area, sizeof(float));
    w->mask = calloc((size_t)width * height, 1);
    if (!w->reference_patch || !w->matches || !w->top || !w->group_noisy || !w->group_basic ||
        !w->samples_noisy || !w->samples_basic || !w->centered_noisy || !w->centered_basic ||
        !w->filtered || !w->mean_noisy || !w->mean_basic || !w->eigenvalues || !w->coefficients ||
        !w->eigenvectors || !w->dual || !w->sym || !w->jac_m || !w->jac_v || !w->order ||
        !w->log_w || !w->w || !w->scores || !w->window || !w->mask) {
        ws_free(w);
        return fail("VNLB: oracle workspace allocation failed");
    }
    prepare_window(w);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Matching: find_similar_patches + select_similar_patches
 * (core.cpp:1200-1362) with the distance scans of core.cpp:1033-1150.      */
static void record_distance(workspace* w, float d) {
    const int K = w->p.similar;
    if (w->top_count < K) { w->top[w->top_count++] = d; return; }
    int worst = 0;
    for (int i = 1; i < K; ++i) if (w->top[worst] < w->top[i]) worst = i;
    if (d < w->top[worst]) w->top[worst] = d;
}

static float top_front(const workspace* w) {
    float m = w->top[0];
    for (int i = 1; i < w->top_count; ++i) if (m < w->top[i]) m = w->top[i];
    return m;
}

typedef struct soft_buffer {
    int cap;
    int worst_index;
    float worst;
} soft_buffer;

static void refresh_worst(workspace* w, soft_buffer* b) {
    int worst = 0;
    for (int i = 1; i < w->match_count; ++i)
        if (w->matches[worst].distance < w->matches[i].distance) worst = i;
    b->worst_index = worst;
    b->worst = w->matches[worst].distance;
}

static void record_match(workspace* w, soft_buffer* b, match m) {
    if (w->match_count < b->cap) {
        w->matches[w->match_count++] = m;
        if (w->match_count == b->cap) refresh_worst(w, b);
        return;
    }
    if (m.distance < b->worst) {
        w->matches[b->worst_index] = m;
        refresh_worst(w, b);
    }
}

static float distance_limit(const workspace* w, const soft_buffer* b) {
    float limit = w->top_count >= w->p.similar ? fmax_std(w->p.tau, top_front(w)) : INFINITY;
    if (w->match_count >= b->cap) limit = fmin_std(limit, b->worst);
    return limit;
}

static void load_reference_patch(workspace* w, const video* src, int channels, int ax, int ay, int af) {
    const int P = w->p.patch_size;
    for (int c = 0; c < channels; ++c)
        for (int t = 0; t < w->p.patch_time; ++t) {
            const float* plane = plane_ptr(src, af + t, c);
            for (int y = 0; y < P; ++y)
                memcpy(w->reference_patch + c * w->patch_dim + (t * P + y) * P,
                       plane + (size_t)(ay + y) * src->width + ax, (size_t)P * sizeof(float));
        }
}

static float candidate_distance(const workspace* w, const video* src, int channels, int cx, int cy,
                                int cf, float limit) {
    const int P = w->p.patch_size;
    float distance = 0.0f;
    for (int c = 0; c < channels; ++c) {
        for (int t = 0; t < w->p.patch_time; ++t) {
            const float* ref_row = w->reference_patch + c * w->patch_dim + t * w->patch_area;
            const float* cand = plane_ptr(src, cf + t, c) + (size_t)cy * src->width + cx;
            for (int y = 0; y < P; ++y) {
                distance = row_ssd(distance, ref_row, cand, P);
                if (distance > limit) return distance;
                ref_row += P;
                cand += src->width;
            }
        }
    }
    return distance;
}

/* ------------------------------------------------------------------------ */
/* Flow-guided search centres: MVToolsVectorGrid::nearest_vector
 * (src/flow/flow.hpp:72-120), round_subpixel_to_pixel (flow.hpp:183-191) and
 * MVToolsFlowProvider::center_for (flow.hpp:341-389).                        */
static int nearest_block_index(int coordinate, int first_center, int step, int count) {
    if (count <= 1) return 0;
    const int shifted = coordinate - first_center;
    const int index = shifted >= 0 ? (shifted + step / 2) / step : -((-shifted + step / 2) / step);
    return index < 0 ? 0 : (index > count - 1 ? count - 1 : index);
}

static int round_subpixel(int value, int pel) {
    if (pel <= 1) return value;
    return value >= 0 ? (value + pel / 2) / pel : -((-value + pel / 2) / pel);
}

/* One frame of the walk: the centre moves by the grid's nearest vector to the
 * patch centre, rounded to whole pixels, then is clamped to the frame. */
static void flow_step(const vnlb_flow_grids* g, int frame, int patch_center, int width, int height, int* cx,
                      int* cy) {
    if (!g->present || !g->usable[frame] || g->pel <= 0 || g->block_size_x <= 0 || g->block_size_y <= 0 ||
        g->block_count_x <= 0 || g->block_count_y <= 0)
        return;
    const int step_x = imax(1, g->block_size_x - imax(0, g->overlap_x));
    const int step_y = imax(1, g->block_size_y - imax(0, g->overlap_y));
    const int bx = nearest_block_index(*cx + patch_center, g->block_size_x / 2, step_x, g->block_count_x);
    const int by = nearest_block_index(*cy + patch_center, g->block_size_y / 2, step_y, g->block_count_y);
    const int* v = g->vectors + (((size_t)frame * g->block_count_y + by) * g->block_count_x + bx) * 2;
    *cx += round_subpixel(v[0], g->pel);
    *cy += round_subpixel(v[1], g->pel);
    if (width > 0) *cx = imin(imax(*cx, 0), width - 1);
    if (height > 0) *cy = imin(imax(*cy, 0), height - 1);
}

/* The search centre of anchor (ax, ay) of frame af in candidate frame cf. */
static void flow_center(const workspace* w, int ax, int ay, int af, int cf, int* cx, int* cy) {
    *cx = ax;
    *cy = ay;
    if (!w->flow || cf == af) return;
    const int patch_center = imax(0, w->p.patch_size / 2);
    if (cf < af) {
        for (int f = af; f > cf; --f) flow_step(&w->flow->fw, f, patch_center, w->width, w->height, cx, cy);
    } else {
        for (int f = af; f < cf; ++f) flow_step(&w->flow->bw, f, patch_center, w->width, w->height, cx, cy);
    }
}

static int find_similar(workspace* w, const video* src, int channels, int ax, int ay, int af) {
    const vnlb_stage_params* p = &w->p;
    if (p->similar <= 1) {
        w->matches[0] = (match){0.0f, ax, ay, af};
        w->match_count = 1;
        return 1;
    }
    int low, high;
    temporal_range(p, w->source_frames, af, &low, &high);
    int schedule[4096];
    int scheduled = 0;
    schedule[scheduled++] = af;
    for (int f = af + 1; f <= high; ++f) schedule[scheduled++] = f;
    for (int f = af - 1; f >= low; --f) schedule[scheduled++] = f;

    soft_buffer b;
    b.cap = imin(cap_of(p->similar, p->similar_cap_factor), p->search_window * p->search_window * scheduled);
    b.worst_index = 0;
    b.worst = INFINITY;
    w->match_count = 0;
    w->top_count = 0;
    for (int s = 0; s < scheduled; ++s) {
        const int cf = schedule[s];
        int xl, xh, yl, yh, ccx, ccy;
        flow_center(w, ax, ay, af, cf, &ccx, &ccy);
        spatial_range(p, ccx, w->width, &xl, &xh);
        spatial_range(p, ccy, w->height, &yl, &yh);
        for (int cy = yl; cy <= yh; ++cy)
            for (int cx = xl; cx <= xh; ++cx) {
                const float limit = distance_limit(w, &b);
                const float d = candidate_distance(w, src, channels, cx, cy, cf, limit);
                if (d <= limit) {
                    record_match(w, &b, (match){d, cx, cy, cf});
                    record_distance(w, d);
                }
            }
    }
    /* select_similar_patches (core.cpp:1200-1243) */
    const int n = w->match_count;
    const int selected = imin(p->similar, n);
    partial_sort_matches(w->matches, selected, n);
    const float threshold = fmax_std(p->tau, w->matches[selected - 1].distance);
    int out = 0;
    for (int i = 0; i < n; ++i)
        if (w->matches[i].distance <= threshold) w->matches[out++] = w->matches[i];
    const int output_cap = imin(cap_of(p->similar, p->similar_cap_factor), n);
    if (out > output_cap) {
        partial_sort_matches(w->matches, output_cap, out);
        out = output_cap;
    }
    w->match_count = out;
    return out;
}

/* ------------------------------------------------------------------------ */
/* linalg (src/linalg/linalg.cpp).                                            */

/* compute_mean (linalg.cpp:275-293) over the first `rows` rows */
static void mean_rows(const float* x, int rows, int cols, float* mean) {
    for (int c = 0; c < cols; ++c) mean[c] = 0.0f;
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) mean[c] += x[(size_t)r * cols + c];
    const float inv = 1.0f / (float)rows;
    for (int c = 0; c < cols; ++c) mean[c] *= inv;
}

/* center_rows (linalg.cpp:295-307) */
static void center(const float* x, int rows, int cols, const float* mean, float* out) {
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) out[(size_t)r * cols + c] = x[(size_t)r * cols + c] - mean[c];
}

/* compute_gram_centered (linalg.cpp:309-337) */
static void gram(const float* x, int rows, int cols, float scale, float* g) {
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c <= r; ++c) {
            const float v = scale * dot8(x + (size_t)r * cols, x + (size_t)c * cols, cols);
            g[r * rows + c] = v;
            g[c * rows + r] = v;
        }
}

/* compute_covariance_centered (linalg.cpp:357-389) */
static void covariance(const float* x, int rows, int cols, float scale, float* cov) {
    memset(cov, 0, (size_t)cols * cols * sizeof(float));
    for (int s = 0; s < rows; ++s) {
        const float* row = x + (size_t)s * cols;
        for (int c0 = 0; c0 < cols; ++c0)
            add_scaled(cov + (size_t)c0 * cols + c0, row + c0, row[c0], cols - c0);
    }
    for (int r = 0; r < cols; ++r)
        for (int c = r; c < cols; ++c) {
            const float v = cov[r * cols + c] * scale;
            cov[r * cols + c] = v;
            cov[c * cols + r] = v;
        }
}

/* jacobi_rotate (linalg.cpp:152-196) */
static void jacobi_rotate(float* m, float* v, int n, int p, int q) {
    const float app = m[p * n + p], aqq = m[q * n + q], apq = m[p * n + q];
    if (apq == 0.0f) return;
    const float tau = (aqq - app) / (2.0f * apq);
    const float tau_abs = fabsf(tau);
    const float t_abs = 1.0f / (tau_abs + sqrtf(1.0f + (tau * tau)));
    const float t = tau < 0.0f ? -t_abs : t_abs;
    const float c = 1.0f / sqrtf(1.0f + (t * t));
    const float s = t * c;
    const float cc = c * c, ss = s * s, cs = c * s;
    for (int r = 0; r < n; ++r) {
        if (r == p || r == q) continue;
        const float arp = m[r * n + p], arq = m[r * n + q];
        const float nrp = (c * arp) - (s * arq);
        const float nrq = (s * arp) + (c * arq);
        m[r * n + p] = nrp; m[p * n + r] = nrp;
        m[r * n + q] = nrq; m[q * n + r] = nrq;
    }
    m[p * n + p] = ((cc * app) - ((2.0f * cs) * apq)) + (ss * aqq);
    m[q * n + q] = ((ss * app) + ((2.0f * cs) * apq)) + (cc * aqq);
    m[p * n + q] = 0.0f;
    m[q * n + p] = 0.0f;
    for (int r = 0; r < n; ++r) {
        const float vrp = v[r * n + p], vrq = v[r * n + q];
        v[r * n + p] = (c * vrp) - (s * vrq);
        v[r * n + q] = (s * vrp) + (c * vrq);
    }
}

/* topk_symmetric_eigen_jacobi (linalg.cpp:447-519) with
 * canonicalize_vector_row (linalg.cpp:198-227). */
static void topk_eigen(workspace* w, const float* sym, int n, int rank, float* values, float* vectors) {
    float* m = w->jac_m;
    float* v = w->jac_v;
    memcpy(m, sym, (size_t)n * n * sizeof(float));
    for (int i = 0; i < n * n; ++i) v[i] = 0.0f;
    for (int i = 0; i < n; ++i) v[i * n + i] = 1.0f;
    float max_abs = 0.0f;
    for (int i = 0; i < n * n; ++i) max_abs = fmax_std(max_abs, fabsf(m[i]));
    const float rel_tol = 64.0f * FLT_EPSILON;
    const float threshold = fmax_std(0.0f, rel_tol * fmax_std(1.0f, max_abs));
    if (n > 1) {
        for (int sweep = 0; sweep < 64; ++sweep) {
            float off = 0.0f;
            for (int r = 0; r < n; ++r)
                for (int c = r + 1; c < n; ++c) off = fmax_std(off, fabsf(m[r * n + c]));
            if (off <= threshold) break;
            for (int p = 0; p + 1 < n; ++p)
                for (int q = p + 1; q < n; ++q)
                    if (fabsf(m[p * n + q]) > threshold) jacobi_rotate(m, v, n, p, q);
        }
    }
    /* stable sort of the diagonal, descending */
    int* order = w->order;
    for (int i = 0; i < n; ++i) {
        int j = i;
        const float key = m[i * n + i];
        while (j > 0 && m[order[j - 1] * n + order[j - 1]] < key) { order[j] = order[j - 1]; --j; }
        order[j] = i;
    }
    for (int out = 0; out < rank; ++out) {
        const int src = order[out];
        values[out] = m[src * n + src];
        float* row = vectors + (size_t)out * n;
        for (int r = 0; r < n; ++r) row[r] = v[r * n + src];
        float norm2 = 0.0f, best = 0.0f;
        int pivot = 0;
        for (int c = 0; c < n; ++c) {
            norm2 += row[c] * row[c];
            const float a = fabsf(row[c]);
            if (a > best) { best = a; pivot = c; }
        }
        if (norm2 <= FLT_MIN) continue;
        float scale = 1.0f / sqrtf(norm2);
        if (row[pivot] < 0.0f) scale = -scale;
        for (int c = 0; c < n; ++c) row[c] *= scale;
    }
}

/* map_dual_eigenvectors_to_basis (linalg.cpp:552-595) */
static void map_dual(const float* x, int rows, int cols, const float* values, const float* dual, int rank,
                     float* basis) {
    const float floor_value = 128.0f * FLT_EPSILON;
    for (int b = 0; b < rank; ++b) {
        float* row = basis + (size_t)b * cols;
        for (int c = 0; c < cols; ++c) row[c] = 0.0f;
        const float lambda = values[b];
        if (lambda <= floor_value) continue;
        for (int s = 0; s < rows; ++s) add_scaled(row, x + (size_t)s * cols, dual[(size_t)b * rows + s], cols);
        const float inv = 1.0f / sqrtf(lambda);
        for (int c = 0; c < cols; ++c) row[c] *= inv;
        const float norm2 = dot8(row, row, cols);
        if (norm2 <= floor_value) {
            for (int c = 0; c < cols; ++c) row[c] = 0.0f;
            continue;
        }
        const float scale = 1.0f / sqrtf(norm2);
        for (int c = 0; c < cols; ++c) row[c] *= scale;
    }
}

/* ------------------------------------------------------------------------ */
/* Group filter (core.cpp:190-412, 578-871).                                  */
static float model_noise2(const workspace* w) {
    const vnlb_stage_params* p = &w->p;
    return w->stage == VNLB_STAGE_FINAL ? (p->beta * p->sigma_basic) * p->sigma_basic
                                        : (p->beta * p->sigma) * p->sigma;
}

static void default_model(workspace* w, int similar) {
    const vnlb_stage_params* p = &w->p;
    const int sample_dim = w->patch_dim * (p->couple_channels && w->channels > 1 ? w->channels : 1);
    const int basis = imin(similar, cap_of(p->similar, p->model_cap_factor));
    const float tau = p->weight_epsilon + ((float)sample_dim / (float)basis);
    const float lgw = p->weight_alpha == 0.0f ? 0.0f : -p->weight_alpha * pin_logf(tau);
    for (int i = 0; i < similar; ++i) w->log_w[i] += lgw;
    w->model_count++;
}

/* accumulate_aggregation_model (core.cpp:326-412) */
static void aggregation_model(workspace* w, const float* centered, int similar, int dim, const float* values,
                              int rank, int basis_similar) {
    const vnlb_stage_params* p = &w->p;
    if (p->weight_alpha == 0.0f && p->weight_beta == 0.0f) { w->model_count++; return; }
    const float mn2 = model_noise2(w);
    const float estimate_noise2 = (p->beta * p->sigma) * p->sigma;
    float trace = 0.0f;
    for (int c = 0; c < rank; ++c) {
        const float diff = values[c] - mn2;
        const float lambda = diff > 0.0f ? diff : 0.0f;
        if (lambda > 0.0f) trace += lambda / (lambda + estimate_noise2);
    }
    const float tau = (p->weight_epsilon + ((float)dim / (float)basis_similar)) + trace;
    const float lgw = p->weight_alpha == 0.0f ? 0.0f : -p->weight_alpha * pin_logf(tau);
    if (p->weight_beta != 0.0f) {
        const float match_sigma = w->stage == VNLB_STAGE_FINAL ? p->sigma_basic : p->sigma;
        const float mem2 = fmax_std(match_sigma * match_sigma, (p->membership_noise_floor * p->sigma) * p->sigma);
        float volume = 0.0f;
        for (int c = 0; c < rank; ++c) {
            const float diff = values[c] - mn2;
            const float lambda = diff > 0.0f ? diff : 0.0f;
            if (lambda > 0.0f) volume += pin_log1pf(lambda / mem2);
        }
        volume /= (float)dim;
        float min_score = INFINITY;
        const float score_scale = sqrtf(2.0f * (float)dim);
        for (int i = 0; i < similar; ++i) {
            const float* row = centered + (size_t)i * dim;
            const float norm2 = dot8(row, row, dim);
            float distance = 0.0f, projected = 0.0f;
            for (int c = 0; c < rank; ++c) {
                const float proj = dot8(row, w->eigenvectors + (size_t)c * dim, dim);
                const float proj2 = proj * proj;
                const float diff = values[c] - mn2;
                const float lambda = diff > 0.0f ? diff : 0.0f;
                distance += proj2 / (lambda + mem2);
                projected += proj2;
            }
            const float res = norm2 - projected;
            distance += (res > 0.0f ? res : 0.0f) / mem2;
            const float score = (distance - (float)dim) / score_scale;
            w->scores[i] = score;
            min_score = fmin_std(min_score, score);
        }
        for (int i = 0; i < similar; ++i) {
            const float diff = w->scores[i] - min_score;
            const float membership = (diff > 0.0f ? diff : 0.0f) + volume;
            w->log_w[i] += lgw - (p->weight_beta * membership);
        }
    } else {
        for (int i = 0; i < similar; ++i) w->log_w[i] += lgw;
    }
    w->model_count++;
}

/* filter_vnlb_samples (core.cpp:638-792); samples are [similar][dim]. */
static int filter_samples(workspace* w, int similar, int dim, int flat) {
    const vnlb_stage_params* p = &w->p;
    const int rank = p->rank;
    const int B = imin(similar, cap_of(p->similar, p->model_cap_factor));
    if (B < imin(dim, rank)) return fail("VNLB: group_size must cover the effective VNLB rank");
    const int final_stage = w->stage == VNLB_STAGE_FINAL;
    const int dual = dim >= 64 && B < dim;
    if (final_stage) {
        mean_rows(w->samples_basic, B, dim, w->mean_basic);
        center(w->samples_basic, similar, dim, w->mean_basic, w->centered_basic);
        if (flat) {
            center(w->samples_noisy, similar, dim, w->mean_basic, w->centered_noisy);
        } else {
            mean_rows(w->samples_noisy, B, dim, w->mean_noisy);
            center(w->samples_noisy, similar, dim, w->mean_noisy, w->centered_noisy);
        }
    } else {
        mean_rows(w->samples_noisy, B, dim, w->mean_noisy);
        center(w->samples_noisy, similar, dim, w->mean_noisy, w->centered_noisy);
    }
    const float* center_vec = (final_stage && flat) ? w->mean_basic : w->mean_noisy;
    const float* membership = final_stage ? w->centered_basic : w->centered_noisy;
    if (rank == 0) {
        for (int i = 0; i < similar; ++i) memcpy(w->filtered + (size_t)i * dim, center_vec, (size_t)dim * sizeof(float));
        aggregation_model(w, membership, similar, dim, NULL, 0, B);
        return 0;
    }
    const float scale = 1.0f / (float)B;
    const float* basis_samples = final_stage ? w->centered_basic : w->centered_noisy;
    if (dual) {
        gram(basis_samples, B, dim, scale, w->sym);
        topk_eigen(w, w->sym, B, rank, w->eigenvalues, w->dual);
        map_dual(basis_samples, B, dim, w->eigenvalues, w->dual, rank, w->eigenvectors);
    } else {
        covariance(basis_samples, B, dim, scale, w->sym);
        topk_eigen(w, w->sym, dim, rank, w->eigenvalues, w->eigenvectors);
    }
    /* compute_filter_coefficients (core.cpp:616-636) */
    {
        const float sigma2 = (p->beta * p->sigma) * p->sigma;
        const float sigma_basic2 = final_stage ? (p->beta * p->sigma_basic) * p->sigma_basic : sigma2;
        const float threshold = p->variance_threshold * sigma2;
        for (int c = 0; c < rank; ++c) {
            float variance = w->eigenvalues[c];
            if (sigma_basic2 > 0.0f) variance -= fmin_std(variance, sigma_basic2);
            w->coefficients[c] = variance > threshold ? 1.0f / (1.0f + (sigma2 / variance)) : 0.0f;
        }
    }
    aggregation_model(w, membership, similar, dim, w->eigenvalues, rank, B);
    /* project_bayes_estimate (core.cpp:578-614) */
    for (int i = 0; i < similar; ++i) {
        const float* in = w->centered_noisy + (size_t)i * dim;
        float* out = w->filtered + (size_t)i * dim;
        for (int c = 0; c < dim; ++c) out[c] = 0.0f;
        for (int c = 0; c < rank; ++c) {
            const float coef = w->coefficients[c];
            if (coef == 0.0f) continue;
            const float* basis = w->eigenvectors + (size_t)c * dim;
            const float proj = dot8(in, basis, dim);
            add_scaled(out, basis, coef * proj, dim);
        }
        for (int c = 0; c < dim; ++c) out[c] += center_vec[c];
    }
    return 0;
}

/* group_variance / samples_channel_variance (core.cpp:491-559) */
static float variance_of(const float* values, int channels, int per_channel, int sample_major, int patch_dim,
                         int similar) {
    float variance = 0.0f;
    if (per_channel <= 1) return 0.0f;
    for (int c = 0; c < channels; ++c) {
        double sum = 0.0, sum2 = 0.0;
        if (sample_major) {
            for (int r = 0; r < similar; ++r)
                for (int q = 0; q < patch_dim; ++q) {
                    const float v = values[(size_t)r * channels * patch_dim + c * patch_dim + q];
                    sum += v;
                    sum2 += (double)v * (double)v;
                }
        } else {
            for (int i = 0; i < per_channel; ++i) {
                const float v = values[(size_t)c * per_channel + i];
                sum += v;
                sum2 += (double)v * (double)v;
            }
        }
        const double count = (double)per_channel;
        variance += (float)((sum2 - (sum * sum / count)) / (count - 1.0));
    }
    return variance / (float)channels;
}

/* ------------------------------------------------------------------------ */
/* One anchor frame: process_anchor_impl (core.cpp:1820-1906).                */
typedef struct record_sink {
    vnlb_group_record* groups;
    int group_capacity;
    int group_count;
    vnlb_match_record* matches;
    int match_capacity;
    int match_count;
} record_sink;

static int process_anchor_frame(workspace* w, const video* noisy, const video* basic, int anchor,
                                const stack_view* stack, record_sink* sink) {
    const vnlb_stage_params* p = &w->p;
    const int P = p->patch_size;
    const int W = w->width, H = w->height, C = w->channels;
    const int final_stage = w->stage == VNLB_STAGE_FINAL;
    const int coupled = p->couple_channels && C > 1;
    const int pd = w->patch_dim;
    for (int c = 0; c < C; ++c)
        for (int s = 0; s < stack->slots; ++s)
            for (int k = 0; k < 2; ++k)
                memset(stack_row(stack, c, s, k, 0), 0, (size_t)W * H * sizeof(float));
    if (anchor < 0 || anchor > w->source_frames - p->patch_time) return 0;
    const int max_x = W - P, max_y = H - P;
    memset(w->mask, 0, (size_t)W * H);
    for (int y = 0; y <= max_y; ++y)
        for (int x = 0; x <= max_x; ++x)
            if (grid_selected(p, W, H, w->source_frames, anchor, x, y)) w->mask[(size_t)y * W + x] = 1;

    const video* search = final_stage ? basic : noisy;
    const int search_channels = final_stage ? C : 1;
    for (int ay = 0; ay <= max_y; ++ay) {
        for (int ax = 0; ax <= max_x; ++ax) {
            if (!w->mask[(size_t)ay * W + ax]) continue;
            load_reference_patch(w, search, search_channels, ax, ay, anchor);
            const int S = find_similar(w, search, search_channels, ax, ay, anchor);
            w->sample_major = 0;
            for (int i = 0; i < S; ++i) { w->log_w[i] = 0.0f; w->w[i] = 1.0f; w->scores[i] = 0.0f; }
            w->model_count = 0;
            if (coupled) {
                /* gather_*_samples_coupled (core.cpp:1425-1585) */
                const int D = C * pd;
                for (int i = 0; i < S; ++i) {
                    const match m = w->matches[i];
                    for (int c = 0; c < C; ++c)
                        for (int t = 0; t < p->patch_time; ++t)
                            for (int y = 0; y < P; ++y) {
                                const size_t src = (size_t)(m.y + y) * W + m.x;
                                const size_t dst = (size_t)i * D + c * pd + (t * P + y) * P;
                                memcpy(w->samples_noisy + dst, plane_ptr(noisy, m.frame + t, c) + src, (size_t)P * 4);
                                if (final_stage)
                                    memcpy(w->samples_basic + dst, plane_ptr(basic, m.frame + t, c) + src, (size_t)P * 4);
                            }
                }
                /* transform_vnlb_coupled_samples (core.cpp:828-846) */
                w->sample_major = 1;
                int equal = S > 1;
                for (int i = 1; i < S && equal; ++i)
                    for (int d = 0; d < D; ++d)
                        if (w->samples_noisy[(size_t)i * D + d] != w->samples_noisy[d]) { equal = 0; break; }
                if (equal) {
                    memcpy(w->filtered, w->samples_noisy, (size_t)S * D * sizeof(float));
                } else {
                    int flat = 0;
                    if (final_stage)
                        flat = p->flat_areas &&
                               variance_of(w->samples_noisy, C, pd * S, 1, pd, S) < (p->sigma * p->sigma) * p->gamma;
                    if (filter_samples(w, S, D, flat) != 0) return -1;
                }
            } else {
                /* gather_basic_group / gather_final_group (core.cpp:1364-1508) */
                for (int c = 0; c < C; ++c) {
                    const int base = c * pd * S;
                    for (int t = 0; t < p->patch_time; ++t)
                        for (int y = 0; y < P; ++y)
                            for (int x = 0; x < P; ++x) {
                                const int pos = (t * P + y) * P + x;
                                for (int i = 0; i < S; ++i) {
                                    const match m = w->matches[i];
                                    const size_t src = (size_t)(m.y + y) * W + m.x + x;
                                    w->group_noisy[base + pos * S + i] = plane_ptr(noisy, m.frame + t, c)[src];
                                    if (final_stage) w->group_basic[base + pos * S + i] = plane_ptr(basic, m.frame + t, c)[src];
                                }
                            }
                }
                /* transform_vnlb_group (core.cpp:848-871) */
                int equal = S > 1;
                for (int c = 0; c < C && equal; ++c)
                    for (int pos = 0; pos < pd && equal; ++pos) {
                        const float v = w->group_noisy[c * pd * S + pos * S];
                        for (int i = 1; i < S; ++i)
                            if (w->group_noisy[c * pd * S + pos * S + i] != v) { equal = 0; break; }
                    }
                if (!equal) {
                    int flat = 0;
                    if (final_stage)
                        flat = p->flat_areas &&
                               variance_of(w->group_noisy, C, pd * S, 0, pd, S) < (p->sigma * p->sigma) * p->gamma;
                    for (int c = 0; c < C; ++c) {
                        /* transform_vnlb_channel (core.cpp:794-808) */
                        for (int i = 0; i < S; ++i)
                            for (int pos = 0; pos < pd; ++pos) {
                                w->samples_noisy[(size_t)i * pd + pos] = w->group_noisy[c * pd * S + pos * S + i];
                                if (final_stage) w->samples_basic[(size_t)i * pd + pos] = w->group_basic[c * pd * S + pos * S + i];
                            }
                        if (filter_samples(w, S, pd, flat) != 0) return -1;
                        for (int i = 0; i < S; ++i)
                            for (int pos = 0; pos < pd; ++pos)
                                w->group_noisy[c * pd * S + pos * S + i] = w->filtered[(size_t)i * pd + pos];
                    }
                }
            }
            /* finalize_aggregation_weights (core.cpp:276-294) */
            if (!(p->weight_alpha != 0.0f || p->weight_beta != 0.0f || p->weight_gamma != 0.0f)) {
                for (int i = 0; i < S; ++i) w->w[i] = 1.0f;
            } else {
                if (w->model_count == 0) default_model(w, S);
                const float inv = 1.0f / (float)w->model_count;
                for (int i = 0; i < S; ++i) {
                    float lw = w->log_w[i] * inv;
                    lw = lw < -80.0f ? -80.0f : (lw > 80.0f ? 80.0f : lw);
                    w->w[i] = pin_expf(lw);
                }
            }
            /* write_*_contributions (core.cpp:1587-1795) */
            const int windowed = p->weight_gamma != 0.0f;
            for (int i = 0; i < S; ++i) {
                const match m = w->matches[i];
                const float pw = w->w[i];
                for (int t = 0; t < p->patch_time; ++t) {
                    const int slot = m.frame + t - anchor + p->search_bwd;
                    if (slot < 0 || slot >= stack->slots) continue;
                    for (int y = 0; y < P; ++y) {
                        const int oy = m.y + y;
                        if (w->sample_major) {
                            const float* row = w->filtered + (size_t)i * C * pd;
                            for (int c = 0; c < C; ++c) {
                                const float* sample = row + c * pd + (t * P + y) * P;
                                float* num = stack_row(stack, c, slot, 0, oy) + m.x;
                                float* wt = stack_row(stack, c, slot, 1, oy) + m.x;
                                if (!windowed) {
                                    add_scaled(num, sample, pw, P);
                                    for (int x = 0; x < P; ++x) wt[x] += pw;
                                } else {
                                    for (int x = 0; x < P; ++x) {
                                        const float cw = pw * w->window[y * P + x];
                                        num[x] += cw * sample[x];
                                        wt[x] += cw;
                                    }
                                }
                            }
                        } else {
                            for (int x = 0; x < P; ++x) {
                                const float cw = pw * w->window[y * P + x];
                                for (int c = 0; c < C; ++c) stack_row(stack, c, slot, 1, oy)[m.x + x] += cw;
                                const int pos = (t * P + y) * P + x;
                                for (int c = 0; c < C; ++c)
                                    stack_row(stack, c, slot, 0, oy)[m.x + x] += cw * w->group_noisy[c * pd * S + pos * S + i];
                            }
                        }
                    }
                }
            }
            if (sink) {
                if (sink->group_count < sink->group_capacity) {
                    sink->groups[sink->group_count] = (vnlb_group_record){ax, ay, S, sink->match_count};
                }
                sink->group_count++;
                for (int i = 0; i < S; ++i) {
                    if (sink->match_count < sink->match_capacity) {
                        const match m = w->matches[i];
                        sink->matches[sink->match_count] = (vnlb_match_record){m.distance, m.x, m.y, m.frame, w->w[i]};
                    }
                    sink->match_count++;
                }
            }
            /* apply_frame_paste_mask (core.cpp:980-1008) */
            for (int i = 0; i < S; ++i) {
                const match m = w->matches[i];
                if (m.frame != anchor) continue;
#define CLEAR(xx, yy) do { const int cx_ = (xx), cy_ = (yy); \
                if (cx_ >= 0 && cx_ < W && cy_ >= 0 && cy_ < H) w->mask[(size_t)cy_ * W + cx_] = 0; } while (0)
                CLEAR(m.x, m.y);
                if (m.y > 2 * P) CLEAR(m.x, m.y - 1);
                if (m.y < H - 2 * P) CLEAR(m.x, m.y + 1);
                if (m.x > 2 * P) CLEAR(m.x - 1, m.y);
                if (m.x < W - 2 * P) CLEAR(m.x + 1, m.y);
#undef CLEAR
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Exported entry points.                                                    */
typedef struct job {
    int stage;
    const vnlb_stage_params* p;
    const vnlb_flow* flow;
    video noisy, basic;
    int first_anchor, anchor_count;
    float* stacks;
    size_t stack_values;
    int next;
    int status;
    pthread_mutex_t lock;
} job;

static void* worker(void* arg) {
    job* j = (job*)arg;
    workspace w;
    memset(&w, 0, sizeof(w));
    if (ws_prepare(&w, j->stage, j->p, j->noisy.width, j->noisy.height, j->noisy.frames, j->noisy.channels) != 0) {
        pthread_mutex_lock(&j->lock); j->status = -1; pthread_mutex_unlock(&j->lock);
        return NULL;
    }
    w.flow = j->flow;
    for (;;) {
        pthread_mutex_lock(&j->lock);
        const int index = j->status == 0 ? j->next++ : j->anchor_count;
        pthread_mutex_unlock(&j->lock);
        if (index >= j->anchor_count) break;
        const stack_view sv = {j->stacks + j->stack_values * (size_t)index, j->noisy.width, j->noisy.height,
                               j->noisy.channels, j->p->search_bwd + j->p->search_fwd + j->p->patch_time,
                               j->p->search_bwd};
        if (process_anchor_frame(&w, &j->noisy, &j->basic, j->first_anchor + index, &sv, NULL) != 0) {
            pthread_mutex_lock(&j->lock); j->status = -1; pthread_mutex_unlock(&j->lock);
        }
    }
    ws_free(&w);
    return NULL;
}

/* vnlb.Basic / vnlb.Final stacks of anchor frames first_anchor .. + count - 1,
 * with flow-guided search centres when flow is not NULL (process_*_anchor_
 * mvtools, src/core/core.cpp:2095-2109). */
int vnlboracle_stage_stacks_flow(int stage, const vnlb_stage_params* params, const float* clip, const float* basic,
                                 int width, int height, int frames, int channels, int first_anchor, int anchor_count,
                                 int threads, const vnlb_flow* flow, float* stacks) {
    if (validate(params, width, height, frames, channels) != 0) return -1;
    if (stage == VNLB_STAGE_FINAL && basic == NULL) return fail("VNLB: ref must be a video node");
    job j;
    memset(&j, 0, sizeof(j));
    j.stage = stage;
    j.p = params;
    j.flow = flow;
    j.noisy = (video){clip, width, height, frames, channels};
    j.basic = (video){basic, width, height, frames, channels};
    j.first_anchor = first_anchor;
    j.anchor_count = anchor_count;
    j.stacks = stacks;
    j.stack_values = (size_t)channels * (params->search_bwd + params->search_fwd + params->patch_time) * 2 *
                     (size_t)height * width;
    pthread_mutex_init(&j.lock, NULL);
    if (threads < 1) threads = 1;
    if (threads > anchor_count) threads = anchor_count > 0 ? anchor_count : 1;
    pthread_t pool[256];
    if (threads > 256) threads = 256;
    for (int t = 0; t < threads; ++t) pthread_create(&pool[t], NULL, worker, &j);
    for (int t = 0; t < threads; ++t) pthread_join(pool[t], NULL);
    pthread_mutex_destroy(&j.lock);
    return j.status;
}

int vnlboracle_stage_stacks(int stage, const vnlb_stage_params* params, const float* clip, const float* basic,
                            int width, int height, int frames, int channels, int first_anchor, int anchor_count,
                            int threads, float* stacks) {
    return vnlboracle_stage_stacks_flow(stage, params, clip, basic, width, height, frames, channels, first_anchor,
                                        anchor_count, threads, NULL, stacks);
}

int vnlboracle_stage_stack(int stage, const vnlb_stage_params* params, const float* clip, const float* basic,
                           int width, int height, int frames, int channels, int anchor_frame, float* stack) {
    return vnlboracle_stage_stacks(stage, params, clip, basic, width, height, frames, channels, anchor_frame, 1, 1,
                                   stack);
}

/* Same as vnlboracle_stage_stack, and also reports every processed group in
 * raster order: its anchor, its rows (CPU row order) and their weights.
 * Returns the number of groups (which may exceed group_capacity), or -1. */
int vnlboracle_anchor_groups_flow(int stage, const vnlb_stage_params* params, const float* clip,
                                  const float* basic, int width, int height, int frames, int channels,
                                  int anchor_frame, const vnlb_flow* flow, float* stack, vnlb_group_record* groups,
                                  int group_capacity, vnlb_match_record* matches, int match_capacity,
                                  int* match_total) {
    if (validate(params, width, height, frames, channels) != 0) return -1;
    workspace w;
    memset(&w, 0, sizeof(w));
    if (ws_prepare(&w, stage, params, width, height, frames, channels) != 0) return -1;
    w.flow = flow;
    const video noisy = {clip, width, height, frames, channels};
    const video ref = {basic, width, height, frames, channels};
    const stack_view sv = {stack, width, height, channels,
                           params->search_bwd + params->search_fwd + params->patch_time, params->search_bwd};
    record_sink sink = {groups, group_capacity, 0, matches, match_capacity, 0};
    const int status = process_anchor_frame(&w, &noisy, &ref, anchor_frame, &sv, &sink);
    ws_free(&w);
    if (status != 0) return -1;
    if (match_total) *match_total = sink.match_count;
    return sink.group_count;
}

int vnlboracle_anchor_groups(int stage, const vnlb_stage_params* params, const float* clip, const float* basic,
                             int width, int height, int frames, int channels, int anchor_frame, float* stack,
                             vnlb_group_record* groups, int group_capacity, vnlb_match_record* matches,
                             int match_capacity, int* match_total) {
    return vnlboracle_anchor_groups_flow(stage, params, clip, basic, width, height, frames, channels, anchor_frame,
                                         NULL, stack, groups, group_capacity, matches, match_capacity, match_total);
}

/* Matches of one anchor alone (no paste mask), rows in CPU order. */
int vnlboracle_match_anchor(int stage, const vnlb_stage_params* params, const float* clip, const float* basic,
                            int width, int height, int frames, int channels, int anchor_frame, int ax, int ay,
                            vnlb_match_record* out, int capacity) {
    if (validate(params, width, height, frames, channels) != 0) return -1;
    workspace w;
    memset(&w, 0, sizeof(w));
    if (ws_prepare(&w, stage, params, width, height, frames, channels) != 0) return -1;
    const video src = {stage == VNLB_STAGE_FINAL ? basic : clip, width, height, frames, channels};
    const int sc = stage == VNLB_STAGE_FINAL ? channels : 1;
    load_reference_patch(&w, &src, sc, ax, ay, anchor_frame);
    const int S = find_similar(&w, &src, sc, ax, ay, anchor_frame);
    for (int i = 0; i < S && i < capacity; ++i)
        out[i] = (vnlb_match_record){w.matches[i].distance, w.matches[i].x, w.matches[i].y, w.matches[i].frame, 1.0f};
    ws_free(&w);
    return S;
}

/* render_aggregate_frame (src/vs/plugin.cpp:966-1045) */
int vnlboracle_aggregate(const float* stacks, const float* source, int width, int height, int frames, int channels,
                         int search_bwd, int search_fwd, int patch_time, float* out) {
    const int slots = search_bwd + search_fwd + patch_time;
    const size_t plane = (size_t)width * height;
    const size_t stack_plane = plane * 2 * (size_t)slots;
    for (int f = 0; f < frames; ++f) {
        const int first = imax(0, f - (search_fwd + patch_time - 1));
        const int last = imin(frames - 1, f + search_bwd);
        for (int c = 0; c < channels; ++c) {
            const float* src = source + ((size_t)f * channels + c) * plane;
            float* dst = out + ((size_t)f * channels + c) * plane;
            for (int y = 0; y < height; ++y)
                for (int x = 0; x < width; ++x) {
                    float num = 0.0f, wt = 0.0f;
                    for (int a = first; a <= last; ++a) {
                        const int slot = f - a + search_bwd;
                        const float* base = stacks + ((size_t)a * channels + c) * stack_plane;
                        const size_t row = (size_t)slot * 2 * height + y;
                        num += base[row * width + x];
                        wt += base[(row + height) * width + x];
                    }
                    const size_t i = (size_t)y * width + x;
                    dst[i] = wt > 0.0f ? num / wt : src[i];
                }
        }
    }
    return 0;
}
