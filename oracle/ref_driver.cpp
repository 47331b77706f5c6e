// Driver that runs the reference's own CPU core without VapourSynth.
//
// TEST INFRASTRUCTURE ONLY (see oracle/vnlb_oracle.h).  It is compiled by
// oracle/Makefile together with the reference sources src/core/core.cpp,
// src/linalg/linalg.cpp and src/aggregate/aggregate.cpp into
// oracle/_ref/libvnlb_ref.so.  It replays what the VapourSynth plugin does
// around the core:
//   * vnlbref_stage_stack   = render_stage_frame   (src/vs/plugin.cpp:616-758)
//   * vnlbref_aggregate     = render_aggregate_frame (src/vs/plugin.cpp:966-1045)
//   * vnlbref_chain         = Basic -> Aggregate -> Final(ref) -> Aggregate,
//                             frames spread over std::threads with one
//                             workspace per thread, as fmParallel does;
//   * vnlbref_stage_stacks_flow: render_stage_frame with mvfw / mvbw clips,
//                             the reference's MVToolsVectorGrid objects of the
//                             anchor's input window handed to its
//                             MVToolsFlowProvider (plugin.cpp:697-729).
#include "vnlb_oracle.h"

#include "aggregate/aggregate.hpp"
#include "core/core.hpp"
#include "flow/flow.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using vnlb::aggregate::ContributionPlaneView;
using vnlb::aggregate::ContributionStackView;
using vnlb::core::ConstPlaneView;
using vnlb::core::ConstVideoView;
using vnlb::core::FrameRange;
using vnlb::core::StageParameters;
using vnlb::core::StageWorkspace;
using vnlb::core::VideoGeometry;

thread_local std::string g_last_error;

StageParameters to_core(const vnlb_stage_params& p) {
    StageParameters s{};
    s.sigma = p.sigma;
    s.patch_size = p.patch_size;
    s.patch_time = p.patch_time;
    s.search_window = p.search_window;
    s.search_bwd = p.search_bwd;
    s.search_fwd = p.search_fwd;
    s.similar = p.similar;
    s.rank = p.rank;
    s.similar_cap_factor = p.similar_cap_factor;
    s.model_cap_factor = p.model_cap_factor;
    s.beta = p.beta;
    s.tau = p.tau;
    s.variance_threshold = p.variance_threshold;
    s.sigma_basic = p.sigma_basic;
    s.gamma = p.gamma;
    s.weight_alpha = p.weight_alpha;
    s.weight_beta = p.weight_beta;
    s.weight_gamma = p.weight_gamma;
    s.weight_epsilon = p.weight_epsilon;
    s.membership_noise_floor = p.membership_noise_floor;
    s.proc_step = p.proc_step;
    s.flat_areas = p.flat_areas != 0;
    s.couple_channels = p.couple_channels != 0;
    return s;
}

int slot_count(const StageParameters& p) {
    return p.search_bwd + p.search_fwd + p.patch_time;
}

// The reference's grid object of one frame of one direction.
vnlb::flow::MVToolsVectorGrid make_grid(const vnlb_flow_grids& g, int frame) {
    vnlb::flow::MVToolsVectorGrid grid;
    grid.analysis.block_size_x = g.block_size_x;
    grid.analysis.block_size_y = g.block_size_y;
    grid.analysis.pel = g.pel;
    grid.analysis.overlap_x = g.overlap_x;
    grid.analysis.overlap_y = g.overlap_y;
    grid.analysis.block_count_x = g.block_count_x;
    grid.analysis.block_count_y = g.block_count_y;
    grid.analysis.delta_frame = 1;
    grid.valid = g.usable[frame] != 0;
    const std::size_t count = static_cast<std::size_t>(g.block_count_x) * g.block_count_y;
    grid.vectors.resize(count);
    const int* v = g.vectors + static_cast<std::size_t>(frame) * count * 2;
    for (std::size_t i = 0; i < count; ++i) {
        grid.vectors[i].x = v[2 * i];
        grid.vectors[i].y = v[2 * i + 1];
    }
    return grid;
}

// render_stage_frame (src/vs/plugin.cpp:616-758) without VapourSynth: the
// local frame window is [range.first, range.last] of the whole clip.
void stage_stack(int stage, const StageParameters& parameters,
                 const float* clip, const float* basic, int width, int height,
                 int frames, int channels, int anchor_frame, float* stack,
                 StageWorkspace& workspace, const vnlb_flow* flow = nullptr) {
    const VideoGeometry full{width, height, frames, channels, 0, frames};
    const auto layout = vnlb::aggregate::make_contribution_layout(
        full, parameters.search_bwd, parameters.search_fwd,
        parameters.patch_time);
    const int slots = layout.slot_count;
    const std::size_t plane_rows = static_cast<std::size_t>(slots) * 2 * height;
    std::vector<ContributionPlaneView> planes(static_cast<std::size_t>(channels));
    for (int c = 0; c < channels; ++c) {
        planes[static_cast<std::size_t>(c)] = ContributionPlaneView{
            stack + static_cast<std::size_t>(c) * plane_rows * width, width};
    }
    const ContributionStackView contributions(
        std::span<ContributionPlaneView>(planes), layout);

    if (anchor_frame > frames - parameters.patch_time) {
        vnlb::aggregate::clear_contributions(contributions);
        return;
    }
    const FrameRange range =
        vnlb::core::input_frame_range_for_anchor(full, parameters, anchor_frame);
    const int local_frames = range.last - range.first + 1;
    std::vector<ConstPlaneView> clip_planes;
    std::vector<ConstPlaneView> ref_planes;
    const std::size_t plane = static_cast<std::size_t>(width) * height;
    for (int f = range.first; f <= range.last; ++f) {
        for (int c = 0; c < channels; ++c) {
            const std::size_t offset =
                (static_cast<std::size_t>(f) * channels + c) * plane;
            clip_planes.push_back(ConstPlaneView{clip + offset, width});
            if (stage == VNLB_STAGE_FINAL) {
                ref_planes.push_back(ConstPlaneView{basic + offset, width});
            }
        }
    }
    const VideoGeometry local{width, height, local_frames, channels,
                              range.first, frames};
    const ConstVideoView clip_view(
        std::span<const ConstPlaneView>(clip_planes), local);
    if (flow != nullptr && (flow->fw.present || flow->bw.present)) {
        // build_mvtools_grid_window + MVToolsFlowProvider(mvfw, mvbw)
        std::vector<vnlb::flow::MVToolsVectorGrid> fw, bw;
        std::vector<const vnlb::flow::MVToolsVectorGrid*> fw_ptrs, bw_ptrs;
        for (int f = range.first; f <= range.last; ++f) {
            if (flow->fw.present) fw.push_back(make_grid(flow->fw, f));
            if (flow->bw.present) bw.push_back(make_grid(flow->bw, f));
        }
        for (auto& g : fw) fw_ptrs.push_back(&g);
        for (auto& g : bw) bw_ptrs.push_back(&g);
        const vnlb::flow::MVToolsFlowProvider provider(
            std::span<const vnlb::flow::MVToolsVectorGrid* const>(fw_ptrs.data(), fw_ptrs.size()), range.first,
            std::span<const vnlb::flow::MVToolsVectorGrid* const>(bw_ptrs.data(), bw_ptrs.size()), range.first);
        if (stage == VNLB_STAGE_BASIC) {
            vnlb::core::process_basic_anchor_mvtools(clip_view, anchor_frame, parameters, provider, contributions,
                                                     workspace);
        } else {
            const ConstVideoView ref_view(std::span<const ConstPlaneView>(ref_planes), local);
            vnlb::core::process_final_anchor_mvtools(clip_view, ref_view, anchor_frame, parameters, provider,
                                                     contributions, workspace);
        }
        return;
    }
    const vnlb::flow::SameLocationProvider flow_same;
    const auto& flow_provider = flow_same;
    if (stage == VNLB_STAGE_BASIC) {
        vnlb::core::process_basic_anchor_no_flow(clip_view, anchor_frame,
                                                 parameters, flow_provider,
                                                 contributions, workspace);
    } else {
        const ConstVideoView ref_view(
            std::span<const ConstPlaneView>(ref_planes), local);
        vnlb::core::process_final_anchor_no_flow(clip_view, ref_view,
                                                 anchor_frame, parameters,
                                                 flow_provider, contributions,
                                                 workspace);
    }
}

// render_aggregate_frame (src/vs/plugin.cpp:966-1045).
void aggregate_frame(const float* stacks, const float* source, int width,
                     int height, int frames, int channels, int search_bwd,
                     int search_fwd, int patch_time, int frame, float* out) {
    const int slots = search_bwd + search_fwd + patch_time;
    const int first_anchor = std::max(0, frame - (search_fwd + patch_time - 1));
    const int last_anchor = std::min(frames - 1, frame + search_bwd);
    const std::size_t plane = static_cast<std::size_t>(width) * height;
    const std::size_t stack_plane = plane * 2 * static_cast<std::size_t>(slots);
    for (int c = 0; c < channels; ++c) {
        const float* src =
            source + (static_cast<std::size_t>(frame) * channels + c) * plane;
        float* dst = out + (static_cast<std::size_t>(frame) * channels + c) * plane;
        for (int y = 0; y < height; ++y) {
            for (int x = 0; x < width; ++x) {
                float numerator = 0.0F;
                float weight = 0.0F;
                for (int anchor = first_anchor; anchor <= last_anchor; ++anchor) {
                    const int slot = frame - anchor + search_bwd;
                    const float* base =
                        stacks + (static_cast<std::size_t>(anchor) * channels + c) *
                                     stack_plane;
                    const std::size_t num_row =
                        static_cast<std::size_t>(slot) * 2 * height + y;
                    numerator += base[num_row * width + x];
                    weight += base[(num_row + height) * width + x];
                }
                const std::size_t i = static_cast<std::size_t>(y) * width + x;
                dst[i] = weight > 0.0F ? numerator / weight : src[i];
            }
        }
    }
}

template <typename Fn> void parallel_frames(int count, int threads, Fn fn) {
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    std::exception_ptr failure;
    std::mutex failure_lock;
    const int workers = std::max(1, std::min(threads, count));
    for (int t = 0; t < workers; ++t) {
        pool.emplace_back([&]() {
            StageWorkspace workspace;
            for (;;) {
                const int index = next.fetch_add(1);
                if (index >= count) {
                    return;
                }
                try {
                    fn(index, workspace);
                } catch (...) {
                    std::lock_guard lock(failure_lock);
                    failure = std::current_exception();
                    next.store(count);
                    return;
                }
            }
        });
    }
    for (auto& worker : pool) {
        worker.join();
    }
    if (failure) {
        std::rethrow_exception(failure);
    }
}

template <typename Fn> int guarded(Fn fn) {
    try {
        fn();
        return 0;
    } catch (const std::exception& error) {
        g_last_error = std::string("VNLB: ") + error.what();
        return -1;
    }
}

} // namespace

extern "C" {

const char* vnlbref_last_error(void) { return g_last_error.c_str(); }

int vnlbref_stage_stack(int stage, const vnlb_stage_params* params,
                        const float* clip, const float* basic, int width,
                        int height, int frames, int channels, int anchor_frame,
                        float* stack) {
    return guarded([&]() {
        StageWorkspace workspace;
        const StageParameters p = to_core(*params);
        vnlb::core::validate_stage_configuration(
            VideoGeometry{width, height, frames, channels, 0, frames}, p);
        stage_stack(stage, p, clip, basic, width, height, frames, channels,
                    anchor_frame, stack, workspace);
    });
}

int vnlbref_stage_stacks(int stage, const vnlb_stage_params* params,
                         const float* clip, const float* basic, int width,
                         int height, int frames, int channels, int first_anchor,
                         int anchor_count, int threads, float* stacks) {
    return guarded([&]() {
        const StageParameters p = to_core(*params);
        vnlb::core::validate_stage_configuration(
            VideoGeometry{width, height, frames, channels, 0, frames}, p);
        const std::size_t stack_values = static_cast<std::size_t>(channels) *
                                         slot_count(p) * 2 * height * width;
        parallel_frames(anchor_count, threads,
                        [&](int index, StageWorkspace& workspace) {
                            stage_stack(stage, p, clip, basic, width, height,
                                        frames, channels, first_anchor + index,
                                        stacks + stack_values * index,
                                        workspace);
                        });
    });
}

int vnlbref_stage_stacks_flow(int stage, const vnlb_stage_params* params,
                              const float* clip, const float* basic, int width,
                              int height, int frames, int channels,
                              int first_anchor, int anchor_count, int threads,
                              const vnlb_flow* flow, float* stacks) {
    return guarded([&]() {
        const StageParameters p = to_core(*params);
        vnlb::core::validate_stage_configuration(
            VideoGeometry{width, height, frames, channels, 0, frames}, p);
        const std::size_t stack_values = static_cast<std::size_t>(channels) *
                                         slot_count(p) * 2 * height * width;
        parallel_frames(anchor_count, threads,
                        [&](int index, StageWorkspace& workspace) {
                            stage_stack(stage, p, clip, basic, width, height,
                                        frames, channels, first_anchor + index,
                                        stacks + stack_values * index,
                                        workspace, flow);
                        });
    });
}

int vnlbref_aggregate(const float* stacks, const float* source, int width,
                      int height, int frames, int channels, int search_bwd,
                      int search_fwd, int patch_time, float* out) {
    return guarded([&]() {
        for (int frame = 0; frame < frames; ++frame) {
            aggregate_frame(stacks, source, width, height, frames, channels,
                            search_bwd, search_fwd, patch_time, frame, out);
        }
    });
}

} // extern "C"
