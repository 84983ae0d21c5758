// State of the batched reference tick (engine_batch.cpp).
#pragma once
#include <vector>

#include "compat.h"
#include "engine.h"

namespace pfsf_b200 {

// What recording one group's schedule does to the per-island state: rbgs
// steps counted (chebyshev_iter), coarse ping-pong flips, PCG slot flips,
// whether a V-cycle rebuilt the coarse inputs.
struct TickEffect {
    int steps = 0, f1 = 0, f2 = 0, fr = 0, downsampled = 0;
};

struct Engine::TickBatch {
    // device: descriptor table, block prefixes (per group, then the whole
    // set), result records; pinned host staging of the table and prefixes
    compat::CIsl* d_tab = nullptr;
    int* d_bs = nullptr;
    TickResult* d_res = nullptr;
    compat::CIsl* h_tab = nullptr;
    int* h_bs = nullptr;
    int cap_isl = 0, cap_bs = 0;
    // captured tick and the structure it was captured for
    cudaGraphExec_t exec = nullptr;
    std::vector<int64_t> key;
    int64_t graph_launches = 0;
    std::vector<TickEffect> effects;  // per group of the captured structure
    // the last tick (pfsf_last_tick_report); the events bracket its stream work
    bool have_tick = false;
    pfsf_tick_report last{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // capture streams of the groups' branches, their join events, the fork
    std::vector<cudaStream_t> lanes;
    std::vector<cudaEvent_t> lane_done;
    cudaEvent_t fork = nullptr;
};

// group branches of one captured tick
constexpr int kLanes = 8;

}  // namespace pfsf_b200
