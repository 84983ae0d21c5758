// Packed device arena of the tolerance solve (one allocation per island set).
#pragma once
#include <vector>

#include "arena_io.h"
#include "engine.h"
#include "kappa.h"

namespace pfsf_b200 {

struct Engine::Arena {
    std::vector<int32_t> ids;        // island ids in arena order
    std::vector<int64_t> active;     // solid voxels per island
    std::vector<KDesc> desc;         // host copy of descriptors
    int prec = -1;
    int64_t nfine = 0, ncoarse = 0;
    void* base = nullptr;            // single device allocation
    size_t bytes = 0;
    KArena dev{};                    // device pointers (into base)
    float* hscratch = nullptr;       // pinned host words (the whole-GPU tier's barrier error flag)
    float* phi_out = nullptr;        // FP32 solution staging (device), aliases e
    std::vector<void*> pinned;       // host ranges registered (mapped) by this arena
    // the islands' kappa-form host arrays as device-mapped addresses, for the
    // one-launch gather of the inputs and scatter of the solution
    std::vector<kappa::IslandIO> io;
    kappa::IslandIO* d_io = nullptr; // device copy (inside base)
    int io_blocks = 0;               // blocks of the gather / scatter launches
    bool io_any = false;             // at least one island is mapped
    bool solved = false;             // x64 holds a forward solution of this island set
    int persistent_ctas = 0;         // CTAs of the last batched launch(es)
    bool b_stale = false;            // b holds an adjoint right-hand side, not the sources
    double* xf = nullptr;            // adjoint: FP64 copy of the forward solution (own allocation)
    KDesc* hdesc = nullptr;          // pinned host copy of the per-island results of the last solve
    // the batched solve's launch sequence (queue reset, persistent launch(es),
    // result copies) as a CUDA graph, captured on the second solve of this
    // arena with the same parameters and replayed after
    bool launched = false;
    bool graph_off = false;          // capture failed once: launch directly from then on
    cudaGraphExec_t solve_exec = nullptr;
    std::vector<double> solve_key;
    int graph_launches = 0, graph_ctas = 0;
    kappa::PlainGraphs plain;        // per-island graphs of the plain solve
};

}  // namespace pfsf_b200
