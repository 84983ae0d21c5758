// Upload and readback of the tolerance solve's arena through the caller's
// pinned, device-mapped host arrays: one kernel gathers every island's
// inputs, one scatters every island's FP32 solution (arena_io.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pfsf_b200 {
namespace kappa {

// One island's host arrays as device-visible addresses (nullptr: the island
// is copied with cudaMemcpyAsync instead) and its place in the arena.
struct IslandIO {
    const uint8_t* h_type;
    const float* h_kappa;
    const float* h_source;
    const float* h_phi;   // initial guess in
    float* h_phi_out;     // solution out (the same caller array)
    int64_t off, n;
    int32_t b0;           // first block of this island in the launches below
    int32_t pad;
};

// type, kappa, source and phi0 of every mapped island into the arena arrays
// (type, k32, b, e); nb = total blocks (last island's b0 + its blocks).
void launch_arena_upload(cudaStream_t s, const IslandIO* io, int nisl, int nb, uint8_t* type, float* k32, float* b,
                         float* e);
// e = (float)x64 over the arena's islands and, for every mapped island, the
// same values into its caller phi array.
void launch_arena_readback(cudaStream_t s, const IslandIO* io, int nisl, int nb, const double* x64, float* e);
constexpr int kArenaIoBlock = 256;

}  // namespace kappa
}  // namespace pfsf_b200
