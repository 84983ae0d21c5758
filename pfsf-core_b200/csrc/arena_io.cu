// Gather / scatter of the tolerance solve's inputs and solution between the
// caller's pinned host arrays (read and written through their device-mapped
// addresses, over the host link) and the packed arena: one launch each for
// all islands, instead of four copies per island in and one out.
#include "arena_io.h"

namespace pfsf_b200 {
namespace kappa {
namespace {

// island of block b: the last island whose first block is <= b
__device__ __forceinline__ int io_island(const IslandIO* __restrict__ io, int nisl) {
    __shared__ int s_q;
    if (threadIdx.x == 0) {
        const int b = (int)blockIdx.x;
        int lo = 0, hi = nisl - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (io[mid].b0 <= b) lo = mid;
            else hi = mid - 1;
        }
        s_q = lo;
    }
    __syncthreads();
    return s_q;
}

__global__ void __launch_bounds__(kArenaIoBlock) k_arena_upload(const IslandIO* __restrict__ io, int nisl,
                                                                 uint8_t* __restrict__ type, float* __restrict__ k32,
                                                                 float* __restrict__ b, float* __restrict__ e) {
    const IslandIO& I = io[io_island(io, nisl)];
    const int64_t t = (int64_t)(blockIdx.x - I.b0) * blockDim.x + threadIdx.x;
    if (t >= I.n || I.h_type == nullptr) return;
    const int64_t o = I.off + t;
    type[o] = I.h_type[t];
    k32[o] = I.h_kappa[t];
    b[o] = I.h_source[t];
    e[o] = I.h_phi[t];
}

__global__ void __launch_bounds__(kArenaIoBlock) k_arena_readback(const IslandIO* __restrict__ io, int nisl,
                                                                   const double* __restrict__ x64,
                                                                   float* __restrict__ e) {
    const IslandIO& I = io[io_island(io, nisl)];
    const int64_t t = (int64_t)(blockIdx.x - I.b0) * blockDim.x + threadIdx.x;
    if (t >= I.n) return;
    const float v = (float)x64[I.off + t];
    e[I.off + t] = v;
    if (I.h_phi_out) I.h_phi_out[t] = v;
}

}  // namespace

void launch_arena_upload(cudaStream_t s, const IslandIO* io, int nisl, int nb, uint8_t* type, float* k32, float* b,
                         float* e) {
    if (nisl > 0 && nb > 0) k_arena_upload<<<(unsigned)nb, kArenaIoBlock, 0, s>>>(io, nisl, type, k32, b, e);
}

void launch_arena_readback(cudaStream_t s, const IslandIO* io, int nisl, int nb, const double* x64, float* e) {
    if (nisl > 0 && nb > 0) k_arena_readback<<<(unsigned)nb, kArenaIoBlock, 0, s>>>(io, nisl, x64, e);
}

}  // namespace kappa
}  // namespace pfsf_b200
