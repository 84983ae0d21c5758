// Adjoint of the tolerance solve.
//
// Forward: A(kappa) phi = s over the solid voxels of an island, with
//     (A phi)_i = sum_j w_ij (phi_i - phi_j),  w_ij = g_k * k_i k_j / (k_i + k_j)
// (g = 2 face, 1 edge, 1/3 corner; anchors phi = 0; air / out-of-box links
// dropped).  For a loss L(phi) with g = dL/dphi, A is symmetric, so one more
// solve A lambda = g gives
//     dL/ds_i     = lambda_i                                   (solid i)
//     dL/dkappa_i = - sum_j dw_ij/dk_i (lambda_i - lambda_j)(phi_i - phi_j)
//     dw_ij/dk_i  = g_k * k_j^2 / (k_i + k_j)^2
// over every non-air voxel i (anchors included: their kappa enters the links
// to their solid neighbours), with lambda = phi = 0 off the solid voxels.
// The edge-product kernel below evaluates both in FP64 from the FP64 forward
// solution and the FP64 adjoint accumulator.
#include <algorithm>

#include "common.cuh"
#include "kappa.h"

#include "kappa_ops.cuh"

namespace pfsf_b200 {
namespace kappa {
namespace {

// adjoint right-hand side: b = g on solid voxels (0 elsewhere), lambda0 = 0
__global__ void k_adj_prepare(const uint8_t* __restrict__ type, float* __restrict__ b, double* __restrict__ x64,
                              int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (type[i] != kSolid) b[i] = 0.0f;
    x64[i] = 0.0;
}

// island of arena voxel g: the last descriptor whose offset is <= g
__device__ __forceinline__ int island_of(const KDesc* __restrict__ desc, int nisl, int64_t g) {
    int lo = 0, hi = nisl - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (desc[mid].off <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_edge_product(const __grid_constant__ KArena A, const double* __restrict__ phi,
                                                      int64_t nfine, float* __restrict__ gk, float* __restrict__ gs) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < nfine; g += stride) {
        const KDesc& D = A.desc[island_of(A.desc, A.nisl, g)];
        const int64_t li = g - D.off;
        if (li >= D.n || A.type[g] == kAir) {  // alignment gap or air
            gk[g] = 0.0f;
            gs[g] = 0.0f;
            continue;
        }
        const Fine F = fine_view(A, D);
        const int i = (int)li;
        const Pos p = decode((unsigned)i, (unsigned)F.lx, (unsigned)F.ly);
        const bool solid = F.type[i] == kSolid;
        const double ki = F.k32[i];
        const double li_ = solid ? F.x64[i] : 0.0;
        const double pi_ = solid ? phi[g] : 0.0;
        double acc = 0.0;
        for_nb(p, F.lx, F.ly, F.lz, [&](int, int, int, int dj, float gsc) {
            const int j = i + dj;
            const uint8_t tj = F.type[j];
            if (tj == kAir) return;
            const double kj = F.k32[j];
            const double s = ki + kj;
            if (!(s > 0.0)) return;
            const double dw = (double)gsc * (kj * kj) / (s * s);
            const double lj = tj == kSolid ? F.x64[j] : 0.0;
            const double pj = tj == kSolid ? phi[g + dj] : 0.0;
            acc += dw * (li_ - lj) * (pi_ - pj);
        });
        gk[g] = (float)(-acc);
        gs[g] = solid ? (float)li_ : 0.0f;
    }
}

}  // namespace

void launch_adjoint_prepare(cudaStream_t s, const KArena& a, int64_t n) {
    k_adj_prepare<<<(unsigned)ceil_div64(n, 256), 256, 0, s>>>(a.type, const_cast<float*>(a.b), a.x64, n);
}

void launch_edge_product(cudaStream_t s, const KArena& a, const double* phi, int64_t nfine, float* gk, float* gs,
                         int num_sms) {
    const int64_t blocks = std::min<int64_t>(ceil_div64(nfine, 256), (int64_t)num_sms * 8);
    k_edge_product<<<(unsigned)std::max<int64_t>(blocks, 1), 256, 0, s>>>(a, phi, nfine, gk, gs);
}

}  // namespace kappa
}  // namespace pfsf_b200
