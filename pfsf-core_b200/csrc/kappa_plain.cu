// Tolerance solve of the symmetric per-link 26-point operator
//     sum_j w_ij (phi_i - phi_j) = s_i,   w_ij = c_k * 2 k_i k_j / (k_i + k_j)
// (c = 1 / 0.5 / 1/6 for face / edge / corner links; anchors phi = 0; air and
// out-of-box links dropped) for many islands.
//
// Numerical scheme (same for both execution modes):
//  * outer iterative refinement: the solution accumulates in FP64 and the
//    residual b - A x is evaluated with FP64 link weights and FP64 sums --
//    an FP32 phi cannot represent a solution whose FP64-evaluated relative
//    residual is 1e-6 once the island is more than ~16 voxels tall, so the
//    convergence test must see the FP64 accumulator;
//  * inner PCG on A e = r with FP32 vectors and FP32 link weights;
//  * preconditioner: one V-cycle of a geometric hierarchy (2x2x2 aggregation,
//    Galerkin coarse operators A_c = P^T A' P), symmetric 8-colour
//    Gauss-Seidel smoothing (colours 0..7 before, 7..0 after the coarse
//    correction), coarse correction weight omega_c; A' uses kappa and coarse
//    coefficients stored in BF16 / FP16 (mixed) or FP32 (plain).  Coarse
//    diagonals are rebuilt from the rounded off-diagonals plus the anchor
//    (Dirichlet) part, which keeps every coarse operator weakly diagonally
//    dominant, hence positive semi-definite, after rounding.
//
// Execution modes:
//  * batched: one persistent launch; each CTA pulls whole islands from a
//    queue (largest first) and runs the full solve for it with CTA barriers
//    between dependent passes -- no grid-wide synchronisation, per-island
//    convergence flags, FP64 (or FP32) CTA reductions;
//  * plain: one island at a time, one grid-wide kernel per operation, FP32
//    inner products, host-side convergence checks.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kappa.h"

#include "kappa_ops.cuh"

namespace pfsf_b200 {
namespace kappa {
namespace {

constexpr int kPlainBlock = 256;
constexpr int kPlainMaxBlocks = 148 * 16;

// ------------------------------------------------------------------ preparation
// k32 = kappa on non-air (0 on air), k16 = rounded copy, b = 0 off solid,
// x64 = phi0 on solid (0 elsewhere)
__global__ void k_prepare(const uint8_t* __restrict__ type, float* __restrict__ k32, uint16_t* __restrict__ k16,
                          float* __restrict__ b, double* __restrict__ x64, const float* __restrict__ phi0, int64_t n,
                          int prec) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t t = type[i];
    const float k = t == kAir ? 0.0f : fmaxf(k32[i], 0.0f);
    k32[i] = k;
    if (prec == 1) k16[i] = __bfloat16_as_ushort(__float2bfloat16_rn(k));
    else if (prec == 2) k16[i] = __half_as_ushort(__float2half_rn(k));
    if (t != kSolid) b[i] = 0.0f;
    x64[i] = t == kSolid ? (double)phi0[i] : 0.0;
}

// ------------------------------------------------------------------ plain per-island kernels (team = grid)
template <int OP, int P>
__global__ void __launch_bounds__(kPlainBlock)
    k_plain(const __grid_constant__ KArena A, int isl, int arg, float fa, float* partial) {
    const KDesc& D = A.desc[isl];
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int T = (int)(gridDim.x * blockDim.x);
    __shared__ float shf[33];
    __shared__ double shd[33];
    if constexpr (OP == 0) {  // outer residual -> partial[2*block] = rr, bb (FP64 as 2 doubles)
        double rr = 0.0, bb = 0.0;
        op_outer_residual(A, D, t, T, rr, bb);
        rr = cta_sum(rr, shd);
        bb = cta_sum(bb, shd);
        if (threadIdx.x == 0) {
            reinterpret_cast<double*>(partial)[2 * blockIdx.x] = rr;
            reinterpret_cast<double*>(partial)[2 * blockIdx.x + 1] = bb;
        }
    } else if constexpr (OP == 1) {
        float pq = 0.0f;
        op_matvec(A, D, t, T, pq);
        pq = cta_sum(pq, shf);
        if (threadIdx.x == 0) partial[blockIdx.x] = pq;
    } else if constexpr (OP == 2) {
        float rr = 0.0f;
        op_update(A, D, t, T, fa, rr);
        rr = cta_sum(rr, shf);
        if (threadIdx.x == 0) partial[blockIdx.x] = rr;
    } else if constexpr (OP == 3) {
        float rz = 0.0f;
        op_dot_rz(A, D, t, T, rz);
        rz = cta_sum(rz, shf);
        if (threadIdx.x == 0) partial[blockIdx.x] = rz;
    } else if constexpr (OP == 4) {
        op_pupdate(A, D, t, T, fa);
    } else if constexpr (OP == 5) {
        op_accumulate(A, D, t, T);
    } else if constexpr (OP == 6) {
        op_smooth0<P>(A, D, t, T, arg);
    } else if constexpr (OP == 7) {
        op_restrict0<P>(A, D, t, T);
    } else if constexpr (OP == 8) {
        op_prolong0(A, D, t, T, fa);
    } else if constexpr (OP == 9) {
        op_build1<P>(A, D, t, T);
    } else if constexpr (OP == 10) {
        op_buildc<P>(A, D, arg, t, T);
    } else if constexpr (OP == 11) {
        op_smoothc<P>(A, D, arg & 0xff, t, T, arg >> 8);
    } else if constexpr (OP == 12) {
        op_restrictc<P>(A, D, arg, t, T);
    } else if constexpr (OP == 13) {
        op_prolongc(A, D, arg, t, T, fa);
    }
}

// sum of n float partials (single block) -> out[0]; FP32 like the plain inner products
__global__ void k_sum_f(const float* __restrict__ p, int64_t n, float* __restrict__ out) {
    __shared__ float sh[33];
    float v = 0.0f;
    for (int64_t k = threadIdx.x; k < n; k += blockDim.x) v += p[k];
    v = cta_sum(v, sh);
    if (threadIdx.x == 0) out[0] = v;
}
__global__ void k_sum_d2(const double* __restrict__ p, int64_t n, double* __restrict__ out) {
    __shared__ double sh[33];
    double a = 0.0, b = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += blockDim.x) { a += p[2 * k]; b += p[2 * k + 1]; }
    a = cta_sum(a, sh);
    b = cta_sum(b, sh);
    if (threadIdx.x == 0) { out[0] = a; out[1] = b; }
}

}  // namespace

namespace {
__global__ void k_to_f32(const double* __restrict__ x, float* __restrict__ out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)x[i];
}
}  // namespace

// phi (FP32) = x64 rounded, staged in a.e for the copy back to the host
void launch_to_f32(cudaStream_t s, const KArena& a, int64_t n) {
    k_to_f32<<<(unsigned)ceil_div64(n, 256), 256, 0, s>>>(a.x64, a.e, n);
}

// Coarsen by 2 per axis until a level has at most 64 cells (or a side of 2,
// or kMaxLevels levels).
int plan_levels(int lx, int ly, int lz, KLevel* lev) {
    int nlev = 1;
    int x = lx, y = ly, z = lz;
    lev[0] = KLevel{lx, ly, lz, 0, 0, (int64_t)lx * ly * lz};
    while (nlev < kMaxLevels && std::max(x, std::max(y, z)) > 2 && (int64_t)x * y * z > 64) {
        x = (x + 1) / 2; y = (y + 1) / 2; z = (z + 1) / 2;
        lev[nlev] = KLevel{x, y, z, 0, 0, (int64_t)x * y * z};
        nlev++;
    }
    return nlev;
}

void launch_prepare(cudaStream_t s, const KArena& a, int64_t n, const int64_t*) {
    // x64 initialised from the phi0 staged in e (reinterpret): caller copies phi into a.e first
    k_prepare<<<(unsigned)ceil_div64(n, 256), 256, 0, s>>>(a.type, const_cast<float*>(a.k32),
                                                          const_cast<uint16_t*>(a.k16), const_cast<float*>(a.b),
                                                          a.x64, a.e, n, a.prec);
}

// host, which computes alpha / beta and tests convergence every iteration.
template <int P>
static int64_t solve_plain_t(cudaStream_t s, const KArena& a, int isl, const KDesc& D, KDesc* res, float* part,
                             float* scal, float* hscal) {
    int64_t launches = 0;
    const int64_t n = D.n;
    auto blocks = [&](int64_t m) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div64(m, kPlainBlock), kPlainMaxBlocks)); };
    const unsigned bf = blocks(n);
#define L(OP, nb, arg, fa) \
    do { k_plain<OP, P><<<nb, kPlainBlock, 0, s>>>(a, isl, arg, fa, part); launches++; } while (0)
    auto vcycle = [&]() {
        const int Lv = D.nlev;
        if (Lv <= 1) {
            for (int sw = 0; sw < a.coarse_sweeps; sw++) {
                for (int c = 0; c < 8; c++) L(6, blocks(n / 8 + 1), c, 0.0f);
                for (int c = 7; c >= 0; c--) L(6, blocks(n / 8 + 1), c, 0.0f);
            }
            return;
        }
        for (int sw = 0; sw < a.nu; sw++)
            for (int c = 0; c < 8; c++) L(6, blocks(n / 8 + 1), c, 0.0f);
        L(7, blocks(D.lev[1].n), 0, 0.0f);
        for (int l = 1; l < Lv - 1; l++) {
            for (int sw = 0; sw < a.nu; sw++)
                for (int c = 0; c < 8; c++) L(11, blocks(D.lev[l].n / 8 + 1), l | (c << 8), 0.0f);
            L(12, blocks(D.lev[l + 1].n), l, 0.0f);
        }
        const int lc = Lv - 1;
        for (int sw = 0; sw < a.coarse_sweeps; sw++) {
            for (int c = 0; c < 8; c++) L(11, blocks(D.lev[lc].n / 8 + 1), lc | (c << 8), 0.0f);
            for (int c = 7; c >= 0; c--) L(11, blocks(D.lev[lc].n / 8 + 1), lc | (c << 8), 0.0f);
        }
        for (int l = Lv - 2; l >= 1; l--) {
            L(13, blocks(D.lev[l].n), l, a.omega_c);
            for (int sw = 0; sw < a.nu; sw++)
                for (int c = 7; c >= 0; c--) L(11, blocks(D.lev[l].n / 8 + 1), l | (c << 8), 0.0f);
        }
        L(8, bf, 0, a.omega_c);
        for (int sw = 0; sw < a.nu; sw++)
            for (int c = 7; c >= 0; c--) L(6, blocks(n / 8 + 1), c, 0.0f);
    };
    auto reduce_f = [&](unsigned nb) -> float {
        k_sum_f<<<1, 256, 0, s>>>(part, nb, scal);
        launches++;
        cudaMemcpyAsync(hscal, scal, sizeof(float), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        return hscal[0];
    };
    if (D.nlev > 1) {
        L(9, blocks(D.lev[1].n), 0, 0.0f);
        for (int l = 1; l < D.nlev - 1; l++) L(10, blocks(D.lev[l + 1].n), l, 0.0f);
    }
    double relres = 1.0, bn = 0.0;
    int inner_total = 0, outer = 0;
    bool conv = false;
    for (outer = 0; outer <= a.max_outer; outer++) {
        L(0, bf, 0, 0.0f);
        k_sum_d2<<<1, 256, 0, s>>>(reinterpret_cast<double*>(part), bf, reinterpret_cast<double*>(scal));
        launches++;
        double hd[2];
        cudaMemcpyAsync(hd, scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        const double rr = hd[0], bb = hd[1];
        bn = sqrt(bb);
        relres = bb > 0.0 ? sqrt(rr / bb) : 0.0;
        if (relres <= a.tol) { conv = true; break; }
        if (outer == a.max_outer || inner_total >= a.max_inner) break;
        const double eta = std::max(a.eta_min, 0.3 * a.tol / relres);
        const double stop2 = eta * eta * rr;
        vcycle();
        L(3, bf, 0, 0.0f);
        float rz = reduce_f(bf);
        L(4, bf, 0, 0.0f);
        for (int it = 0; it < a.max_inner - inner_total; it++) {
            L(1, bf, 0, 0.0f);
            const float pq = reduce_f(bf);
            const float alpha = pq > 0.0f ? rz / pq : 0.0f;
            L(2, bf, 0, alpha);
            const float rri = reduce_f(bf);
            inner_total++;
            if ((double)rri <= stop2 || !(pq > 0.0f)) break;
            vcycle();
            L(3, bf, 0, 0.0f);
            const float rzn = reduce_f(bf);
            const float beta = rz > 0.0f ? rzn / rz : 0.0f;
            rz = rzn;
            L(4, bf, 0, beta);
        }
        L(5, bf, 0, 0.0f);
    }
#undef L
    *res = D;
    res->relres = relres;
    res->bnorm = bn;
    res->inner_iters = inner_total;
    res->outer_iters = outer;
    res->converged = conv ? 1 : 0;
    cudaMemcpyAsync(a.desc + isl, res, sizeof(KDesc), cudaMemcpyHostToDevice, s);
    return launches;
}

int64_t solve_plain(cudaStream_t s, const KArena& a, int isl, const KDesc& hdesc, KDesc* hres) {
    // a.scratch: 2 doubles per block (<= kPlainMaxBlocks blocks) of partials, then 64 floats of scalars
    float* part = a.scratch;
    float* scal = a.scratch + 4 * kPlainMaxBlocks;
    switch (a.prec) {
        case 1: return solve_plain_t<1>(s, a, isl, hdesc, hres, part, scal, a.hscratch);
        case 2: return solve_plain_t<2>(s, a, isl, hdesc, hres, part, scal, a.hscratch);
        default: return solve_plain_t<0>(s, a, isl, hdesc, hres, part, scal, a.hscratch);
    }
}

int64_t plain_scratch_floats() { return 4 * kPlainMaxBlocks + 64; }

}  // namespace kappa
}  // namespace pfsf_b200
