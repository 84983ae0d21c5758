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
//    inner products; the refinement and PCG loops run as while-nodes of a
//    per-island CUDA graph with the convergence decisions on the device.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "kappa.h"

#include "kappa_ops.cuh"

namespace pfsf_b200 {
namespace kappa {
namespace {

constexpr int kPlainBlock = 256;
constexpr int kPlainMaxBlocks = 148 * 16;
// bound on the loop passes of one plain solve, independent of its own
// iteration counters (outer and inner budgets end the loops long before)
constexpr int kPlainMaxPasses = 4096;

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
// Control record of one island's plain solve, in device memory: the scalars
// of the outer refinement and the inner PCG, and the flags that gate the
// kernels of the current loop pass.  The loops themselves are conditional
// while-nodes of a CUDA graph (solve_plain); the control kernels below set
// their conditions, so nothing returns to the host until the island is done.
struct PlainCtl {
    double rr, bb, relres, stop2, bn;
    float rz, rzn, pq, alpha, beta, rri;
    int outer, inner, conv;
    int active;   // the outer pass continues past its residual (not converged, budget left)
    int iactive;  // the inner pass continues past its update (PCG not stopped)
    int passes;   // loop passes so far (a bound independent of the solve's own counters)
};
static_assert(sizeof(PlainCtl) <= 64 * sizeof(float), "the control record lives in 64 floats of scratch");
// gate of a plain kernel: 0 always runs, 1 runs while ctl->active, 2 while ctl->iactive
__device__ __forceinline__ bool plain_gated(const PlainCtl* ctl, int gate) {
    return (gate == 1 && !ctl->active) || (gate == 2 && !ctl->iactive);
}
// scalar argument of a plain kernel: 0 the literal fa, 1 ctl->alpha, 2 ctl->beta
__device__ __forceinline__ float plain_scalar(const PlainCtl* ctl, int fsrc, float fa) {
    return fsrc == 1 ? ctl->alpha : (fsrc == 2 ? ctl->beta : fa);
}

template <int OP, int P>
__global__ void __launch_bounds__(kPlainBlock)
    k_plain(const __grid_constant__ KArena A, int isl, int arg, float fa, float* partial, const PlainCtl* ctl,
            int gate, int fsrc) {
    if (plain_gated(ctl, gate)) return;  // uniform over the grid
    const KDesc& D = A.desc[isl];
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int T = (int)(gridDim.x * blockDim.x);
    const float f = plain_scalar(ctl, fsrc, fa);
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
        op_update(A, D, t, T, f, rr);
        rr = cta_sum(rr, shf);
        if (threadIdx.x == 0) partial[blockIdx.x] = rr;
    } else if constexpr (OP == 3) {
        float rz = 0.0f;
        op_dot_rz(A, D, t, T, rz);
        rz = cta_sum(rz, shf);
        if (threadIdx.x == 0) partial[blockIdx.x] = rz;
    } else if constexpr (OP == 4) {
        op_pupdate(A, D, t, T, f);
    } else if constexpr (OP == 5) {
        op_accumulate(A, D, t, T);
    } else if constexpr (OP == 6) {
        op_smooth0<P>(A, D, t, T, arg);
    } else if constexpr (OP == 7) {
        op_restrict0<P>(A, D, t, T);
    } else if constexpr (OP == 8) {
        op_prolong0(A, D, t, T, f);
    } else if constexpr (OP == 9) {
        op_build1<P>(A, D, t, T);
    } else if constexpr (OP == 10) {
        op_buildc<P>(A, D, arg, t, T);
    } else if constexpr (OP == 11) {
        op_smoothc<P>(A, D, arg & 0xff, t, T, arg >> 8);
    } else if constexpr (OP == 12) {
        op_restrictc<P>(A, D, arg, t, T);
    } else if constexpr (OP == 13) {
        op_prolongc(A, D, arg, t, T, f);
    }
}

// sum of n float partials (single block) -> *out; FP32 like the plain inner products
__global__ void k_sum_f(const float* __restrict__ p, int64_t n, float* __restrict__ out, const PlainCtl* ctl,
                        int gate) {
    if (plain_gated(ctl, gate)) return;
    __shared__ float sh[33];
    float v = 0.0f;
    for (int64_t k = threadIdx.x; k < n; k += blockDim.x) v += p[k];
    v = cta_sum(v, sh);
    if (threadIdx.x == 0) *out = v;
}
__global__ void k_sum_d2(const double* __restrict__ p, int64_t n, PlainCtl* ctl) {
    __shared__ double sh[33];
    double a = 0.0, b = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += blockDim.x) { a += p[2 * k]; b += p[2 * k + 1]; }
    a = cta_sum(a, sh);
    b = cta_sum(b, sh);
    if (threadIdx.x == 0) { ctl->rr = a; ctl->bb = b; }
}

// ---- control kernels (one thread each)
__global__ void k_ctl_init(PlainCtl* ctl) {
    *ctl = PlainCtl{};
}
// After the outer residual: converged, out of budget, or one more correction
// (eta and the inner stopping threshold); sets both loop conditions.
__global__ void k_ctl_outer(PlainCtl* ctl, double tol, double eta_min, int max_outer, int max_inner,
                            cudaGraphConditionalHandle h_outer, cudaGraphConditionalHandle h_inner) {
    PlainCtl& c = *ctl;
    c.bn = sqrt(c.bb);
    c.relres = c.bb > 0.0 ? sqrt(c.rr / c.bb) : 0.0;
    c.passes++;
    bool go = true;
    if (c.relres <= tol) {
        c.conv = 1;
        go = false;
    } else if (c.outer >= max_outer || c.inner >= max_inner || c.passes > kPlainMaxPasses) {
        go = false;
    } else {
        const double eta = fmax(eta_min, 0.3 * tol / c.relres);
        c.stop2 = eta * eta * c.rr;
    }
    c.active = go ? 1 : 0;
    c.iactive = go ? 1 : 0;
    cudaGraphSetConditional(h_outer, go ? 1u : 0u);
    cudaGraphSetConditional(h_inner, go ? 1u : 0u);
}
__global__ void k_ctl_alpha(PlainCtl* ctl) {
    ctl->alpha = ctl->pq > 0.0f ? ctl->rz / ctl->pq : 0.0f;
}
// After the inner update: stop the PCG at the threshold, on breakdown, or at
// the iteration budget.
__global__ void k_ctl_inner(PlainCtl* ctl, int max_inner, cudaGraphConditionalHandle h_inner) {
    PlainCtl& c = *ctl;
    c.inner++;
    c.passes++;
    const bool stop = (double)c.rri <= c.stop2 || !(c.pq > 0.0f) || c.inner >= max_inner ||
                      c.passes > kPlainMaxPasses;
    c.iactive = stop ? 0 : 1;
    cudaGraphSetConditional(h_inner, stop ? 0u : 1u);
}
__global__ void k_ctl_beta(PlainCtl* ctl) {
    if (!ctl->iactive) return;
    ctl->beta = ctl->rz > 0.0f ? ctl->rzn / ctl->rz : 0.0f;
    ctl->rz = ctl->rzn;
}
__global__ void k_ctl_next(PlainCtl* ctl) {
    if (ctl->active) ctl->outer++;
}
// the island's result record
__global__ void k_ctl_finish(const __grid_constant__ KArena A, int isl, const PlainCtl* ctl) {
    KDesc& D = A.desc[isl];
    D.relres = ctl->relres;
    D.bnorm = ctl->bn;
    D.inner_iters = ctl->inner;
    D.outer_iters = ctl->outer;
    D.converged = ctl->conv;
    D.team = 0;
    D.team_ctas = 0;
}

}  // namespace

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

namespace {

// The per-island plain solve as a CUDA graph: the Galerkin build, then a
// while-node over the outer FP64 refinement whose body holds a while-node
// over the inner PCG iterations.  The control kernels set both loop
// conditions on the device; every other kernel of a pass is gated by the
// control record, so a pass that ends early does no work.  The graph is
// built once per island (captured on two auxiliary streams into the loop
// bodies) and replayed on every later solve with the same parameters.
template <int P>
static cudaGraphExec_t build_plain_graph(cudaStream_t s, cudaStream_t s2, cudaStream_t s3, const KArena& a, int isl,
                                         const KDesc& D, float* part, PlainCtl* ctl) {
    auto blocks = [&](int64_t m) {
        return (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div64(m, kPlainBlock), kPlainMaxBlocks));
    };
    const int64_t n = D.n;
    const unsigned bf = blocks(n);
#define L(st, OP, nb, arg, fa, gate, fsrc) \
    k_plain<OP, P><<<nb, kPlainBlock, 0, st>>>(a, isl, arg, fa, part, ctl, gate, fsrc)
    auto vcycle = [&](cudaStream_t st, int gate) {
        const int Lv = D.nlev;
        if (Lv <= 1) {
            for (int sw = 0; sw < a.coarse_sweeps; sw++) {
                for (int c = 0; c < 8; c++) L(st, 6, blocks(n / 8 + 1), c, 0.0f, gate, 0);
                for (int c = 7; c >= 0; c--) L(st, 6, blocks(n / 8 + 1), c, 0.0f, gate, 0);
            }
            return;
        }
        for (int sw = 0; sw < a.nu; sw++)
            for (int c = 0; c < 8; c++) L(st, 6, blocks(n / 8 + 1), c, 0.0f, gate, 0);
        L(st, 7, blocks(D.lev[1].n), 0, 0.0f, gate, 0);
        for (int l = 1; l < Lv - 1; l++) {
            for (int sw = 0; sw < a.nu; sw++)
                for (int c = 0; c < 8; c++) L(st, 11, blocks(D.lev[l].n / 8 + 1), l | (c << 8), 0.0f, gate, 0);
            L(st, 12, blocks(D.lev[l + 1].n), l, 0.0f, gate, 0);
        }
        const int lc = Lv - 1;
        for (int sw = 0; sw < a.coarse_sweeps; sw++) {
            for (int c = 0; c < 8; c++) L(st, 11, blocks(D.lev[lc].n / 8 + 1), lc | (c << 8), 0.0f, gate, 0);
            for (int c = 7; c >= 0; c--) L(st, 11, blocks(D.lev[lc].n / 8 + 1), lc | (c << 8), 0.0f, gate, 0);
        }
        for (int l = Lv - 2; l >= 1; l--) {
            L(st, 13, blocks(D.lev[l].n), l, a.omega_c, gate, 0);
            for (int sw = 0; sw < a.nu; sw++)
                for (int c = 7; c >= 0; c--) L(st, 11, blocks(D.lev[l].n / 8 + 1), l | (c << 8), 0.0f, gate, 0);
        }
        L(st, 8, bf, 0, a.omega_c, gate, 0);
        for (int sw = 0; sw < a.nu; sw++)
            for (int c = 7; c >= 0; c--) L(st, 6, blocks(n / 8 + 1), c, 0.0f, gate, 0);
    };
    // a while-node appended to the graph stream st is capturing into; returns
    // its body graph (or nullptr)
    auto add_while = [&](cudaStream_t st, cudaGraphConditionalHandle h) -> cudaGraph_t {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd) != cudaSuccess ||
            cs != cudaStreamCaptureStatusActive)
            return nullptr;
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, g, deps, nd, &np) != cudaSuccess) return nullptr;
        if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
            return nullptr;
        return np.conditional.phGraph_out[0];
    };
    auto capture_graph = [](cudaStream_t st, cudaGraph_t g) {
        return st && g && cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
                              cudaSuccess;
    };
    cudaGraph_t top = nullptr;
    if (cudaGraphCreate(&top, 0) != cudaSuccess) return nullptr;
    bool ok = capture_graph(s, top);
    if (ok) {
        if (D.nlev > 1) {
            L(s, 9, blocks(D.lev[1].n), 0, 0.0f, 0, 0);
            for (int l = 1; l < D.nlev - 1; l++) L(s, 10, blocks(D.lev[l + 1].n), l, 0.0f, 0, 0);
        }
        k_ctl_init<<<1, 1, 0, s>>>(ctl);
        cudaGraphConditionalHandle h_outer = 0, h_inner = 0;
        ok = cudaGraphConditionalHandleCreate(&h_outer, top, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraph_t body_o = ok ? add_while(s, h_outer) : nullptr;
        ok = ok && body_o && cudaGraphConditionalHandleCreate(&h_inner, body_o, 0, 0) == cudaSuccess;
        ok = ok && capture_graph(s2, body_o);
        if (ok) {
            // outer pass: FP64 residual, decision, the first V-cycle and direction
            L(s2, 0, bf, 0, 0.0f, 0, 0);
            k_sum_d2<<<1, 256, 0, s2>>>(reinterpret_cast<double*>(part), bf, ctl);
            k_ctl_outer<<<1, 1, 0, s2>>>(ctl, a.tol, a.eta_min, a.max_outer, a.max_inner, h_outer, h_inner);
            vcycle(s2, 1);
            L(s2, 3, bf, 0, 0.0f, 1, 0);
            k_sum_f<<<1, 256, 0, s2>>>(part, bf, &ctl->rz, ctl, 1);
            L(s2, 4, bf, 0, 0.0f, 1, 0);
            cudaGraph_t body_i = add_while(s2, h_inner);
            ok = body_i && capture_graph(s3, body_i);
            if (ok) {
                // inner pass: matvec, alpha, update, stop test, V-cycle, beta, direction
                L(s3, 1, bf, 0, 0.0f, 0, 0);
                k_sum_f<<<1, 256, 0, s3>>>(part, bf, &ctl->pq, ctl, 0);
                k_ctl_alpha<<<1, 1, 0, s3>>>(ctl);
                L(s3, 2, bf, 0, 0.0f, 0, 1);
                k_sum_f<<<1, 256, 0, s3>>>(part, bf, &ctl->rri, ctl, 0);
                k_ctl_inner<<<1, 1, 0, s3>>>(ctl, a.max_inner, h_inner);
                vcycle(s3, 2);
                L(s3, 3, bf, 0, 0.0f, 2, 0);
                k_sum_f<<<1, 256, 0, s3>>>(part, bf, &ctl->rzn, ctl, 2);
                k_ctl_beta<<<1, 1, 0, s3>>>(ctl);
                L(s3, 4, bf, 0, 0.0f, 2, 2);
                cudaGraph_t g3 = nullptr;
                ok = cudaStreamEndCapture(s3, &g3) == cudaSuccess;
            }
            L(s2, 5, bf, 0, 0.0f, 1, 0);
            k_ctl_next<<<1, 1, 0, s2>>>(ctl);
            cudaGraph_t g2 = nullptr;
            ok = (cudaStreamEndCapture(s2, &g2) == cudaSuccess) && ok;
        }
        k_ctl_finish<<<1, 1, 0, s>>>(a, isl, ctl);
        cudaGraph_t g1 = nullptr;
        ok = (cudaStreamEndCapture(s, &g1) == cudaSuccess) && ok;
    }
#undef L
    cudaGraphExec_t exec = nullptr;
    if (ok && cudaGraphInstantiate(&exec, top, 0) != cudaSuccess) exec = nullptr;
    cudaGraphDestroy(top);
    if (!exec) {
        std::fprintf(stderr, "[libpfsf] plain solve graph for island %d could not be built: %s\n", isl,
                     cudaGetErrorString(cudaGetLastError()));
    }
    return exec;
}

}  // namespace

void free_plain_graphs(PlainGraphs& g) {
    for (cudaGraphExec_t e : g.exec)
        if (e) cudaGraphExecDestroy(e);
    g.exec.clear();
    g.key.clear();
    for (cudaStream_t& st : g.aux) {
        if (st) cudaStreamDestroy(st);
        st = nullptr;
    }
}

// One island's plain solve: its graph (built on first use for the current
// parameters) launched on s.  Returns the graph launches issued (0 when the
// graph cannot be built: the island's record then says not converged).
int64_t solve_plain(cudaStream_t s, const KArena& a, int isl, const KDesc& hdesc, PlainGraphs& cache) {
    const std::vector<double> key = {a.tol, a.eta_min, (double)a.max_inner, (double)a.max_outer, (double)a.omega_c,
                                     (double)a.nu, (double)a.coarse_sweeps, (double)a.prec, (double)a.nisl};
    if (cache.key != key) {
        cudaStreamSynchronize(s);
        for (cudaGraphExec_t e : cache.exec)
            if (e) cudaGraphExecDestroy(e);
        cache.exec.assign(a.nisl, nullptr);
        cache.key = key;
    }
    for (cudaStream_t& st : cache.aux)
        if (!st && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
    // a.scratch: 2 doubles per block (<= kPlainMaxBlocks blocks) of partials, then the control record
    float* part = a.scratch;
    PlainCtl* ctl = reinterpret_cast<PlainCtl*>(a.scratch + 4 * kPlainMaxBlocks);
    cudaGraphExec_t& exec = cache.exec[isl];
    if (!exec) {
        switch (a.prec) {
            case 1: exec = build_plain_graph<1>(s, cache.aux[0], cache.aux[1], a, isl, hdesc, part, ctl); break;
            case 2: exec = build_plain_graph<2>(s, cache.aux[0], cache.aux[1], a, isl, hdesc, part, ctl); break;
            default: exec = build_plain_graph<0>(s, cache.aux[0], cache.aux[1], a, isl, hdesc, part, ctl); break;
        }
        if (!exec) return 0;
    }
    if (cudaGraphLaunch(exec, s) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return 1;
}

int64_t plain_scratch_floats() { return 4 * kPlainMaxBlocks + 64; }


}  // namespace kappa
}  // namespace pfsf_b200
