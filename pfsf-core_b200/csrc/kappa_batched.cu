// Batched tolerance solve: one persistent launch solves every island.
//
// Work distribution.  Islands are ordered largest first.  Giant islands
// (PFSF_GRID_MIN_VOXELS and up) are solved first, one at a time, by a
// cooperative launch of the whole GPU (k_grid: a software grid barrier with a
// bounded wait between dependent passes).  The rest go to k_batched, launched
// with thread-block clusters of C CTAs (C = 1 disables the cluster phase).
// Phase 1: each cluster takes the next "big" island from a queue and its C
// CTAs solve it together -- cluster barriers (barrier.cluster, release/acquire
// at cluster scope) between dependent passes, inner products reduced across
// the cluster through distributed shared memory.  Phase 2: when the big queue
// is empty every CTA independently takes islands from a second queue and
// solves each with CTA barriers only; phase 3 does the same per warp for the
// smallest islands.  k_batched has no grid-wide synchronisation, so there is
// nothing to wait on across clusters, and every island carries its own
// convergence state.
//
// Each island's solve: Galerkin hierarchy build, then outer FP64 refinement
// around an inner FP32 PCG preconditioned by one V-cycle (see kappa_ops.cuh).
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>

#include "kappa_flat.cuh"

namespace cg = cooperative_groups;

namespace pfsf_b200 {
namespace kappa {
namespace {

// 512 threads, two CTAs (two islands) per SM: the passes are latency bound
// (L2 round trips between CTA barriers), so warps per SM matter more than
// registers per thread (measured: 256 x 2 with 128 registers took 1.8x longer),
// but not at any price in spills (3 CTAs per SM at 40 registers, with twice
// the spill traffic, took 11 % longer on the 4096-island solve).
#ifndef PFSF_BATCHED_MIN_BLOCKS
#define PFSF_BATCHED_MIN_BLOCKS 2
#endif
constexpr int kBatchedThreads = 512;
constexpr int kBatchedMinBlocks = PFSF_BATCHED_MIN_BLOCKS;
static_assert(kBatchedThreads == kFlatThreads, "the tile marching passes assume one CTA of kFlatThreads");

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

struct SharedScratch {
    double shd[34];
    float shf[34];
    double slotd[2][16];
    float slotf[2][16];
    int next;
};

// Team = one CTA.
struct CtaTeam {
    static constexpr bool kFlat = true;  // fine passes by tile marching (kappa_flat.cuh)
    static constexpr int kKind = 3;      // PFSF_TEAM_CTA
    SharedScratch* sh;
    FlatSmem* fs;
    __device__ int cta() const { return 0; }
    __device__ int ncta() const { return 1; }
    __device__ int ctas() const { return 1; }
    __device__ int64_t t() const { return threadIdx.x; }
    __device__ int64_t T() const { return blockDim.x; }
    __device__ bool leader() const { return threadIdx.x == 0; }
    __device__ bool leader_warp() const { return threadIdx.x < 32; }
    __device__ void sync() const { __syncthreads(); }
    __device__ double sum(double v) { return cta_sum(v, sh->shd); }
    __device__ float sum(float v) { return cta_sum(v, sh->shf); }
};

// Team = one warp (small islands): warp barriers only, shuffle reductions.
struct WarpTeam {
    static constexpr bool kFlat = false;  // fine passes by the generic per-voxel ops
    static constexpr int kKind = 4;  // PFSF_TEAM_WARP
    __device__ int ctas() const { return 0; }
    __device__ int64_t t() const { return threadIdx.x & 31; }
    __device__ int64_t T() const { return 32; }
    __device__ bool leader() const { return (threadIdx.x & 31) == 0; }
    __device__ bool leader_warp() const { return true; }
    __device__ void sync() const { __syncwarp(); }
    __device__ double sum(double v) { return __shfl_sync(0xffffffffu, warp_sum(v), 0); }
    __device__ float sum(float v) { return __shfl_sync(0xffffffffu, warp_sum(v), 0); }
};

// Team = thread-block cluster of C CTAs.  Inner products: CTA reduction, then
// each CTA's partial is written into rank 0's shared slots (double-buffered
// by call parity, so one cluster barrier per reduction suffices) and summed in
// rank order by every CTA -- identical, deterministic results everywhere.
template <int C>
struct ClusterTeam {
    static constexpr bool kFlat = true;
    static constexpr int kKind = 2;  // PFSF_TEAM_CLUSTER
    SharedScratch* sh;
    FlatSmem* fs;
    int parity = 0;
    __device__ int cta() const { return (int)cg::this_cluster().block_rank(); }
    __device__ int ncta() const { return C; }
    __device__ int ctas() const { return C; }
    __device__ int64_t t() const { return (int64_t)cg::this_cluster().block_rank() * blockDim.x + threadIdx.x; }
    __device__ int64_t T() const { return (int64_t)C * blockDim.x; }
    __device__ bool leader() const { return cg::this_cluster().block_rank() == 0 && threadIdx.x == 0; }
    __device__ bool leader_warp() const { return cg::this_cluster().block_rank() == 0 && threadIdx.x < 32; }
    __device__ void sync() const { cg::this_cluster().sync(); }
    template <class R>
    __device__ R xsum(R v, R* local, R (*slots)[16]) {
        cg::cluster_group cl = cg::this_cluster();
        const R part = cta_sum(v, local);
        if (threadIdx.x == 0) {
            R* dst = cl.map_shared_rank(&slots[parity][0], 0);
            dst[cl.block_rank()] = part;
        }
        cl.sync();
        if (threadIdx.x < 32) {
            const R* src = cl.map_shared_rank(&slots[parity][0], 0);
            R s = threadIdx.x < C ? src[threadIdx.x] : R(0);
            s = warp_sum(s);
            if (threadIdx.x == 0) local[33] = s;
        }
        __syncthreads();
        parity ^= 1;
        return local[33];
    }
    __device__ double sum(double v) { return xsum<double>(v, sh->shd, sh->slotd); }
    __device__ float sum(float v) { return xsum<float>(v, sh->shf, sh->slotf); }
};

// Team = the whole grid (giant islands, one at a time).  The kernel is
// launched cooperatively, so every CTA is resident; the barrier is a
// generation barrier on two global words with a bounded wait: a CTA that
// waits longer than kGridSpinLimit polls (about a second) sets the error
// word and stops waiting, after which every later barrier returns at once and
// the solve runs out its bounded iteration counts; the host reports the
// error.  Inner products: CTA partials in a global double-buffered slot array,
// summed in block order by every CTA (deterministic, identical everywhere).
constexpr unsigned kGridSpinLimit = 1u << 22;
constexpr int kGridMaxBlocks = 1024;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

struct GridTeam {
    static constexpr bool kFlat = true;
    static constexpr int kKind = 1;  // PFSF_TEAM_GRID
    SharedScratch* sh;
    unsigned* count;  // arrivals at the current barrier
    unsigned* gen;    // barrier generation
    int* err;         // set on a timed-out wait
    double* slots;    // [2][kGridMaxBlocks] CTA partials
    FlatSmem* fs;
    int parity = 0;
    __device__ int cta() const { return blockIdx.x; }
    __device__ int ncta() const { return gridDim.x; }
    __device__ int ctas() const { return gridDim.x; }
    __device__ int64_t t() const { return (int64_t)blockIdx.x * blockDim.x + threadIdx.x; }
    __device__ int64_t T() const { return (int64_t)gridDim.x * blockDim.x; }
    __device__ bool leader() const { return blockIdx.x == 0 && threadIdx.x == 0; }
    __device__ bool leader_warp() const { return blockIdx.x == 0 && threadIdx.x < 32; }
    __device__ void sync() const {
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned g = ld_acquire_gpu(gen);
            __threadfence();
            if (atomicAdd(count, 1u) == gridDim.x - 1) {
                atomicExch(count, 0u);
                __threadfence();
                atomicAdd(gen, 1u);
            } else {
                unsigned spins = 0;
                while (ld_acquire_gpu(gen) == g) {
                    if (*(volatile int*)err) break;
                    if (++spins > kGridSpinLimit) {
                        atomicExch(err, 1);
                        break;
                    }
                    __nanosleep(32);
                }
            }
            __threadfence();
        }
        __syncthreads();
    }
    template <class R>
    __device__ R gsum(R v, R* local) {
        const R part = cta_sum(v, local);
        double* s = slots + parity * kGridMaxBlocks;
        if (threadIdx.x == 0) s[blockIdx.x] = (double)part;
        sync();
        if (threadIdx.x < 32) {
            double a = 0.0;
            for (unsigned k = threadIdx.x; k < gridDim.x; k += 32) a += __ldcg(s + k);
            a = warp_sum(a);
            if (threadIdx.x == 0) local[33] = (R)a;
        }
        __syncthreads();
        parity ^= 1;
        return local[33];
    }
    __device__ double sum(double v) { return gsum<double>(v, sh->shd); }
    __device__ float sum(float v) { return gsum<float>(v, sh->shf); }
};

// Fine-level passes: tile marching / four-wide streaming for CTA-granular
// teams, the generic per-voxel ops for warp teams.  The FP64 outer residual
// (a few passes per solve) always takes the generic op.
template <class TeamT>
__device__ __forceinline__ void t_outer_residual(const KArena& A, const KDesc& D, TeamT& tm, double& rr, double& bb) {
    op_outer_residual(A, D, (int)tm.t(), (int)tm.T(), rr, bb);
}
template <class R, class TeamT>
__device__ __forceinline__ void t_matvec(const KArena& A, const KDesc& D, TeamT& tm, R& pq) {
    if constexpr (TeamT::kFlat) fop_matvec(A, D, *tm.fs, tm.cta(), tm.ncta(), pq);
    else op_matvec(A, D, (int)tm.t(), (int)tm.T(), pq);
}
template <class R, class TeamT>
__device__ __forceinline__ void t_update(const KArena& A, const KDesc& D, TeamT& tm, float alpha, R& rr) {
    if constexpr (TeamT::kFlat) vop_update(A, D, (int)tm.t(), (int)tm.T(), alpha, rr);
    else op_update(A, D, (int)tm.t(), (int)tm.T(), alpha, rr);
}
template <class R, class TeamT>
__device__ __forceinline__ void t_dot_rz(const KArena& A, const KDesc& D, TeamT& tm, R& rz) {
    if constexpr (TeamT::kFlat) vop_dot_rz(A, D, (int)tm.t(), (int)tm.T(), rz);
    else op_dot_rz(A, D, (int)tm.t(), (int)tm.T(), rz);
}
template <class TeamT>
__device__ __forceinline__ void t_pupdate(const KArena& A, const KDesc& D, TeamT& tm, float beta) {
    if constexpr (TeamT::kFlat) vop_pupdate(A, D, (int)tm.t(), (int)tm.T(), beta);
    else op_pupdate(A, D, (int)tm.t(), (int)tm.T(), beta);
}
template <class TeamT>
__device__ __forceinline__ void t_accumulate(const KArena& A, const KDesc& D, TeamT& tm) {
    if constexpr (TeamT::kFlat) vop_accumulate(A, D, (int)tm.t(), (int)tm.T());
    else op_accumulate(A, D, (int)tm.t(), (int)tm.T());
}
template <int P, class TeamT>
__device__ __forceinline__ void t_restrict0(const KArena& A, const KDesc& D, TeamT& tm) {
    if constexpr (TeamT::kFlat) fop_restrict0<P>(A, D, *tm.fs, tm.cta(), tm.ncta());
    else op_restrict0<P>(A, D, (int)tm.t(), (int)tm.T());
}
template <class TeamT>
__device__ __forceinline__ void t_cheb0_first(const KArena& A, const KDesc& D, TeamT& tm, float c2, float* zout) {
    if constexpr (TeamT::kFlat) vop_cheb0_first(A, D, (int)tm.t(), (int)tm.T(), c2, zout);
    else op_cheb0_first(A, D, (int)tm.t(), (int)tm.T(), c2, zout);
}
template <int P, class TeamT>
__device__ __forceinline__ void t_cheb0_dz(const KArena& A, const KDesc& D, TeamT& tm, const float* zin, float* zout,
                                           float c1, float c2) {
    if constexpr (TeamT::kFlat) fop_cheb0_dz<P>(A, D, *tm.fs, tm.cta(), tm.ncta(), zin, zout, c1, c2);
    else op_cheb0_dz<P>(A, D, (int)tm.t(), (int)tm.T(), zin, zout, c1, c2);
}
template <class TeamT>
__device__ __forceinline__ void t_copy(const KDesc& D, TeamT& tm, const float* src, float* dst) {
    if constexpr (TeamT::kFlat) vop_copy((int)tm.t(), (int)tm.T(), (int)D.n, src, dst);
    else op_copy((int)tm.t(), (int)tm.T(), (int)D.n, src, dst);
}

// One V-cycle z = M r.  Levels above A.tail_cells cells are processed by
// the whole team; from the first level at or below it the rest of the cycle
// runs on one warp of the leader CTA (warp barriers only).
template <int P, class TeamT>
__device__ void team_vcycle(const KArena& A, const KDesc& D, TeamT& tm) {
    const int t = (int)tm.t(), T = (int)tm.T();
    const int L = D.nlev;
    if (L <= 1) {
        for (int s = 0; s < A.coarse_sweeps; s++) {
            for (int c = 0; c < 8; c++) { op_smooth0<P>(A, D, t, T, c); tm.sync(); }
            for (int c = 7; c >= 0; c--) { op_smooth0<P>(A, D, t, T, c); tm.sync(); }
        }
        return;
    }
    int l0 = 1;
    while (l0 < L - 1 && D.lev[l0].n > A.tail_cells) l0++;
    for (int s = 0; s < A.nu; s++)
        for (int c = 0; c < 8; c++) { op_smooth0<P>(A, D, t, T, c); tm.sync(); }
    op_restrict0<P>(A, D, t, T);
    tm.sync();
    for (int l = 1; l < l0; l++) {
        for (int s = 0; s < A.nu; s++)
            for (int c = 0; c < 8; c++) { op_smoothc<P>(A, D, l, t, T, c); tm.sync(); }
        op_restrictc<P>(A, D, l, t, T);
        tm.sync();
    }
    if (D.lev[l0].n <= A.tail_cells) {
        if (tm.leader_warp()) warp_tail_vcycle<P>(A, D, l0, A.nu, A.coarse_sweeps, A.omega_c);
        tm.sync();
    } else {  // coarsest level still large: team sweeps
        for (int s = 0; s < A.coarse_sweeps; s++) {
            for (int c = 0; c < 8; c++) { op_smoothc<P>(A, D, L - 1, t, T, c); tm.sync(); }
            for (int c = 7; c >= 0; c--) { op_smoothc<P>(A, D, L - 1, t, T, c); tm.sync(); }
        }
    }
    for (int l = l0 - 1; l >= 1; l--) {
        op_prolongc(A, D, l, t, T, A.omega_c);
        tm.sync();
        for (int s = 0; s < A.nu; s++)
            for (int c = 7; c >= 0; c--) { op_smoothc<P>(A, D, l, t, T, c); tm.sync(); }
    }
    op_prolong0(A, D, t, T, A.omega_c);
    tm.sync();
    for (int s = 0; s < A.nu; s++)
        for (int c = 7; c >= 0; c--) { op_smooth0<P>(A, D, t, T, c); tm.sync(); }
}

// Chebyshev smoothing of degree A.cheb_k on the fine level (from z = 0 when
// `from_zero`), one pass per step: the steps ping-pong z between the z array
// and the q array (free while the preconditioner runs).  z is in the z array
// on exit; on entry it is in the z array, or in q when `in_q`.  From zero, the
// first step writes whichever array makes the last step land in z.
template <int P, class TeamT>
__device__ void team_cheb0(const KArena& A, const KDesc& D, TeamT& tm, bool from_zero, bool in_q = false) {
    float* zz = A.z + D.off;
    float* zq = A.q + D.off;
    bool cur_q = in_q;
    int j = 0;
    if (from_zero) {
        cur_q = ((A.cheb_k - 1) & 1) != 0;
        t_cheb0_first(A, D, tm, A.cheb_c2[0], cur_q ? zq : zz);
        tm.sync();
        j = 1;
    }
    for (; j < A.cheb_k; j++) {
        t_cheb0_dz<P>(A, D, tm, cur_q ? zq : zz, cur_q ? zz : zq, j == 0 ? 0.0f : A.cheb_c1[j], A.cheb_c2[j]);
        tm.sync();
        cur_q = !cur_q;
    }
    if (cur_q) {
        t_copy(D, tm, zq, zz);
        tm.sync();
    }
}
template <int P, class TeamT>
__device__ void team_chebc(const KArena& A, const KDesc& D, int l, TeamT& tm, bool from_zero, bool in_x2 = false) {
    // as team_cheb0, ping-ponging the level's x and x2 arrays; x on exit
    const int t = (int)tm.t(), T = (int)tm.T();
    float* xa = A.cx + D.lev[l].off;
    float* xb = A.cx2 + D.lev[l].off;
    const int n = (int)D.lev[l].n;
    bool cur_b = in_x2;
    int j = 0;
    if (from_zero) {
        cur_b = ((A.cheb_k - 1) & 1) != 0;
        op_chebc_first(A, D, l, t, T, A.cheb_c2[0], cur_b ? xb : xa);
        tm.sync();
        j = 1;
    }
    for (; j < A.cheb_k; j++) {
        op_chebc_dx<P>(A, D, l, t, T, cur_b ? xb : xa, cur_b ? xa : xb, j == 0 ? 0.0f : A.cheb_c1[j], A.cheb_c2[j]);
        tm.sync();
        cur_b = !cur_b;
    }
    if (cur_b) {
        op_copy(t, T, n, xb, xa);
        tm.sync();
    }
}

// The rest of the V-cycle from coarse level l0 (<= A.tail_cells cells) on
// one warp with Chebyshev smoothing: cheb_k passes per smoothing instead of
// the 16 colour passes of two Gauss-Seidel sweeps, coarse_sweeps smoothings
// on the coarsest level.
template <int P>
__device__ void warp_tail_cheb(const KArena& A, const KDesc& D, int l0) {
    WarpTeam wt;
    const int t = (int)wt.t(), T = (int)wt.T();
    const int L = D.nlev;
    const bool odd = (A.cheb_k & 1) != 0;
    for (int l = l0; l < L - 1; l++) {
        team_chebc<P>(A, D, l, wt, true);
        op_restrictc<P>(A, D, l, t, T);
        __syncwarp();
    }
    team_chebc<P>(A, D, L - 1, wt, true);
    for (int s = 1; s < A.coarse_sweeps; s++) team_chebc<P>(A, D, L - 1, wt, false);
    for (int l = L - 2; l >= l0; l--) {
        float* xa = A.cx + D.lev[l].off;
        op_prolongc_to(A, D, l, t, T, A.omega_c, xa, odd ? A.cx2 + D.lev[l].off : xa);
        __syncwarp();
        team_chebc<P>(A, D, l, wt, false, odd);
    }
}

// V-cycle with Chebyshev smoothing on every level (same structure as
// team_vcycle).  Time spent in each part (the leader's clock, between
// barriers) accumulates in the island's descriptor: the leader keeps its lap
// marks there, in global memory, so that no thread of the team carries
// timestamps in registers through the passes.
template <class TeamT>
__device__ __forceinline__ void tmark(const TeamT& tm, const KDesc& D, unsigned long long KDesc::*mark) {
    if (tm.leader()) const_cast<KDesc&>(D).*mark = globaltimer();
}
template <class TeamT>
__device__ __forceinline__ void tlap(const TeamT& tm, const KDesc& D, unsigned long long KDesc::*mark,
                                     unsigned long long KDesc::*acc) {
    if (tm.leader()) {
        KDesc& d = const_cast<KDesc&>(D);
        const unsigned long long now = globaltimer();
        d.*acc += now - d.*mark;
        d.*mark = now;
    }
}

template <int P, class TeamT>
__device__ void team_vcycle_cheb(const KArena& A, const KDesc& D, TeamT& tm) {
    const int t = (int)tm.t(), T = (int)tm.T();
    const int L = D.nlev;
    tmark(tm, D, &KDesc::t_mark);
    if (L <= 1) {
        team_cheb0<P>(A, D, tm, true);
        team_cheb0<P>(A, D, tm, false);
        tlap(tm, D, &KDesc::t_mark, &KDesc::t_vfine);
        return;
    }
    int l0 = 1;
    while (l0 < L - 1 && D.lev[l0].n > A.tail_cells) l0++;
    team_cheb0<P>(A, D, tm, true);
    t_restrict0<P>(A, D, tm);
    tm.sync();
    tlap(tm, D, &KDesc::t_mark, &KDesc::t_vfine);
    for (int l = 1; l < l0; l++) {
        team_chebc<P>(A, D, l, tm, true);
        op_restrictc<P>(A, D, l, t, T);
        tm.sync();
    }
    tlap(tm, D, &KDesc::t_mark, &KDesc::t_vcoarse);
    if (D.lev[l0].n <= A.tail_cells) {
        if (tm.leader_warp()) warp_tail_cheb<P>(A, D, l0);
        tm.sync();
    } else {
        team_chebc<P>(A, D, L - 1, tm, true);
        for (int s = 1; s < A.coarse_sweeps; s++) team_chebc<P>(A, D, L - 1, tm, false);
    }
    tlap(tm, D, &KDesc::t_mark, &KDesc::t_vtail);
    // prolongate into whichever array makes the post-smoothing end in x / z
    const bool odd = (A.cheb_k & 1) != 0;
    for (int l = l0 - 1; l >= 1; l--) {
        float* xa = A.cx + D.lev[l].off;
        op_prolongc_to(A, D, l, t, T, A.omega_c, xa, odd ? A.cx2 + D.lev[l].off : xa);
        tm.sync();
        team_chebc<P>(A, D, l, tm, false, odd);
    }
    // W-cycle: a second visit of the levels below level 1 (the reference's
    // second W leg, dispatcher_vcycle.cpp:315-340, 373-374): smooth level 1
    // from its current x, restrict its residual, the same descent, tail and
    // ascent, then prolongate into level 1 and smooth it again
    if (A.wcycle && l0 >= 2) {
        team_chebc<P>(A, D, 1, tm, false, false);
        op_restrictc<P>(A, D, 1, t, T);
        tm.sync();
        for (int l = 2; l < l0; l++) {
            team_chebc<P>(A, D, l, tm, true);
            op_restrictc<P>(A, D, l, t, T);
            tm.sync();
        }
        if (D.lev[l0].n <= A.tail_cells) {
            if (tm.leader_warp()) warp_tail_cheb<P>(A, D, l0);
            tm.sync();
        } else {
            team_chebc<P>(A, D, L - 1, tm, true);
            for (int s = 1; s < A.coarse_sweeps; s++) team_chebc<P>(A, D, L - 1, tm, false);
        }
        for (int l = l0 - 1; l >= 1; l--) {
            float* xa = A.cx + D.lev[l].off;
            op_prolongc_to(A, D, l, t, T, A.omega_c, xa, odd ? A.cx2 + D.lev[l].off : xa);
            tm.sync();
            team_chebc<P>(A, D, l, tm, false, odd);
        }
    }
    tlap(tm, D, &KDesc::t_mark, &KDesc::t_vcoarse);
    op_prolong0_to(A, D, t, T, A.omega_c, A.z + D.off, odd ? A.q + D.off : A.z + D.off);
    tm.sync();
    team_cheb0<P>(A, D, tm, false, odd);
    tlap(tm, D, &KDesc::t_mark, &KDesc::t_vfine);
}

template <int P, class TeamT>
__device__ __forceinline__ void precondition(const KArena& A, const KDesc& D, TeamT& tm) {
    if (A.smoother == 1) team_vcycle_cheb<P>(A, D, tm);
    else team_vcycle<P>(A, D, tm);
}

// The island's inputs straight from the caller's mapped host arrays into
// the arena, prepared as k_prepare prepares them (kappa_plain.cu): kappa
// clamped at 0 and 0 on air, its preconditioner rounding, the source 0 off
// solid voxels, x64 = phi0 on solid voxels (0 elsewhere, 0 everywhere with
// a cold start).  Each team reads its own island while the other teams
// solve theirs, so the host-link transfer overlaps the solve.
__device__ __forceinline__ void team_ingest(const KArena& A, const KDesc& D, const kappa::IslandIO& io, int t,
                                            int T) {
    uint8_t* type = const_cast<uint8_t*>(A.type) + D.off;
    float* k32 = const_cast<float*>(A.k32) + D.off;
    uint16_t* k16 = const_cast<uint16_t*>(A.k16) + D.off;
    float* b = const_cast<float*>(A.b) + D.off;
    double* x64 = A.x64 + D.off;
    const int64_t n = D.n;
#pragma unroll 4
    for (int64_t i = t; i < n; i += T) {
        const uint8_t ty = io.h_type[i];
        const float kin = io.h_kappa[i], src = io.h_source[i], phi0 = io.h_phi[i];
        const float k = ty == kAir ? 0.0f : fmaxf(kin, 0.0f);
        type[i] = ty;
        k32[i] = k;
        if (A.prec == 1) k16[i] = __bfloat16_as_ushort(__float2bfloat16_rn(k));
        else if (A.prec == 2) k16[i] = __half_as_ushort(__float2half_rn(k));
        b[i] = ty == kSolid ? src : 0.0f;
        x64[i] = (ty == kSolid && !A.cold) ? (double)phi0 : 0.0;
    }
}

// The island's FP32 solution into the arena's e and, for a mapped island,
// into the caller's phi array (posted writes over the host link).
__device__ __forceinline__ void team_emit(const KArena& A, const KDesc& D, const kappa::IslandIO& io, int t, int T) {
    const double* x64 = A.x64 + D.off;
    float* e = A.e + D.off;
    const int64_t n = D.n;
    for (int64_t i = t; i < n; i += T) {
        const float v = (float)x64[i];
        e[i] = v;
        if (io.h_phi_out) io.h_phi_out[i] = v;
    }
}

template <int P, class R, class TeamT>
__device__ void team_solve(const KArena& A, KDesc& D, TeamT& tm) {
    const int t = (int)tm.t(), T = (int)tm.T();
    if (tm.leader()) {
        D.t_start = globaltimer();
        D.t_precond = D.t_vfine = D.t_vcoarse = D.t_vtail = 0;
    }
    const kappa::IslandIO* io = (A.ingest || A.emit) ? &A.io[&D - A.desc] : nullptr;
    if (A.ingest && io->h_type) {
        team_ingest(A, D, *io, t, T);
        tm.sync();
    }
    if (D.nlev > 1) {
        op_build1<P>(A, D, t, T);
        tm.sync();
        for (int l = 1; l < D.nlev - 1; l++) {
            op_buildc<P>(A, D, l, t, T);
            tm.sync();
        }
    }
    if (A.smoother == 1) {
        op_dinv0<P>(A, D, t, T);
        tm.sync();
    }
    if constexpr (TeamT::kFlat) {
        // the marching passes never write non-solid voxels: q starts at zero
        vop_zero(t, T, (int)D.n, A.q + D.off);
        op_rk<P>(A, D, t, T);
        flat_lists(A, D, *tm.fs, tm);  // ends with a team barrier
    }
    if (tm.leader()) D.t_setup = globaltimer() - D.t_start;
    // time in V-cycles (the leader's clock, between barriers)
    auto timed_precondition = [&]() {
        tmark(tm, D, &KDesc::t_pmark);
        precondition<P>(A, D, tm);
        tlap(tm, D, &KDesc::t_pmark, &KDesc::t_precond);
    };
    double relres = 1.0, bn = 0.0;
    int inner_total = 0, outer = 0;
    bool conv = false;
    for (outer = 0; outer <= A.max_outer; outer++) {
        double rr = 0.0, bb = 0.0;
        t_outer_residual(A, D, tm, rr, bb);
        rr = tm.sum(rr);
        bb = tm.sum(bb);
        bn = sqrt(bb);
        relres = bb > 0.0 ? sqrt(rr / bb) : 0.0;
        if (relres <= A.tol) { conv = true; break; }
        if (outer == A.max_outer || inner_total >= A.max_inner) break;
        // inner PCG on A e = r, stopping at ||r_in|| <= eta ||r_out||
        const double eta = fmax(A.eta_min, 0.3 * A.tol / relres);
        const R stop2 = (R)(eta * eta * rr);
        timed_precondition();
        R rz = 0;
        t_dot_rz(A, D, tm, rz);
        rz = tm.sum(rz);
        t_pupdate(A, D, tm, 0.0f);
        tm.sync();
        for (int it = 0; it < A.max_inner - inner_total; it++) {
            R pq = 0;
            t_matvec(A, D, tm, pq);
            pq = tm.sum(pq);
            const float alpha = pq > (R)0 ? (float)(rz / pq) : 0.0f;
            R rri = 0;
            t_update(A, D, tm, alpha, rri);
            rri = tm.sum(rri);
            inner_total++;
            if (rri <= stop2 || !(pq > (R)0)) break;
            timed_precondition();
            R rzn = 0;
            t_dot_rz(A, D, tm, rzn);
            rzn = tm.sum(rzn);
            const float beta = rz > (R)0 ? (float)(rzn / rz) : 0.0f;
            rz = rzn;
            t_pupdate(A, D, tm, beta);
            tm.sync();
        }
        t_accumulate(A, D, tm);
        tm.sync();
    }
    if (A.emit) team_emit(A, D, *io, t, T);
    if (tm.leader()) {
        D.relres = relres;
        D.bnorm = bn;
        D.inner_iters = inner_total;
        D.outer_iters = outer;
        D.converged = conv ? 1 : 0;
        D.t_end = globaltimer();
        D.team = TeamT::kKind;
        D.team_ctas = tm.ctas();
    }
}

// Giant islands (a.order[0 .. ngiant)): the whole grid solves them one after
// another.  Barrier words and partial slots live in the arena's queue and
// scratch regions (zeroed by the host before the launch).
template <int P>
__global__ void __launch_bounds__(kBatchedThreads, kBatchedMinBlocks)
    k_grid(const __grid_constant__ KArena A, int ngiant) {
    __shared__ SharedScratch sh;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    FlatSmem& fs = *reinterpret_cast<FlatSmem*>(dyn_smem);
    GridTeam tm{&sh, reinterpret_cast<unsigned*>(A.queue + 8), reinterpret_cast<unsigned*>(A.queue + 9), A.queue + 10,
                reinterpret_cast<double*>(A.scratch), &fs};
    for (int q = 0; q < ngiant; q++) {
        KDesc& D = A.desc[A.order[q]];
        if (A.fp64_dots) team_solve<P, double>(A, D, tm);
        else team_solve<P, float>(A, D, tm);
        tm.sync();
    }
}

// Islands a.order[base ..): queue[0] hands the next nbig ones to clusters,
// queue[1] the following ones to single CTAs, queue[2] the last nsmall ones
// to single warps.
template <int P, int C>
__global__ void __launch_bounds__(kBatchedThreads, kBatchedMinBlocks)
    k_batched(const __grid_constant__ KArena A, int base, int nbig, int nsmall) {
    __shared__ SharedScratch sh;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    FlatSmem& fs = *reinterpret_cast<FlatSmem*>(dyn_smem);
    if constexpr (C > 1) {
        cg::cluster_group cl = cg::this_cluster();
        ClusterTeam<C> tm{&sh, &fs};
        for (;;) {
            if (cl.block_rank() == 0 && threadIdx.x == 0) sh.next = atomicAdd(&A.queue[0], 1);
            cl.sync();
            const int k = *cl.map_shared_rank(&sh.next, 0);
            if (k >= nbig) break;
            KDesc& D = A.desc[A.order[base + k]];
            if (A.fp64_dots) team_solve<P, double>(A, D, tm);
            else team_solve<P, float>(A, D, tm);
            cl.sync();
        }
        cl.sync();  // no CTA leaves while a peer may still read its shared memory
    }
    CtaTeam tm{&sh, &fs};
    const int nmid_end = A.nisl - nsmall;
    for (;;) {
        if (threadIdx.x == 0) sh.next = atomicAdd(&A.queue[1], 1);
        __syncthreads();
        const int q = base + nbig + sh.next;
        __syncthreads();
        if (q >= nmid_end) break;
        KDesc& D = A.desc[A.order[q]];
        if (A.fp64_dots) team_solve<P, double>(A, D, tm);
        else team_solve<P, float>(A, D, tm);
        __syncthreads();
    }
    // small islands: every warp on its own, no CTA barrier from here on
    WarpTeam wt;
    for (;;) {
        int k = 0;
        if ((threadIdx.x & 31) == 0) k = atomicAdd(&A.queue[2], 1);
        k = __shfl_sync(0xffffffffu, k, 0);
        const int q = nmid_end + k;
        if (q >= A.nisl) break;
        KDesc& D = A.desc[A.order[q]];
        if (A.fp64_dots) team_solve<P, double>(A, D, wt);
        else team_solve<P, float>(A, D, wt);
        __syncwarp();
    }
}

// Cooperative launch of k_grid: one resident grid of per_sm CTAs per SM.
template <int P>
cudaError_t launch_grid(cudaStream_t s, const KArena& a, int ngiant, int num_sms) {
    auto kern = k_grid<P>;
    int per_sm = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FlatSmem)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchedThreads, sizeof(FlatSmem)) !=
            cudaSuccess ||
        per_sm <= 0)
        return cudaErrorInvalidConfiguration;
    const int ctas = std::min(num_sms * per_sm, kGridMaxBlocks);
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(kBatchedThreads);
    cfg.dynamicSmemBytes = sizeof(FlatSmem);
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, a, ngiant);
}

// k_batched with clusters of C CTAs: as many CTAs as can be resident (at
// most max_ctas when > 0); *ctas = CTAs launched, *slots = CTAs the GPU could
// hold without clusters.
template <int P, int C>
cudaError_t launch_one(cudaStream_t s, const KArena& a, int base, int nbig, int nsmall, int num_sms, int max_ctas,
                       int* ctas_out, int* slots_out) {
    auto kern = k_batched<P, C>;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    cfg.blockDim = dim3(kBatchedThreads);
    cfg.dynamicSmemBytes = sizeof(FlatSmem);
    cfg.stream = s;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FlatSmem)) !=
        cudaSuccess)
        return cudaErrorInvalidConfiguration;
    int per_sm = kBatchedMinBlocks;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchedThreads, sizeof(FlatSmem)) !=
            cudaSuccess ||
        per_sm <= 0) {
        cudaGetLastError();
        per_sm = 1;
    }
    *slots_out = num_sms * per_sm;
    int ctas = num_sms * per_sm;
    if (C > 1) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cfg.gridDim = dim3(C);
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters <= 0) {
            cudaGetLastError();
            return cudaErrorInvalidConfiguration;
        }
        ctas = clusters * C;
    } else {
        cfg.attrs = nullptr;
        cfg.numAttrs = 0;
    }
    if (max_ctas > 0) ctas = std::min(ctas, max_ctas);
    const int rest = std::max(1, a.nisl - base);
    ctas = std::max(C, std::min(ctas, std::max(C, rest * C)));
    cfg.gridDim = dim3(ctas);
    *ctas_out = ctas;
    return cudaLaunchKernelEx(&cfg, kern, a, base, nbig, nsmall);
}

// Clusters of C CTAs cannot fill every CTA slot of a GPC (an 18-SM GPC
// holds 36 CTAs of this kernel but only 4 clusters of 8), so the slots a
// clustered launch leaves free get a second, cluster-less launch on the
// side stream: it takes CTA- and warp-sized islands from the same queues
// from the start.  Neither launch waits on the other (islands are handed
// out by atomic counters), so they need not run at the same time; the fork
// is recorded before the clustered launch, so that the side launch depends
// only on the work before both (recorded after it, the side launch would
// wait for the clustered kernel to finish and find the queues empty).
template <int P, int C>
cudaError_t launch_clustered(cudaStream_t s, const SideStream& side, const KArena& a, int base, int nbig,
                             int nsmall, int num_sms, int* ctas, int* launches) {
    const int nmid = a.nisl - base - nbig - nsmall;
    const bool fork = side.stream && nmid + nsmall > 0;
    if (fork &&
        (cudaEventRecord(side.fork, s) != cudaSuccess || cudaStreamWaitEvent(side.stream, side.fork, 0) != cudaSuccess))
        return cudaErrorLaunchFailure;
    int used = 0, slots = 0;
    cudaError_t e = launch_one<P, C>(s, a, base, nbig, nsmall, num_sms, 0, &used, &slots);
    if (e != cudaSuccess) return e;
    *ctas = used;
    *launches = 1;
    if (fork) {
        int used2 = 0, slots2 = 0;
        if (slots > used)
            e = launch_one<P, 1>(side.stream, a, base, nbig, nsmall, num_sms, slots - used, &used2, &slots2);
        if (e != cudaSuccess) return e;
        if (cudaEventRecord(side.join, side.stream) != cudaSuccess || cudaStreamWaitEvent(s, side.join, 0) != cudaSuccess)
            return cudaErrorLaunchFailure;
        *ctas += used2;
        *launches += used2 > 0 ? 1 : 0;
    }
    return cudaSuccess;
}

template <int P>
cudaError_t launch_p(cudaStream_t s, const SideStream& side, const KArena& a, int ngiant, int nbig, int nsmall,
                     int cluster, int num_sms, int* ctas, int* launches) {
    *ctas = 0;
    *launches = 0;
    if (ngiant > 0) {
        const cudaError_t e = launch_grid<P>(s, a, ngiant, num_sms);
        if (e != cudaSuccess) return e;
        *launches = 1;
        if (ngiant >= a.nisl) return cudaSuccess;
    }
    int c = 0, l = 0;
    cudaError_t e = cudaErrorInvalidConfiguration;
    if (nbig > 0 && cluster >= 8) e = launch_clustered<P, 8>(s, side, a, ngiant, nbig, nsmall, num_sms, &c, &l);
    if (e != cudaSuccess && nbig > 0 && cluster >= 4) {
        cudaGetLastError();
        e = launch_clustered<P, 4>(s, side, a, ngiant, nbig, nsmall, num_sms, &c, &l);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        int slots = 0;
        l = 1;
        e = launch_one<P, 1>(s, a, ngiant, 0, nsmall, num_sms, 0, &c, &slots);
    }
    *ctas = c;
    *launches += l;
    return e;
}

// One fine-level pass of the whole-GPU tier, `reps` times in a row with a
// grid barrier between repetitions, on island a.order-independent index isl
// of the last solve (its solid lists and inverse diagonal are still in the
// arena): pass 0 = one Chebyshev step (zin = z, zout = q), pass 1 = the FP32
// matvec q = A p.  For measuring a pass alone; the arrays it writes (q, d)
// are scratch between solves.
template <int P>
__global__ void __launch_bounds__(kBatchedThreads, kBatchedMinBlocks)
    k_pass(const __grid_constant__ KArena A, int isl, int pass, int reps) {
    __shared__ SharedScratch sh;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    FlatSmem& fs = *reinterpret_cast<FlatSmem*>(dyn_smem);
    GridTeam tm{&sh, reinterpret_cast<unsigned*>(A.queue + 8), reinterpret_cast<unsigned*>(A.queue + 9), A.queue + 10,
                reinterpret_cast<double*>(A.scratch), &fs};
    const KDesc& D = A.desc[isl];
    for (int r = 0; r < reps; r++) {
        if (pass == 0) {
            fop_cheb0_dz<P>(A, D, fs, tm.cta(), tm.ncta(), A.z + D.off, A.q + D.off, A.cheb_c1[1], A.cheb_c2[1]);
        } else {
            float pq = 0.0f;
            fop_matvec(A, D, fs, tm.cta(), tm.ncta(), pq);
        }
        tm.sync();
    }
}

template <int P>
cudaError_t launch_pass_p(cudaStream_t s, const KArena& a, int isl, int pass, int reps, int num_sms) {
    auto kern = k_pass<P>;
    int per_sm = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FlatSmem)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBatchedThreads, sizeof(FlatSmem)) !=
            cudaSuccess ||
        per_sm <= 0)
        return cudaErrorInvalidConfiguration;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3(std::min(num_sms * per_sm, kGridMaxBlocks));
    cfg.blockDim = dim3(kBatchedThreads);
    cfg.dynamicSmemBytes = sizeof(FlatSmem);
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, a, isl, pass, reps);
}

}  // namespace

int launch_pass(cudaStream_t s, const KArena& a, int isl, int pass, int reps, int num_sms) {
    cudaError_t e;
    switch (a.prec) {
        case 1: e = launch_pass_p<1>(s, a, isl, pass, reps, num_sms); break;
        case 2: e = launch_pass_p<2>(s, a, isl, pass, reps, num_sms); break;
        default: e = launch_pass_p<0>(s, a, isl, pass, reps, num_sms); break;
    }
    return e == cudaSuccess ? 0 : -1;
}

int batched_threads() { return kBatchedThreads; }

// ngiant: leading islands (in a.order) solved by the whole grid; nbig: the
// next ones, solved by whole clusters; nsmall: trailing islands solved by
// single warps.
int launch_batched(cudaStream_t s, const SideStream& side, const KArena& a, int ngiant, int nbig, int nsmall,
                   int cluster, int num_sms, int* launches) {
    cudaError_t e;
    int ctas = 0;
    switch (a.prec) {
        case 1: e = launch_p<1>(s, side, a, ngiant, nbig, nsmall, cluster, num_sms, &ctas, launches); break;
        case 2: e = launch_p<2>(s, side, a, ngiant, nbig, nsmall, cluster, num_sms, &ctas, launches); break;
        default: e = launch_p<0>(s, side, a, ngiant, nbig, nsmall, cluster, num_sms, &ctas, launches); break;
    }
    if (e != cudaSuccess) {
        std::fprintf(stderr, "[libpfsf] batched solve launch failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return ctas;
}

}  // namespace kappa
}  // namespace pfsf_b200
