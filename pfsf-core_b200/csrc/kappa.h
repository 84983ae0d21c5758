// Tolerance solve of the symmetric harmonic-mean 26-point operator.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "arena_io.h"

namespace pfsf_b200 {

// Levels of the hierarchy (fine + 4 coarse).  Measured with 8 (coarsest
// levels of <= 64 cells): the 256x256x128 island took as many PCG iterations
// and 6 % longer per tick (the extra levels run on one warp while the rest of
// the GPU waits), so the coarsest level of a giant island stays large and is
// smoothed by the whole team.
constexpr int kMaxLevels = 5;

// Fine-level stencil passes of CTA-granular teams march over plane tiles of
// tx x ty columns (kappa_flat.cuh); a tile plane with its one-voxel halo has
// at most kFlatCap cells, one CTA of kFlatThreads threads stages it in
// shared memory.  tx and ty are even unless they cover the whole island
// side, so every 2 x 2 x 2 aggregate of the next level lies in one tile.
constexpr int kFlatCap = 2048;
constexpr int kFlatThreads = 512;
constexpr int kFlatMaxTX = 126;
constexpr int kFlatZ = 16;  // planes per work item when several CTAs share an island
__host__ __device__ inline void flat_tile(int lx, int ly, int& tx, int& ty) {
    // wider islands: the fewest tiles of at most kFlatMaxTX columns, equal
    // widths rounded up to even (no sliver tile at the far edge)
    const int ntx = (lx + kFlatMaxTX - 1) / kFlatMaxTX;
    tx = ntx <= 1 ? lx : ((((lx + ntx - 1) / ntx) + 1) & ~1);
    ty = (kFlatCap / (tx + 2) - 2) & ~1;
    if (ty >= ly) ty = ly;
}
// entries of an island's per-(tile, plane) solid-list offset table
__host__ __device__ inline int64_t flat_starts(int lx, int ly, int lz) {
    int tx, ty;
    flat_tile(lx, ly, tx, ty);
    return (int64_t)((lx + tx - 1) / tx) * ((ly + ty - 1) / ty) * lz + 1;
}

struct KLevel {
    int lx, ly, lz;
    int pad;
    int64_t off;  // first cell of this level in the coarse arrays
    int64_t n;    // cells
};

// Per-island descriptor (device resident).
struct KDesc {
    int lx, ly, lz, nlev;
    int64_t off;  // first voxel in the fine arrays
    int64_t n;
    int64_t soff;  // first entry of the island's solid-list offset table
    KLevel lev[kMaxLevels];  // lev[0] unused (fine level), 1..nlev-1 coarse
    // results
    double relres;
    double bnorm;
    int inner_iters, outer_iters, converged, status;
    unsigned long long t_start, t_end;  // %globaltimer (ns) around the island's solve
    unsigned long long t_setup, t_precond;  // ns in the hierarchy build / in V-cycles (batched mode)
    unsigned long long t_vfine, t_vcoarse, t_vtail;  // V-cycle split: fine level, team coarse levels, tail
    unsigned long long t_mark, t_pmark;  // the team leader's last lap marks (timing scratch)
    int team, team_ctas;  // pfsf_island_team of the solving team and its CTAs (batched mode)
};

// Device pointers and parameters of one batched solve.
struct KArena {
    const uint8_t* type;
    const float* k32;      // sanitised kappa (0 on air), FP32
    const uint16_t* k16;   // kappa rounded to BF16 / FP16 (preconditioner)
    const float* b;        // source (0 off solid voxels)
    double* x64;           // solution accumulator
    float *r, *e, *z, *p, *q;
    float* cdiag;          // coarse diagonal (FP32)
    uint16_t* coef16;      // coarse off-diagonals, 26 per cell (16-bit)
    float* coef32;         // coarse off-diagonals, 26 per cell (FP32)
    float *cx, *cb;        // coarse solution / right-hand side
    float* cx2;            // second coarse solution array (out-of-place Chebyshev steps)
    KDesc* desc;
    const int* order;      // island processing order (largest first)
    int* queue;            // work counter
    int nisl;
    int prec;              // 0 fp32, 1 bf16, 2 fp16 (preconditioner storage)
    double tol;
    double eta_min;
    int max_inner, max_outer;
    float omega_c;
    int nu;                // pre/post smoothing sweeps
    int coarse_sweeps;     // symmetric sweeps on the coarsest level
    int fp64_dots;         // inner products in FP64 (1) or FP32 (0)
    float* scratch;        // block partials + the plain solve's control record (device)
    // Chebyshev smoother (smoother == 1): fine-level inverse diagonal and
    // update vectors, coarse update vector, per-step coefficients
    float* dinv0;
    float* d0;
    // per fine voxel: 1/kappa of the preconditioner's kappa and of the FP32
    // kappa (rcp.approx: +inf on air), written once per solve; the marching
    // passes copy them into shared memory with cp.async
    float* rkp;
    float* rk32;
    float* cd;
    int smoother;          // 0 symmetric 8-colour Gauss-Seidel, 1 Chebyshev
    int wcycle;            // 1: W-cycle (levels below level 1 visited twice), 0: V-cycle
    int cheb_k;            // polynomial degree (stencil passes per smoothing)
    int tail_cells;        // coarse levels of at most this many cells run on one warp
    float cheb_c1[4], cheb_c2[4];
    // per island: solid voxels of each (tile, plane) as packed tile columns
    // (cx | cy << 16), island-relative at desc.off, and the table of list
    // offsets per (tile, plane) at desc.soff (built by each solve)
    uint32_t* flist;
    int* fstart;
    // the caller's host arrays, device-mapped, per island (arena_io.h).
    // ingest: each team reads its island's inputs from there before the
    // solve (prepared as k_prepare does; x64 = 0 with cold); emit: each team
    // writes its FP32 solution into e and the caller's phi array after it.
    const kappa::IslandIO* io;
    int ingest, cold, emit;
};

struct KappaState {
    bool registered = false;
    void* h_phi = nullptr;
    void* h_src = nullptr;
    void* h_kappa = nullptr;
    void* h_type = nullptr;
};

namespace kappa {
// Plans levels for an island (host).
int plan_levels(int lx, int ly, int lz, KLevel* lev);
// A second stream and two events for the cluster-less launch that fills the
// CTA slots a clustered launch leaves free (stream may be null: no fill).
struct SideStream {
    cudaStream_t stream;
    cudaEvent_t fork, join;
};
// Batched solve over all islands in the arena: the first ngiant islands of
// a.order are solved one at a time by a cooperative launch of the whole GPU,
// the next nbig by thread-block clusters of `cluster` CTAs (8, 4 or 1) in
// one persistent launch, the last nsmall by single warps, the rest by single
// CTAs.  a.queue[0..15] must be zero.  Returns the CTAs of the persistent
// launch(es) (kernel launches in *launches), -1 on a launch failure; a
// timed-out grid barrier is reported later through a.queue[10] != 0.
int launch_batched(cudaStream_t s, const SideStream& side, const KArena& a, int ngiant, int nbig, int nsmall,
                   int cluster, int num_sms, int* launches);
// Prepare kernels: sanitise kappa, round to 16-bit, zero non-solid source.
void launch_prepare(cudaStream_t s, const KArena& a, int64_t nfine_total, const int64_t* dummy);
// Per-island CUDA graphs of the plain solve, kept with the arena.
struct PlainGraphs {
    std::vector<cudaGraphExec_t> exec;  // per island (nullptr: not built yet)
    std::vector<double> key;            // solve parameters the graphs were built for
    cudaStream_t aux[2] = {nullptr, nullptr};  // capture streams of the loop bodies
};
void free_plain_graphs(PlainGraphs& g);
// Per-island plain solve (one grid-wide kernel per operation, loops on the
// device): launches the island's graph, building it on first use.  Writes
// the results into desc (device).  Returns the graph launches issued, 0 if
// the graph could not be built or launched.
int64_t solve_plain(cudaStream_t s, const KArena& a, int isl, const KDesc& hdesc, PlainGraphs& cache);
int batched_threads();
// One fine-level pass of the whole-GPU tier (0: Chebyshev step, 1: FP32
// matvec) `reps` times over island isl of the last solve (its lists and
// inverse diagonal still in the arena); a.queue[8..10] must be zero.
// Returns 0, -1 on a launch failure.
int launch_pass(cudaStream_t s, const KArena& a, int isl, int pass, int reps, int num_sms);
int64_t plain_scratch_floats();
// Adjoint: b = g on solid voxels, x64 = 0 (kappa_adjoint.cu).
void launch_adjoint_prepare(cudaStream_t s, const KArena& a, int64_t nfine_total);
// dL/dkappa -> gk, dL/ds -> gs for every arena voxel, from the forward
// solution phi (FP64) and the adjoint solution in a.x64.
void launch_edge_product(cudaStream_t s, const KArena& a, const double* phi, int64_t nfine_total, float* gk,
                         float* gs, int num_sms);
}  // namespace kappa

}  // namespace pfsf_b200
