// Host launchers of the reference-schedule kernels (compat_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pfsf_b200 {
namespace compat {

int64_t pcg_blocks(int64_t n);
int64_t fail_compact_blocks(int64_t n);

void fail_compact(cudaStream_t s, const uint8_t* fail, int lx, int ly, int lz, int ox, int oy, int oz,
                  int32_t* counts, int32_t* offsets, int32_t* total, int32_t* tuples, int32_t cap);

void sparse_scatter(cudaStream_t s, const void* records, int count, int64_t n, float* source, float* cond,
                    uint8_t* type, float* maxphi, float* rcomp, float* rtens);

// ---------------------------------------------------------------- batched tick
// All dirty islands of a tick whose schedules are the same (an island group)
// run each step of that schedule in ONE launch: block b of a launch finds its
// island by binary search over the group's per-kind block prefix, then runs
// the per-voxel body of the reference-schedule kernel for that island.
//
// Device descriptor of one island (pointers to its device arrays, the
// device-visible mappings of the caller's pinned host arrays, and the
// per-island schedule state at the start of the tick).
struct CIsl {
    int lx, ly, lz, ox, oy, oz;
    int l1x, l1y, l1z, l2x, l2y, l2z;
    int64_t n, nmb, n1, n2;
    float *phi, *src, *sigma, *rcomp, *rtens, *maxphi, *hyd, *H, *D, *Dold;
    uint8_t *type, *fail;
    uint32_t* macro;
    float* res_macro;      // tick result: max macro residual
    int32_t* res_fail;     // tick result: failed voxels
    uint32_t* res_phimax;  // tick result: max phi (order-preserving key)
    int32_t *fcounts, *foffsets, *tuples;  // failed voxels per 256-voxel block, their offsets, tuples
    int32_t tuple_cap;
    int32_t iter0;         // chebyshev_iter at the start of the tick
    int32_t cur1, cur2;    // coarse ping-pong slots at the start of the tick
    int32_t rcur;          // PCG residual slot at the start of the tick
    int32_t pad;
    float *phi1[2], *src1, *sig1, *phi2[2], *src2, *sig2;
    uint8_t *type1, *type2;
    float *r[2], *p, *ap, *invdiag, *partial, *red;
    // aggregation correction (nullptr / 0: not part of this tick)
    int32_t* agg;
    float *aw, *adc, *aec;
    int64_t anc;           // aggregates: ceil(lx/2) ceil(ly/2) ceil(lz/2)
    // caller's host arrays as device-visible pointers (nullptr: not uploaded
    // by the batched upload; h_curing nullptr keeps hydration)
    const float *h_phi, *h_src, *h_sigma, *h_rcomp, *h_rtens, *h_maxphi, *h_curing;
    const uint8_t* h_type;
    float* h_stress;       // stress readback target (device-visible), nullptr: none
    int64_t stress_n;
    const float* phi_in;   // tolerance tick: the solved phi to take (device), nullptr: none
};

// Block-count kinds of a batched launch: grid voxels, the voxels of each of
// the 8 colours, the two coarse levels, macro blocks, aggregates.
enum BKind : int { kbN = 0, kbC0 = 1, kbN1 = 9, kbN2 = 10, kbMB = 11, kbAG = 12, kbKinds = 13 };

// One island group as the launchers see it.
struct BGroup {
    const CIsl* tab;       // device: nisl descriptors
    const int* bstart;     // device: kbKinds x (nisl + 1) block prefixes
    int nisl;
    int blocks[kbKinds];   // total blocks per kind
};

// Blocks of kind k for island I (host and device agree on these).
int64_t batch_blocks(const CIsl& I, int kind);

namespace batch {
void upload(cudaStream_t s, const BGroup& g);
void macro_fill(cudaStream_t s, const BGroup& g);
// damping of a step: the island's chebyshev_iter at the step (iter0 + sidx)
// >= warm ? dampf : 0
void rbgs_color(cudaStream_t s, const BGroup& g, int color, int sidx, int warm, float dampf);
void jacobi(cudaStream_t s, const BGroup& g, int level, int flip, int sidx, int warm, float dampf);
// level 1: fine -> L1, level 2: L1 -> L2 (flips: ping-pong counts so far)
void restrict_to(cudaStream_t s, const BGroup& g, int level, int f1, int f2);
// level 1: L1 -> fine, level 2: L2 -> L1
void prolong_from(cudaStream_t s, const BGroup& g, int level, int f1, int f2);
void downsample(cudaStream_t s, const BGroup& g, int level);
void pcg_precompute(cudaStream_t s, const BGroup& g);
// which 0: ap = A phi (no partials); 1: ap = A p with p.Ap partials
void pcg_matvec(cudaStream_t s, const BGroup& g, int which);
void pcg_update(cudaStream_t s, const BGroup& g, int is_init, int fr);
void finalize(cudaStream_t s, const BGroup& g, int slot, int rotate);
void pcg_direction(cudaStream_t s, const BGroup& g, int fr);
// aggregation correction (dispatcher_amg.cpp:83-161): the aggregates,
// weights and coarse diagonal from sigma and type (amg_builder.cpp:9-63);
// e_c = (P^T r) / D_c per aggregate from the PCG start's residual slot fr;
// phi += P e_c
void amg_build(cudaStream_t s, const BGroup& g);
void amg_coarse(cudaStream_t s, const BGroup& g, int fr);
void amg_prolong(cudaStream_t s, const BGroup& g);
void copy_damage(cudaStream_t s, const BGroup& g);
void phase_field(cudaStream_t s, const BGroup& g, float l0, float gc, float relax, int split);
void history(cudaStream_t s, const BGroup& g);
void take_phi(cudaStream_t s, const BGroup& g);
// failure codes, macro residual and phi maxima, failed-voxel block counts
void failure_scan(cudaStream_t s, const BGroup& g);
// scan of the block counts and the tuple write (after failure_scan)
void fail_compact(cudaStream_t s, const BGroup& g);
void stress_out(cudaStream_t s, const BGroup& g);
}  // namespace batch

}  // namespace compat
}  // namespace pfsf_b200
