// Host launchers of the reference-schedule kernels (compat_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pfsf_b200 {
namespace compat {

int64_t pcg_blocks(int64_t n);
int64_t fail_compact_blocks(int64_t n);

void rbgs_color(cudaStream_t s, int lx, int ly, int lz, float* phi, const float* rho, const float* sigma,
                const uint8_t* type, float* H, const uint32_t* macro, int color, float damping);
void jacobi_coarse(cudaStream_t s, int lx, int ly, int lz, float* phi_out, const float* phi_in, const float* rho,
                   const float* sigma, const uint8_t* type, float* Hfine, float damping);
void restrict_level(cudaStream_t s, int fx, int fy, int fz, const float* phi_f, const float* rho_f,
                    const float* sig_f, const uint8_t* type_f, int cx, int cy, int cz, float* phi_c, float* rho_c);
void prolong_level(cudaStream_t s, int fx, int fy, int fz, float* phi_f, int cx, int cy, int cz,
                   const float* phi_c);
void downsample(cudaStream_t s, int sx, int sy, int sz, const float* cond, const uint8_t* type, int dx, int dy,
                int dz, float* out_cond, uint8_t* out_type);
void pcg_precompute(cudaStream_t s, int lx, int ly, int lz, const float* sigma, float* invdiag);
void pcg_matvec(cudaStream_t s, int lx, int ly, int lz, const float* in, float* out, const float* sigma,
                const uint8_t* type, float* partial);
void pcg_update(cudaStream_t s, int lx, int ly, int lz, float* phi, const float* r_in, float* r_out, float* p,
                const float* ap, const float* src, const uint8_t* type, const float* sigma, const float* invdiag,
                const float* red, int is_init, int64_t rtz_limit, float* partial);
void pcg_direction(cudaStream_t s, int lx, int ly, int lz, const float* r, float* p, const uint8_t* type,
                   const float* red, const float* sigma);
void finalize(cudaStream_t s, const float* partial, int64_t count, float* red, int slot, int rotate);
void phase_field(cudaStream_t s, int lx, int ly, int lz, const float* phi, const float* H, float* D,
                 const float* Dold, const float* sigma, const uint8_t* type, uint8_t* fail, const float* hyd,
                 float l0, float gc, float relax, int split);
void history(cudaStream_t s, int lx, int ly, int lz, const float* phi, const float* sigma, const uint8_t* type,
             float* H);
void failure_scan(cudaStream_t s, int lx, int ly, int lz, const float* phi, const float* sigma, const float* rcomp,
                  const uint8_t* type, uint8_t* fail, const float* rtens, uint32_t* macro, const float* rho);
void macro_fill(cudaStream_t s, uint32_t* macro, int64_t nmb);
void macro_max(cudaStream_t s, const uint32_t* macro, int64_t nmb, float* out);
void fail_compact(cudaStream_t s, const uint8_t* fail, int lx, int ly, int lz, int ox, int oy, int oz,
                  int32_t* counts, int32_t* offsets, int32_t* total, int32_t* tuples, int32_t cap);

void sparse_scatter(cudaStream_t s, const void* records, int count, int64_t n, float* source, float* cond,
                    uint8_t* type, float* maxphi, float* rcomp, float* rtens);

}  // namespace compat
}  // namespace pfsf_b200
