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

namespace pfsf_b200 {
namespace kappa {
namespace {

constexpr int kBatchedThreads = 512;
constexpr int kPlainBlock = 256;
constexpr int kPlainMaxBlocks = 148 * 16;

// ------------------------------------------------------------------ helpers
template <int P>
__device__ __forceinline__ float kload(const KArena& A, int64_t g) {
    if constexpr (P == 0) return A.k32[g];
    else if constexpr (P == 1) return __bfloat162float(__ushort_as_bfloat16(A.k16[g]));
    else return __half2float(__ushort_as_half(A.k16[g]));
}
template <int P>
__device__ __forceinline__ float cload(const KArena& A, int64_t idx) {
    if constexpr (P == 0) return A.coef32[idx];
    else if constexpr (P == 1) return __bfloat162float(__ushort_as_bfloat16(A.coef16[idx]));
    else return __half2float(__ushort_as_half(A.coef16[idx]));
}
template <int P>
__device__ __forceinline__ float cround(float v) {  // value as stored
    if constexpr (P == 0) return v;
    else if constexpr (P == 1) return __bfloat162float(__float2bfloat16_rn(v));
    else return __half2float(__float2half_rn(v));
}
template <int P>
__device__ __forceinline__ void cstore(const KArena& A, int64_t idx, float v) {
    if constexpr (P == 0) A.coef32[idx] = v;
    else if constexpr (P == 1) A.coef16[idx] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
    else A.coef16[idx] = __half_as_ushort(__float2half_rn(v));
}

// k * k' / (k + k'), 0 when both are 0 (air)
__device__ __forceinline__ float hm(float a, float b) {
    const float s = a + b;
    return s > 0.0f ? __fdividef(a * b, s) : 0.0f;
}
__device__ __forceinline__ double hm64(double a, double b) {
    const double s = a + b;
    return s > 0.0 ? (a * b) / s : 0.0;
}
// group scale of 2ab/(a+b) * c_k: face 2, edge 1, corner 1/3
__host__ __device__ constexpr float gscale(int dx, int dy, int dz) {
    return (dx != 0) + (dy != 0) + (dz != 0) == 1 ? 2.0f : ((dx != 0) + (dy != 0) + (dz != 0) == 2 ? 1.0f : 1.0f / 3.0f);
}
// 26-neighbour index k of offset (dx,dy,dz) in {-1,0,1}^3 \ 0 (lexicographic, centre skipped)
__host__ __device__ constexpr int nbk(int dx, int dy, int dz) {
    const int q = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
    return q < 13 ? q : q - 1;
}
__device__ __forceinline__ void nboff(int k, int& dx, int& dy, int& dz) {
    const int q = k < 13 ? k : k + 1;
    dx = q % 3 - 1;
    dy = (q / 3) % 3 - 1;
    dz = q / 9 - 1;
}

struct Pos {
    int x, y, z;
};
__device__ __forceinline__ Pos decode(int64_t i, int lx, int ly) {
    Pos p;
    p.x = (int)(i % lx);
    const int64_t r = i / lx;
    p.y = (int)(r % ly);
    p.z = (int)(r / ly);
    return p;
}

// Visit the in-box 26 neighbours: f(dx, dy, dz, delta_index, group_scale)
template <class F>
__device__ __forceinline__ void for_nb(const Pos& p, int lx, int ly, int lz, F f) {
    const int64_t sy = lx, sz = (int64_t)lx * ly;
#pragma unroll
    for (int dz = -1; dz <= 1; dz++) {
        if ((dz < 0 && p.z == 0) || (dz > 0 && p.z + 1 >= lz)) continue;
#pragma unroll
        for (int dy = -1; dy <= 1; dy++) {
            if ((dy < 0 && p.y == 0) || (dy > 0 && p.y + 1 >= ly)) continue;
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                if ((dx < 0 && p.x == 0) || (dx > 0 && p.x + 1 >= lx)) continue;
                f(dx, dy, dz, dx + dy * sy + dz * sz, gscale(dx, dy, dz));
            }
        }
    }
}

// ------------------------------------------------------------------ reductions
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
// CTA-wide sum; every thread receives the result.
template <class T>
__device__ T cta_sum(T v, T* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        T s = lane < nw ? sh[lane] : T(0);
        s = warp_sum(s);
        if (lane == 0) sh[32] = s;
    }
    __syncthreads();
    return sh[32];
}

// ------------------------------------------------------------------ fine-level ops
// All ops take (t, T): this thread's index and the team size.

// r = b - A x (FP64 weights and sums), e = z = 0; returns (r.r, b.b) partials.
__device__ void op_outer_residual(const KArena& A, const KDesc& D, int64_t t, int64_t T, double& rr, double& bb) {
    const int lx = D.lx, ly = D.ly, lz = D.lz;
    for (int64_t i = t; i < D.n; i += T) {
        const int64_t g = D.off + i;
        if (A.type[g] != kSolid) {
            A.r[g] = 0.0f; A.e[g] = 0.0f; A.z[g] = 0.0f;
            continue;
        }
        const Pos p = decode(i, lx, ly);
        const double ki = A.k32[g], xi = A.x64[g];
        double acc = 0.0;
        for_nb(p, lx, ly, lz, [&](int, int, int, int64_t dj, float gs) {
            const double kj = A.k32[g + dj];
            const double w = (double)gs * hm64(ki, kj);
            acc += w * (xi - A.x64[g + dj]);
        });
        const double bi = A.b[g];
        const double ri = bi - acc;
        A.r[g] = (float)ri;
        A.e[g] = 0.0f;
        A.z[g] = 0.0f;
        rr += ri * ri;
        bb += bi * bi;
    }
}

// q = A p (FP32 weights); returns p.q partial
template <class R>
__device__ void op_matvec(const KArena& A, const KDesc& D, int64_t t, int64_t T, R& pq) {
    const int lx = D.lx, ly = D.ly, lz = D.lz;
    for (int64_t i = t; i < D.n; i += T) {
        const int64_t g = D.off + i;
        if (A.type[g] != kSolid) { A.q[g] = 0.0f; continue; }
        const Pos p = decode(i, lx, ly);
        const float ki = A.k32[g], pi = A.p[g];
        float acc = 0.0f;
        for_nb(p, lx, ly, lz, [&](int, int, int, int64_t dj, float gs) {
            acc += gs * hm(ki, A.k32[g + dj]) * (pi - A.p[g + dj]);
        });
        A.q[g] = acc;
        pq += (R)pi * (R)acc;
    }
}

// e += alpha p, r -= alpha q; returns r.r partial
template <class R>
__device__ void op_update(const KArena& A, const KDesc& D, int64_t t, int64_t T, float alpha, R& rr) {
    for (int64_t i = t; i < D.n; i += T) {
        const int64_t g = D.off + i;
        const float ri = A.r[g] - alpha * A.q[g];
        A.e[g] += alpha * A.p[g];
        A.r[g] = ri;
        rr += (R)ri * (R)ri;
    }
}

template <class R>
__device__ void op_dot_rz(const KArena& A, const KDesc& D, int64_t t, int64_t T, R& rz) {
    for (int64_t i = t; i < D.n; i += T) {
        const int64_t g = D.off + i;
        rz += (R)A.r[g] * (R)A.z[g];
    }
}

// p = z + beta p; z = 0 (ready for the next V-cycle)
__device__ void op_pupdate(const KArena& A, const KDesc& D, int64_t t, int64_t T, float beta) {
    for (int64_t i = t; i < D.n; i += T) {
        const int64_t g = D.off + i;
        const float zi = A.z[g];
        A.p[g] = beta == 0.0f ? zi : zi + beta * A.p[g];
        A.z[g] = 0.0f;
    }
}

// x64 += e
__device__ void op_accumulate(const KArena& A, const KDesc& D, int64_t t, int64_t T) {
    for (int64_t i = t; i < D.n; i += T) {
        const int64_t g = D.off + i;
        A.x64[g] += (double)A.e[g];
    }
}

// ---- level-0 Gauss-Seidel colour pass on A' z = r (kappa storage P)
template <int P>
__device__ void op_smooth0(const KArena& A, const KDesc& D, int64_t t, int64_t T, int color) {
    const int lx = D.lx, ly = D.ly, lz = D.lz;
    const int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    const int ncx = (lx - cx + 1) >> 1, ncy = (ly - cy + 1) >> 1, ncz = (lz - cz + 1) >> 1;
    const int64_t nc = (int64_t)ncx * ncy * ncz;
    for (int64_t v = t; v < nc; v += T) {
        const int xi = (int)(v % ncx);
        const int64_t rem = v / ncx;
        Pos p;
        p.x = 2 * xi + cx;
        p.y = 2 * (int)(rem % ncy) + cy;
        p.z = 2 * (int)(rem / ncy) + cz;
        const int64_t g = D.off + p.x + (int64_t)lx * (p.y + (int64_t)ly * p.z);
        if (A.type[g] != kSolid) continue;
        const float ki = kload<P>(A, g);
        float d = 0.0f, s = 0.0f;
        for_nb(p, lx, ly, lz, [&](int, int, int, int64_t dj, float gs) {
            const float w = gs * hm(ki, kload<P>(A, g + dj));
            d += w;
            s += w * A.z[g + dj];
        });
        A.z[g] = d > 0.0f ? (A.r[g] + s) / d : 0.0f;
    }
}

// residual of level 0 (operator A') restricted to level 1 by aggregation; x1 = 0
template <int P>
__device__ void op_restrict0(const KArena& A, const KDesc& D, int64_t t, int64_t T) {
    const KLevel& C = D.lev[1];
    const int lx = D.lx, ly = D.ly, lz = D.lz;
    for (int64_t c = t; c < C.n; c += T) {
        const Pos pc = decode(c, C.lx, C.ly);
        float sum = 0.0f;
        for (int a = 0; a < 8; a++) {
            Pos p;
            p.x = 2 * pc.x + (a & 1);
            p.y = 2 * pc.y + ((a >> 1) & 1);
            p.z = 2 * pc.z + ((a >> 2) & 1);
            if (p.x >= lx || p.y >= ly || p.z >= lz) continue;
            const int64_t g = D.off + p.x + (int64_t)lx * (p.y + (int64_t)ly * p.z);
            if (A.type[g] != kSolid) continue;
            const float ki = kload<P>(A, g), zi = A.z[g];
            float az = 0.0f;
            for_nb(p, lx, ly, lz, [&](int, int, int, int64_t dj, float gs) {
                az += gs * hm(ki, kload<P>(A, g + dj)) * (zi - A.z[g + dj]);
            });
            sum += A.r[g] - az;
        }
        A.cb[C.off + c] = sum;
        A.cx[C.off + c] = 0.0f;
    }
}

// z_i += omega * x1[cell(i)] on solid voxels
__device__ void op_prolong0(const KArena& A, const KDesc& D, int64_t t, int64_t T, float omega) {
    const KLevel& C = D.lev[1];
    for (int64_t i = t; i < D.n; i += T) {
        const int64_t g = D.off + i;
        if (A.type[g] != kSolid) continue;
        const Pos p = decode(i, D.lx, D.ly);
        const int64_t c = (p.x >> 1) + (int64_t)C.lx * ((p.y >> 1) + (int64_t)C.ly * (p.z >> 1));
        A.z[g] += omega * A.cx[C.off + c];
    }
}

// ---- Galerkin level 1 from the fine operator A' (kappa storage P).
template <int P>
__device__ void op_build1(const KArena& A, const KDesc& D, int64_t t, int64_t T) {
    const KLevel& C = D.lev[1];
    const int lx = D.lx, ly = D.ly, lz = D.lz;
    for (int64_t c = t; c < C.n; c += T) {
        const Pos pc = decode(c, C.lx, C.ly);
        float W[26];
#pragma unroll
        for (int k = 0; k < 26; k++) W[k] = 0.0f;
        float anchor = 0.0f;
        for (int a = 0; a < 8; a++) {
            Pos p;
            p.x = 2 * pc.x + (a & 1);
            p.y = 2 * pc.y + ((a >> 1) & 1);
            p.z = 2 * pc.z + ((a >> 2) & 1);
            if (p.x >= lx || p.y >= ly || p.z >= lz) continue;
            const int64_t g = D.off + p.x + (int64_t)lx * (p.y + (int64_t)ly * p.z);
            if (A.type[g] != kSolid) continue;
            const float ki = kload<P>(A, g);
            for_nb(p, lx, ly, lz, [&](int dx, int dy, int dz, int64_t dj, float gs) {
                const uint8_t tj = A.type[g + dj];
                if (tj == kAir) return;
                const float w = gs * hm(ki, kload<P>(A, g + dj));
                if (tj == kAnchor) { anchor += w; return; }
                const int ddx = ((p.x + dx) >> 1) - pc.x, ddy = ((p.y + dy) >> 1) - pc.y, ddz = ((p.z + dz) >> 1) - pc.z;
                if (ddx == 0 && ddy == 0 && ddz == 0) return;
                W[nbk(ddx, ddy, ddz)] += w;
            });
        }
        float diag = anchor;
#pragma unroll
        for (int k = 0; k < 26; k++) {
            cstore<P>(A, 26 * C.off + (int64_t)k * C.n + c, W[k]);
            diag += cround<P>(W[k]);
        }
        A.cdiag[C.off + c] = diag;
    }
}

// Galerkin level l+1 from the explicit coefficients of level l.
template <int P>
__device__ void op_buildc(const KArena& A, const KDesc& D, int l, int64_t t, int64_t T) {
    const KLevel& F = D.lev[l];
    const KLevel& C = D.lev[l + 1];
    for (int64_t c = t; c < C.n; c += T) {
        const Pos pc = decode(c, C.lx, C.ly);
        float W[26];
#pragma unroll
        for (int k = 0; k < 26; k++) W[k] = 0.0f;
        float anchor = 0.0f;
        for (int a = 0; a < 8; a++) {
            const int fx = 2 * pc.x + (a & 1), fy = 2 * pc.y + ((a >> 1) & 1), fz = 2 * pc.z + ((a >> 2) & 1);
            if (fx >= F.lx || fy >= F.ly || fz >= F.lz) continue;
            const int64_t f = fx + (int64_t)F.lx * (fy + (int64_t)F.ly * fz);
            const float dg = A.cdiag[F.off + f];
            if (!(dg > 0.0f)) continue;
            float off = 0.0f;
            for (int k = 0; k < 26; k++) {
                const float w = cload<P>(A, 26 * F.off + (int64_t)k * F.n + f);
                if (w == 0.0f) continue;
                off += w;
                int dx, dy, dz;
                nboff(k, dx, dy, dz);
                const int ddx = ((fx + dx) >> 1) - pc.x, ddy = ((fy + dy) >> 1) - pc.y, ddz = ((fz + dz) >> 1) - pc.z;
                if (ddx == 0 && ddy == 0 && ddz == 0) continue;
                W[nbk(ddx, ddy, ddz)] += w;
            }
            anchor += fmaxf(dg - off, 0.0f);
        }
        float diag = anchor;
#pragma unroll
        for (int k = 0; k < 26; k++) {
            cstore<P>(A, 26 * C.off + (int64_t)k * C.n + c, W[k]);
            diag += cround<P>(W[k]);
        }
        A.cdiag[C.off + c] = diag;
    }
}

// Gauss-Seidel colour pass on coarse level l
template <int P>
__device__ void op_smoothc(const KArena& A, const KDesc& D, int l, int64_t t, int64_t T, int color) {
    const KLevel& L = D.lev[l];
    const int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    const int ncx = (L.lx - cx + 1) >> 1, ncy = (L.ly - cy + 1) >> 1, ncz = (L.lz - cz + 1) >> 1;
    const int64_t nc = (int64_t)ncx * ncy * ncz;
    for (int64_t v = t; v < nc; v += T) {
        const int xi = (int)(v % ncx);
        const int64_t rem = v / ncx;
        Pos p;
        p.x = 2 * xi + cx;
        p.y = 2 * (int)(rem % ncy) + cy;
        p.z = 2 * (int)(rem / ncy) + cz;
        const int64_t c = p.x + (int64_t)L.lx * (p.y + (int64_t)L.ly * p.z);
        const float dg = A.cdiag[L.off + c];
        if (!(dg > 0.0f)) continue;
        float s = 0.0f;
        for_nb(p, L.lx, L.ly, L.lz, [&](int dx, int dy, int dz, int64_t dj, float) {
            s += cload<P>(A, 26 * L.off + (int64_t)nbk(dx, dy, dz) * L.n + c) * A.cx[L.off + c + dj];
        });
        A.cx[L.off + c] = (A.cb[L.off + c] + s) / dg;
    }
}

// residual of level l restricted to level l+1; x_{l+1} = 0
template <int P>
__device__ void op_restrictc(const KArena& A, const KDesc& D, int l, int64_t t, int64_t T) {
    const KLevel& F = D.lev[l];
    const KLevel& C = D.lev[l + 1];
    for (int64_t c = t; c < C.n; c += T) {
        const Pos pc = decode(c, C.lx, C.ly);
        float sum = 0.0f;
        for (int a = 0; a < 8; a++) {
            Pos p;
            p.x = 2 * pc.x + (a & 1);
            p.y = 2 * pc.y + ((a >> 1) & 1);
            p.z = 2 * pc.z + ((a >> 2) & 1);
            if (p.x >= F.lx || p.y >= F.ly || p.z >= F.lz) continue;
            const int64_t f = p.x + (int64_t)F.lx * (p.y + (int64_t)F.ly * p.z);
            const float dg = A.cdiag[F.off + f];
            if (!(dg > 0.0f)) continue;
            float s = 0.0f;
            for_nb(p, F.lx, F.ly, F.lz, [&](int dx, int dy, int dz, int64_t dj, float) {
                s += cload<P>(A, 26 * F.off + (int64_t)nbk(dx, dy, dz) * F.n + f) * A.cx[F.off + f + dj];
            });
            sum += A.cb[F.off + f] - (dg * A.cx[F.off + f] - s);
        }
        A.cb[C.off + c] = sum;
        A.cx[C.off + c] = 0.0f;
    }
}

// x_l += omega * x_{l+1}[parent] on active cells
__device__ void op_prolongc(const KArena& A, const KDesc& D, int l, int64_t t, int64_t T, float omega) {
    const KLevel& F = D.lev[l];
    const KLevel& C = D.lev[l + 1];
    for (int64_t f = t; f < F.n; f += T) {
        if (!(A.cdiag[F.off + f] > 0.0f)) continue;
        const Pos p = decode(f, F.lx, F.ly);
        const int64_t c = (p.x >> 1) + (int64_t)C.lx * ((p.y >> 1) + (int64_t)C.ly * (p.z >> 1));
        A.cx[F.off + f] += omega * A.cx[C.off + c];
    }
}

// ------------------------------------------------------------------ batched solve (team = CTA)
template <int P>
__device__ void cta_vcycle(const KArena& A, const KDesc& D) {
    const int64_t t = threadIdx.x, T = blockDim.x;
    const int L = D.nlev;
    if (L <= 1) {
        for (int s = 0; s < A.coarse_sweeps; s++) {
            for (int c = 0; c < 8; c++) { op_smooth0<P>(A, D, t, T, c); __syncthreads(); }
            for (int c = 7; c >= 0; c--) { op_smooth0<P>(A, D, t, T, c); __syncthreads(); }
        }
        return;
    }
    for (int s = 0; s < A.nu; s++)
        for (int c = 0; c < 8; c++) { op_smooth0<P>(A, D, t, T, c); __syncthreads(); }
    op_restrict0<P>(A, D, t, T);
    __syncthreads();
    for (int l = 1; l < L - 1; l++) {
        for (int s = 0; s < A.nu; s++)
            for (int c = 0; c < 8; c++) { op_smoothc<P>(A, D, l, t, T, c); __syncthreads(); }
        op_restrictc<P>(A, D, l, t, T);
        __syncthreads();
    }
    for (int s = 0; s < A.coarse_sweeps; s++) {
        for (int c = 0; c < 8; c++) { op_smoothc<P>(A, D, L - 1, t, T, c); __syncthreads(); }
        for (int c = 7; c >= 0; c--) { op_smoothc<P>(A, D, L - 1, t, T, c); __syncthreads(); }
    }
    for (int l = L - 2; l >= 1; l--) {
        op_prolongc(A, D, l, t, T, A.omega_c);
        __syncthreads();
        for (int s = 0; s < A.nu; s++)
            for (int c = 7; c >= 0; c--) { op_smoothc<P>(A, D, l, t, T, c); __syncthreads(); }
    }
    op_prolong0(A, D, t, T, A.omega_c);
    __syncthreads();
    for (int s = 0; s < A.nu; s++)
        for (int c = 7; c >= 0; c--) { op_smooth0<P>(A, D, t, T, c); __syncthreads(); }
}

template <int P, class R>
__device__ void cta_solve(const KArena& A, KDesc& D, R* shr, double* shd) {
    const int64_t t = threadIdx.x, T = blockDim.x;
    // hierarchy
    if (D.nlev > 1) {
        op_build1<P>(A, D, t, T);
        __syncthreads();
        for (int l = 1; l < D.nlev - 1; l++) {
            op_buildc<P>(A, D, l, t, T);
            __syncthreads();
        }
    }
    double relres = 1.0, bn = 0.0;
    int inner_total = 0, outer = 0;
    bool conv = false;
    for (outer = 0; outer <= A.max_outer; outer++) {
        double rr = 0.0, bb = 0.0;
        op_outer_residual(A, D, t, T, rr, bb);
        rr = cta_sum(rr, shd);
        bb = cta_sum(bb, shd);
        bn = sqrt(bb);
        relres = bb > 0.0 ? sqrt(rr / bb) : 0.0;
        if (relres <= A.tol) { conv = true; break; }
        if (outer == A.max_outer || inner_total >= A.max_inner) break;
        // inner PCG on A e = r, stopping at ||r_in|| <= eta ||r_out||
        const double eta = fmax(A.eta_min, 0.3 * A.tol / relres);
        const R stop2 = (R)(eta * eta * rr);
        cta_vcycle<P>(A, D);
        R rz = 0;
        op_dot_rz(A, D, t, T, rz);
        rz = cta_sum(rz, shr);
        op_pupdate(A, D, t, T, 0.0f);
        __syncthreads();
        for (int it = 0; it < A.max_inner - inner_total; it++) {
            R pq = 0;
            op_matvec(A, D, t, T, pq);
            pq = cta_sum(pq, shr);
            const float alpha = pq > (R)0 ? (float)(rz / pq) : 0.0f;
            R rri = 0;
            op_update(A, D, t, T, alpha, rri);
            rri = cta_sum(rri, shr);
            inner_total++;
            if (rri <= stop2 || !(pq > (R)0)) break;
            cta_vcycle<P>(A, D);
            R rzn = 0;
            op_dot_rz(A, D, t, T, rzn);
            rzn = cta_sum(rzn, shr);
            const float beta = rz > (R)0 ? (float)(rzn / rz) : 0.0f;
            rz = rzn;
            op_pupdate(A, D, t, T, beta);
            __syncthreads();
        }
        op_accumulate(A, D, t, T);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        D.relres = relres;
        D.bnorm = bn;
        D.inner_iters = inner_total;
        D.outer_iters = outer;
        D.converged = conv ? 1 : 0;
    }
}

template <int P>
__global__ void __launch_bounds__(kBatchedThreads, 2) k_batched(KArena A) {
    __shared__ double shd[33];
    __shared__ float shf[33];
    __shared__ int next;
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(A.queue, 1);
        __syncthreads();
        const int q = next;
        __syncthreads();
        if (q >= A.nisl) break;
        KDesc& D = A.desc[A.order[q]];
        if (A.fp64_dots) cta_solve<P, double>(A, D, shd, shd);
        else cta_solve<P, float>(A, D, shf, shd);
        __syncthreads();
    }
}

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
__global__ void __launch_bounds__(kPlainBlock) k_plain(KArena A, int isl, int arg, float fa, float* partial) {
    const KDesc& D = A.desc[isl];
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
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

int batched_threads() { return kBatchedThreads; }

int plan_levels(int lx, int ly, int lz, KLevel* lev) {
    int nlev = 1;
    int x = lx, y = ly, z = lz;
    lev[0] = KLevel{lx, ly, lz, 0, 0, (int64_t)lx * ly * lz};
    while (nlev < kMaxLevels && std::max(x, std::max(y, z)) > 2) {
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

void launch_batched(cudaStream_t s, const KArena& a, int ctas, int threads) {
    (void)threads;
    switch (a.prec) {
        case 1: k_batched<1><<<ctas, kBatchedThreads, 0, s>>>(a); break;
        case 2: k_batched<2><<<ctas, kBatchedThreads, 0, s>>>(a); break;
        default: k_batched<0><<<ctas, kBatchedThreads, 0, s>>>(a); break;
    }
}

// Host-driven plain solve of island `isl`: one grid-wide kernel per
// operation, FP32 inner products reduced on the device and read back by the
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
