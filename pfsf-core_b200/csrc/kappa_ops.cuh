// Device operations of the tolerance solve, shared by the batched
// (kappa_batched.cu) and per-island (kappa_plain.cu) execution modes.
// Every op is a loop over a team: thread index t of T threads (a warp, a
// CTA, a thread-block cluster or a whole grid); callers place the barriers.
//
// Indexing is 32-bit inside an island (N < 2^31): each op first forms
// per-island base pointers (the island's arena offset added once in 64-bit
// pointer arithmetic), then decodes voxel coordinates with 32-bit
// division.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "kappa.h"

namespace pfsf_b200 {
namespace kappa {
namespace {

// ------------------------------------------------------------------ storage
template <int P>
__device__ __forceinline__ float k16f(uint16_t v) {
    if constexpr (P == 1) return __bfloat162float(__ushort_as_bfloat16(v));
    else return __half2float(__ushort_as_half(v));
}
template <int P>
__device__ __forceinline__ float cround(float v) {  // value as stored
    if constexpr (P == 0) return v;
    else if constexpr (P == 1) return __bfloat162float(__float2bfloat16_rn(v));
    else return __half2float(__float2half_rn(v));
}

// Fine level of one island (pointers already offset to the island).
struct Fine {
    const uint8_t* type;
    const float* k32;
    const uint16_t* k16;
    const float* b;
    double* x64;
    float *r, *e, *z, *p, *q;
    int lx, ly, lz, n;
};
__device__ __forceinline__ Fine fine_view(const KArena& A, const KDesc& D) {
    const int64_t o = D.off;
    return Fine{A.type + o, A.k32 + o, A.k16 + o, A.b + o, A.x64 + o, A.r + o, A.e + o,
                A.z + o, A.p + o, A.q + o, D.lx, D.ly, D.lz, (int)D.n};
}
template <int P>
__device__ __forceinline__ float kpre(const Fine& F, int g) {  // preconditioner kappa
    if constexpr (P == 0) return F.k32[g];
    else return k16f<P>(F.k16[g]);
}

// Coarse level l of one island: 26 off-diagonals per cell (SoA, stride n).
struct Coarse {
    float* diag;
    float* c32;
    uint16_t* c16;
    float *x, *b;
    int lx, ly, lz, n;
};
__device__ __forceinline__ Coarse coarse_view(const KArena& A, const KDesc& D, int l) {
    const KLevel& L = D.lev[l];
    return Coarse{A.cdiag + L.off, A.coef32 + 26 * L.off, A.coef16 + 26 * L.off, A.cx + L.off, A.cb + L.off,
                  L.lx, L.ly, L.lz, (int)L.n};
}
template <int P>
__device__ __forceinline__ float cget(const Coarse& C, int k, int c) {
    if constexpr (P == 0) return C.c32[k * C.n + c];
    else return k16f<P>(C.c16[k * C.n + c]);
}
template <int P>
__device__ __forceinline__ void cput(const Coarse& C, int k, int c, float v) {
    if constexpr (P == 0) C.c32[k * C.n + c] = v;
    else if constexpr (P == 1) C.c16[k * C.n + c] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
    else C.c16[k * C.n + c] = __half_as_ushort(__float2half_rn(v));
}

// k * k' / (k + k'), 0 when both are 0 (air)
__device__ __forceinline__ float hm(float a, float b) {
    const float s = a + b;
    return s > 0.0f ? __fdividef(a * b, s) : 0.0f;
}
// 1/s for s > 0: the hardware approximation (rcp.approx.ftz.f64, about 2^-23
// relative) refined by two Newton steps r <- r + r(1 - s r), each squaring
// the relative error, to within an ulp of the correctly rounded quotient --
// far below what the FP64 residual needs (link weights to ~1e-12).  The FP64
// residual pass measured 2.7x faster than with IEEE double division.  The
// approximation flushes subnormal inputs (1/s = inf, and the Newton step
// then gives NaN) and subnormal results (s near DBL_MAX gives 0), so s
// outside [2^-1022, 2^1020] takes the IEEE division; kappa sums of the solve
// (kappa normalised to mean 1) never get near either end.
__device__ __forceinline__ double rcp64(double s) {
    if (!(s >= 0x1p-1022 && s <= 0x1p+1020)) return 1.0 / s;
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(s));
    double e = fma(-s, r, 1.0);
    r = fma(r, e, r);
    e = fma(-s, r, 1.0);
    return fma(r, e, r);
}
__device__ __forceinline__ double hm64(double a, double b) {
    const double s = a + b;
    return s > 0.0 ? (a * b) * rcp64(s) : 0.0;
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
__device__ __forceinline__ Pos decode(unsigned i, unsigned lx, unsigned ly) {
    Pos p;
    const unsigned r = i / lx;
    p.x = (int)(i - r * lx);
    const unsigned zz = r / ly;
    p.y = (int)(r - zz * ly);
    p.z = (int)zz;
    return p;
}
// v-th voxel of colour c on an (lx, ly, lz) grid
__device__ __forceinline__ Pos decode_color(unsigned v, unsigned ncx, unsigned ncy, int cx, int cy, int cz) {
    const Pos q = decode(v, ncx, ncy);
    return Pos{2 * q.x + cx, 2 * q.y + cy, 2 * q.z + cz};
}
__device__ __forceinline__ unsigned color_count(int lx, int ly, int lz, int color, unsigned& ncx, unsigned& ncy) {
    const int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    ncx = (unsigned)((lx - cx + 1) >> 1);
    ncy = (unsigned)((ly - cy + 1) >> 1);
    const unsigned ncz = (unsigned)((lz - cz + 1) >> 1);
    return ncx * ncy * ncz;
}

// Visit the in-box 26 neighbours: f(dx, dy, dz, delta_index, group_scale)
template <class F>
__device__ __forceinline__ void for_nb(const Pos& p, int lx, int ly, int lz, F f) {
    const int sy = lx, sz = lx * ly;
    // planes one at a time: 9 neighbours' loads in flight per plane keeps the
    // batched kernel inside 64 registers at 1024 threads per SM
#pragma unroll 1
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
// r = b - A x (FP64 weights and sums), e = z = 0; accumulates (r.r, b.b).
__device__ void op_outer_residual(const KArena& A, const KDesc& D, int t, int T, double& rr, double& bb) {
    const Fine F = fine_view(A, D);
    for (int i = t; i < F.n; i += T) {
        if (F.type[i] != kSolid) {
            F.r[i] = 0.0f; F.e[i] = 0.0f; F.z[i] = 0.0f;
            continue;
        }
        const Pos p = decode((unsigned)i, (unsigned)F.lx, (unsigned)F.ly);
        const double ki = F.k32[i], xi = F.x64[i];
        double acc = 0.0;
        for_nb(p, F.lx, F.ly, F.lz, [&](int, int, int, int dj, float gs) {
            const double w = (double)gs * hm64(ki, (double)F.k32[i + dj]);
            acc += w * (xi - F.x64[i + dj]);
        });
        const double bi = F.b[i];
        const double ri = bi - acc;
        F.r[i] = (float)ri;
        F.e[i] = 0.0f;
        F.z[i] = 0.0f;
        rr += ri * ri;
        bb += bi * bi;
    }
}

// q = A p (FP32 weights); accumulates p.q
template <class R>
__device__ void op_matvec(const KArena& A, const KDesc& D, int t, int T, R& pq) {
    const Fine F = fine_view(A, D);
    for (int i = t; i < F.n; i += T) {
        if (F.type[i] != kSolid) { F.q[i] = 0.0f; continue; }
        const Pos p = decode((unsigned)i, (unsigned)F.lx, (unsigned)F.ly);
        const float ki = F.k32[i], pi = F.p[i];
        float acc = 0.0f;
        for_nb(p, F.lx, F.ly, F.lz, [&](int, int, int, int dj, float gs) {
            acc += gs * hm(ki, F.k32[i + dj]) * (pi - F.p[i + dj]);
        });
        F.q[i] = acc;
        pq += (R)pi * (R)acc;
    }
}

// e += alpha p, r -= alpha q; accumulates r.r
template <class R>
__device__ void op_update(const KArena& A, const KDesc& D, int t, int T, float alpha, R& rr) {
    const Fine F = fine_view(A, D);
    for (int i = t; i < F.n; i += T) {
        const float ri = F.r[i] - alpha * F.q[i];
        F.e[i] += alpha * F.p[i];
        F.r[i] = ri;
        rr += (R)ri * (R)ri;
    }
}

template <class R>
__device__ void op_dot_rz(const KArena& A, const KDesc& D, int t, int T, R& rz) {
    const Fine F = fine_view(A, D);
    for (int i = t; i < F.n; i += T) rz += (R)F.r[i] * (R)F.z[i];
}

// p = z + beta p; z = 0 (ready for the next V-cycle)
__device__ void op_pupdate(const KArena& A, const KDesc& D, int t, int T, float beta) {
    const Fine F = fine_view(A, D);
    for (int i = t; i < F.n; i += T) {
        const float zi = F.z[i];
        F.p[i] = beta == 0.0f ? zi : zi + beta * F.p[i];
        F.z[i] = 0.0f;
    }
}

// x64 += e
__device__ void op_accumulate(const KArena& A, const KDesc& D, int t, int T) {
    const Fine F = fine_view(A, D);
    for (int i = t; i < F.n; i += T) F.x64[i] += (double)F.e[i];
}

// ---- level-0 Gauss-Seidel colour pass on A' z = r (kappa storage P)
template <int P>
__device__ void op_smooth0(const KArena& A, const KDesc& D, int t, int T, int color) {
    const Fine F = fine_view(A, D);
    unsigned ncx, ncy;
    const unsigned nc = color_count(F.lx, F.ly, F.lz, color, ncx, ncy);
    const int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    for (unsigned v = t; v < nc; v += T) {
        const Pos p = decode_color(v, ncx, ncy, cx, cy, cz);
        const int i = p.x + F.lx * (p.y + F.ly * p.z);
        if (F.type[i] != kSolid) continue;
        const float ki = kpre<P>(F, i);
        float d = 0.0f, s = 0.0f;
        for_nb(p, F.lx, F.ly, F.lz, [&](int, int, int, int dj, float gs) {
            const float w = gs * hm(ki, kpre<P>(F, i + dj));
            d += w;
            s += w * F.z[i + dj];
        });
        F.z[i] = d > 0.0f ? (F.r[i] + s) / d : 0.0f;
    }
}

// residual of level 0 (operator A') summed over each 2x2x2 aggregate into level 1; x1 = 0
template <int P>
__device__ void op_restrict0(const KArena& A, const KDesc& D, int t, int T) {
    const Fine F = fine_view(A, D);
    const Coarse C = coarse_view(A, D, 1);
    for (int c = t; c < C.n; c += T) {
        const Pos pc = decode((unsigned)c, (unsigned)C.lx, (unsigned)C.ly);
        float sum = 0.0f;
        for (int a = 0; a < 8; a++) {
            const Pos p{2 * pc.x + (a & 1), 2 * pc.y + ((a >> 1) & 1), 2 * pc.z + ((a >> 2) & 1)};
            if (p.x >= F.lx || p.y >= F.ly || p.z >= F.lz) continue;
            const int i = p.x + F.lx * (p.y + F.ly * p.z);
            if (F.type[i] != kSolid) continue;
            const float ki = kpre<P>(F, i), zi = F.z[i];
            float az = 0.0f;
            for_nb(p, F.lx, F.ly, F.lz, [&](int, int, int, int dj, float gs) {
                az += gs * hm(ki, kpre<P>(F, i + dj)) * (zi - F.z[i + dj]);
            });
            sum += F.r[i] - az;
        }
        C.b[c] = sum;
        C.x[c] = 0.0f;
    }
}

// z_i += omega * x1[aggregate(i)] on solid voxels
__device__ void op_prolong0(const KArena& A, const KDesc& D, int t, int T, float omega) {
    const Fine F = fine_view(A, D);
    const Coarse C = coarse_view(A, D, 1);
    for (int i = t; i < F.n; i += T) {
        if (F.type[i] != kSolid) continue;
        const Pos p = decode((unsigned)i, (unsigned)F.lx, (unsigned)F.ly);
        const int c = (p.x >> 1) + C.lx * ((p.y >> 1) + C.ly * (p.z >> 1));
        F.z[i] += omega * C.x[c];
    }
}

// ---- Galerkin level 1 from the fine operator A' (kappa storage P).
template <int P>
__device__ void op_build1(const KArena& A, const KDesc& D, int t, int T) {
    const Fine F = fine_view(A, D);
    const Coarse C = coarse_view(A, D, 1);
    for (int c = t; c < C.n; c += T) {
        const Pos pc = decode((unsigned)c, (unsigned)C.lx, (unsigned)C.ly);
        float W[26];
#pragma unroll
        for (int k = 0; k < 26; k++) W[k] = 0.0f;
        float anchor = 0.0f;
        for (int a = 0; a < 8; a++) {
            const Pos p{2 * pc.x + (a & 1), 2 * pc.y + ((a >> 1) & 1), 2 * pc.z + ((a >> 2) & 1)};
            if (p.x >= F.lx || p.y >= F.ly || p.z >= F.lz) continue;
            const int i = p.x + F.lx * (p.y + F.ly * p.z);
            if (F.type[i] != kSolid) continue;
            const float ki = kpre<P>(F, i);
            for_nb(p, F.lx, F.ly, F.lz, [&](int dx, int dy, int dz, int dj, float gs) {
                const uint8_t tj = F.type[i + dj];
                if (tj == kAir) return;
                const float w = gs * hm(ki, kpre<P>(F, i + dj));
                if (tj == kAnchor) { anchor += w; return; }
                const int ddx = ((p.x + dx) >> 1) - pc.x, ddy = ((p.y + dy) >> 1) - pc.y, ddz = ((p.z + dz) >> 1) - pc.z;
                if (ddx == 0 && ddy == 0 && ddz == 0) return;
                W[nbk(ddx, ddy, ddz)] += w;
            });
        }
        float diag = anchor;
#pragma unroll
        for (int k = 0; k < 26; k++) {
            cput<P>(C, k, c, W[k]);
            diag += cround<P>(W[k]);
        }
        C.diag[c] = diag;
    }
}

// Galerkin level l+1 from the explicit coefficients of level l.
template <int P>
__device__ void op_buildc(const KArena& A, const KDesc& D, int l, int t, int T) {
    const Coarse F = coarse_view(A, D, l);
    const Coarse C = coarse_view(A, D, l + 1);
    for (int c = t; c < C.n; c += T) {
        const Pos pc = decode((unsigned)c, (unsigned)C.lx, (unsigned)C.ly);
        float W[26];
#pragma unroll
        for (int k = 0; k < 26; k++) W[k] = 0.0f;
        float anchor = 0.0f;
        for (int a = 0; a < 8; a++) {
            const int fx = 2 * pc.x + (a & 1), fy = 2 * pc.y + ((a >> 1) & 1), fz = 2 * pc.z + ((a >> 2) & 1);
            if (fx >= F.lx || fy >= F.ly || fz >= F.lz) continue;
            const int f = fx + F.lx * (fy + F.ly * fz);
            const float dg = F.diag[f];
            if (!(dg > 0.0f)) continue;
            float off = 0.0f;
            for (int k = 0; k < 26; k++) {
                const float w = cget<P>(F, k, f);
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
            cput<P>(C, k, c, W[k]);
            diag += cround<P>(W[k]);
        }
        C.diag[c] = diag;
    }
}

// Gauss-Seidel colour pass on coarse level l
template <int P>
__device__ void op_smoothc(const KArena& A, const KDesc& D, int l, int t, int T, int color) {
    const Coarse L = coarse_view(A, D, l);
    unsigned ncx, ncy;
    const unsigned nc = color_count(L.lx, L.ly, L.lz, color, ncx, ncy);
    const int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    for (unsigned v = t; v < nc; v += T) {
        const Pos p = decode_color(v, ncx, ncy, cx, cy, cz);
        const int c = p.x + L.lx * (p.y + L.ly * p.z);
        const float dg = L.diag[c];
        if (!(dg > 0.0f)) continue;
        float s = 0.0f;
        for_nb(p, L.lx, L.ly, L.lz, [&](int dx, int dy, int dz, int dj, float) {
            s += cget<P>(L, nbk(dx, dy, dz), c) * L.x[c + dj];
        });
        L.x[c] = (L.b[c] + s) / dg;
    }
}

// residual of level l summed per aggregate into level l+1; x_{l+1} = 0
template <int P>
__device__ void op_restrictc(const KArena& A, const KDesc& D, int l, int t, int T) {
    const Coarse F = coarse_view(A, D, l);
    const Coarse C = coarse_view(A, D, l + 1);
    for (int c = t; c < C.n; c += T) {
        const Pos pc = decode((unsigned)c, (unsigned)C.lx, (unsigned)C.ly);
        float sum = 0.0f;
        for (int a = 0; a < 8; a++) {
            const Pos p{2 * pc.x + (a & 1), 2 * pc.y + ((a >> 1) & 1), 2 * pc.z + ((a >> 2) & 1)};
            if (p.x >= F.lx || p.y >= F.ly || p.z >= F.lz) continue;
            const int f = p.x + F.lx * (p.y + F.ly * p.z);
            const float dg = F.diag[f];
            if (!(dg > 0.0f)) continue;
            float s = 0.0f;
            for_nb(p, F.lx, F.ly, F.lz, [&](int dx, int dy, int dz, int dj, float) {
                s += cget<P>(F, nbk(dx, dy, dz), f) * F.x[f + dj];
            });
            sum += F.b[f] - (dg * F.x[f] - s);
        }
        C.b[c] = sum;
        C.x[c] = 0.0f;
    }
}

// x_l += omega * x_{l+1}[parent] on active cells
__device__ void op_prolongc(const KArena& A, const KDesc& D, int l, int t, int T, float omega) {
    const Coarse F = coarse_view(A, D, l);
    const Coarse C = coarse_view(A, D, l + 1);
    for (int f = t; f < F.n; f += T) {
        if (!(F.diag[f] > 0.0f)) continue;
        const Pos p = decode((unsigned)f, (unsigned)F.lx, (unsigned)F.ly);
        const int c = (p.x >> 1) + C.lx * ((p.y >> 1) + C.ly * (p.z >> 1));
        F.x[f] += omega * C.x[c];
    }
}
// xout = xin + omega * x_{l+1}[parent] on active cells of level l, xout = xin elsewhere
__device__ void op_prolongc_to(const KArena& A, const KDesc& D, int l, int t, int T, float omega, const float* xin,
                               float* xout) {
    const Coarse F = coarse_view(A, D, l);
    const Coarse C = coarse_view(A, D, l + 1);
    for (int f = t; f < F.n; f += T) {
        float v = xin[f];
        if (F.diag[f] > 0.0f) {
            const Pos p = decode((unsigned)f, (unsigned)F.lx, (unsigned)F.ly);
            v += omega * C.x[(p.x >> 1) + C.lx * ((p.y >> 1) + C.ly * (p.z >> 1))];
        }
        xout[f] = v;
    }
}

// ---- Chebyshev smoothing (polynomial in D^-1 A' on [lambda_max/10, lambda_max],
// lambda_max = 2, the Gershgorin bound of a weakly diagonally dominant
// operator).  One step: d = c1 d + c2 D^-1 (b - A' x), then x += d, as two
// passes (the second after a barrier) so no pass reads what it writes.

// fine level: inverse diagonal of A' (solid voxels), once per solve
template <int P>
__device__ void op_dinv0(const KArena& A, const KDesc& D, int t, int T) {
    const Fine F = fine_view(A, D);
    float* dinv = A.dinv0 + D.off;
    for (int i = t; i < F.n; i += T) {
        if (F.type[i] != kSolid) { dinv[i] = 0.0f; continue; }
        const Pos p = decode((unsigned)i, (unsigned)F.lx, (unsigned)F.ly);
        const float ki = kpre<P>(F, i);
        float d = 0.0f;
        for_nb(p, F.lx, F.ly, F.lz, [&](int, int, int, int dj, float gs) { d += gs * hm(ki, kpre<P>(F, i + dj)); });
        dinv[i] = d > 0.0f ? 1.0f / d : 0.0f;
    }
}
// first pre-smoothing step from z = 0: d = c2 D^-1 r, zout = d (dinv is 0 off
// solid voxels, so zout is too)
__device__ void op_cheb0_first(const KArena& A, const KDesc& D, int t, int T, float c2, float* zout) {
    const Fine F = fine_view(A, D);
    const float* dinv = A.dinv0 + D.off;
    float* d = A.d0 + D.off;
    for (int i = t; i < F.n; i += T) {
        const float v = c2 * dinv[i] * F.r[i];
        d[i] = v;
        zout[i] = v;
    }
}
// One whole Chebyshev step in one pass, out of place:
//   d = c1 d + c2 D^-1 (r - A' zin),  zout = zin + d     (solid voxels; zout = zin elsewhere)
// (zin and zout are different arrays, so the pass reads nothing it writes)
template <int P>
__device__ void op_cheb0_dz(const KArena& A, const KDesc& D, int t, int T, const float* zin, float* zout, float c1,
                            float c2) {
    const Fine F = fine_view(A, D);
    const float* dinv = A.dinv0 + D.off;
    float* d = A.d0 + D.off;
    for (int i = t; i < F.n; i += T) {
        const float zi = zin[i];
        if (F.type[i] != kSolid) {
            zout[i] = zi;
            continue;
        }
        const Pos p = decode((unsigned)i, (unsigned)F.lx, (unsigned)F.ly);
        const float ki = kpre<P>(F, i);
        float az = 0.0f;
        for_nb(p, F.lx, F.ly, F.lz, [&](int, int, int, int dj, float gs) {
            az += gs * hm(ki, kpre<P>(F, i + dj)) * (zi - zin[i + dj]);
        });
        const float upd = c2 * dinv[i] * (F.r[i] - az);
        const float dn = c1 == 0.0f ? upd : c1 * d[i] + upd;
        d[i] = dn;
        zout[i] = zi + dn;
    }
}
// zout = zin + omega * x1[aggregate(i)] on solid voxels, zout = zin elsewhere
__device__ void op_prolong0_to(const KArena& A, const KDesc& D, int t, int T, float omega, const float* zin,
                               float* zout) {
    const Fine F = fine_view(A, D);
    const Coarse C = coarse_view(A, D, 1);
    for (int i = t; i < F.n; i += T) {
        float v = zin[i];
        if (F.type[i] == kSolid) {
            const Pos p = decode((unsigned)i, (unsigned)F.lx, (unsigned)F.ly);
            v += omega * C.x[(p.x >> 1) + C.lx * ((p.y >> 1) + C.ly * (p.z >> 1))];
        }
        zout[i] = v;
    }
}
__device__ void op_copy(int t, int T, int n, const float* src, float* dst) {
    for (int i = t; i < n; i += T) dst[i] = src[i];
}
// coarse level l: first step from x = 0
// coarse level l: first step from x = 0 into xout (the level's x or x2 array)
__device__ void op_chebc_first(const KArena& A, const KDesc& D, int l, int t, int T, float c2, float* xout) {
    const Coarse L = coarse_view(A, D, l);
    float* d = A.cd + D.lev[l].off;
    for (int c = t; c < L.n; c += T) {
        const float dg = L.diag[c];
        const float v = dg > 0.0f ? c2 * L.b[c] / dg : 0.0f;
        d[c] = v;
        xout[c] = v;
    }
}
// one whole coarse Chebyshev step out of place:
//   d = c1 d + c2 (b - A_c xin) / diag,  xout = xin + d   (active cells; xout = xin elsewhere)
template <int P>
__device__ void op_chebc_dx(const KArena& A, const KDesc& D, int l, int t, int T, const float* xin, float* xout,
                            float c1, float c2) {
    const Coarse L = coarse_view(A, D, l);
    float* d = A.cd + D.lev[l].off;
    for (int c = t; c < L.n; c += T) {
        const float dg = L.diag[c], xc = xin[c];
        if (!(dg > 0.0f)) {
            xout[c] = xc;
            continue;
        }
        const Pos p = decode((unsigned)c, (unsigned)L.lx, (unsigned)L.ly);
        float s = 0.0f;
        for_nb(p, L.lx, L.ly, L.lz, [&](int dx, int dy, int dz, int dj, float) {
            s += cget<P>(L, nbk(dx, dy, dz), c) * xin[c + dj];
        });
        const float upd = c2 * (L.b[c] - (dg * xc - s)) / dg;
        const float dn = c1 == 0.0f ? upd : c1 * d[c] + upd;
        d[c] = dn;
        xout[c] = xc + dn;
    }
}

// One warp runs the V-cycle from coarse level l0 down to the coarsest level
// and back (pre-smoothing at l0 through post-smoothing at l0), with warp
// barriers between dependent passes.  Used once a level is small enough
// (A.tail_cells, tuned) that team-wide barriers would cost more than the work.
template <int P>
__device__ void warp_tail_vcycle(const KArena& A, const KDesc& D, int l0, int nu, int coarse_sweeps, float omega) {
    const int t = threadIdx.x & 31, T = 32;
    const int L = D.nlev;
    for (int l = l0; l < L - 1; l++) {
        for (int s = 0; s < nu; s++)
            for (int c = 0; c < 8; c++) { op_smoothc<P>(A, D, l, t, T, c); __syncwarp(); }
        op_restrictc<P>(A, D, l, t, T);
        __syncwarp();
    }
    for (int s = 0; s < coarse_sweeps; s++) {
        for (int c = 0; c < 8; c++) { op_smoothc<P>(A, D, L - 1, t, T, c); __syncwarp(); }
        for (int c = 7; c >= 0; c--) { op_smoothc<P>(A, D, L - 1, t, T, c); __syncwarp(); }
    }
    for (int l = L - 2; l >= l0; l--) {
        op_prolongc(A, D, l, t, T, omega);
        __syncwarp();
        for (int s = 0; s < nu; s++)
            for (int c = 7; c >= 0; c--) { op_smoothc<P>(A, D, l, t, T, c); __syncwarp(); }
    }
}

}  // namespace
}  // namespace kappa
}  // namespace pfsf_b200
