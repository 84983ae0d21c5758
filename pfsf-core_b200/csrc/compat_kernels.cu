// Reference-schedule ("compat") kernels: the per-tick solve on the SoA-6 face
// conductivity layout the libpfsf C ABI receives (pfsf_island_buffers).
//
// Each kernel restates one reference compute shader; SH below is
// Block Reality/api/src/main/resources/assets/blockreality/shaders/compute/pfsf.
// Arithmetic follows the shader's operation order so results agree with the
// FP32 CPU restatement to rounding; this file is compiled with -fmad=false
// so products and sums round as written.
//
// B200 layout decisions (not in the reference):
//  * voxel type and failure flags are uint8 on the device (the reference
//    widens type to uint32 on the host every upload);
//  * an RBGS colour pass launches only the N/8 voxels of that colour instead
//    of a full-grid dispatch that discards 7/8 of its threads;
//  * dot products are fused into the kernel that produces their operands and
//    finished by a one-block deterministic reduction;
//  * failure flags are compacted to {x,y,z,type} tuples on the device.
#include "common.cuh"
#include "compat.h"

namespace pfsf_b200 {
namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ int64_t gidx(int x, int y, int z, int lx, int ly) {
    return (int64_t)x + (int64_t)lx * ((int64_t)y + (int64_t)ly * z);
}
__device__ __forceinline__ bool inb(int x, int y, int z, int lx, int ly, int lz) {
    return x >= 0 && x < lx && y >= 0 && y < ly && z >= 0 && z < lz;
}

// Accumulate the 26-point Gauss-Seidel sums of voxel i (SH/rbgs_smooth.comp.glsl:125-176).
// phi_nb supplies neighbour values; nphi6 returns the face neighbours (0 off-grid).
__device__ __forceinline__ void gs_accumulate(const float* __restrict__ phi_nb, const float s6[6],
                                              int x, int y, int z, int lx, int ly, int lz,
                                              float& sum_sigma, float& sum_nb, float nphi6[6]) {
    const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
    float ss = 0.0f, sn = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++) {
        const int nx = x + kOfs(d, 0), ny = y + kOfs(d, 1), nz = z + kOfs(d, 2);
        nphi6[d] = inb(nx, ny, nz, lx, ly, lz) ? phi_nb[gidx(nx, ny, nz, lx, ly)] : 0.0f;
    }
#pragma unroll
    for (int d = 0; d < 6; d++) {
        if (!valid[d]) continue;
        const float s = s6[d];
        if (s > 0.0f) {
            const float np = nphi6[d];
            if (finite_f(np)) { ss = __fadd_rn(ss, s); sn = __fadd_rn(sn, __fmul_rn(s, np)); }
        }
    }
#pragma unroll
    for (int e = 0; e < 12; e++) {
        if (!(valid[kEdgeDir(e, 0)] && valid[kEdgeDir(e, 1)])) continue;
        const float es = edge_weight(s6, e);
        if (es > 0.0f) {
            const float ep = phi_nb[gidx(x + kOfs(6 + e, 0), y + kOfs(6 + e, 1), z + kOfs(6 + e, 2), lx, ly)];
            if (finite_f(ep)) { ss = __fadd_rn(ss, es); sn = __fadd_rn(sn, __fmul_rn(es, ep)); }
        }
    }
#pragma unroll
    for (int ci = 0; ci < 8; ci++) {
        const int nx = x + kOfs(18 + ci, 0), ny = y + kOfs(18 + ci, 1), nz = z + kOfs(18 + ci, 2);
        if (!inb(nx, ny, nz, lx, ly, lz)) continue;
        const float cs = corner_weight(s6, ci);
        if (cs > 0.0f) {
            const float cp = phi_nb[gidx(nx, ny, nz, lx, ly)];
            if (finite_f(cp)) { ss = __fadd_rn(ss, cs); sn = __fadd_rn(sn, __fmul_rn(cs, cp)); }
        }
    }
    sum_sigma = ss;
    sum_nb = sn;
}

// Amor split psi_e (rbgs_smooth.comp.glsl:189-203).
__device__ __forceinline__ float amor_psi(const float s6[6], const float nphi6[6], int x, int y, int z,
                                          int lx, int ly, int lz, float phi_new) {
    const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
    float fin = 0.0f, fout = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++) {
        if (!valid[d]) continue;
        const float s = s6[d];
        if (s <= 0.0f) continue;
        const float flow = s * (nphi6[d] - phi_new);
        if (flow > 0.0f) fin += flow;
        else fout -= flow;
    }
    const float k_comp = (fin > 3.0f * fout) ? 0.01f : 1.0f;
    return 0.5f * phi_new * phi_new * k_comp;
}

__device__ __forceinline__ void load_s6(const float* __restrict__ sigma, int64_t n, int64_t i, float s6[6]) {
#pragma unroll
    for (int d = 0; d < 6; d++) s6[d] = __ldg(sigma + d * n + i);
}

// ---------------------------------------------------------------- RBGS colour
// SH/rbgs_smooth.comp.glsl:73-211.  One thread per voxel of colour `color`.
__device__ __forceinline__ void d_rbgs_color(int lx, int ly, int lz, float* __restrict__ phi,
                                             const float* __restrict__ rho, const float* __restrict__ sigma,
                                             const uint8_t* __restrict__ type, float* __restrict__ H,
                                             const uint32_t* __restrict__ macro, int color, float damping,
                                             int64_t t) {
    const int cx = color & 1, cy = (color >> 1) & 1, cz = (color >> 2) & 1;
    const int ncx = (lx - cx + 1) >> 1, ncy = (ly - cy + 1) >> 1, ncz = (lz - cz + 1) >> 1;
    const int64_t nc = (int64_t)ncx * ncy * ncz;
    if (t >= nc) return;
    const int xi = (int)(t % ncx);
    const int64_t rem = t / ncx;
    const int yi = (int)(rem % ncy), zi = (int)(rem / ncy);
    const int x = 2 * xi + cx, y = 2 * yi + cy, z = 2 * zi + cz;
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t i = gidx(x, y, z, lx, ly);
    {
        const int mbx = (lx + kMacroBlock - 1) / kMacroBlock, mby = (ly + kMacroBlock - 1) / kMacroBlock;
        const int64_t mb = (x / kMacroBlock) + (int64_t)mbx * ((y / kMacroBlock) + (int64_t)mby * (z / kMacroBlock));
        if (__uint_as_float(__ldg(macro + mb)) < 1e-4f) return;
    }
    const uint8_t tp = type[i];
    if (tp == kAnchor || tp == kAir) { phi[i] = 0.0f; return; }
    float s6[6], nphi6[6], ss, sn;
    load_s6(sigma, n, i, s6);
    gs_accumulate(phi, s6, x, y, z, lx, ly, lz, ss, sn, nphi6);
    const float phi_gs = (ss > 0.0f) ? (rho[i] + sn) / ss : 0.0f;
    if (phi_gs > 0.0f) {
        const float psi = amor_psi(s6, nphi6, x, y, z, lx, ly, lz, phi_gs);
        H[i] = fmaxf(H[i], psi);
    }
    float result = clamp_f(phi_gs, 0.0f, 1e7f);
    if (damping > 0.0f) result *= damping;
    if (isnan(result)) result = phi[i];
    phi[i] = result;
}


// ---------------------------------------------------------------- history
// H = max(H, psi_e(phi)) on solid voxels with phi > 0 -- the history update
// the reference performs inside every RBGS / Jacobi sweep
// (SH/rbgs_smooth.comp.glsl:177-191), applied once to a given phi (the
// tolerance tick, whose phi does not come from sweeps).
__device__ __forceinline__ void d_history(int lx, int ly, int lz, const float* __restrict__ phi,
                                          const float* __restrict__ sigma, const uint8_t* __restrict__ type,
                                          float* __restrict__ H, int64_t i) {
    const int64_t n = (int64_t)lx * ly * lz;
    if (i >= n || type[i] != kSolid) return;
    const float p = phi[i];
    if (!(p > 0.0f)) return;
    const int x = (int)(i % lx), y = (int)((i / lx) % ly), z = (int)(i / ((int64_t)lx * ly));
    float s6[6], nphi6[6];
    load_s6(sigma, n, i, s6);
#pragma unroll
    for (int d = 0; d < 6; d++) {
        const int nx = x + kOfs(d, 0), ny = y + kOfs(d, 1), nz = z + kOfs(d, 2);
        nphi6[d] = inb(nx, ny, nz, lx, ly, lz) ? phi[gidx(nx, ny, nz, lx, ly)] : 0.0f;
    }
    H[i] = fmaxf(H[i], amor_psi(s6, nphi6, x, y, z, lx, ly, lz, p));
}

// ---------------------------------------------------------------- coarse Jacobi
// SH/jacobi_smooth.comp.glsl:60-227, omega = 1, reading phi_in (a snapshot)
// and writing every voxel of phi_out.  Hfine is the fine-level history buffer,
// which the reference binds at every level (coarse cell i updates Hfine[i]).
__device__ __forceinline__ void d_jacobi_coarse(int lx, int ly, int lz, float* __restrict__ phi_out,
                                                const float* __restrict__ phi_in, const float* __restrict__ rho,
                                                const float* __restrict__ sigma, const uint8_t* __restrict__ type,
                                                float* __restrict__ Hfine, float damping, int64_t i) {
    const int64_t n = (int64_t)lx * ly * lz;
    if (i >= n) return;
    const int x = (int)(i % lx);
    const int64_t rem = i / lx;
    const int y = (int)(rem % ly), z = (int)(rem / ly);
    const uint8_t tp = type[i];
    if (tp == kAnchor || tp == kAir) { phi_out[i] = 0.0f; return; }
    float s6[6], nphi6[6], ss, sn;
    load_s6(sigma, n, i, s6);
    gs_accumulate(phi_in, s6, x, y, z, lx, ly, lz, ss, sn, nphi6);
    const float phi_j = (ss > 0.0f) ? (rho[i] + sn) / ss : 1e7f;
    const float psi = amor_psi(s6, nphi6, x, y, z, lx, ly, lz, phi_j);
    Hfine[i] = fmaxf(Hfine[i], psi);
    const float prev = phi_in[i];
    float result = 1.0f * (phi_j - prev) + prev;
    if (damping > 0.0f) result *= damping;
    result = clamp_f(result, 0.0f, 1e7f);
    if (isnan(result)) result = prev;
    phi_out[i] = result;
}

// ---------------------------------------------------------------- restriction
// residual r = rho + L26 phi (SH/mg_restrict.comp.glsl:53-116)
__device__ float restrict_residual(const float* __restrict__ phi, const float* __restrict__ rho,
                                   const float* __restrict__ sigma, const uint8_t* __restrict__ type,
                                   int x, int y, int z, int lx, int ly, int lz) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t i = gidx(x, y, z, lx, ly);
    if (type[i] != kSolid) return 0.0f;
    const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
    float s6[6];
    load_s6(sigma, n, i, s6);
    const float phi_i = phi[i];
    float L = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++)
        if (valid[d] && s6[d] > 0.0f)
            L += s6[d] * (phi[gidx(x + kOfs(d, 0), y + kOfs(d, 1), z + kOfs(d, 2), lx, ly)] - phi_i);
#pragma unroll
    for (int e = 0; e < 12; e++) {
        if (!(valid[kEdgeDir(e, 0)] && valid[kEdgeDir(e, 1)])) continue;
        const float es = edge_weight(s6, e);
        if (es > 0.0f)
            L += es * (phi[gidx(x + kOfs(6 + e, 0), y + kOfs(6 + e, 1), z + kOfs(6 + e, 2), lx, ly)] - phi_i);
    }
#pragma unroll
    for (int ci = 0; ci < 8; ci++) {
        const int nx = x + kOfs(18 + ci, 0), ny = y + kOfs(18 + ci, 1), nz = z + kOfs(18 + ci, 2);
        if (!inb(nx, ny, nz, lx, ly, lz)) continue;
        const float cs = corner_weight(s6, ci);
        if (cs > 0.0f) L += cs * (phi[gidx(nx, ny, nz, lx, ly)] - phi_i);
    }
    return rho[i] + L;
}
__device__ __forceinline__ float face_cond_sum(const float* __restrict__ sigma, int64_t n, int64_t i) {
    float w = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++) {
        const float s = sigma[d * n + i];
        if (s > 0.0f) w += s;
    }
    return w;
}

// SH/mg_restrict.comp.glsl:118-195
__device__ __forceinline__ void d_restrict(int fx_, int fy_, int fz_, const float* __restrict__ phi_f,
                                                     const float* __restrict__ rho_f,
                                                     const float* __restrict__ sig_f,
                                                     const uint8_t* __restrict__ type_f, int cx_, int cy_,
                                                     int cz_, float* __restrict__ phi_c,
                                                     float* __restrict__ rho_c, int64_t gt_, int64_t blk_) {
    const int64_t nc = (int64_t)cx_ * cy_ * cz_;
    const int64_t c = gt_;
    if (c >= nc) return;
    const int cx = (int)(c % cx_);
    const int64_t rem = c / cx_;
    const int cy = (int)(rem % cy_), cz = (int)(rem / cy_);
    const int64_t nf = (int64_t)fx_ * fy_ * fz_;
    float swr = 0.0f, tw = 0.0f, sur = 0.0f;
    int count = 0;
    for (int dz = 0; dz < 2; dz++)
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                const int x = cx * 2 + dx, y = cy * 2 + dy, z = cz * 2 + dz;
                if (x < fx_ && y < fy_ && z < fz_) {
                    const float r = restrict_residual(phi_f, rho_f, sig_f, type_f, x, y, z, fx_, fy_, fz_);
                    const float w = face_cond_sum(sig_f, nf, gidx(x, y, z, fx_, fy_));
                    swr += w * r; tw += w; sur += r; count++;
                }
            }
    rho_c[c] = (tw > 1e-20f) ? (swr / tw) * (float)count : (count > 0 ? sur : 0.0f);
    float swp = 0.0f, tpw = 0.0f, sp = 0.0f;
    count = 0;
    for (int dz = 0; dz < 2; dz++)
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                const int x = cx * 2 + dx, y = cy * 2 + dy, z = cz * 2 + dz;
                if (x < fx_ && y < fy_ && z < fz_) {
                    const int64_t i = gidx(x, y, z, fx_, fy_);
                    const float p = phi_f[i], w = face_cond_sum(sig_f, nf, i);
                    swp += w * p; tpw += w; sp += p; count++;
                }
            }
    phi_c[c] = (tpw > 1e-20f) ? swp / tpw : (count > 0 ? sp / (float)count : 0.0f);
}

// SH/mg_prolong.comp.glsl:233-275 -- phi_f += trilinear(phi_c) at x/2
__device__ __forceinline__ void d_prolong(int fx_, int fy_, int fz_, float* __restrict__ phi_f, int cx_,
                                                    int cy_, int cz_, const float* __restrict__ phi_c, int64_t gt_, int64_t blk_) {
    const int64_t nf = (int64_t)fx_ * fy_ * fz_;
    const int64_t i = gt_;
    if (i >= nf) return;
    const int x = (int)(i % fx_);
    const int64_t rem = i / fx_;
    const int y = (int)(rem % fy_), z = (int)(rem / fy_);
    const float cxf = (float)x * 0.5f, cyf = (float)y * 0.5f, czf = (float)z * 0.5f;
    const int x0 = (int)floorf(cxf), y0 = (int)floorf(cyf), z0 = (int)floorf(czf);
    const float wx = cxf - (float)x0, wy = cyf - (float)y0, wz = czf - (float)z0;
    float c[2][2][2];
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const int ax = min(max(x0 + q, 0), cx_ - 1);
                const int ay = min(max(y0 + j, 0), cy_ - 1);
                const int az = min(max(z0 + k, 0), cz_ - 1);
                c[k][j][q] = phi_c[gidx(ax, ay, az, cx_, cy_)];
            }
#define MIXF(a, b, t) ((a) * (1.0f - (t)) + (b) * (t))
    const float corr = MIXF(MIXF(MIXF(c[0][0][0], c[0][0][1], wx), MIXF(c[0][1][0], c[0][1][1], wx), wy),
                            MIXF(MIXF(c[1][0][0], c[1][0][1], wx), MIXF(c[1][1][0], c[1][1][1], wx), wy), wz);
#undef MIXF
    phi_f[i] += corr;
}

// island_buffer.cpp:600-700 (downsampleLevel), on the device: coarse
// sigma_d = mean of the children, type = ANCHOR if any anchor child, SOLID
// if solid children > contributing/2, else AIR.
__device__ __forceinline__ void d_downsample(int sx, int sy, int sz, const float* __restrict__ src_cond,
                                                       const uint8_t* __restrict__ src_type, int dx_, int dy_,
                                                       int dz_, float* __restrict__ out_cond,
                                                       uint8_t* __restrict__ out_type, int64_t gt_, int64_t blk_) {
    const int64_t dn = (int64_t)dx_ * dy_ * dz_;
    const int64_t ci = gt_;
    if (ci >= dn) return;
    const int cx = (int)(ci % dx_);
    const int64_t rem = ci / dx_;
    const int cy = (int)(rem % dy_), cz = (int)(rem / dy_);
    const int64_t sn = (int64_t)sx * sy * sz;
    float sum[6] = {0, 0, 0, 0, 0, 0};
    int contrib = 0, solid = 0, anchor = 0;
    for (int ddz = 0; ddz < 2 && cz * 2 + ddz < sz; ddz++)
        for (int ddy = 0; ddy < 2 && cy * 2 + ddy < sy; ddy++)
            for (int ddx = 0; ddx < 2 && cx * 2 + ddx < sx; ddx++) {
                const int64_t fi = gidx(cx * 2 + ddx, cy * 2 + ddy, cz * 2 + ddz, sx, sy);
                contrib++;
                const uint8_t t = src_type[fi];
                if (t == kAnchor) anchor++;
                else if (t == kSolid) solid++;
#pragma unroll
                for (int d = 0; d < 6; d++) sum[d] += src_cond[d * sn + fi];
            }
    const float inv = contrib > 0 ? 1.0f / (float)contrib : 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++) out_cond[d * dn + ci] = contrib > 0 ? sum[d] * inv : 0.0f;
    out_type[ci] = anchor > 0 ? kAnchor : (solid > contrib / 2 ? kSolid : kAir);
}

// ---------------------------------------------------------------- PCG
// 26-point diagonal with bounds-checked faces (pcg_update/pcg_direction computeDiag)
__device__ __forceinline__ float diag26_valid(const float s6[6], int x, int y, int z, int lx, int ly, int lz) {
    const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
    float diag = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++) if (valid[d] && s6[d] > 0.0f) diag += s6[d];
#pragma unroll
    for (int e = 0; e < 12; e++)
        if (valid[kEdgeDir(e, 0)] && valid[kEdgeDir(e, 1)]) diag += edge_weight(s6, e);
#pragma unroll
    for (int ci = 0; ci < 8; ci++) {
        if (!inb(x + kOfs(18 + ci, 0), y + kOfs(18 + ci, 1), z + kOfs(18 + ci, 2), lx, ly, lz)) continue;
        diag += corner_weight(s6, ci);
    }
    return diag;
}

// SH/pcg_precompute.comp.glsl:24-86 (faces summed without a bounds check)
__device__ __forceinline__ void d_pcg_precompute(int lx, int ly, int lz, const float* __restrict__ sigma,
                                                           float* __restrict__ invdiag, int64_t gt_, int64_t blk_) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t i = gt_;
    if (i >= n) return;
    const int x = (int)(i % lx);
    const int64_t rem = i / lx;
    const int y = (int)(rem % ly), z = (int)(rem / ly);
    const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
    float s6[6];
    load_s6(sigma, n, i, s6);
    float d26 = s6[0] + s6[1] + s6[2] + s6[3] + s6[4] + s6[5];
#pragma unroll
    for (int e = 0; e < 12; e++)
        if (valid[kEdgeDir(e, 0)] && valid[kEdgeDir(e, 1)]) d26 += edge_weight(s6, e);
#pragma unroll
    for (int ci = 0; ci < 8; ci++) {
        if (!inb(x + kOfs(18 + ci, 0), y + kOfs(18 + ci, 1), z + kOfs(18 + ci, 2), lx, ly, lz)) continue;
        d26 += corner_weight(s6, ci);
    }
    invdiag[i] = (d26 > 1e-20f) ? (1.0f / d26) : 0.0f;
}

// Block-wide float sum (fixed shuffle tree, deterministic).  Result valid in thread 0.
__device__ __forceinline__ float block_sum(float v) {
    __shared__ float warp_part[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_part[w] = v;
    __syncthreads();
    float s = 0.0f;
    if (w == 0) {
        s = lane < (kBlock / 32) ? warp_part[lane] : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    return s;
}

// SH/pcg_matvec.comp.glsl:128-214: out = sum_j w_ij (in_i - in_j); air/anchor rows 0.
// If partial != nullptr, also emits per-block sums of in_i * out_i (pcg_dot pass 1
// fused: the p.Ap product of pcg_dot.comp.glsl).
__device__ __forceinline__ void d_pcg_matvec(int lx, int ly, int lz, const float* __restrict__ in,
                                                       float* __restrict__ out, const float* __restrict__ sigma,
                                                       const uint8_t* __restrict__ type,
                                                       float* __restrict__ partial, int64_t gt_, int64_t blk_) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t i = gt_;
    float prod = 0.0f;
    if (i < n) {
        const int x = (int)(i % lx);
        const int64_t rem = i / lx;
        const int y = (int)(rem % ly), z = (int)(rem / ly);
        const uint8_t tp = type[i];
        float res = 0.0f;
        if (tp != kAir && tp != kAnchor) {
            const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
            float s6[6];
            load_s6(sigma, n, i, s6);
            const float c = in[i];
#pragma unroll
            for (int d = 0; d < 6; d++) {
                if (!valid[d]) continue;
                if (s6[d] > 0.0f) {
                    const float nv = in[gidx(x + kOfs(d, 0), y + kOfs(d, 1), z + kOfs(d, 2), lx, ly)];
                    if (finite_f(nv)) res += s6[d] * (c - nv);
                }
            }
#pragma unroll
            for (int e = 0; e < 12; e++) {
                if (!(valid[kEdgeDir(e, 0)] && valid[kEdgeDir(e, 1)])) continue;
                const float es = edge_weight(s6, e);
                if (es > 0.0f) {
                    const float ep = in[gidx(x + kOfs(6 + e, 0), y + kOfs(6 + e, 1), z + kOfs(6 + e, 2), lx, ly)];
                    if (finite_f(ep)) res += es * (c - ep);
                }
            }
#pragma unroll
            for (int ci = 0; ci < 8; ci++) {
                const int nx = x + kOfs(18 + ci, 0), ny = y + kOfs(18 + ci, 1), nz = z + kOfs(18 + ci, 2);
                if (!inb(nx, ny, nz, lx, ly, lz)) continue;
                const float cs = corner_weight(s6, ci);
                if (cs > 0.0f) {
                    const float cp = in[gidx(nx, ny, nz, lx, ly)];
                    if (finite_f(cp)) res += cs * (c - cp);
                }
            }
            if (!finite_f(res)) res = 0.0f;
        }
        out[i] = res;
        prod = in[i] * res;
    }
    if (partial != nullptr) {
        const float s = block_sum(prod);
        if (threadIdx.x == 0) partial[blk_] = s;
    }
}

// SH/pcg_update.comp.glsl:116-211.  Init: r = s - Ap, z = r/diag, p = z.
// Iteration: alpha = red[0]/red[1]; phi += alpha p (clamped), r = r_in - alpha Ap,
// z = r/diag + (sum_d sigma_d r_in[j] invdiag[j]) / diag where r_in is r before
// this dispatch.  Per-block partial of r.z over voxels i < rtz_limit.
__device__ __forceinline__ void d_pcg_update(int lx, int ly, int lz, float* __restrict__ phi,
                                                       const float* __restrict__ r_in, float* __restrict__ r_out,
                                                       float* __restrict__ p, const float* __restrict__ ap,
                                                       const float* __restrict__ src,
                                                       const uint8_t* __restrict__ type,
                                                       const float* __restrict__ sigma,
                                                       const float* __restrict__ invdiag,
                                                       const float* __restrict__ red, int is_init,
                                                       int64_t rtz_limit, float* __restrict__ partial, int64_t gt_, int64_t blk_) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t i = gt_;
    float rz = 0.0f;
    if (i < n) {
        const int x = (int)(i % lx);
        const int64_t rem = i / lx;
        const int y = (int)(rem % ly), z = (int)(rem / ly);
        const uint8_t tp = type[i];
        float s6[6];
        if (is_init) {
            if (tp == kSolid) {
                float ri = src[i] - ap[i];
                if (!finite_f(ri)) ri = 0.0f;
                r_out[i] = ri;
                load_s6(sigma, n, i, s6);
                const float diag = diag26_valid(s6, x, y, z, lx, ly, lz);
                float zi = (diag > 1e-20f) ? ri / diag : ri;
                if (!finite_f(zi)) zi = 0.0f;
                p[i] = zi;
                rz = ri * zi;
            } else {
                r_out[i] = 0.0f;
                p[i] = 0.0f;
            }
        } else if (tp == kSolid) {
            const float rtz_old = red[0], pap = red[1];
            const float alpha = (pap > 1e-30f) ? rtz_old / pap : 0.0f;
            load_s6(sigma, n, i, s6);
            const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
            const int64_t lxly = (int64_t)lx * ly;
            const int64_t nb[6] = {i - 1, i + 1, i - lx, i + lx, i - lxly, i + lxly};
            float corr = 0.0f;
#pragma unroll
            for (int d = 0; d < 6; d++)
                if (valid[d]) corr += s6[d] * (r_in[nb[d]] * invdiag[nb[d]]);
            float ph = phi[i] + alpha * p[i];
            float ri = r_in[i] - alpha * ap[i];
            ph = clamp_f(ph, 0.0f, 1e7f);
            if (isnan(ph)) ph = 0.0f;
            phi[i] = ph;
            if (!finite_f(ri)) ri = 0.0f;
            r_out[i] = ri;
            const float diag = diag26_valid(s6, x, y, z, lx, ly, lz);
            const float zj = (diag > 1e-20f) ? ri / diag : ri;
            float zi = zj + ((diag > 1e-20f) ? corr / diag : 0.0f);
            if (!finite_f(zi)) zi = zj;
            rz = ri * zi;
        } else {
            r_out[i] = r_in[i];
        }
        if (i >= rtz_limit) rz = 0.0f;
    }
    const float s = block_sum(rz);
    if (threadIdx.x == 0) partial[blk_] = s;
}

// SH/pcg_direction.comp.glsl:336-379
__device__ __forceinline__ void d_pcg_direction(int lx, int ly, int lz, const float* __restrict__ r,
                                                          float* __restrict__ p, const uint8_t* __restrict__ type,
                                                          const float* __restrict__ red,
                                                          const float* __restrict__ sigma, int64_t gt_, int64_t blk_) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t i = gt_;
    if (i >= n) return;
    if (type[i] != kSolid) { p[i] = 0.0f; return; }
    const int x = (int)(i % lx);
    const int64_t rem = i / lx;
    const int y = (int)(rem % ly), z = (int)(rem / ly);
    const float rtz_old = red[0], rtz_new = red[2];
    float beta = (rtz_old > 1e-30f) ? rtz_new / rtz_old : 0.0f;
    beta = clamp_f(beta, 0.0f, 10.0f);
    float s6[6];
    load_s6(sigma, n, i, s6);
    const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
    const int64_t lxly = (int64_t)lx * ly;
    const int64_t nb[6] = {i - 1, i + 1, i - lx, i + lx, i - lxly, i + lxly};
    const float ri = r[i];
    const float diag = diag26_valid(s6, x, y, z, lx, ly, lz);
    float corr = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++) {
        if (!valid[d]) continue;
        const int64_t j = nb[d];
        const float rj = r[j];
        const float d6j = sigma[0 * n + j] + sigma[1 * n + j] + sigma[2 * n + j] + sigma[3 * n + j] +
                          sigma[4 * n + j] + sigma[5 * n + j];
        corr += s6[d] * ((d6j > 1e-20f) ? rj / d6j : 0.0f);
    }
    const float zj = (diag > 1e-20f) ? ri / diag : ri;
    float zi = zj + ((diag > 1e-20f) ? corr / diag : 0.0f);
    if (!finite_f(zi)) zi = zj;
    float np = zi + beta * p[i];
    if (!finite_f(np)) np = zi;
    p[i] = np;
}

// ---- aggregation correction (NP/src/solver/dispatcher_amg.cpp:83-161)
//
// An aggregate is the 2x2x2 block of the L1 coarsening (amg_builder.cpp:9-63).
// One thread per aggregate visits its voxels (2cx+dx, 2cy+dy, 2cz+dz) in
// increasing voxel index, the order of the builder's sequential loops, so
// every sum below adds in the reference builder's order.  The restriction
// gathers instead of the shader's atomic scatter (amg_scatter_restrict
// adds in no fixed order): no zero fill, no atomics, one deterministic sum.
__device__ __forceinline__ bool amg_voxel(int lx, int ly, int lz, int cx, int cy, int cz, int k, int64_t& i) {
    const int x = 2 * cx + (k & 1), y = 2 * cy + ((k >> 1) & 1), z = 2 * cz + (k >> 2);
    if (x >= lx || y >= ly || z >= lz) return false;
    i = x + (int64_t)lx * (y + (int64_t)ly * z);
    return true;
}

// amg_builder.cpp:23-61: diag6 = sum of the six face conductivities; a
// voxel joins its aggregate unless it is an anchor or diag6 < 1e-20; weight
// = diag6 / (aggregate's diag6 sum); D_c = sum of weight^2 * diag6.
__device__ __forceinline__ void d_amg_build(int lx, int ly, int lz, const float* __restrict__ sigma,
                                            const uint8_t* __restrict__ type, int32_t* __restrict__ agg,
                                            float* __restrict__ w, float* __restrict__ dc, int64_t gt_) {
    const int ax = (lx + 1) >> 1, ay = (ly + 1) >> 1, az = (lz + 1) >> 1;
    const int64_t j = gt_;
    if (j >= (int64_t)ax * ay * az) return;
    const int cx = (int)(j % ax);
    const int64_t rem = j / ax;
    const int cy = (int)(rem % ay), cz = (int)(rem / ay);
    const int64_t n = (int64_t)lx * ly * lz;
    float d6[8];
    float asum = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        int64_t i;
        d6[k] = -1.0f;
        if (!amg_voxel(lx, ly, lz, cx, cy, cz, k, i)) continue;
        float t = 0.0f;
#pragma unroll
        for (int d = 0; d < 6; d++) t = __fadd_rn(t, sigma[d * n + i]);
        const bool in = type[i] != 2 && !(t < 1e-20f);
        agg[i] = in ? (int32_t)j : -1;
        w[i] = 0.0f;
        if (in) {
            asum = __fadd_rn(asum, t);
            d6[k] = t;
        }
    }
    float dcj = 0.0f;
    if (!(asum < 1e-20f)) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            int64_t i;
            if (d6[k] < 0.0f || !amg_voxel(lx, ly, lz, cx, cy, cz, k, i)) continue;
            const float pi = __fdiv_rn(d6[k], asum);
            w[i] = pi;
            dcj = __fadd_rn(dcj, __fmul_rn(__fmul_rn(pi, pi), d6[k]));
        }
    }
    dc[j] = dcj;
}

// amg_scatter_restrict.comp.glsl:51-60 + amg_coarse_jacobi.comp.glsl:33-40:
// e_c = (sum of w_i r_i over the aggregate) / D_c, 0 where D_c <= 1e-20
__device__ __forceinline__ void d_amg_coarse(int lx, int ly, int lz, const int32_t* __restrict__ agg,
                                             const float* __restrict__ w, const float* __restrict__ dc,
                                             const float* __restrict__ r, float* __restrict__ ec, int64_t gt_) {
    const int ax = (lx + 1) >> 1, ay = (ly + 1) >> 1, az = (lz + 1) >> 1;
    const int64_t j = gt_;
    if (j >= (int64_t)ax * ay * az) return;
    const int cx = (int)(j % ax);
    const int64_t rem = j / ax;
    const int cy = (int)(rem % ay), cz = (int)(rem / ay);
    float rc = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        int64_t i;
        if (!amg_voxel(lx, ly, lz, cx, cy, cz, k, i) || agg[i] < 0) continue;
        rc = __fadd_rn(rc, __fmul_rn(w[i], r[i]));
    }
    const float d = dc[j];
    ec[j] = d > 1e-20f ? __fdiv_rn(rc, d) : 0.0f;
}

// amg_gather_prolong.comp.glsl:44-71: phi += w e_c[agg] at aggregated voxels
__device__ __forceinline__ void d_amg_prolong(int64_t n, const int32_t* __restrict__ agg,
                                              const float* __restrict__ w, const float* __restrict__ ec,
                                              float* __restrict__ phi, int64_t gt_) {
    const int64_t i = gt_;
    if (i >= n) return;
    const int32_t a = agg[i];
    if (a < 0) return;
    phi[i] = __fadd_rn(phi[i], __fmul_rn(w[i], ec[a]));
}

// Single-block sum of `count` partials into red[slot].  rotate: first copy
// red[2] -> red[0] (the rTz slot rotation of dispatcher_pcg.cpp recordReductionRotate).
__device__ __forceinline__ void d_finalize(const float* __restrict__ partial, int64_t count,
                                                     float* __restrict__ red, int slot, int rotate, int64_t gt_, int64_t blk_) {
    float v = 0.0f;
    for (int64_t k = threadIdx.x; k < count; k += kBlock) v += partial[k];
    const float s = block_sum(v);
    if (threadIdx.x == 0) {
        if (rotate) red[0] = red[2];
        red[slot] = s;
    }
}

// ---------------------------------------------------------------- phase field
// SH/phase_field_evolve.comp.glsl:246-364.  The shader rewrites dField in place
// while neighbours read it (a race); here every d_j comes from Dold, a copy of
// the field taken before the pass.
__device__ __forceinline__ void d_phase_field(int lx, int ly, int lz, const float* __restrict__ phi,
                                                        const float* __restrict__ H, float* __restrict__ D,
                                                        const float* __restrict__ Dold,
                                                        const float* __restrict__ sigma,
                                                        const uint8_t* __restrict__ type,
                                                        uint8_t* __restrict__ fail, const float* __restrict__ hyd,
                                                        float l0, float gc, float relax, int split, int64_t gt_, int64_t blk_) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t i = gt_;
    if (i >= n) return;
    const uint8_t tp = type[i];
    if (tp == kAir || tp == kAnchor) return;
    if (fail[i] != 0) return;
    const int x = (int)(i % lx);
    const int64_t rem = i / lx;
    const int y = (int)(rem % ly), z = (int)(rem / ly);
    const float phi_i = phi[i], d_i = Dold[i];
    float sum_sigma = 0.0f, lap_phi = 0.0f, lap_d = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++) {
        const int nx = x + kOfs(d, 0), ny = y + kOfs(d, 1), nz = z + kOfs(d, 2);
        if (!inb(nx, ny, nz, lx, ly, lz)) continue;
        const int64_t j = gidx(nx, ny, nz, lx, ly);
        if (type[j] == kAir) continue;
        const float s = sigma[d * n + i], pj = phi[j], dj = Dold[j];
        if (finite_f(pj)) { lap_phi += (pj - phi_i); sum_sigma += s; }
        if (finite_f(dj)) lap_d += (dj - d_i);
    }
    const float hv = H[i];
    if (hv <= 0.0f) return;
    const float hdeg = clamp_f(hyd[i], 0.01f, 1.0f);
    const float gce = gc * powf(hdeg, 1.5f);
    float heff = hv;
    if (split) {
        const float sd = fmaxf(sum_sigma, 1e-12f);
        const float fo = fmaxf(lap_phi, 0.0f);
        heff = fmaxf(hv, fo / sd);
    }
    const float num = 2.0f * heff + gce * l0 * lap_d;
    float den = 2.0f * heff + gce / l0;
    den = fmaxf(den, 1e-8f);
    float dn = clamp_f(num / den, d_i, 1.0f);
    dn = d_i * (1.0f - relax) + dn * relax;
    dn = clamp_f(dn, 0.0f, 1.0f);
    if (!finite_f(dn)) dn = d_i;
    D[i] = dn;
    if (dn > 0.95f) fail[i] = 1;
}

// ---------------------------------------------------------------- failure scan
// SH/failure_scan.comp.glsl:36-196
// Failure code of voxel i (SH/failure_scan.comp.glsl:36-196): 0 intact, 2
// crushing (compressive inflow above rcomp), 3 no support (no live face or
// phi above the orphan level), 4 tension (outflow above rtens); air and
// anchors 0.  For an intact solid voxel also its residual |fin - fout + rho|
// (res, else -1) and its macro block (mb), which the reference feeds into
// the macro-residual maximum.
__device__ __forceinline__ uint8_t d_fail_code(int lx, int ly, int lz, const float* __restrict__ phi,
                                               const float* __restrict__ sigma, const float* __restrict__ rcomp,
                                               const uint8_t* __restrict__ type, const float* __restrict__ rtens,
                                               const float* __restrict__ rho, float phi_orphan, int64_t i,
                                               float& res, int64_t& mb) {
    const int64_t n = (int64_t)lx * ly * lz;
    res = -1.0f;
    mb = 0;
    if (type[i] != kSolid) return 0;
    const float p = phi[i];
    float s6[6];
    load_s6(sigma, n, i, s6);
    const float sum6 = s6[0] + s6[1] + s6[2] + s6[3] + s6[4] + s6[5];
    if (sum6 == 0.0f || p > phi_orphan) return 3;
    const int x = (int)(i % lx);
    const int64_t rem = i / lx;
    const int y = (int)(rem % ly), z = (int)(rem / ly);
    const bool valid[6] = {x > 0, x + 1 < lx, y > 0, y + 1 < ly, z > 0, z + 1 < lz};
    float fin = 0.0f, fout = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; d++) {
        if (!valid[d]) continue;
        if (s6[d] > 0.0f) {
            const float dphi = phi[gidx(x + kOfs(d, 0), y + kOfs(d, 1), z + kOfs(d, 2), lx, ly)] - p;
            if (dphi > 0.0f) fin += s6[d] * dphi;
            else if (dphi < 0.0f) fout += s6[d] * (-dphi);
        }
    }
    const float sxa = (s6[0] + s6[1]) * 0.5f, sya = (s6[2] + s6[3]) * 0.5f, sza = (s6[4] + s6[5]) * 0.5f;
    const float ew[3] = {sqrtf(fmaxf(sxa * sya, 0.0f)) * kEdgeP, sqrtf(fmaxf(sxa * sza, 0.0f)) * kEdgeP,
                         sqrtf(fmaxf(sya * sza, 0.0f)) * kEdgeP};
#pragma unroll
    for (int plane = 0; plane < 3; plane++) {
        if (!(ew[plane] > 0.0f)) continue;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int e = plane * 4 + k;
            if (!(valid[kEdgeDir(e, 0)] && valid[kEdgeDir(e, 1)])) continue;
            const float dphi = phi[gidx(x + kOfs(6 + e, 0), y + kOfs(6 + e, 1), z + kOfs(6 + e, 2), lx, ly)] - p;
            if (dphi > 0.0f) fin += ew[plane] * dphi;
            else fout += ew[plane] * (-dphi);
        }
    }
    const float cw = cbrtf(fmaxf(sxa * sya * sza, 0.0f)) * kCornerP;
    if (cw > 0.0f) {
#pragma unroll
        for (int ci = 0; ci < 8; ci++) {
            const int nx = x + kOfs(18 + ci, 0), ny = y + kOfs(18 + ci, 1), nz = z + kOfs(18 + ci, 2);
            if (!inb(nx, ny, nz, lx, ly, lz)) continue;
            const float dphi = phi[gidx(nx, ny, nz, lx, ly)] - p;
            if (dphi > 0.0f) fin += cw * dphi;
            else fout += cw * (-dphi);
        }
    }
    const float rc = rcomp[i], rt = rtens[i];
    if (rc > 0.0f && fin > rc) return 2;
    if (rt > 0.0f && fout > rt) return 4;
    res = fabsf(fin - fout + rho[i]);
    const int mbx = (lx + kMacroBlock - 1) / kMacroBlock, mby = (ly + kMacroBlock - 1) / kMacroBlock;
    mb = (x / kMacroBlock) + (int64_t)mbx * ((y / kMacroBlock) + (int64_t)mby * (z / kMacroBlock));
    return 0;
}

// Order-preserving map of a float onto uint32 (atomicMax over keys = max over
// floats, negatives included); 0 is below every key.
__device__ __forceinline__ uint32_t float_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Block-wide max (valid in thread 0).
__device__ __forceinline__ float block_max(float v) {
    __shared__ float warp_part[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_part[w] = v;
    __syncthreads();
    float m = -INFINITY;
    if (w == 0) {
        m = lane < (kBlock / 32) ? warp_part[lane] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    }
    return m;
}

__device__ __forceinline__ void d_macro_fill(uint32_t* __restrict__ macro, int64_t nmb, int64_t gt_, int64_t blk_) {
    const int64_t i = gt_;
    if (i < nmb) macro[i] = kMacroSeedBits;
}

// max over macro blocks as float (readbackMacroResidualMax, island_buffer.cpp:1012-1090),
// single block; writes out[0].

// ---------------------------------------------------------------- failure compaction
constexpr int kCompactChunk = 4096;  // voxels per block

__device__ __forceinline__ void d_fail_count(const uint8_t* __restrict__ fail, int64_t n,
                                                       int32_t* __restrict__ counts, int64_t gt_, int64_t blk_) {
    const int64_t base = (int64_t)blk_ * kCompactChunk;
    int c = 0;
    for (int k = threadIdx.x; k < kCompactChunk; k += kBlock) {
        const int64_t i = base + k;
        if (i < n && fail[i] != 0) c++;
    }
    const float s = block_sum((float)c);
    if (threadIdx.x == 0) counts[blk_] = (int32_t)s;
}
__global__ void __launch_bounds__(kBlock) k_fail_count(const uint8_t* __restrict__ fail, int64_t n,
                                                       int32_t* __restrict__ counts) {
    d_fail_count(fail, n, counts, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)blockIdx.x);
}

// exclusive scan of block counts (single block, sequential over chunks of 256);
// writes offsets[] and total[0].
__device__ __forceinline__ void d_fail_scan(const int32_t* __restrict__ counts, int64_t nblocks,
                                                      int32_t* __restrict__ offsets, int32_t* __restrict__ total, int64_t gt_, int64_t blk_) {
    __shared__ int32_t buf[kBlock];
    __shared__ int32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nblocks; base += kBlock) {
        const int64_t k = base + threadIdx.x;
        const int32_t v = k < nblocks ? counts[k] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < kBlock; o <<= 1) {
            const int32_t t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        if (k < nblocks) offsets[k] = carry + buf[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == kBlock - 1) carry += buf[kBlock - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) total[0] = carry;
}
__global__ void __launch_bounds__(kBlock) k_fail_scan(const int32_t* __restrict__ counts, int64_t nblocks,
                                                      int32_t* __restrict__ offsets, int32_t* __restrict__ total) {
    d_fail_scan(counts, nblocks, offsets, total, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)blockIdx.x);
}

// write {x+ox, y+oy, z+oz, code} tuples in index order; tuples beyond cap are dropped.
__device__ __forceinline__ void d_fail_write(const uint8_t* __restrict__ fail, int lx, int ly, int lz,
                                                       int ox, int oy, int oz,
                                                       const int32_t* __restrict__ offsets,
                                                       int32_t* __restrict__ tuples, int32_t cap, int64_t gt_, int64_t blk_) {
    __shared__ int32_t warp_cnt[kBlock / 32];
    __shared__ int32_t run;
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t base = (int64_t)blk_ * kCompactChunk;
    if (threadIdx.x == 0) run = offsets[blk_];
    __syncthreads();
    for (int k0 = 0; k0 < kCompactChunk; k0 += kBlock) {
        const int64_t i = base + k0 + threadIdx.x;
        const uint8_t f = (i < n) ? fail[i] : 0;
        const unsigned ballot = __ballot_sync(0xffffffffu, f != 0);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) warp_cnt[w] = __popc(ballot);
        __syncthreads();
        int before = 0;
        for (int q = 0; q < w; q++) before += warp_cnt[q];
        const int pos = run + before + __popc(ballot & ((1u << lane) - 1u));
        if (f != 0 && pos < cap) {
            int32_t* t = tuples + 4 * (int64_t)pos;
            t[0] = ox + (int)(i % lx);
            t[1] = oy + (int)((i / lx) % ly);
            t[2] = oz + (int)(i / ((int64_t)lx * ly));
            t[3] = f;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int q = 0; q < kBlock / 32; q++) tot += warp_cnt[q];
            run += tot;
        }
        __syncthreads();
    }
}
__global__ void __launch_bounds__(kBlock) k_fail_write(const uint8_t* __restrict__ fail, int lx, int ly, int lz,
                                                       int ox, int oy, int oz,
                                                       const int32_t* __restrict__ offsets,
                                                       int32_t* __restrict__ tuples, int32_t cap) {
    d_fail_write(fail, lx, ly, lz, ox, oy, oz, offsets, tuples, cap, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, (int64_t)blockIdx.x);
}

// SH/sparse_scatter.comp.glsl: 48-byte records {u32 idx, f32 source, u32 type,
// f32 maxPhi, f32 rcomp, f32 rtens, f32 cond[6]} scattered into the SoA arrays.
// Records whose index is outside the island are skipped (the shader has no
// bounds check).
__global__ void k_sparse_scatter(const uint32_t* __restrict__ rec, int count, int64_t n,
                                 float* __restrict__ source, float* __restrict__ cond, uint8_t* __restrict__ type,
                                 float* __restrict__ maxphi, float* __restrict__ rcomp, float* __restrict__ rtens) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= count) return;
    const uint32_t* r = rec + 12 * (int64_t)u;
    const int64_t i = r[0];
    if (i >= n) return;
    source[i] = __uint_as_float(r[1]);
    type[i] = (uint8_t)r[2];
    maxphi[i] = __uint_as_float(r[3]);
    rcomp[i] = __uint_as_float(r[4]);
    rtens[i] = __uint_as_float(r[5]);
#pragma unroll
    for (int d = 0; d < 6; d++) cond[d * n + i] = __uint_as_float(r[6 + d]);
}

// ---------------------------------------------------------------- batched forms
using compat::CIsl;
// Block b of a batched launch belongs to the island q whose block range
// [bs[q], bs[q+1]) holds it (islands with no blocks of this kind are
// skipped by the search); found once per block by thread 0.
__device__ __forceinline__ int b_island(const int* __restrict__ bs, int nisl) {
    __shared__ int s_q;
    if (threadIdx.x == 0) {
        const int b = (int)blockIdx.x;
        int lo = 0, hi = nisl - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (bs[mid] <= b) lo = mid;
            else hi = mid - 1;
        }
        s_q = lo;
    }
    __syncthreads();
    return s_q;
}

#define BATCH_ISLAND                                                   \
    const int q_ = b_island(bs, nisl);                                 \
    const CIsl& I = tab[q_];                                           \
    const int64_t lb_ = (int64_t)blockIdx.x - (int64_t)bs[q_];         \
    const int64_t t_ = lb_ * (int64_t)blockDim.x + threadIdx.x;

__device__ __forceinline__ float b_damping(const CIsl& I, int sidx, int warm, float dampf) {
    return I.iter0 + sidx >= warm ? dampf : 0.0f;
}

// The caller's arrays into the device arrays (uploadFromHosts), read through
// the device-visible mappings of the pinned host buffers.
__global__ void __launch_bounds__(kBlock) kb_upload(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                    int nisl) {
    BATCH_ISLAND
    if (t_ >= I.n || I.h_phi == nullptr) return;
    const int64_t i = t_, n = I.n;
    I.phi[i] = I.h_phi[i];
    I.src[i] = I.h_src[i];
#pragma unroll
    for (int d = 0; d < 6; d++) I.sigma[d * n + i] = I.h_sigma[d * n + i];
    I.type[i] = I.h_type[i];
    I.rcomp[i] = I.h_rcomp[i];
    I.rtens[i] = I.h_rtens[i];
    I.maxphi[i] = I.h_maxphi[i];
    if (I.h_curing) I.hyd[i] = I.h_curing[i];
}
__global__ void __launch_bounds__(kBlock) kb_macro_fill(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                        int nisl) {
    BATCH_ISLAND
    d_macro_fill(I.macro, I.nmb, t_, lb_);
    if (t_ == 0) {  // the island records the failure pass reduces into
        *I.res_macro = __uint_as_float(kMacroSeedBits);
        *I.res_phimax = 0u;
    }
}
__global__ void __launch_bounds__(kBlock) kb_rbgs_color(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                        int nisl, int color, int sidx, int warm, float dampf) {
    BATCH_ISLAND
    d_rbgs_color(I.lx, I.ly, I.lz, I.phi, I.src, I.sigma, I.type, I.H, I.macro, color,
                 b_damping(I, sidx, warm, dampf), t_);
}
__global__ void __launch_bounds__(kBlock) kb_jacobi(const CIsl* __restrict__ tab, const int* __restrict__ bs, int nisl,
                                                    int level, int flip, int sidx, int warm, float dampf) {
    BATCH_ISLAND
    const float damping = b_damping(I, sidx, warm, dampf);
    if (level == 1) {
        const int c = (I.cur1 + flip) & 1;
        d_jacobi_coarse(I.l1x, I.l1y, I.l1z, I.phi1[1 - c], I.phi1[c], I.src1, I.sig1, I.type1, I.H, damping, t_);
    } else {
        const int c = (I.cur2 + flip) & 1;
        d_jacobi_coarse(I.l2x, I.l2y, I.l2z, I.phi2[1 - c], I.phi2[c], I.src2, I.sig2, I.type2, I.H, damping, t_);
    }
}
__global__ void __launch_bounds__(kBlock) kb_restrict(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                      int nisl, int level, int f1, int f2) {
    BATCH_ISLAND
    const int c1 = (I.cur1 + f1) & 1, c2 = (I.cur2 + f2) & 1;
    if (level == 1)
        d_restrict(I.lx, I.ly, I.lz, I.phi, I.src, I.sigma, I.type, I.l1x, I.l1y, I.l1z, I.phi1[c1], I.src1, t_, lb_);
    else
        d_restrict(I.l1x, I.l1y, I.l1z, I.phi1[c1], I.src1, I.sig1, I.type1, I.l2x, I.l2y, I.l2z, I.phi2[c2], I.src2,
                   t_, lb_);
}
__global__ void __launch_bounds__(kBlock) kb_prolong(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                     int nisl, int level, int f1, int f2) {
    BATCH_ISLAND
    const int c1 = (I.cur1 + f1) & 1, c2 = (I.cur2 + f2) & 1;
    if (level == 1) d_prolong(I.lx, I.ly, I.lz, I.phi, I.l1x, I.l1y, I.l1z, I.phi1[c1], t_, lb_);
    else d_prolong(I.l1x, I.l1y, I.l1z, I.phi1[c1], I.l2x, I.l2y, I.l2z, I.phi2[c2], t_, lb_);
}
__global__ void __launch_bounds__(kBlock) kb_downsample(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                        int nisl, int level) {
    BATCH_ISLAND
    if (level == 1) d_downsample(I.lx, I.ly, I.lz, I.sigma, I.type, I.l1x, I.l1y, I.l1z, I.sig1, I.type1, t_, lb_);
    else d_downsample(I.l1x, I.l1y, I.l1z, I.sig1, I.type1, I.l2x, I.l2y, I.l2z, I.sig2, I.type2, t_, lb_);
}
__global__ void __launch_bounds__(kBlock) kb_pcg_precompute(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                            int nisl) {
    BATCH_ISLAND
    d_pcg_precompute(I.lx, I.ly, I.lz, I.sigma, I.invdiag, t_, lb_);
}
__global__ void __launch_bounds__(kBlock) kb_pcg_matvec(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                        int nisl, int which) {
    BATCH_ISLAND
    if (which == 0) d_pcg_matvec(I.lx, I.ly, I.lz, I.phi, I.ap, I.sigma, I.type, nullptr, t_, lb_);
    else d_pcg_matvec(I.lx, I.ly, I.lz, I.p, I.ap, I.sigma, I.type, I.partial, t_, lb_);
}
__global__ void __launch_bounds__(kBlock) kb_pcg_update(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                        int nisl, int is_init, int fr) {
    BATCH_ISLAND
    const int c = (I.rcur + fr) & 1;
    const int64_t g = (I.n + 511) / 512;
    const int64_t rtz = I.n < 256 * g ? I.n : 256 * g;
    d_pcg_update(I.lx, I.ly, I.lz, I.phi, I.r[c], is_init ? I.r[c] : I.r[1 - c], I.p, I.ap, I.src, I.type, I.sigma,
                 I.invdiag, I.red, is_init, rtz, I.partial, t_, lb_);
}
// one block per island
__global__ void __launch_bounds__(kBlock) kb_finalize(const CIsl* __restrict__ tab, int slot, int rotate) {
    const CIsl& I = tab[blockIdx.x];
    d_finalize(I.partial, ceil_div64(I.n, kBlock), I.red, slot, rotate, 0, 0);
}
__global__ void __launch_bounds__(kBlock) kb_pcg_direction(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                           int nisl, int fr) {
    BATCH_ISLAND
    d_pcg_direction(I.lx, I.ly, I.lz, I.r[(I.rcur + fr) & 1], I.p, I.type, I.red, I.sigma, t_, lb_);
}
__global__ void __launch_bounds__(kBlock) kb_amg_build(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                       int nisl) {
    BATCH_ISLAND
    d_amg_build(I.lx, I.ly, I.lz, I.sigma, I.type, I.agg, I.aw, I.adc, t_);
}
__global__ void __launch_bounds__(kBlock) kb_amg_coarse(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                        int nisl, int fr) {
    BATCH_ISLAND
    d_amg_coarse(I.lx, I.ly, I.lz, I.agg, I.aw, I.adc, I.r[(I.rcur + fr) & 1], I.aec, t_);
}
__global__ void __launch_bounds__(kBlock) kb_amg_prolong(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                         int nisl) {
    BATCH_ISLAND
    d_amg_prolong(I.n, I.agg, I.aw, I.aec, I.phi, t_);
}
__global__ void __launch_bounds__(kBlock) kb_copy_damage(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                         int nisl) {
    BATCH_ISLAND
    if (t_ < I.n) I.Dold[t_] = I.D[t_];
}
__global__ void __launch_bounds__(kBlock) kb_phase_field(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                         int nisl, float l0, float gc, float relax, int split) {
    BATCH_ISLAND
    d_phase_field(I.lx, I.ly, I.lz, I.phi, I.H, I.D, I.Dold, I.sigma, I.type, I.fail, I.hyd, l0, gc, relax, split,
                  t_, lb_);
}
__global__ void __launch_bounds__(kBlock) kb_take_phi(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                      int nisl) {
    BATCH_ISLAND
    if (I.phi_in && t_ < I.n) I.phi[t_] = I.phi_in[t_];
}
__global__ void __launch_bounds__(kBlock) kb_history(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                     int nisl) {
    BATCH_ISLAND
    d_history(I.lx, I.ly, I.lz, I.phi, I.sigma, I.type, I.H, t_);
}
// One pass over the voxels after the phase field: failure code, macro
// residual (per macro block and the island's maximum, the readback of
// island_buffer.cpp:968-1090), the island's phi maximum (SH/phi_reduce_max.comp.glsl,
// the divergence check's input) and the failed voxels of each 256-voxel
// block (the counts the compaction scans).  NaN residuals and NaN phi do not
// enter the island maxima.
__global__ void __launch_bounds__(kBlock) kb_failure_scan(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                          int nisl) {
    BATCH_ISLAND
    float res = -1.0f, ph = -INFINITY;
    uint8_t code = 0;
    if (t_ < I.n) {
        int64_t mb = 0;
        code = d_fail_code(I.lx, I.ly, I.lz, I.phi, I.sigma, I.rcomp, I.type, I.rtens, I.src, kPhiOrphan, t_, res, mb);
        I.fail[t_] = code;
        if (res >= 0.0f || isnan(res)) atomicMax(I.macro + mb, __float_as_uint(res));
        ph = I.phi[t_];
        if (isnan(ph)) ph = -INFINITY;
        if (isnan(res)) res = -1.0f;
    }
    const int failed = __syncthreads_count(code != 0);
    const float mres = block_max(res);
    __syncthreads();
    const float mphi = block_max(ph);
    if (threadIdx.x == 0) {
        I.fcounts[lb_] = failed;
        if (mres >= 0.0f) atomicMax(reinterpret_cast<uint32_t*>(I.res_macro), __float_as_uint(mres));
        if (mphi > -INFINITY) atomicMax(I.res_phimax, float_key(mphi));
    }
}
// one block per island: exclusive scan of the 256-voxel block counts
__global__ void __launch_bounds__(kBlock) kb_fail_scan(const CIsl* __restrict__ tab) {
    const CIsl& I = tab[blockIdx.x];
    d_fail_scan(I.fcounts, ceil_div64(I.n, kBlock), I.foffsets, I.res_fail, 0, 0);
}
// {x, y, z, code} tuples of one 256-voxel block at its scanned offset, in
// voxel order; tuples at or beyond the island's capacity are dropped.
__global__ void __launch_bounds__(kBlock) kb_fail_write(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                        int nisl) {
    BATCH_ISLAND
    __shared__ int32_t warp_cnt[kBlock / 32];
    const uint8_t f = t_ < I.n ? I.fail[t_] : 0;
    const unsigned ballot = __ballot_sync(0xffffffffu, f != 0);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_cnt[w] = __popc(ballot);
    __syncthreads();
    int before = 0;
    for (int q = 0; q < w; q++) before += warp_cnt[q];
    const int64_t pos = (int64_t)I.foffsets[lb_] + before + __popc(ballot & ((1u << lane) - 1u));
    if (f != 0 && I.tuples && pos < I.tuple_cap) {
        int32_t* t = I.tuples + 4 * pos;
        t[0] = I.ox + (int)(t_ % I.lx);
        t[1] = I.oy + (int)((t_ / I.lx) % I.ly);
        t[2] = I.oz + (int)(t_ / ((int64_t)I.lx * I.ly));
        t[3] = f;
    }
}
// phi into the caller's stress readback buffer (device-visible host memory)
__global__ void __launch_bounds__(kBlock) kb_stress_out(const CIsl* __restrict__ tab, const int* __restrict__ bs,
                                                        int nisl) {
    BATCH_ISLAND
    if (I.h_stress && t_ < I.stress_n) I.h_stress[t_] = I.phi[t_];
}
#undef BATCH_ISLAND

inline unsigned grid_for(int64_t n) { return (unsigned)ceil_div64(n, kBlock); }

}  // namespace

// ============================================================ launchers
namespace compat {

int64_t fail_compact_blocks(int64_t n) { return ceil_div64(n, kCompactChunk); }

int64_t pcg_blocks(int64_t n) { return grid_for(n); }
void fail_compact(cudaStream_t s, const uint8_t* fail, int lx, int ly, int lz, int ox, int oy, int oz,
                  int32_t* counts, int32_t* offsets, int32_t* total, int32_t* tuples, int32_t cap) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t nb = fail_compact_blocks(n);
    k_fail_count<<<(unsigned)nb, kBlock, 0, s>>>(fail, n, counts);
    k_fail_scan<<<1, kBlock, 0, s>>>(counts, nb, offsets, total);
    k_fail_write<<<(unsigned)nb, kBlock, 0, s>>>(fail, lx, ly, lz, ox, oy, oz, offsets, tuples, cap);
}

int64_t batch_blocks(const CIsl& I, int kind) {
    if (kind == kbN) return ceil_div64(I.n, kBlock);
    if (kind >= kbC0 && kind < kbC0 + 8) {
        const int c = kind - kbC0;
        const int cx = c & 1, cy = (c >> 1) & 1, cz = (c >> 2) & 1;
        const int64_t nc = (int64_t)((I.lx - cx + 1) >> 1) * ((I.ly - cy + 1) >> 1) * ((I.lz - cz + 1) >> 1);
        return nc > 0 ? ceil_div64(nc, kBlock) : 0;
    }
    if (kind == kbN1) return ceil_div64(I.n1, kBlock);
    if (kind == kbN2) return ceil_div64(I.n2, kBlock);
    if (kind == kbMB) return ceil_div64(I.nmb, kBlock);
    if (kind == kbAG) return ceil_div64(I.anc, kBlock);
    return 0;
}

namespace batch {
namespace {
inline const int* row(const BGroup& g, int kind) { return g.bstart + (int64_t)kind * (g.nisl + 1); }
}  // namespace
#define BLAUNCH(kind, kern, ...)                                                                         \
    do {                                                                                                 \
        if (g.nisl > 0 && g.blocks[kind] > 0)                                                           \
            kern<<<(unsigned)g.blocks[kind], kBlock, 0, s>>>(g.tab, row(g, kind), g.nisl, ##__VA_ARGS__); \
    } while (0)

void upload(cudaStream_t s, const BGroup& g) { BLAUNCH(kbN, kb_upload); }
void macro_fill(cudaStream_t s, const BGroup& g) { BLAUNCH(kbMB, kb_macro_fill); }
void rbgs_color(cudaStream_t s, const BGroup& g, int color, int sidx, int warm, float dampf) {
    BLAUNCH(kbC0 + color, kb_rbgs_color, color, sidx, warm, dampf);
}
void jacobi(cudaStream_t s, const BGroup& g, int level, int flip, int sidx, int warm, float dampf) {
    BLAUNCH(level == 1 ? kbN1 : kbN2, kb_jacobi, level, flip, sidx, warm, dampf);
}
void restrict_to(cudaStream_t s, const BGroup& g, int level, int f1, int f2) {
    BLAUNCH(level == 1 ? kbN1 : kbN2, kb_restrict, level, f1, f2);
}
void prolong_from(cudaStream_t s, const BGroup& g, int level, int f1, int f2) {
    BLAUNCH(level == 1 ? kbN : kbN1, kb_prolong, level, f1, f2);
}
void downsample(cudaStream_t s, const BGroup& g, int level) { BLAUNCH(level == 1 ? kbN1 : kbN2, kb_downsample, level); }
void pcg_precompute(cudaStream_t s, const BGroup& g) { BLAUNCH(kbN, kb_pcg_precompute); }
void pcg_matvec(cudaStream_t s, const BGroup& g, int which) { BLAUNCH(kbN, kb_pcg_matvec, which); }
void pcg_update(cudaStream_t s, const BGroup& g, int is_init, int fr) { BLAUNCH(kbN, kb_pcg_update, is_init, fr); }
void amg_build(cudaStream_t s, const BGroup& g) { BLAUNCH(kbAG, kb_amg_build); }
void amg_coarse(cudaStream_t s, const BGroup& g, int fr) { BLAUNCH(kbAG, kb_amg_coarse, fr); }
void amg_prolong(cudaStream_t s, const BGroup& g) { BLAUNCH(kbN, kb_amg_prolong); }
void finalize(cudaStream_t s, const BGroup& g, int slot, int rotate) {
    if (g.nisl > 0) kb_finalize<<<(unsigned)g.nisl, kBlock, 0, s>>>(g.tab, slot, rotate);
}
void pcg_direction(cudaStream_t s, const BGroup& g, int fr) { BLAUNCH(kbN, kb_pcg_direction, fr); }
void copy_damage(cudaStream_t s, const BGroup& g) { BLAUNCH(kbN, kb_copy_damage); }
void phase_field(cudaStream_t s, const BGroup& g, float l0, float gc, float relax, int split) {
    BLAUNCH(kbN, kb_phase_field, l0, gc, relax, split);
}
void history(cudaStream_t s, const BGroup& g) { BLAUNCH(kbN, kb_history); }
void take_phi(cudaStream_t s, const BGroup& g) { BLAUNCH(kbN, kb_take_phi); }
void failure_scan(cudaStream_t s, const BGroup& g) { BLAUNCH(kbN, kb_failure_scan); }
void fail_compact(cudaStream_t s, const BGroup& g) {
    if (g.nisl > 0) kb_fail_scan<<<(unsigned)g.nisl, kBlock, 0, s>>>(g.tab);
    BLAUNCH(kbN, kb_fail_write);
}
void stress_out(cudaStream_t s, const BGroup& g) { BLAUNCH(kbN, kb_stress_out); }
#undef BLAUNCH
}  // namespace batch

void sparse_scatter(cudaStream_t s, const void* records, int count, int64_t n, float* source, float* cond,
                    uint8_t* type, float* maxphi, float* rcomp, float* rtens) {
    if (count <= 0) return;
    k_sparse_scatter<<<(count + 63) / 64, 64, 0, s>>>((const uint32_t*)records, count, n, source, cond, type, maxphi,
                                                      rcomp, rtens);
}

}  // namespace compat
}  // namespace pfsf_b200
