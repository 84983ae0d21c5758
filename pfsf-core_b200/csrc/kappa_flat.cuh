// Fine-level passes of CTA-granular teams (one CTA, a thread-block cluster,
// the whole GPU): plane-tile marching over per-plane solid-voxel lists, and
// four-wide streaming ops.
//
// The generic ops in kappa_ops.cuh give every thread a strided list of
// voxels and gather each voxel's 26 neighbours from global memory; within
// 64 registers per thread they keep only one plane's loads in flight, so the
// passes are latency bound, and the lanes of air voxels idle through the
// stencil arithmetic of their solid neighbours in the warp.  Here a CTA takes
// a work item of tx x ty columns (kFlatCap cells per plane with the one-voxel
// halo, see flat_tile) by a run of planes and marches up the planes with a
// 4-plane ring of the input vector and of 1/kappa in shared memory: plane
// z+2 is copied by cp.async (no registers) into the slot plane z-2 used
// while plane z is computed.  Plane z is computed only at its solid voxels,
// taken from a list per (tile, plane) built once per solve (flat_lists), so
// every active lane does stencil work.
//
// Link weight.  The harmonic mean is evaluated as kappa_i kappa_j /
// (kappa_i + kappa_j) = 1 / (1/kappa_i + 1/kappa_j), with the reciprocals
// written once per solve (op_rk; rcp.approx: 1/0 = +inf, so an air or
// out-of-box neighbour gets weight 1/(r_i + inf) = 0 with no test), and the 26 terms
// are summed per link class (faces x2, edges x1, corners x1/3).  Results
// equal the generic ops' up to FP32 rounding; both are the same operator.
//
// Invariant relied on: the vectors marched here (z, q, p) are zero on every
// non-solid voxel.  The outer residual zeroes z, p = z + beta p keeps p's
// zeros, and the solve clears q once at its start (team_solve), so the
// passes never write non-solid voxels.
#pragma once
#include "kappa_ops.cuh"

namespace pfsf_b200 {
namespace kappa {
namespace {

// Ring of kFlatRing planes: z-1, z, z+1 in use, z+2 landed or landing,
// planes up to z + kFlatAhead in flight (plane z + kFlatAhead issued at step
// z).  Measured on the 4096-island solve: 4 slots 333 ms, 5 slots 344 ms,
// 6 slots 368 ms -- the shared memory of two CTAs per SM comes out of the
// L1 that the rest of the solve relies on.
#ifndef PFSF_FLAT_RING
#define PFSF_FLAT_RING 4
#endif
constexpr int kFlatRing = PFSF_FLAT_RING;
constexpr int kFlatAhead = kFlatRing - 2;
static_assert(kFlatRing >= 4, "three planes in use and one landing");
struct FlatSmem {
    float v[kFlatRing][kFlatCap];  // vector ring
    float w[kFlatRing][kFlatCap];  // 1/kappa ring
};

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ int fslot(int z) { return (z + kFlatRing) % kFlatRing; }

// 4-byte global -> shared copies that bypass registers (completion per
// thread by commit groups; a CTA barrier after the wait publishes them)
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

struct FlatGeom {
    int tx, ty, hx, hp, ntx, ntiles, zc, nwork;
};
// Tiles of the island, and work items of zc planes: the whole depth for a
// single-CTA team; when ncta CTAs share the island, the run length that
// minimises rounds x (zc + 3) plane steps for the busiest CTA (a work item
// re-reads 3 planes), over runs of about kFlatZ / 2 planes and more.  zc is
// even, so plane pairs of one aggregate stay together.
__device__ __forceinline__ FlatGeom flat_geom(const KDesc& D, int ncta) {
    FlatGeom G;
    flat_tile(D.lx, D.ly, G.tx, G.ty);
    G.hx = G.tx + 2;
    G.hp = G.hx * (G.ty + 2);
    G.ntx = (D.lx + G.tx - 1) / G.tx;
    G.ntiles = G.ntx * ((D.ly + G.ty - 1) / G.ty);
    if (ncta == 1) {
        G.zc = D.lz;
    } else {
        int best = 0x7fffffff;
        G.zc = kFlatZ;
        const int nzmax = max(1, D.lz / (kFlatZ / 2));
        for (int nz = 1; nz <= nzmax; nz++) {
            const int c = max(2, (((D.lz + nz - 1) / nz) + 1) & ~1);
            const int rounds = (G.ntiles * ((D.lz + c - 1) / c) + ncta - 1) / ncta;
            const int cost = rounds * (c + 3);
            if (cost < best) {
                best = cost;
                G.zc = c;
            }
        }
    }
    G.nwork = G.ntiles * ((D.lz + G.zc - 1) / G.zc);
    return G;
}

struct FlatPlanes {
    const float *vm, *v0, *vp, *wm, *w0, *wp;
    float* spare;  // the vector slot of plane z-1: free once this step's stencils have read it
};

// 26-neighbour sum of w_ij (z_i - z_j) at halo cell hc
__device__ __forceinline__ float flat_az(const FlatPlanes& P, int hc, int hx, float zi, float ri) {
    float af = 0.0f, ae = 0.0f, ac = 0.0f;
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
#pragma unroll
        for (int dy = -1; dy <= 1; dy++)
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                const int o = hc + dy * hx + dx;
                const float zj = (dz < 0 ? P.vm : (dz > 0 ? P.vp : P.v0))[o];
                const float rj = (dz < 0 ? P.wm : (dz > 0 ? P.wp : P.w0))[o];
                const float t = rcp_approx(ri + rj) * (zi - zj);
                const int g = (dx != 0) + (dy != 0) + (dz != 0);
                if (g == 1) af += t;
                else if (g == 2) ae += t;
                else ac += t;
            }
    return 2.0f * af + ae + (1.0f / 3.0f) * ac;
}

// This thread's entries of one (tile, plane) solid list (bounds b0, b1):
// at most kFlatCap / kFlatThreads, ~0u past the end.
__device__ __forceinline__ void flat_entries(const uint32_t* L, int b0, int b1,
                                             uint32_t (&e)[kFlatCap / kFlatThreads]) {
#pragma unroll
    for (int k = 0; k < kFlatCap / kFlatThreads; k++) {
        const int j = b0 + (int)threadIdx.x + kFlatThreads * k;
        e[k] = j < b1 ? L[j] : ~0u;
    }
}

// March over every work item this CTA owns (cta, cta + ncta, ...).
// body(tile, x0, y0, z, z0, z1, planes, entries) runs on every thread once
// per plane (it may hold CTA barriers); vsrc and wsrc are the island's
// vector and 1/kappa arrays.  The planes stream into a shared-memory ring by
// cp.async three planes ahead of the one computed, so a plane step waits on
// no global load of its own (out-of-box cells are stored directly: vector 0,
// 1/kappa +inf, which gives their links weight 0).  With kList the march
// also pipelines the solid lists (L, st): entries of plane z+1 and the list
// bounds of plane z+2 load while plane z is computed.
template <bool kList, class Body>
__device__ void flat_march(const KDesc& D, const FlatGeom& G, FlatSmem& S, int cta, int ncta, const uint32_t* L,
                           const int* st, const float* vsrc, const float* wsrc, Body body) {
    constexpr int J = kFlatCap / kFlatThreads;
    const int tid = threadIdx.x;
    const int lxly = D.lx * D.ly;
    for (int w = cta; w < G.nwork; w += ncta) {
        const int tile = w % G.ntiles, zk = w / G.ntiles;
        const int x0 = (tile % G.ntx) * G.tx, y0 = (tile / G.ntx) * G.ty;
        const int z0 = zk * G.zc, z1 = min(z0 + G.zc, D.lz);
        // this thread's cells of the halo plane: column index in the island,
        // -1 outside the island's box, -2 past the plane
        int col[J];
#pragma unroll
        for (int j = 0; j < J; j++) {
            const int e = tid + kFlatThreads * j;
            col[j] = -2;
            if (e < G.hp) {
                const int hy = e / G.hx, hx = e - hy * G.hx;
                const int x = x0 - 1 + hx, y = y0 - 1 + hy;
                col[j] = (x < 0 || x >= D.lx || y < 0 || y >= D.ly) ? -1 : x + D.lx * y;
            }
        }
        auto issue = [&](int z) {
            float* vs = S.v[fslot(z)];
            float* ws = S.w[fslot(z)];
            const bool inz = z >= 0 && z < D.lz;
#pragma unroll
            for (int j = 0; j < J; j++) {
                const int e = tid + kFlatThreads * j;
                if (col[j] == -2) continue;
                if (col[j] < 0 || !inz) {
                    vs[e] = 0.0f;
                    ws[e] = __int_as_float(0x7f800000);
                } else {
                    const int g = col[j] + lxly * z;
                    cp_async4(vs + e, vsrc + g);
                    cp_async4(ws + e, wsrc + g);
                }
            }
            cp_async_commit();
        };
        uint32_t cur[J], nxt[J];
        int nb0 = 0, nb1 = 0;  // list bounds of plane z+1 (then z+2)
        if constexpr (kList) {
            const int p = tile * D.lz + z0;
            flat_entries(L, st[p], st[p + 1], cur);
            if (z0 + 1 < z1) {
                nb0 = st[p + 1];
                nb1 = st[p + 2];
            }
        }
        for (int pz = z0 - 1; pz < z0 + kFlatAhead; pz++) issue(pz);
        cp_async_wait<kFlatAhead - 2>();  // planes z0-1 .. z0+1 landed
        __syncthreads();
        for (int z = z0; z < z1; z++) {
            issue(z + kFlatAhead);  // into the slot of plane z-2, last read in step z-1
            if constexpr (kList) {
                flat_entries(L, nb0, nb1, nxt);
                const int p2 = tile * D.lz + z + 2;
                nb0 = z + 2 < z1 ? st[p2] : 0;
                nb1 = z + 2 < z1 ? st[p2 + 1] : 0;
            }
            const FlatPlanes P{S.v[fslot(z - 1)], S.v[fslot(z)], S.v[fslot(z + 1)],
                               S.w[fslot(z - 1)], S.w[fslot(z)], S.w[fslot(z + 1)], S.v[fslot(z - 1)]};
            body(tile, x0, y0, z, z0, z1, P, cur);
            if constexpr (kList) {
#pragma unroll
                for (int j = 0; j < J; j++) cur[j] = nxt[j];
            }
            cp_async_wait<kFlatAhead - 2>();  // plane z+2 landed (later ones may still be in flight)
            __syncthreads();
        }
        cp_async_wait<0>();  // nothing in flight into the ring past this work item
        __syncthreads();
    }
}

// 1/kappa of every voxel of the island, for the marching passes (the values
// they staged per plane before: rcp.approx of the preconditioner's kappa and
// of the FP32 kappa, +inf on air)
template <int P>
__device__ void op_rk(const KArena& A, const KDesc& D, int t, int T) {
    const Fine F = fine_view(A, D);
    float* rkp = A.rkp + D.off;
    float* rk32 = A.rk32 + D.off;
    for (int i = t; i < F.n; i += T) {
        rkp[i] = rcp_approx(kpre<P>(F, i));
        rk32[i] = rcp_approx(F.k32[i]);
    }
}

// ---- the per-(tile, plane) solid lists

// Builds the island's lists: counts per (tile, plane), an inclusive scan by
// the team's first CTA, then each (tile, plane) writes its solid columns in
// column order (deterministic).  Ends with a team barrier.
template <class TeamT>
__device__ void flat_lists(const KArena& A, const KDesc& D, FlatSmem& S, TeamT& tm) {
    const FlatGeom G = flat_geom(D, 1);
    const int m = G.ntiles * D.lz, cells = G.tx * G.ty;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint8_t* type = A.type + D.off;
    int* st = A.fstart + D.soff;
    uint32_t* L = A.flist + D.off;
    int* sm = reinterpret_cast<int*>(S.v[0]);  // no march in progress
    auto solid_at = [&](int p, int c, uint32_t& pc) {
        const int tile = p / D.lz, z = p - tile * D.lz;
        const int cy = c / G.tx, cx = c - cy * G.tx;
        const int x = (tile % G.ntx) * G.tx + cx, y = (tile / G.ntx) * G.ty + cy;
        pc = (uint32_t)cx | ((uint32_t)cy << 16);
        return c < cells && x < D.lx && y < D.ly && type[x + D.lx * (y + D.ly * z)] == kSolid;
    };
    for (int p = tm.cta(); p < m; p += tm.ncta()) {
        int cnt = 0;
        for (int c0 = 0; c0 < cells; c0 += kFlatThreads) {
            uint32_t pc;
            cnt += __syncthreads_count(solid_at(p, c0 + tid, pc));
        }
        if (tid == 0) st[p + 1] = cnt;
    }
    tm.sync();
    if (tm.cta() == 0) {
        int carry = 0;
        for (int c0 = 0; c0 < m; c0 += kFlatThreads) {
            const int k = c0 + tid;
            int v = k < m ? st[k + 1] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += u;
            }
            if (lane == 31) sm[wid] = v;
            __syncthreads();
            if (wid == 0) {
                int s = lane < kFlatThreads / 32 ? sm[lane] : 0;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, s, o);
                    if (lane >= o) s += u;
                }
                if (lane < kFlatThreads / 32) sm[32 + lane] = s;
            }
            __syncthreads();
            v += carry + (wid > 0 ? sm[32 + wid - 1] : 0);
            if (k < m) st[k + 1] = v;
            carry += sm[32 + kFlatThreads / 32 - 1];
            __syncthreads();
        }
        if (tid == 0) st[0] = 0;
    }
    tm.sync();
    for (int p = tm.cta(); p < m; p += tm.ncta()) {
        int base = st[p];
        for (int c0 = 0; c0 < cells; c0 += kFlatThreads) {
            uint32_t pc;
            const bool s = solid_at(p, c0 + tid, pc);
            const unsigned ball = __ballot_sync(0xffffffffu, s);
            if (lane == 0) sm[wid] = __popc(ball);
            __syncthreads();
            int off = base + __popc(ball & ((1u << lane) - 1u));
            int total = 0;
            for (int k = 0; k < kFlatThreads / 32; k++) {
                const int c = sm[k];
                off += k < wid ? c : 0;
                total += c;
            }
            if (s) L[off] = pc;
            base += total;
            __syncthreads();
        }
    }
    tm.sync();
}

// ---- the marching forms of the fine-level stencil ops

// one whole Chebyshev step out of place (op_cheb0_dz), solid voxels only
template <int P>
__device__ void fop_cheb0_dz(const KArena& A, const KDesc& D, FlatSmem& S, int cta, int ncta, const float* zin,
                             float* zout, float c1, float c2) {
    const Fine F = fine_view(A, D);
    const float* dinv = A.dinv0 + D.off;
    float* d = A.d0 + D.off;
    const uint32_t* L = A.flist + D.off;
    const int* st = A.fstart + D.soff;
    const FlatGeom G = flat_geom(D, ncta);
    flat_march<true>(D, G, S, cta, ncta, L, st, zin, A.rkp + D.off,
                     [&](int, int x0, int y0, int z, int, int, const FlatPlanes& Pl, const uint32_t(&ent)[kFlatCap / kFlatThreads]) {
#pragma unroll
                         for (int k = 0; k < kFlatCap / kFlatThreads; k++) {
                             const uint32_t pc = ent[k];
                             if (pc == ~0u) break;
                             const int cx = (int)(pc & 0xffffu), cy = (int)(pc >> 16);
                             const int i = x0 + cx + F.lx * (y0 + cy + F.ly * z);
                             const int hc = (cy + 1) * G.hx + cx + 1;
                             const float zi = Pl.v0[hc];
                             const float az = flat_az(Pl, hc, G.hx, zi, Pl.w0[hc]);
                             const float upd = c2 * dinv[i] * (F.r[i] - az);
                             const float dn = c1 == 0.0f ? upd : c1 * d[i] + upd;
                             d[i] = dn;
                             zout[i] = zi + dn;
                         }
                     });
}

// q = A p (FP32 kappa) at solid voxels; returns this thread's share of p.q
template <class R>
__device__ void fop_matvec(const KArena& A, const KDesc& D, FlatSmem& S, int cta, int ncta, R& pq) {
    const Fine F = fine_view(A, D);
    const uint32_t* L = A.flist + D.off;
    const int* st = A.fstart + D.soff;
    const FlatGeom G = flat_geom(D, ncta);
    flat_march<true>(D, G, S, cta, ncta, L, st, F.p, A.rk32 + D.off,
                     [&](int, int x0, int y0, int z, int, int, const FlatPlanes& Pl, const uint32_t(&ent)[kFlatCap / kFlatThreads]) {
#pragma unroll
                         for (int k = 0; k < kFlatCap / kFlatThreads; k++) {
                             const uint32_t pc = ent[k];
                             if (pc == ~0u) break;
                             const int cx = (int)(pc & 0xffffu), cy = (int)(pc >> 16);
                             const int i = x0 + cx + F.lx * (y0 + cy + F.ly * z);
                             const int hc = (cy + 1) * G.hx + cx + 1;
                             const float pi = Pl.v0[hc];
                             const float acc = flat_az(Pl, hc, G.hx, pi, Pl.w0[hc]);
                             F.q[i] = acc;
                             pq += (R)pi * (R)acc;
                         }
                     });
}

// Residual of level 0 (operator A') summed over each 2x2x2 aggregate into
// level 1, x1 = 0.  Every column of the tile, solid or not, keeps one thread
// for the whole march: plane pairs add in registers, then the 2 x 2 column
// groups through the vector slot of plane z-1 (no longer needed once the
// plane's stencils are done).  Tiles and work items start on even x, y, z,
// so every aggregate lies in one work item.  (Summation order differs from
// op_restrict0's child order: equal up to FP32 rounding.)
template <int P>
__device__ void fop_restrict0(const KArena& A, const KDesc& D, FlatSmem& S, int cta, int ncta) {
    constexpr int J = kFlatCap / kFlatThreads;
    const Fine F = fine_view(A, D);
    const Coarse C = coarse_view(A, D, 1);
    const FlatGeom G = flat_geom(D, ncta);
    const int tid = threadIdx.x, cells = G.tx * G.ty;
    const int ctx = (G.tx + 1) >> 1, cty = (G.ty + 1) >> 1;
    int cxj[J], cyj[J];
#pragma unroll
    for (int j = 0; j < J; j++) {
        const int c = tid + kFlatThreads * j;
        cyj[j] = c / G.tx;
        cxj[j] = c - cyj[j] * G.tx;
    }
    float hold[J];
    flat_march<false>(D, G, S, cta, ncta, nullptr, nullptr, F.z, A.rkp + D.off,
                      [&](int, int x0, int y0, int z, int z0, int z1, const FlatPlanes& Pl,
                          const uint32_t(&)[kFlatCap / kFlatThreads]) {
                   const bool second = ((z - z0) & 1) != 0;
#pragma unroll
                   for (int j = 0; j < J; j++) {
                       const int c = tid + kFlatThreads * j;
                       const int x = x0 + cxj[j], y = y0 + cyj[j];
                       float res = 0.0f;
                       if (c < cells && x < F.lx && y < F.ly) {
                           const int i = x + F.lx * (y + F.ly * z);
                           if (F.type[i] == kSolid) {
                               const int hc = (cyj[j] + 1) * G.hx + cxj[j] + 1;
                               const float zi = Pl.v0[hc];
                               res = F.r[i] - flat_az(Pl, hc, G.hx, zi, Pl.w0[hc]);
                           }
                       }
                       hold[j] = second ? hold[j] + res : res;
                   }
                   if (!second && z != z1 - 1) return;
                   __syncthreads();  // every stencil of this plane has read plane z-1
#pragma unroll
                   for (int j = 0; j < J; j++) {
                       const int c = tid + kFlatThreads * j;
                       if (c < cells) Pl.spare[c] = hold[j];
                   }
                   __syncthreads();
                   const int gz = z >> 1;
                   for (int cc = tid; cc < ctx * cty; cc += kFlatThreads) {
                       const int ccy = cc / ctx, ccx = cc - ccy * ctx;
                       float s = 0.0f;
#pragma unroll
                       for (int dy = 0; dy < 2; dy++)
#pragma unroll
                           for (int dx = 0; dx < 2; dx++) {
                               const int ux = 2 * ccx + dx, uy = 2 * ccy + dy;
                               if (ux < G.tx && uy < G.ty) s += Pl.spare[uy * G.tx + ux];
                           }
                       const int gx = (x0 >> 1) + ccx, gy = (y0 >> 1) + ccy;
                       if (gx < C.lx && gy < C.ly && gz < C.lz) {
                           const int c = gx + C.lx * (gy + C.ly * gz);
                           C.b[c] = s;
                           C.x[c] = 0.0f;
                       }
                   }
                   __syncthreads();  // the slot is refilled by the next step's copies
               });
}

// ---- streaming ops, four voxels per access (island arrays start 128-byte aligned)
template <class R>
__device__ void vop_update(const KArena& A, const KDesc& D, int t, int T, float alpha, R& rr) {
    const Fine F = fine_view(A, D);
    const int n4 = F.n >> 2;
    float4* r4 = reinterpret_cast<float4*>(F.r);
    float4* e4 = reinterpret_cast<float4*>(F.e);
    const float4* q4 = reinterpret_cast<const float4*>(F.q);
    const float4* p4 = reinterpret_cast<const float4*>(F.p);
    for (int j = t; j < n4; j += T) {
        float4 r = r4[j], e = e4[j];
        const float4 q = q4[j], p = p4[j];
        r.x -= alpha * q.x; r.y -= alpha * q.y; r.z -= alpha * q.z; r.w -= alpha * q.w;
        e.x += alpha * p.x; e.y += alpha * p.y; e.z += alpha * p.z; e.w += alpha * p.w;
        r4[j] = r;
        e4[j] = e;
        rr += (R)r.x * (R)r.x + (R)r.y * (R)r.y + (R)r.z * (R)r.z + (R)r.w * (R)r.w;
    }
    for (int i = 4 * n4 + t; i < F.n; i += T) {
        const float ri = F.r[i] - alpha * F.q[i];
        F.e[i] += alpha * F.p[i];
        F.r[i] = ri;
        rr += (R)ri * (R)ri;
    }
}

template <class R>
__device__ void vop_dot_rz(const KArena& A, const KDesc& D, int t, int T, R& rz) {
    const Fine F = fine_view(A, D);
    const int n4 = F.n >> 2;
    const float4* r4 = reinterpret_cast<const float4*>(F.r);
    const float4* z4 = reinterpret_cast<const float4*>(F.z);
    for (int j = t; j < n4; j += T) {
        const float4 r = r4[j], z = z4[j];
        rz += (R)r.x * (R)z.x + (R)r.y * (R)z.y + (R)r.z * (R)z.z + (R)r.w * (R)z.w;
    }
    for (int i = 4 * n4 + t; i < F.n; i += T) rz += (R)F.r[i] * (R)F.z[i];
}

__device__ void vop_pupdate(const KArena& A, const KDesc& D, int t, int T, float beta) {
    const Fine F = fine_view(A, D);
    const int n4 = F.n >> 2;
    float4* p4 = reinterpret_cast<float4*>(F.p);
    float4* z4 = reinterpret_cast<float4*>(F.z);
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int j = t; j < n4; j += T) {
        const float4 z = z4[j];
        float4 p;
        if (beta == 0.0f) {
            p = z;
        } else {
            p = p4[j];
            p.x = z.x + beta * p.x; p.y = z.y + beta * p.y; p.z = z.z + beta * p.z; p.w = z.w + beta * p.w;
        }
        p4[j] = p;
        z4[j] = zero;
    }
    for (int i = 4 * n4 + t; i < F.n; i += T) {
        const float zi = F.z[i];
        F.p[i] = beta == 0.0f ? zi : zi + beta * F.p[i];
        F.z[i] = 0.0f;
    }
}

// zout: F.z or the q array (both island arrays, 128-byte aligned)
__device__ void vop_cheb0_first(const KArena& A, const KDesc& D, int t, int T, float c2, float* zout) {
    const Fine F = fine_view(A, D);
    const int n4 = F.n >> 2;
    const float4* dv4 = reinterpret_cast<const float4*>(A.dinv0 + D.off);
    const float4* r4 = reinterpret_cast<const float4*>(F.r);
    float4* d4 = reinterpret_cast<float4*>(A.d0 + D.off);
    float4* z4 = reinterpret_cast<float4*>(zout);
    for (int j = t; j < n4; j += T) {
        const float4 dv = dv4[j], r = r4[j];
        const float4 v = make_float4(c2 * dv.x * r.x, c2 * dv.y * r.y, c2 * dv.z * r.z, c2 * dv.w * r.w);
        d4[j] = v;
        z4[j] = v;
    }
    const float* dinv = A.dinv0 + D.off;
    float* d = A.d0 + D.off;
    for (int i = 4 * n4 + t; i < F.n; i += T) {
        const float v = c2 * dinv[i] * F.r[i];
        d[i] = v;
        zout[i] = v;
    }
}

__device__ void vop_zero(int t, int T, int n, float* dst) {
    const int n4 = n >> 2;
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (int j = t; j < n4; j += T) d4[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int i = 4 * n4 + t; i < n; i += T) dst[i] = 0.0f;
}

__device__ void vop_copy(int t, int T, int n, const float* src, float* dst) {
    const int n4 = n >> 2;
    const float4* s4 = reinterpret_cast<const float4*>(src);
    float4* d4 = reinterpret_cast<float4*>(dst);
    for (int j = t; j < n4; j += T) d4[j] = s4[j];
    for (int i = 4 * n4 + t; i < n; i += T) dst[i] = src[i];
}

__device__ void vop_accumulate(const KArena& A, const KDesc& D, int t, int T) {
    const Fine F = fine_view(A, D);
    const int n4 = F.n >> 2;
    const float4* e4 = reinterpret_cast<const float4*>(F.e);
    double2* x2 = reinterpret_cast<double2*>(F.x64);
    for (int j = t; j < n4; j += T) {
        const float4 e = e4[j];
        double2 a = x2[2 * j], b = x2[2 * j + 1];
        a.x += (double)e.x; a.y += (double)e.y; b.x += (double)e.z; b.y += (double)e.w;
        x2[2 * j] = a;
        x2[2 * j + 1] = b;
    }
    for (int i = 4 * n4 + t; i < F.n; i += T) F.x64[i] += (double)F.e[i];
}

}  // namespace
}  // namespace kappa
}  // namespace pfsf_b200
