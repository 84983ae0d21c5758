// Plane-marching fine-level stencil passes for CTA-granular teams (the
// whole-GPU team of giant islands).
//
// The generic ops in kappa_ops.cuh give every thread a strided list of
// voxels and gather each voxel's 26 neighbours from global memory: three
// dependent rounds of L2 latency per voxel and nothing in flight across
// voxels, so a large island's pass runs at a small fraction of HBM
// bandwidth.  Here each CTA takes work items of 32 x 16 columns by ZC planes
// and marches up the planes keeping a 4-plane ring of the input vector and
// the link kappa (with a one-voxel halo, 34 x 18 per plane) in shared
// memory: plane z+2 is fetched into registers while plane z is computed
// from shared memory, then stored into the ring slot plane z-2 used.  One
// thread per column; coalesced 34-wide rows; halo overhead ~1.2x.
//
// Out-of-box neighbours enter the ring as kappa = 0 (link weight 0), air
// voxels carry kappa = 0 already, so the stencil needs no neighbour type or
// bounds test, and its neighbour order (dz, dy, dx ascending, centre
// skipped) is the generic ops' order: results are bitwise those of
// kappa_ops.cuh.
#pragma once
#include "kappa_ops.cuh"

namespace pfsf_b200 {
namespace kappa {
namespace {

constexpr int kMX = 32, kMY = 16;               // columns per work item (= 512 threads)
constexpr int kMHX = kMX + 2, kMHY = kMY + 2;   // with halo
constexpr int kMPlane = kMHX * kMHY;            // 612
constexpr int kMZ = 16;                         // planes per work item

struct MarchTile {
    union {
        float f[4][kMPlane];
        double d[4][kMPlane];
    } v;
    float k[4][kMPlane];
    float pair[kMY / 2 * kMX / 2];  // restriction: y-pair exchange
};

__device__ __forceinline__ int mslot(int z) { return (z + 4) & 3; }

// One plane of the ring: element e of the 34 x 18 halo plane -> global voxel.
template <class V, class VLoad, class KLoad>
__device__ __forceinline__ void mfetch(const Fine& F, int x0, int y0, int z, int e, VLoad vload, KLoad kload, V& v,
                                       float& k) {
    v = V(0);
    k = 0.0f;
    if (e >= kMPlane || z < 0 || z >= F.lz) return;
    const int hy = e / kMHX, hx = e - hy * kMHX;
    const int x = x0 - 1 + hx, y = y0 - 1 + hy;
    if (x < 0 || x >= F.lx || y < 0 || y >= F.ly) return;
    const int g = x + F.lx * (y + F.ly * z);
    v = vload(g);
    k = kload(g);
}

template <class V>
__device__ __forceinline__ V* mplane(MarchTile& S, int slot) {
    if constexpr (sizeof(V) == 8) return reinterpret_cast<V*>(S.v.d[slot]);
    else return reinterpret_cast<V*>(S.v.f[slot]);
}

// March over every work item this CTA owns (cta, cta + ncta, ...).
// body(i, vc, kc, nb) is called for each in-box voxel i of a plane (vc, kc:
// its own vector value and kappa),
// with nb(dx, dy, dz, v, k) giving a neighbour's vector value and kappa.
template <class V, class VLoad, class KLoad, class Body>
__device__ void march(const Fine& F, MarchTile& S, int cta, int ncta, VLoad vload, KLoad kload, Body body) {
    const int tid = threadIdx.x;
    const int tx = tid & (kMX - 1), ty = tid / kMX;
    const int ntx = (F.lx + kMX - 1) / kMX, nty = (F.ly + kMY - 1) / kMY, nzc = (F.lz + kMZ - 1) / kMZ;
    const int nwork = ntx * nty * nzc;
    const int hc = (ty + 1) * kMHX + (tx + 1);
    for (int w = cta; w < nwork; w += ncta) {
        const int x0 = (w % ntx) * kMX, y0 = ((w / ntx) % nty) * kMY, z0 = (w / (ntx * nty)) * kMZ;
        const int z1 = min(z0 + kMZ, F.lz);
        for (int pz = z0 - 1; pz <= z0 + 1; pz++) {
            V a, b;
            float ka, kb;
            mfetch<V>(F, x0, y0, pz, tid, vload, kload, a, ka);
            mfetch<V>(F, x0, y0, pz, tid + 512, vload, kload, b, kb);
            V* pv = mplane<V>(S, mslot(pz));
            float* pk = S.k[mslot(pz)];
            pv[tid] = a;
            pk[tid] = ka;
            if (tid + 512 < kMPlane) {
                pv[tid + 512] = b;
                pk[tid + 512] = kb;
            }
        }
        __syncthreads();
        const int x = x0 + tx, y = y0 + ty;
        const bool col = x < F.lx && y < F.ly;
        for (int z = z0; z < z1; z++) {
            V a, b;
            float ka, kb;
            mfetch<V>(F, x0, y0, z + 2, tid, vload, kload, a, ka);
            mfetch<V>(F, x0, y0, z + 2, tid + 512, vload, kload, b, kb);
            if (col) {
                const V* pm = mplane<V>(S, mslot(z - 1));
                const V* p0 = mplane<V>(S, mslot(z));
                const V* pp = mplane<V>(S, mslot(z + 1));
                const float* km = S.k[mslot(z - 1)];
                const float* k0 = S.k[mslot(z)];
                const float* kp = S.k[mslot(z + 1)];
                auto nb = [&](int dx, int dy, int dz, V& v, float& k) {
                    const int o = hc + dy * kMHX + dx;
                    const V* pv = dz < 0 ? pm : (dz > 0 ? pp : p0);
                    const float* pk = dz < 0 ? km : (dz > 0 ? kp : k0);
                    v = pv[o];
                    k = pk[o];
                };
                body(x + F.lx * (y + F.ly * z), p0[hc], k0[hc], nb);
            }
            V* pv = mplane<V>(S, mslot(z + 2));
            float* pk = S.k[mslot(z + 2)];
            pv[tid] = a;
            pk[tid] = ka;
            if (tid + 512 < kMPlane) {
                pv[tid + 512] = b;
                pk[tid + 512] = kb;
            }
            __syncthreads();
        }
    }
}

// sum over the 26 neighbours in the generic ops' order (dz, dy, dx ascending)
template <class V, class NB, class F>
__device__ __forceinline__ void mfor_nb(NB& nb, F f) {
#pragma unroll
    for (int dz = -1; dz <= 1; dz++)
#pragma unroll
        for (int dy = -1; dy <= 1; dy++)
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                V v;
                float k;
                nb(dx, dy, dz, v, k);
                f(v, k, gscale(dx, dy, dz));
            }
}

// ---- the marching forms of the fine-level stencil ops

// one whole Chebyshev step out of place (op_cheb0_dz)
template <int P>
__device__ void mop_cheb0_dz(const KArena& A, const KDesc& D, MarchTile& S, int cta, int ncta, const float* zin,
                             float* zout, float c1, float c2) {
    const Fine F = fine_view(A, D);
    const float* dinv = A.dinv0 + D.off;
    float* d = A.d0 + D.off;
    march<float>(F, S, cta, ncta, [&](int g) { return zin[g]; }, [&](int g) { return kpre<P>(F, g); },
                 [&](int i, float zi, float ki, auto& nb) {
                     if (F.type[i] != kSolid) {
                         zout[i] = zi;
                         return;
                     }
                     float az = 0.0f;
                     mfor_nb<float>(nb, [&](float zj, float kj, float gs) { az += gs * hm(ki, kj) * (zi - zj); });
                     const float upd = c2 * dinv[i] * (F.r[i] - az);
                     const float dn = c1 == 0.0f ? upd : c1 * d[i] + upd;
                     d[i] = dn;
                     zout[i] = zi + dn;
                 });
}

// q = A p (FP32 kappa); returns this thread's share of p.q
template <class R>
__device__ void mop_matvec(const KArena& A, const KDesc& D, MarchTile& S, int cta, int ncta, R& pq) {
    const Fine F = fine_view(A, D);
    march<float>(F, S, cta, ncta, [&](int g) { return F.p[g]; }, [&](int g) { return F.k32[g]; },
                 [&](int i, float pi, float ki, auto& nb) {
                     if (F.type[i] != kSolid) {
                         F.q[i] = 0.0f;
                         return;
                     }
                     float acc = 0.0f;
                     mfor_nb<float>(nb, [&](float pj, float kj, float gs) { acc += gs * hm(ki, kj) * (pi - pj); });
                     F.q[i] = acc;
                     pq += (R)pi * (R)acc;
                 });
    // voxels outside every work item's columns do not exist; q of air inside
    // the box is written above
}

// r = b - A x (FP64 weights and sums), e = z = 0; accumulates (r.r, b.b)
__device__ void mop_outer_residual(const KArena& A, const KDesc& D, MarchTile& S, int cta, int ncta, double& rr,
                                   double& bb) {
    const Fine F = fine_view(A, D);
    march<double>(F, S, cta, ncta, [&](int g) { return F.x64[g]; }, [&](int g) { return F.k32[g]; },
                  [&](int i, double xi, float kif, auto& nb) {
                      F.e[i] = 0.0f;
                      F.z[i] = 0.0f;
                      if (F.type[i] != kSolid) {
                          F.r[i] = 0.0f;
                          return;
                      }
                      const double ki = kif;
                      double acc = 0.0;
                      mfor_nb<double>(nb, [&](double xj, float kj, float gs) {
                          acc += (double)gs * hm64(ki, (double)kj) * (xi - xj);
                      });
                      const double bi = F.b[i];
                      const double ri = bi - acc;
                      F.r[i] = (float)ri;
                      rr += ri * ri;
                      bb += bi * bi;
                  });
}

// Residual of level 0 (operator A') summed over each 2x2x2 aggregate into
// level 1, x1 = 0.  Work items start on even x, y, z, so every aggregate lies
// in one item: a column adds its two planes, lanes x-pairs by shuffle, warps
// y-pairs through shared memory.  (The summation order differs from
// op_restrict0's child order: equal up to FP32 rounding.)
template <int P>
__device__ void mop_restrict0(const KArena& A, const KDesc& D, MarchTile& S, int cta, int ncta) {
    const Fine F = fine_view(A, D);
    const Coarse C = coarse_view(A, D, 1);
    const int tid = threadIdx.x;
    const int tx = tid & (kMX - 1), ty = tid / kMX;
    const int ntx = (F.lx + kMX - 1) / kMX, nty = (F.ly + kMY - 1) / kMY, nzc = (F.lz + kMZ - 1) / kMZ;
    const int nwork = ntx * nty * nzc;
    const int hc = (ty + 1) * kMHX + (tx + 1);
    auto vload = [&](int g) { return F.z[g]; };
    auto kload = [&](int g) { return kpre<P>(F, g); };
    for (int w = cta; w < nwork; w += ncta) {
        const int x0 = (w % ntx) * kMX, y0 = ((w / ntx) % nty) * kMY, z0 = (w / (ntx * nty)) * kMZ;
        const int z1 = min(z0 + kMZ, F.lz);
        for (int pz = z0 - 1; pz <= z0 + 1; pz++) {
            float a, b, ka, kb;
            mfetch<float>(F, x0, y0, pz, tid, vload, kload, a, ka);
            mfetch<float>(F, x0, y0, pz, tid + 512, vload, kload, b, kb);
            S.v.f[mslot(pz)][tid] = a;
            S.k[mslot(pz)][tid] = ka;
            if (tid + 512 < kMPlane) {
                S.v.f[mslot(pz)][tid + 512] = b;
                S.k[mslot(pz)][tid + 512] = kb;
            }
        }
        __syncthreads();
        const int x = x0 + tx, y = y0 + ty;
        const bool col = x < F.lx && y < F.ly;
        float hold = 0.0f;
        // planes run in pairs; a last unpaired plane (odd lz) pairs with zero
        const int zend = z0 + ((z1 - z0 + 1) & ~1);
        for (int z = z0; z < zend; z++) {
            float a = 0.0f, b = 0.0f, ka = 0.0f, kb = 0.0f;
            if (z < z1) {
                mfetch<float>(F, x0, y0, z + 2, tid, vload, kload, a, ka);
                mfetch<float>(F, x0, y0, z + 2, tid + 512, vload, kload, b, kb);
            }
            float res = 0.0f;
            if (col && z < z1) {
                const int i = x + F.lx * (y + F.ly * z);
                if (F.type[i] == kSolid) {
                    const float* pm = S.v.f[mslot(z - 1)];
                    const float* p0 = S.v.f[mslot(z)];
                    const float* pp = S.v.f[mslot(z + 1)];
                    const float* km = S.k[mslot(z - 1)];
                    const float* k0 = S.k[mslot(z)];
                    const float* kp = S.k[mslot(z + 1)];
                    auto nb = [&](int dx, int dy, int dz, float& v, float& k) {
                        const int o = hc + dy * kMHX + dx;
                        v = (dz < 0 ? pm : (dz > 0 ? pp : p0))[o];
                        k = (dz < 0 ? km : (dz > 0 ? kp : k0))[o];
                    };
                    const float ki = k0[hc], zi = p0[hc];
                    float az = 0.0f;
                    mfor_nb<float>(nb, [&](float zj, float kj, float gs) { az += gs * hm(ki, kj) * (zi - zj); });
                    res = F.r[i] - az;
                }
            }
            if (z < z1) {
                S.v.f[mslot(z + 2)][tid] = a;
                S.k[mslot(z + 2)][tid] = ka;
                if (tid + 512 < kMPlane) {
                    S.v.f[mslot(z + 2)][tid + 512] = b;
                    S.k[mslot(z + 2)][tid + 512] = kb;
                }
            }
            if (((z - z0) & 1) == 0) {
                hold = res;
            } else {
                float s = hold + res;
                s += __shfl_xor_sync(0xffffffffu, s, 1);
                if ((ty & 1) && !(tx & 1)) S.pair[(ty >> 1) * (kMX / 2) + (tx >> 1)] = s;
                __syncthreads();
                if (!(ty & 1) && !(tx & 1)) {
                    s += S.pair[(ty >> 1) * (kMX / 2) + (tx >> 1)];
                    const int cx = (x0 + tx) >> 1, cy = (y0 + ty) >> 1, cz = z >> 1;
                    if (cx < C.lx && cy < C.ly && cz < C.lz) {
                        const int c = cx + C.lx * (cy + C.ly * cz);
                        C.b[c] = s;
                        C.x[c] = 0.0f;
                    }
                }
            }
            __syncthreads();
        }
    }
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
