// Host-side data-assembly primitives of the frozen ABI (pfsf_compute.h).
//
// These run on the caller's thread over caller-owned (Java DirectByteBuffer)
// arrays, exactly like the reference's libpfsf_compute; they feed the
// per-tick solve but are not on the device.  Every function keeps the
// reference's arithmetic order so results are bit-identical to it (the
// library is compiled without FMA contraction).  Flat index everywhere:
// i = x + lx * (y + ly * z); SoA-6 direction order -X,+X,-Y,+Y,-Z,+Z.
//
// Reference semantics followed (project-relative paths):
//   normalize_soa6        L1-native/libpfsf/src/compute/normalize.cpp:37-62
//   apply_wind_bias       L1-native/libpfsf/src/compute/wind_bias.cpp:30-40 (no-op)
//   compute_conductivity  L1-native/libpfsf/src/compute/conductivity.cpp:66-152
//   timoshenko factor     L1-native/libpfsf/src/compute/timoshenko.cpp:26-48
//   wind_pressure_source  L1-native/libpfsf/src/compute/wind_pressure.cpp:19-29
//   compute_arm_map       L1-native/libpfsf/src/compute/arm_map.cpp:30-93
//   arch_factor_map       L1-native/libpfsf/src/compute/arch_factor.cpp:88-185
//   inject_phantom_edges  L1-native/libpfsf/src/compute/phantom_edges.cpp:66-133
//   downsample_2to1       L1-native/libpfsf/src/compute/downsample.cpp:33-98
//   morton / tiled layout L1-native/libpfsf/src/compute/morton.cpp:22-115
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "pfsf/pfsf_compute.h"

namespace {

// Physical constants shared with the Java policy layer
// (L1-native/libpfsf/src/compute/constants.h:14-38).
constexpr float kBlockVolume = 1.0f;
constexpr float kWindBasePressureMPa = 0.5f * 1.225f * 1.2f * 1e-6f;  // rho_air/2 * Cp, MPa
constexpr float kTimoshenkoCap = 10.0f;
constexpr float kNormalizeMin = 1.0f;

struct Box {
    int32_t lx, ly, lz;
    int64_t n;
    Box(int32_t x, int32_t y, int32_t z) : lx(x), ly(y), lz(z), n(int64_t(x) * y * z) {}
    bool valid() const { return lx > 0 && ly > 0 && lz > 0; }
    int64_t at(int32_t x, int32_t y, int32_t z) const { return int64_t(x) + int64_t(lx) * (int64_t(y) + int64_t(ly) * z); }
    bool inside(int32_t x, int32_t y, int32_t z) const {
        return x >= 0 && x < lx && y >= 0 && y < ly && z >= 0 && z < lz;
    }
    void coords(int64_t i, int32_t& x, int32_t& y, int32_t& z) const {
        const int64_t plane = int64_t(lx) * ly;
        z = int32_t(i / plane);
        const int64_t r = i - int64_t(z) * plane;
        y = int32_t(r / lx);
        x = int32_t(r - int64_t(y) * lx);
    }
};

// Face neighbour offsets in SoA-6 order.
constexpr int kFace[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

// Multi-source breadth-first distance over `members`, stepping along the
// given neighbour offsets.  dist must be negative on entry for every voxel
// the search may claim; sources are seeded at 0.
void bfs_distance(const Box& b, const uint8_t* members, const int (*steps)[3], int nsteps,
                  const std::vector<int64_t>& sources, int32_t* dist) {
    std::vector<int64_t> queue;
    queue.reserve(sources.size() + 1024);
    for (int64_t s : sources) {
        dist[s] = 0;
        queue.push_back(s);
    }
    for (size_t head = 0; head < queue.size(); ++head) {
        const int64_t cur = queue[head];
        int32_t x, y, z;
        b.coords(cur, x, y, z);
        const int32_t next = dist[cur] + 1;
        for (int k = 0; k < nsteps; ++k) {
            const int32_t nx = x + steps[k][0], ny = y + steps[k][1], nz = z + steps[k][2];
            if (!b.inside(nx, ny, nz)) continue;
            const int64_t j = b.at(nx, ny, nz);
            if (!members[j] || dist[j] >= 0) continue;
            dist[j] = next;
            queue.push_back(j);
        }
    }
}

constexpr int kHorizontal[4][3] = {{-1, 0, 0}, {1, 0, 0}, {0, 0, -1}, {0, 0, 1}};

// a < b ? a : b, spelled out: with a NaN or a signed zero this differs from
// std::min, and the reference's choice is part of its results.
inline float lesser(float a, float b) { return a < b ? a : b; }

}  // namespace

extern "C" {

PFSF_API void pfsf_normalize_soa6(float* source, float* rcomp, float* rtens, float* conductivity,
                                  const float* /*hydration: reserved by the reference, unused*/, int32_t n,
                                  float* out_sigma_max) {
    if (n <= 0 || !source || !rcomp || !rtens || !conductivity) {
        if (out_sigma_max) *out_sigma_max = 1.0f;
        return;
    }
    const int64_t n6 = 6 * int64_t(n);
    float smax = 1.0f;
    for (int64_t j = 0; j < n6; ++j) smax = conductivity[j] > smax ? conductivity[j] : smax;
    if (smax > kNormalizeMin) {
        const float inv = 1.0f / smax;
        for (int32_t j = 0; j < n; ++j) {
            source[j] *= inv;
            rcomp[j] *= inv;
            rtens[j] *= inv;
        }
        for (int64_t j = 0; j < n6; ++j) conductivity[j] *= inv;
    }
    if (out_sigma_max) *out_sigma_max = smax;
}

// The reference turned the upwind bias into a no-op: scaling opposite faces
// differently makes the operator non-symmetric, which breaks PCG.  Wind acts
// through the source term instead.  Kept as an exported no-op.
PFSF_API void pfsf_apply_wind_bias(float*, int32_t, pfsf_vec3, float) {}

PFSF_API void pfsf_compute_conductivity(float* conductivity, const float* rcomp, const float* rtens,
                                        const uint8_t* type, int32_t lx, int32_t ly, int32_t lz, pfsf_vec3 wind,
                                        float upwind_factor) {
    const Box b(lx, ly, lz);
    if (!conductivity || !rcomp || !rtens || !type || !b.valid()) return;
    const float wind_scale = 1.0f + upwind_factor;
    for (int d = 0; d < 6; ++d) {
        float* out = conductivity + int64_t(d) * b.n;
        const int ox = kFace[d][0], oy = kFace[d][1], oz = kFace[d][2];
        const bool vertical = oy != 0;  // Y is up
        // horizontal step projected on the wind's xz plane
        const float along = float(ox) * wind.x + float(oz) * wind.z;
        for (int32_t z = 0; z < lz; ++z)
            for (int32_t y = 0; y < ly; ++y)
                for (int32_t x = 0; x < lx; ++x) {
                    const int64_t i = b.at(x, y, z);
                    float s = 0.0f;
                    const int32_t nx = x + ox, ny = y + oy, nz = z + oz;
                    if (type[i] != PFSF_VOXEL_AIR && b.inside(nx, ny, nz)) {
                        const int64_t j = b.at(nx, ny, nz);
                        const float base = lesser(rcomp[i], rcomp[j]);
                        if (type[j] != PFSF_VOXEL_AIR && base > 0.0f) {
                            if (vertical) {
                                s = base;
                            } else {
                                const float mean_t = 0.5f * (rtens[i] + rtens[j]);
                                float ratio = mean_t / (base > 1.0f ? base : 1.0f);
                                if (ratio > 1.0f) ratio = 1.0f;
                                s = base * ratio;
                                if (along > 0.0f)
                                    s *= wind_scale;
                                else if (along < 0.0f)
                                    s /= wind_scale;
                                if (!std::isfinite(s)) s = 0.0f;
                            }
                        }
                    }
                    out[i] = s;
                }
    }
}

PFSF_API float pfsf_timoshenko_moment_factor(float b, float h, int32_t arm, float youngs_gpa, float nu) {
    if (arm <= 0 || h <= 0.0f) return 1.0f;
    const float w = std::max(b, 1.0f);
    const float d = std::max(h, 1.0f);
    const float inertia = w * d * d * d / 12.0f;                   // b h^3 / 12
    const float v = std::max(0.0f, std::min(nu, 0.5f));
    const float k_shear = 10.0f * (1.0f + v) / (12.0f + 11.0f * v);  // rectangular section
    const float g_pa = youngs_gpa * 1.0e9f / (2.0f * (1.0f + v));
    const float a = float(arm);
    const float shear = a * a * d / (k_shear * g_pa * inertia + 1.0e-10f) * 1.0e6f;
    return 1.0f + std::min(shear, kTimoshenkoCap);
}

PFSF_API float pfsf_wind_pressure_source(float wind_speed, float density, bool exposed) {
    if (!exposed || wind_speed <= 0.0f || density <= 0.0f) return 0.0f;
    const float q_pa = kWindBasePressureMPa * wind_speed * wind_speed * 1.0e6f;
    return q_pa / (density * kBlockVolume);
}

PFSF_API pfsf_result pfsf_compute_arm_map(const uint8_t* members, const uint8_t* anchors, int32_t lx, int32_t ly,
                                          int32_t lz, int32_t* out_arm) {
    const Box b(lx, ly, lz);
    if (!members || !anchors || !out_arm || !b.valid()) return PFSF_ERROR_INVALID_ARG;
    std::vector<int64_t> seeds;
    for (int64_t i = 0; i < b.n; ++i) {
        out_arm[i] = members[i] ? -1 : 0;
        if (members[i] && anchors[i]) seeds.push_back(i);
    }
    bfs_distance(b, members, kHorizontal, 4, seeds, out_arm);
    for (int64_t i = 0; i < b.n; ++i)
        if (out_arm[i] < 0) out_arm[i] = 0;  // no horizontal path to an anchor
    return PFSF_OK;
}

PFSF_API pfsf_result pfsf_compute_arch_factor_map(const uint8_t* members, const uint8_t* anchors, int32_t lx,
                                                  int32_t ly, int32_t lz, float* out_arch) {
    const Box b(lx, ly, lz);
    if (!members || !anchors || !out_arch || !b.valid()) return PFSF_ERROR_INVALID_ARG;
    std::fill(out_arch, out_arch + b.n, 0.0f);
    std::vector<int64_t> anchor_list;
    for (int64_t i = 0; i < b.n; ++i)
        if (anchors[i] && members[i]) anchor_list.push_back(i);
    if (anchor_list.size() < 2) return PFSF_OK;

    // Group anchors that touch horizontally (flood fill over anchor voxels,
    // groups numbered by their first anchor in flat order).
    std::vector<int32_t> group(size_t(b.n), -1);
    std::vector<std::vector<int64_t>> groups;
    std::vector<int64_t> stack;
    for (int64_t a : anchor_list) {
        if (group[a] >= 0) continue;
        const int32_t g = int32_t(groups.size());
        groups.emplace_back();
        group[a] = g;
        stack.assign(1, a);
        while (!stack.empty()) {
            const int64_t c = stack.back();
            stack.pop_back();
            int32_t x, y, z;
            b.coords(c, x, y, z);
            for (const auto& s : kHorizontal) {
                const int32_t nx = x + s[0], nz = z + s[2];
                if (!b.inside(nx, y, nz)) continue;
                const int64_t j = b.at(nx, y, nz);
                if (anchors[j] && members[j] && group[j] < 0) {
                    group[j] = g;
                    stack.push_back(j);
                }
            }
        }
    }
    if (groups.size() < 2) return PFSF_OK;
    // members of a group in flat order (the BFS seeds their queue in that order)
    for (auto& g : groups) g.clear();
    for (int64_t a : anchor_list) groups[size_t(group[a])].push_back(a);
    // The two largest groups.  Which of several equal-sized groups wins is
    // whatever std::sort's permutation gives for groups listed in
    // first-anchor order (the reference sorts that same sequence with the
    // same comparison), so std::sort is used here too, not a stable sort.
    std::vector<int32_t> order(groups.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = int32_t(k);
    std::sort(order.begin(), order.end(),
              [&](int32_t p, int32_t q) { return groups[size_t(p)].size() > groups[size_t(q)].size(); });

    std::vector<int32_t> da(size_t(b.n), -1), db(size_t(b.n), -1);
    bfs_distance(b, members, kFace, 6, groups[size_t(order[0])], da.data());
    bfs_distance(b, members, kFace, 6, groups[size_t(order[1])], db.data());
    for (int64_t i = 0; i < b.n; ++i) {
        if (!members[i] || da[i] < 0 || db[i] < 0) continue;
        const float fa = float(da[i]), fb = float(db[i]);
        const float lo = std::min(fa, fb), hi = std::max(fa, fb);
        out_arch[i] = hi > 0.0f ? lo / hi : 1.0f;
    }
    return PFSF_OK;
}

// Diagonal neighbour tables.  The injection order is part of the result
// (the first neighbour that reaches a still-empty face slot writes it), so
// both tables keep the Java source builder's order
// (PFSFSourceBuilder.EDGE_OFFSETS / CORNER_OFFSETS).
PFSF_API int32_t pfsf_inject_phantom_edges(const uint8_t* members, float* conductivity, const float* rcomp,
                                           int32_t lx, int32_t ly, int32_t lz, float edge_penalty,
                                           float corner_penalty) {
    static constexpr int8_t kEdge[12][3] = {{1, 1, 0},  {1, -1, 0},  {-1, 1, 0}, {-1, -1, 0},
                                            {1, 0, 1},  {1, 0, -1},  {-1, 0, 1}, {-1, 0, -1},
                                            {0, 1, 1},  {0, 1, -1},  {0, -1, 1}, {0, -1, -1}};
    static constexpr int8_t kCorner[8][3] = {{1, 1, 1},  {1, 1, -1},  {1, -1, 1},  {1, -1, -1},
                                             {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
    const Box b(lx, ly, lz);
    if (!members || !conductivity || !rcomp || !b.valid()) return 0;
    int32_t injected = 0;
    auto put = [&](int64_t self, int64_t nb, int dir, float penalty) {
        float* slot = conductivity + int64_t(dir) * b.n + self;
        if (*slot == 0.0f) {
            *slot = lesser(rcomp[self], rcomp[nb]) * penalty;
            ++injected;
        }
    };
    for (int32_t z = 0; z < lz; ++z)
        for (int32_t y = 0; y < ly; ++y)
            for (int32_t x = 0; x < lx; ++x) {
                const int64_t self = b.at(x, y, z);
                if (!members[self]) continue;
                for (const auto& o : kEdge) {
                    if (!b.inside(x + o[0], y + o[1], z + o[2])) continue;
                    const int64_t nb = b.at(x + o[0], y + o[1], z + o[2]);
                    if (!members[nb]) continue;
                    // the face slot used is the first non-zero axis of the offset
                    const int dir = o[0] ? (o[0] > 0 ? 1 : 0) : o[1] ? (o[1] > 0 ? 3 : 2) : (o[2] > 0 ? 5 : 4);
                    put(self, nb, dir, edge_penalty);
                }
                for (const auto& o : kCorner) {
                    if (!b.inside(x + o[0], y + o[1], z + o[2])) continue;
                    const int64_t nb = b.at(x + o[0], y + o[1], z + o[2]);
                    if (!members[nb]) continue;
                    put(self, nb, o[0] > 0 ? 1 : 0, corner_penalty);  // corners always use the X faces
                }
            }
    return injected;
}

PFSF_API void pfsf_downsample_2to1(const float* fine, const uint8_t* fine_type, int32_t lxf, int32_t lyf,
                                   int32_t lzf, float* coarse, uint8_t* coarse_type) {
    const Box f(lxf, lyf, lzf);
    if (!fine || !coarse || !f.valid()) return;
    const Box c((lxf + 1) / 2, (lyf + 1) / 2, (lzf + 1) / 2);
    for (int32_t zc = 0; zc < c.lz; ++zc)
        for (int32_t yc = 0; yc < c.ly; ++yc)
            for (int32_t xc = 0; xc < c.lx; ++xc) {
                float sum = 0.0f;
                int count = 0, n_anchor = 0, n_solid = 0, n_air = 0;
                for (int dz = 0; dz < 2; ++dz)
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx) {
                            const int32_t x = 2 * xc + dx, y = 2 * yc + dy, z = 2 * zc + dz;
                            if (x >= lxf || y >= lyf || z >= lzf) continue;
                            const int64_t i = f.at(x, y, z);
                            sum += fine[i];
                            ++count;
                            if (fine_type) {
                                const uint8_t t = fine_type[i];
                                n_anchor += t == PFSF_VOXEL_ANCHOR;
                                n_solid += t == PFSF_VOXEL_SOLID;
                                n_air += t != PFSF_VOXEL_ANCHOR && t != PFSF_VOXEL_SOLID;
                            }
                        }
                const int64_t ci = c.at(xc, yc, zc);
                coarse[ci] = count > 0 ? sum / float(count) : 0.0f;
                if (coarse_type) {
                    // majority vote; ties go to the stronger type (anchor > solid > air)
                    uint8_t t = PFSF_VOXEL_AIR;
                    if (n_anchor >= n_solid && n_anchor >= n_air)
                        t = PFSF_VOXEL_ANCHOR;
                    else if (n_solid >= n_air)
                        t = PFSF_VOXEL_SOLID;
                    coarse_type[ci] = t;
                }
            }
}

// Morton (Z-order) code with 10 bits per axis: bit k of x lands at 3k, of y
// at 3k+1, of z at 3k+2.  Spread/gather by the classic magic-mask doubling
// (MortonCode.java:19-56 defines the same code).
static inline uint32_t spread3(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

static inline uint32_t gather3(uint32_t v) {
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030C30C3u;
    v = (v | (v >> 4)) & 0x0300F00Fu;
    v = (v | (v >> 8)) & 0x030000FFu;
    v = (v | (v >> 16)) & 0x3FFu;
    return v;
}

PFSF_API uint32_t pfsf_morton_encode(uint32_t x, uint32_t y, uint32_t z) {
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

PFSF_API void pfsf_morton_decode(uint32_t code, uint32_t* x, uint32_t* y, uint32_t* z) {
    if (x) *x = gather3(code);
    if (y) *y = gather3(code >> 1);
    if (z) *z = gather3(code >> 2);
}

// Re-lays a linear field into 8^3 tiles (tiles in x-fastest order, voxels
// inside a tile in x-fastest order); partial tiles are zero-filled.  Any
// other tile size is a no-op, as in the reference.
PFSF_API void pfsf_tiled_layout_build(const float* linear, int32_t lx, int32_t ly, int32_t lz, int32_t tile,
                                      float* out) {
    const Box b(lx, ly, lz);
    if (!linear || !out || !b.valid() || tile != 8) return;
    constexpr int T = 8, T3 = T * T * T;
    const int32_t tx = (lx + T - 1) / T, ty = (ly + T - 1) / T, tz = (lz + T - 1) / T;
    std::memset(out, 0, size_t(tx) * ty * tz * T3 * sizeof(float));
    for (int32_t z = 0; z < lz; ++z)
        for (int32_t y = 0; y < ly; ++y)
            for (int32_t x = 0; x < lx; ++x) {
                const int64_t t = (int64_t(z / T) * ty + y / T) * tx + x / T;
                const int64_t in = (int64_t(z % T) * T + y % T) * T + x % T;
                out[t * T3 + in] = linear[b.at(x, y, z)];
            }
}

}  // extern "C"
