// Extension surface of the frozen ABI: version/feature discovery,
// the per-island augmentation registry and hook table, the element-wise
// augmentation updates, and the tick-plan opcode interpreter that strings
// the host primitives together in one call.
//
// Reference semantics followed (project-relative paths):
//   version / features   L1-native/libpfsf/src/compute/version.cpp:20-113
//   augmentation table   L1-native/libpfsf/src/ext/augmentation.cpp:27-151
//   hook table           L1-native/libpfsf/src/ext/hooks.cpp:22-105
//   augmentation updates L1-native/libpfsf/src/compute/aug_kernels.cpp:40-125
//   plan interpreter     L1-native/libpfsf/src/ext/plan_dispatcher.cpp:174-896
//   plan binary format   L1-native/libpfsf/include/pfsf/pfsf_plan.h:14-31
#include <array>
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <shared_mutex>
#include <unordered_map>
#include <utility>

#include "pfsf/pfsf_compute.h"
#include "pfsf/pfsf_diagnostics.h"
#include "pfsf/pfsf_extension.h"
#include "pfsf/pfsf_plan.h"
#include "pfsf/pfsf_trace.h"
#include "pfsf/pfsf_version.h"

// ─── version and feature flags ──────────────────────────────────────────────

namespace {

// Features this library reports true.  The first block is what the frozen
// ABI requires (its feature_flags_required_true list plus the POSIX crash
// handler); the second block names this build's additions.
const char* const kFeatures[] = {
    "compute.v1", "compute.v2", "compute.v3", "compute.v4", "compute.v5", "compute.v6", "compute.v7",
    "compute.v8", "diagnostics.v1", "extension.v1", "plan.v1", "plan.v1.1", "plan_buffer", "trace.ring",
    "abi.v1", "crash.handler", "crash.handler.test",
    // additions
    "cuda.sm100", "solve.tolerance", "solve.batched", "precision.bf16", "precision.fp16", "compact.noalloc",
};

}  // namespace

extern "C" {

// The reference's internal phase counter 0.10.0; the externally checked
// contract is pfsf_abi_contract_version().
PFSF_API uint32_t pfsf_abi_version(void) { return (0u << 16) | (10u << 8) | 0u; }

PFSF_API bool pfsf_has_feature(const char* name) {
    if (!name) return false;
    for (const char* f : kFeatures)
        if (std::strcmp(f, name) == 0) return true;
    return false;
}

PFSF_API const char* pfsf_build_info(void) { return "libpfsf b200 (cuda sm_100a, host scalar)"; }

PFSF_API const char* pfsf_abi_contract_version(void) { return "1.5.0"; }

}  // extern "C"

// ─── augmentation registry ──────────────────────────────────────────────────

namespace {

constexpr int kAugKinds = 9;  // PFSF_AUG_THERMAL_FIELD (1) .. PFSF_AUG_LOADPATH_HINT (9)

struct AugTable {
    std::array<pfsf_aug_slot, kAugKinds + 1> slot{};  // indexed by kind; [0] unused
    std::array<bool, kAugKinds + 1> used{};
    int32_t count = 0;
};

std::shared_mutex g_aug_mu;
std::unordered_map<int32_t, AugTable> g_aug;

bool aug_kind_ok(int32_t k) { return k >= 1 && k <= kAugKinds; }

struct HookTable {
    pfsf_hook_fn fn[PFSF_HOOK_POINT_COUNT] = {};
    void* ud[PFSF_HOOK_POINT_COUNT] = {};
};

std::shared_mutex g_hook_mu;
std::unordered_map<int32_t, HookTable> g_hooks;

bool hook_point_ok(int32_t p) { return p >= 0 && p < PFSF_HOOK_POINT_COUNT; }

}  // namespace

extern "C" {

PFSF_API pfsf_result pfsf_aug_register(int32_t island_id, const pfsf_aug_slot* slot) {
    if (!slot || !aug_kind_ok(int32_t(slot->kind))) return PFSF_ERROR_INVALID_ARG;
    // a caller struct must reach at least through `version`; a larger
    // (future) struct is truncated to ours, a non-positive size means ours
    const int32_t need = int32_t(offsetof(pfsf_aug_slot, version) + sizeof(int32_t));
    if (slot->struct_bytes > 0 && slot->struct_bytes < need) return PFSF_ERROR_INVALID_ARG;
    pfsf_aug_slot copy{};
    size_t take = sizeof(pfsf_aug_slot);
    if (slot->struct_bytes > 0 && size_t(slot->struct_bytes) < take) take = size_t(slot->struct_bytes);
    std::memcpy(&copy, slot, take);
    copy.struct_bytes = int32_t(sizeof(pfsf_aug_slot));
    std::unique_lock<std::shared_mutex> lk(g_aug_mu);
    AugTable& t = g_aug[island_id];
    const int k = int(copy.kind);
    if (!t.used[k]) {
        t.used[k] = true;
        ++t.count;
    }
    t.slot[k] = copy;
    return PFSF_OK;
}

PFSF_API void pfsf_aug_clear(int32_t island_id, pfsf_augmentation_kind kind) {
    if (!aug_kind_ok(int32_t(kind))) return;
    std::unique_lock<std::shared_mutex> lk(g_aug_mu);
    auto it = g_aug.find(island_id);
    if (it == g_aug.end()) return;
    AugTable& t = it->second;
    if (t.used[kind]) {
        t.used[kind] = false;
        t.slot[kind] = pfsf_aug_slot{};
        --t.count;
    }
    if (t.count <= 0) g_aug.erase(it);
}

PFSF_API void pfsf_aug_clear_island(int32_t island_id) {
    std::unique_lock<std::shared_mutex> lk(g_aug_mu);
    g_aug.erase(island_id);
}

PFSF_API int32_t pfsf_aug_query(int32_t island_id, pfsf_augmentation_kind kind, pfsf_aug_slot* out) {
    if (!out || !aug_kind_ok(int32_t(kind))) return 0;
    std::shared_lock<std::shared_mutex> lk(g_aug_mu);
    auto it = g_aug.find(island_id);
    if (it == g_aug.end() || !it->second.used[kind]) return 0;
    *out = it->second.slot[kind];
    return 1;
}

PFSF_API int32_t pfsf_aug_island_count(int32_t island_id) {
    std::shared_lock<std::shared_mutex> lk(g_aug_mu);
    auto it = g_aug.find(island_id);
    return it == g_aug.end() ? 0 : it->second.count;
}

// Engine-handle forms: the registry is process-global, the handle is ignored.
PFSF_API pfsf_result pfsf_register_augmentation(pfsf_engine, int32_t island_id, const pfsf_aug_slot* slot) {
    return pfsf_aug_register(island_id, slot);
}

PFSF_API void pfsf_clear_augmentation(pfsf_engine, int32_t island_id, pfsf_augmentation_kind kind) {
    pfsf_aug_clear(island_id, kind);
}

PFSF_API void pfsf_hook_set(int32_t island_id, pfsf_hook_point pt, pfsf_hook_fn fn, void* user_data) {
    if (!hook_point_ok(int32_t(pt))) return;
    std::unique_lock<std::shared_mutex> lk(g_hook_mu);
    HookTable& t = g_hooks[island_id];
    t.fn[pt] = fn;
    t.ud[pt] = user_data;
}

PFSF_API int32_t pfsf_hook_fire(int32_t island_id, pfsf_hook_point pt, int64_t epoch) {
    if (!hook_point_ok(int32_t(pt))) return 0;
    pfsf_hook_fn fn = nullptr;
    void* ud = nullptr;
    {
        std::shared_lock<std::shared_mutex> lk(g_hook_mu);
        auto it = g_hooks.find(island_id);
        if (it == g_hooks.end()) return 0;
        fn = it->second.fn[pt];
        ud = it->second.ud[pt];
    }
    if (!fn) return 0;
    fn(island_id, epoch, ud);  // outside the lock: a hook may re-enter the table
    return 1;
}

PFSF_API void pfsf_hook_clear(int32_t island_id, pfsf_hook_point pt) {
    if (!hook_point_ok(int32_t(pt))) return;
    std::unique_lock<std::shared_mutex> lk(g_hook_mu);
    auto it = g_hooks.find(island_id);
    if (it == g_hooks.end()) return;
    it->second.fn[pt] = nullptr;
    it->second.ud[pt] = nullptr;
}

PFSF_API void pfsf_hook_clear_island(int32_t island_id) {
    std::unique_lock<std::shared_mutex> lk(g_hook_mu);
    g_hooks.erase(island_id);
}

// Engine-handle form: installs on the island-less slot (id -1).
PFSF_API void pfsf_set_hook(pfsf_engine, pfsf_hook_point pt, pfsf_hook_fn fn, void* user_data) {
    pfsf_hook_set(-1, pt, fn, user_data);
}

}  // extern "C"

// ─── augmentation updates ───────────────────────────────────────────────────
// Each clamps the slot sample to [lo, hi] as min(max(v, lo), hi) (a NaN
// sample passes through and counts as clamped) and returns how many voxels
// were clamped.

namespace {

inline float clamp_sample(float v, float lo, float hi) {
    const float a = v < lo ? lo : v;  // std::max(v, lo)
    return hi < a ? hi : a;           // std::min(a, hi)
}

int32_t aug_source_add(float* dst, const float* s, int32_t n, float lo, float hi) {
    int32_t c = 0;
    for (int32_t i = 0; i < n; ++i) {
        const float v = clamp_sample(s[i], lo, hi);
        c += s[i] != v;
        dst[i] += v;
    }
    return c;
}

int32_t aug_scale(float* dst, const float* s, int32_t n, float lo, float hi) {
    int32_t c = 0;
    for (int32_t i = 0; i < n; ++i) {
        const float v = clamp_sample(s[i], lo, hi);
        c += s[i] != v;
        dst[i] *= v;
    }
    return c;
}

// every SoA-6 face of voxel i scaled by the clamped slot sample i
int32_t aug_cond_scale(float* cond, const float* s, int32_t n, float lo, float hi) {
    const int32_t c = aug_scale(cond, s, n, lo, hi);
    for (int d = 1; d < 6; ++d) aug_scale(cond + size_t(d) * size_t(n), s, n, lo, hi);
    return c;
}

// face d of voxel i scaled by clamp(1 + k * (unit normal of d . wind_i))
int32_t aug_wind_bias(float* cond, const float* w3, int32_t n, float k, float lo, float hi) {
    static constexpr float kNx[6] = {-1.0f, 1.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    static constexpr float kNy[6] = {0.0f, 0.0f, -1.0f, 1.0f, 0.0f, 0.0f};
    static constexpr float kNz[6] = {0.0f, 0.0f, 0.0f, 0.0f, -1.0f, 1.0f};
    int32_t c = 0;
    for (int32_t i = 0; i < n; ++i) {
        const float wx = w3[3 * size_t(i)], wy = w3[3 * size_t(i) + 1], wz = w3[3 * size_t(i) + 2];
        bool hit = false;
        for (int d = 0; d < 6; ++d) {
            const float f = 1.0f + k * (kNx[d] * wx + kNy[d] * wy + kNz[d] * wz);
            const float v = clamp_sample(f, lo, hi);
            hit |= f != v;
            cond[size_t(d) * size_t(n) + size_t(i)] *= v;
        }
        c += hit;
    }
    return c;
}

}  // namespace

// ─── plan interpreter ───────────────────────────────────────────────────────

namespace {

std::atomic<int64_t> g_plan_counter{0};

std::shared_mutex g_test_hook_mu;
std::map<std::pair<int32_t, int32_t>, int64_t> g_test_hook_hits;

void plan_test_hook_cb(int32_t island_id, int64_t, void* ud) {
    const int32_t point = int32_t(reinterpret_cast<intptr_t>(ud));
    std::unique_lock<std::shared_mutex> lk(g_test_hook_mu);
    auto it = g_test_hook_hits.find({island_id, point});
    if (it != g_test_hook_hits.end()) ++it->second;
}

// Little-endian field reads from an opcode's argument block (byte-wise, so
// unaligned records and big-endian hosts read the same values).
struct Args {
    const uint8_t* p;
    uint32_t u32(int o) const {
        return uint32_t(p[o]) | uint32_t(p[o + 1]) << 8 | uint32_t(p[o + 2]) << 16 | uint32_t(p[o + 3]) << 24;
    }
    int32_t i32(int o) const { return int32_t(u32(o)); }
    int64_t i64(int o) const { return int64_t(uint64_t(u32(o)) | uint64_t(u32(o + 4)) << 32); }
    float f32(int o) const {
        const uint32_t b = u32(o);
        float f;
        std::memcpy(&f, &b, 4);
        return f;
    }
    template <class T>
    T* ptr(int o) const {
        return reinterpret_cast<T*>(uintptr_t(i64(o)));
    }
};

bool dims_ok(int32_t x, int32_t y, int32_t z) { return x > 0 && y > 0 && z > 0 && x <= 512 && y <= 512 && z <= 512; }

// A published slot is used only if its stride is what the opcode consumes
// and it holds n samples; otherwise the opcode is skipped with a warning.
bool slot_fits(const pfsf_aug_slot& s, int32_t stride, int32_t n, int32_t island, int32_t kind) {
    if (s.stride_bytes != stride) {
        pfsf_trace_emit(PFSF_TRACE_WARN, 0, -1, island, s.stride_bytes, kind, "plan: aug stride mismatch");
        return false;
    }
    if (s.dbb_bytes < int64_t(n) * stride) {
        pfsf_trace_emit(PFSF_TRACE_WARN, 0, -1, island, int32_t(s.dbb_bytes), kind, "plan: aug dbb too small");
        return false;
    }
    return true;
}

enum class Step { Ok, Bad, Fail };  // Fail carries its own result code

// Runs one opcode.  Returns Ok, Bad (malformed: INVALID_ARG) or Fail with
// *rc set (a primitive's own error).
Step run_op(uint16_t op, uint32_t len, const Args& a, int32_t island, int32_t& hooks, pfsf_result& rc) {
    switch (op) {
        case PFSF_OP_NO_OP:
            return Step::Ok;
        case PFSF_OP_INCR_COUNTER:
            if (len < 4) return Step::Bad;
            g_plan_counter.fetch_add(a.i32(0), std::memory_order_relaxed);
            return Step::Ok;
        case PFSF_OP_CLEAR_AUG:
            if (len < 4) return Step::Bad;
            pfsf_aug_clear(island, pfsf_augmentation_kind(a.i32(0)));
            return Step::Ok;
        case PFSF_OP_CLEAR_AUG_ISLAND:
            pfsf_aug_clear_island(island);
            return Step::Ok;
        case PFSF_OP_FIRE_HOOK:
            if (len < 12) return Step::Bad;
            hooks += pfsf_hook_fire(island, pfsf_hook_point(a.i32(0)), a.i64(4));
            return Step::Ok;
        case PFSF_OP_NORMALIZE_SOA6: {
            if (len < 52) return Step::Bad;
            const int32_t n = a.i32(48);
            if (!a.i64(0) || !a.i64(8) || !a.i64(16) || !a.i64(24) || !a.i64(40) || n < 0 || n > 1000000)
                return Step::Bad;
            pfsf_normalize_soa6(a.ptr<float>(0), a.ptr<float>(8), a.ptr<float>(16), a.ptr<float>(24),
                                a.ptr<const float>(32), n, a.ptr<float>(40));
            return Step::Ok;
        }
        case PFSF_OP_APPLY_WIND_BIAS: {
            if (len < 32) return Step::Bad;
            const int32_t n = a.i32(8);
            if (!a.i64(0) || n < 0 || n > 1000000) return Step::Bad;
            pfsf_apply_wind_bias(a.ptr<float>(0), n, pfsf_vec3{a.f32(16), a.f32(20), a.f32(24)}, a.f32(28));
            return Step::Ok;
        }
        case PFSF_OP_COMPUTE_CONDUCTIVITY: {
            if (len < 64) return Step::Bad;
            if (!a.i64(0) || !a.i64(8) || !a.i64(16) || !a.i64(24) || !dims_ok(a.i32(32), a.i32(36), a.i32(40)))
                return Step::Bad;
            pfsf_compute_conductivity(a.ptr<float>(0), a.ptr<const float>(8), a.ptr<const float>(16),
                                      a.ptr<const uint8_t>(24), a.i32(32), a.i32(36), a.i32(40),
                                      pfsf_vec3{a.f32(48), a.f32(52), a.f32(56)}, a.f32(60));
            return Step::Ok;
        }
        case PFSF_OP_ARM_MAP:
        case PFSF_OP_ARCH_FACTOR: {
            if (len < 40) return Step::Bad;
            if (!a.i64(0) || !a.i64(8) || !a.i64(16) || !dims_ok(a.i32(24), a.i32(28), a.i32(32))) return Step::Bad;
            rc = op == PFSF_OP_ARM_MAP
                     ? pfsf_compute_arm_map(a.ptr<const uint8_t>(0), a.ptr<const uint8_t>(8), a.i32(24), a.i32(28),
                                            a.i32(32), a.ptr<int32_t>(16))
                     : pfsf_compute_arch_factor_map(a.ptr<const uint8_t>(0), a.ptr<const uint8_t>(8), a.i32(24),
                                                    a.i32(28), a.i32(32), a.ptr<float>(16));
            return rc == PFSF_OK ? Step::Ok : Step::Fail;
        }
        case PFSF_OP_PHANTOM_EDGES: {
            if (len < 56) return Step::Bad;
            if (!a.i64(0) || !a.i64(8) || !a.i64(16) || !dims_ok(a.i32(32), a.i32(36), a.i32(40))) return Step::Bad;
            const int32_t k = pfsf_inject_phantom_edges(a.ptr<const uint8_t>(0), a.ptr<float>(8),
                                                        a.ptr<const float>(16), a.i32(32), a.i32(36), a.i32(40),
                                                        a.f32(48), a.f32(52));
            if (a.i64(24)) *a.ptr<int32_t>(24) = k;
            return Step::Ok;
        }
        case PFSF_OP_DOWNSAMPLE_2TO1: {
            if (len < 48) return Step::Bad;
            if (!a.i64(0) || !a.i64(8) || !a.i64(16) || !a.i64(24) || !dims_ok(a.i32(32), a.i32(36), a.i32(40)))
                return Step::Bad;
            pfsf_downsample_2to1(a.ptr<const float>(0), a.ptr<const uint8_t>(8), a.i32(32), a.i32(36), a.i32(40),
                                 a.ptr<float>(16), a.ptr<uint8_t>(24));
            return Step::Ok;
        }
        case PFSF_OP_TILED_LAYOUT: {
            if (len < 32) return Step::Bad;
            if (!a.i64(0) || !a.i64(8) || a.i32(28) <= 0 || !dims_ok(a.i32(16), a.i32(20), a.i32(24)))
                return Step::Bad;
            pfsf_tiled_layout_build(a.ptr<const float>(0), a.i32(16), a.i32(20), a.i32(24), a.i32(28),
                                    a.ptr<float>(8));
            return Step::Ok;
        }
        case PFSF_OP_CHEBYSHEV:
            if (len < 20 || !a.i64(0)) return Step::Bad;
            *a.ptr<float>(0) = pfsf_chebyshev_omega(a.i32(8), a.f32(16));
            return Step::Ok;
        case PFSF_OP_CHECK_DIVERGENCE: {
            if (len < 40) return Step::Bad;
            const int32_t mcount = a.i32(28);
            if (!a.i64(0) || !a.i64(16) || mcount < 0) return Step::Bad;
            // the state block is the int[7] view Java keeps (floats as raw bits)
            static_assert(sizeof(pfsf_divergence_state) == 28, "divergence state is 7 x 4 bytes");
            pfsf_divergence_state st;
            std::memcpy(&st, a.ptr<void>(0), sizeof st);
            st.struct_bytes = int32_t(sizeof st);
            const int32_t kind =
                pfsf_check_divergence(&st, a.f32(24), a.ptr<const float>(8), mcount, a.f32(32), a.f32(36));
            std::memcpy(a.ptr<void>(0), &st, sizeof st);
            *a.ptr<int32_t>(16) = kind;
            return Step::Ok;
        }
        case PFSF_OP_EXTRACT_FEATURES: {
            if (len < 72) return Step::Bad;
            const int32_t lx = a.i32(16), ly = a.i32(20), lz = a.i32(24), mcount = a.i32(56);
            if (!a.i64(8) || lx <= 0 || ly <= 0 || lz <= 0 || mcount < 0) return Step::Bad;
            pfsf_extract_island_features(lx, ly, lz, a.i32(28), a.f32(64), a.f32(68), a.i32(32), a.i32(36),
                                         a.i32(40), a.i32(44), a.i32(48), a.i32(52), a.ptr<const float>(0), mcount,
                                         a.ptr<float>(8));
            return Step::Ok;
        }
        case PFSF_OP_WIND_PRESSURE:
            if (len < 24 || !a.i64(0)) return Step::Bad;
            *a.ptr<float>(0) = pfsf_wind_pressure_source(a.f32(8), a.f32(12), a.i32(16) != 0);
            return Step::Ok;
        case PFSF_OP_TIMOSHENKO:
            if (len < 28 || !a.i64(0)) return Step::Bad;
            *a.ptr<float>(0) = pfsf_timoshenko_moment_factor(a.f32(8), a.f32(12), a.i32(16), a.f32(20), a.f32(24));
            return Step::Ok;
        case PFSF_OP_AUG_SOURCE_ADD:
        case PFSF_OP_AUG_COND_MUL:
        case PFSF_OP_AUG_RCOMP_MUL:
        case PFSF_OP_AUG_WIND_3D_BIAS: {
            // island i64 @0, kind i32 @8, target i64 @12, n i32 @20, then
            // [k f32 @24 for the wind form] lo, hi
            const bool wind = op == PFSF_OP_AUG_WIND_3D_BIAS;
            if (len < (wind ? 36u : 32u)) return Step::Bad;
            const int32_t isl = int32_t(a.i64(0)), kind = a.i32(8), n = a.i32(20);
            const int lo_at = wind ? 28 : 24;
            const float lo = a.f32(lo_at), hi = a.f32(lo_at + 4);
            if (!a.i64(12) || n < 0 || !(hi >= lo)) return Step::Bad;
            pfsf_aug_slot s{};
            s.struct_bytes = int32_t(sizeof s);
            if (!pfsf_aug_query(isl, pfsf_augmentation_kind(kind), &s) || !s.dbb_addr) return Step::Ok;  // not published
            if (!slot_fits(s, wind ? 12 : 4, n, isl, kind)) return Step::Ok;
            const float* src = static_cast<const float*>(s.dbb_addr);
            float* dst = a.ptr<float>(12);
            int32_t clamped = 0;
            if (n > 0) {
                if (op == PFSF_OP_AUG_SOURCE_ADD)
                    clamped = aug_source_add(dst, src, n, lo, hi);
                else if (op == PFSF_OP_AUG_RCOMP_MUL)
                    clamped = aug_scale(dst, src, n, lo, hi);
                else if (op == PFSF_OP_AUG_COND_MUL)
                    clamped = aug_cond_scale(dst, src, n, lo, hi);
                else
                    clamped = aug_wind_bias(dst, src, n, a.f32(24), lo, hi);
            }
            if (clamped > 0) pfsf_trace_emit(PFSF_TRACE_WARN, 0, -1, isl, clamped, kind, "plan: aug clamp");
            return Step::Ok;
        }
        default:
            return Step::Bad;
    }
}

}  // namespace

extern "C" {

PFSF_API pfsf_result pfsf_plan_execute(const void* plan, int64_t plan_bytes, pfsf_plan_result* out) {
    pfsf_plan_result scratch;
    pfsf_plan_result& r = out ? *out : scratch;
    r.struct_bytes = int32_t(sizeof(pfsf_plan_result));
    r.executed_count = 0;
    r.failed_index = -1;
    r.error_code = PFSF_OK;
    r.hook_fire_count = 0;
    if (!plan || plan_bytes < PFSF_PLAN_HEADER_BYTES) {
        r.error_code = PFSF_ERROR_INVALID_ARG;
        return PFSF_ERROR_INVALID_ARG;
    }
    const Args hdr{static_cast<const uint8_t*>(plan)};
    const uint32_t magic = hdr.u32(0);
    const uint32_t version = hdr.u32(4) & 0xFFFFu;  // u16 version, u16 flags (reserved)
    const int32_t island = hdr.i32(8);
    const int32_t ops = hdr.i32(12);
    if (magic != PFSF_PLAN_MAGIC || version != PFSF_PLAN_VERSION || ops < 0) {
        r.error_code = PFSF_ERROR_INVALID_ARG;
        pfsf_trace_emit(PFSF_TRACE_ERROR, 0, -1, island, -1, PFSF_ERROR_INVALID_ARG, "plan: bad header");
        return PFSF_ERROR_INVALID_ARG;
    }
    auto fail = [&](int32_t i, pfsf_result code) {
        r.failed_index = i;
        r.error_code = code;
        return code;
    };
    int64_t at = PFSF_PLAN_HEADER_BYTES;
    int32_t hooks = 0;
    for (int32_t i = 0; i < ops; ++i) {
        if (at + PFSF_PLAN_OP_HEADER_BYTES > plan_bytes) return fail(i, PFSF_ERROR_INVALID_ARG);
        const Args rec{static_cast<const uint8_t*>(plan) + at};
        const uint16_t op = uint16_t(rec.u32(0) & 0xFFFFu);
        const uint32_t len = rec.u32(0) >> 16;
        if (at + PFSF_PLAN_OP_HEADER_BYTES + int64_t(len) > plan_bytes) return fail(i, PFSF_ERROR_INVALID_ARG);
        pfsf_result rc = PFSF_OK;
        const Step s = run_op(op, len, Args{rec.p + PFSF_PLAN_OP_HEADER_BYTES}, island, hooks, rc);
        if (s == Step::Fail) return fail(i, rc);
        if (s == Step::Bad) {
            if (op > PFSF_OP_AUG_WIND_3D_BIAS)
                pfsf_trace_emit(PFSF_TRACE_ERROR, 0, -1, island, i, PFSF_ERROR_INVALID_ARG, "plan: unknown opcode");
            return fail(i, PFSF_ERROR_INVALID_ARG);
        }
        at += PFSF_PLAN_OP_HEADER_BYTES + int64_t(len);
        ++r.executed_count;
    }
    r.hook_fire_count = hooks;
    return PFSF_OK;
}

PFSF_API int64_t pfsf_plan_test_counter_read_reset(void) { return g_plan_counter.exchange(0); }

PFSF_API void pfsf_plan_test_hook_install(int32_t island_id, int32_t point) {
    {
        std::unique_lock<std::shared_mutex> lk(g_test_hook_mu);
        g_test_hook_hits[{island_id, point}] = 0;
    }
    pfsf_hook_set(island_id, pfsf_hook_point(point), &plan_test_hook_cb,
                  reinterpret_cast<void*>(static_cast<intptr_t>(point)));
}

PFSF_API int64_t pfsf_plan_test_hook_count_read_reset(int32_t island_id, int32_t point) {
    std::unique_lock<std::shared_mutex> lk(g_test_hook_mu);
    auto it = g_test_hook_hits.find({island_id, point});
    if (it == g_test_hook_hits.end()) return 0;
    return std::exchange(it->second, 0);
}

}  // extern "C"
