// extern "C" entry points of pfsf.h / pfsf_b200.h (reference C ABI wrapper:
// L1-native/libpfsf/src/pfsf_api.cpp).  Each call checks the handle
// (NULL -> PFSF_ERROR_INVALID_ARG) and forwards to the engine.
#include <cstring>
#include <new>

#include "engine.h"
#include "labels.h"

using pfsf_b200::Engine;

struct pfsf_engine_t {
    Engine* eng;
};

namespace {
Engine* E(pfsf_engine e) { return e ? e->eng : nullptr; }

// pfsf_api.cpp:23-31 defaults
pfsf_config default_config() {
    pfsf_config c{};
    c.max_island_size = 50000;
    c.tick_budget_ms = 8;
    c.vram_budget_bytes = 512LL * 1024 * 1024;
    c.enable_phase_field = true;
    c.enable_multigrid = true;
    return c;
}
}  // namespace

extern "C" {

PFSF_API pfsf_engine pfsf_create(const pfsf_config* config) {
    pfsf_config c = config ? *config : default_config();
    auto* h = new (std::nothrow) pfsf_engine_t{nullptr};
    if (!h) return nullptr;
    h->eng = new (std::nothrow) Engine(c);
    if (!h->eng) {
        delete h;
        return nullptr;
    }
    return h;
}

PFSF_API pfsf_engine pfsf_create_with_vulkan(const pfsf_config*, const pfsf_vulkan_handles*) { return nullptr; }

PFSF_API pfsf_result pfsf_init(pfsf_engine e) {
    Engine* g = E(e);
    return g ? g->init() : PFSF_ERROR_INVALID_ARG;
}

PFSF_API void pfsf_shutdown(pfsf_engine e) {
    if (Engine* g = E(e)) g->shutdown();
}

PFSF_API void pfsf_destroy(pfsf_engine e) {
    if (!e) return;
    delete e->eng;
    delete e;
}

PFSF_API bool pfsf_is_available(pfsf_engine e) {
    Engine* g = E(e);
    return g && g->available();
}

PFSF_API pfsf_result pfsf_get_stats(pfsf_engine e, pfsf_stats* out) {
    Engine* g = E(e);
    return g ? g->get_stats(out) : PFSF_ERROR_INVALID_ARG;
}

// The DBB tick path reads precomputed buffers; lookup callbacks are stored by
// the reference but never consulted on that path (pfsf_engine.cpp:135-149).
PFSF_API void pfsf_set_material_lookup(pfsf_engine, pfsf_material_fn, void*) {}
PFSF_API void pfsf_set_anchor_lookup(pfsf_engine, pfsf_anchor_fn, void*) {}
PFSF_API void pfsf_set_fill_ratio_lookup(pfsf_engine, pfsf_fill_ratio_fn, void*) {}
PFSF_API void pfsf_set_curing_lookup(pfsf_engine, pfsf_curing_fn, void*) {}

PFSF_API void pfsf_set_wind(pfsf_engine e, const pfsf_vec3* wind) {
    if (Engine* g = E(e)) g->set_wind(wind);
}

PFSF_API void pfsf_set_pcg_enabled(pfsf_engine e, int enabled) {
    if (Engine* g = E(e)) g->set_pcg_enabled(enabled != 0);
}

PFSF_API pfsf_result pfsf_add_island(pfsf_engine e, const pfsf_island_desc* desc) {
    Engine* g = E(e);
    return g ? g->add_island(desc) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API void pfsf_remove_island(pfsf_engine e, int32_t id) {
    if (Engine* g = E(e)) g->remove_island(id);
}

PFSF_API pfsf_result pfsf_notify_block_change(pfsf_engine e, int32_t id, const pfsf_voxel_update* u) {
    Engine* g = E(e);
    return g ? g->notify_block_change(id, u) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API void pfsf_mark_full_rebuild(pfsf_engine e, int32_t id) {
    if (Engine* g = E(e)) g->mark_full_rebuild(id);
}

PFSF_API pfsf_result pfsf_tick(pfsf_engine e, const int32_t* ids, int32_t count, int64_t, pfsf_tick_result* result) {
    Engine* g = E(e);
    return g ? g->tick(ids, count, result, nullptr, 0) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_read_stress(pfsf_engine e, int32_t id, float* out, int32_t cap, int32_t* count) {
    Engine* g = E(e);
    return g ? g->read_stress(id, out, cap, count) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_register_island_buffers(pfsf_engine e, int32_t id, const pfsf_island_buffers* b) {
    Engine* g = E(e);
    return g ? g->register_buffers(id, b) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_register_island_lookups(pfsf_engine e, int32_t id, const pfsf_island_lookups* l) {
    Engine* g = E(e);
    return g ? g->register_lookups(id, l) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_register_stress_readback(pfsf_engine e, int32_t id, void* addr, int64_t bytes) {
    Engine* g = E(e);
    return g ? g->register_stress(id, addr, bytes) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_tick_dbb(pfsf_engine e, const int32_t* ids, int32_t count, int64_t, void* fail_addr,
                                   int64_t fail_bytes) {
    // pre-zero the header so the caller sees count = 0 on every early return
    if (fail_addr && fail_bytes >= (int64_t)sizeof(int32_t)) *static_cast<int32_t*>(fail_addr) = 0;
    Engine* g = E(e);
    return g ? g->tick(ids, count, nullptr, fail_addr, fail_bytes) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API int32_t pfsf_drain_callbacks(pfsf_engine, int32_t*, int32_t) { return 0; }

PFSF_API pfsf_result pfsf_get_sparse_upload_buffer(pfsf_engine e, int32_t id, void** out_addr, int64_t* out_bytes) {
    Engine* g = E(e);
    return g ? g->get_sparse_buffer(id, out_addr, out_bytes) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_notify_sparse_updates(pfsf_engine e, int32_t id, int32_t count) {
    Engine* g = E(e);
    return g ? g->notify_sparse(id, count) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API const char* pfsf_version(void) { return "0.4.0-b200"; }

// ---- pfsf_b200.h ----
PFSF_API pfsf_result pfsf_register_island_kappa(pfsf_engine e, int32_t id, const pfsf_island_kappa_buffers* b) {
    Engine* g = E(e);
    return g ? g->register_kappa(id, b) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API void pfsf_set_precision_mode(pfsf_engine e, pfsf_precision mode) {
    if (Engine* g = E(e)) g->set_precision(mode);
}

PFSF_API void pfsf_set_solve_mode(pfsf_engine e, pfsf_solve_mode mode) {
    if (Engine* g = E(e)) g->set_solve_mode(mode);
}

PFSF_API pfsf_result pfsf_solve_to_tolerance(pfsf_engine e, const int32_t* ids, int32_t count, double rel_tol,
                                             int32_t max_iter, uint32_t flags, pfsf_solve_stats* out) {
    Engine* g = E(e);
    return g ? g->solve_to_tolerance(ids, count, rel_tol, max_iter, flags, out) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_tick_tolerance(pfsf_engine e, const int32_t* ids, int32_t count, int64_t, void* fail_addr,
                                         int64_t fail_bytes, double rel_tol, int32_t max_iter, pfsf_solve_stats* out) {
    if (fail_addr && fail_bytes >= (int64_t)sizeof(int32_t)) *static_cast<int32_t*>(fail_addr) = 0;
    Engine* g = E(e);
    return g ? g->tick_tolerance(ids, count, fail_addr, fail_bytes, rel_tol, max_iter, out) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_island_solve_report(pfsf_engine e, int32_t id, pfsf_island_report* out) {
    Engine* g = E(e);
    return g ? g->island_report(id, out) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API void pfsf_set_mg_cycle(pfsf_engine e, pfsf_mg_cycle cycle) {
    if (Engine* g = E(e)) g->set_mg_cycle((int)cycle);
}

PFSF_API void pfsf_set_amg(pfsf_engine e, int32_t enable) {
    if (Engine* g = E(e)) g->set_amg(enable != 0);
}

PFSF_API pfsf_result pfsf_get_tuning(pfsf_engine e, pfsf_tuning* out) {
    Engine* g = E(e);
    return g ? g->get_tuning(out) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_set_tuning(pfsf_engine e, const pfsf_tuning* in) {
    Engine* g = E(e);
    return g ? g->set_tuning(in) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_island_phi_max(pfsf_engine e, int32_t id, float* out) {
    Engine* g = E(e);
    return g ? g->island_phi_max(id, out) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_debug_time_pass(pfsf_engine e, int32_t id, int32_t pass, int32_t reps, float* ms,
                                          double* bytes) {
    Engine* g = E(e);
    return g ? g->debug_time_pass(id, pass, reps, ms, bytes) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_last_tick_report(pfsf_engine e, pfsf_tick_report* out) {
    Engine* g = E(e);
    return g ? g->last_tick_report(out) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_read_solution64(pfsf_engine e, int32_t id, double* out, int64_t cap, int64_t* count) {
    Engine* g = E(e);
    return g ? g->read_solution64(id, out, cap, count) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_register_island_adjoint(pfsf_engine e, int32_t id, const pfsf_island_adjoint_buffers* b) {
    Engine* g = E(e);
    return g ? g->register_adjoint(id, b) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_adjoint_to_tolerance(pfsf_engine e, const int32_t* ids, int32_t count, double rel_tol,
                                               int32_t max_iter, uint32_t flags, pfsf_solve_stats* out) {
    Engine* g = E(e);
    return g ? g->adjoint_to_tolerance(ids, count, rel_tol, max_iter, flags, out) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API pfsf_result pfsf_label_components(pfsf_engine e, const uint8_t* type, int32_t lx, int32_t ly, int32_t lz,
                                           uint32_t* labels, pfsf_label_component* comps, int32_t capacity,
                                           int32_t* count, int32_t* overflow) {
    Engine* g = E(e);
    if (!g) return PFSF_ERROR_INVALID_ARG;
    if (!g->available()) return PFSF_ERROR_NOT_INIT;
    return pfsf_b200::labels::label_components(g->stream(), g->num_sms(), type, lx, ly, lz, labels, comps, capacity,
                                               count, overflow);
}

PFSF_API pfsf_result pfsf_debug_read_field(pfsf_engine e, int32_t id, int32_t field, void* out, int64_t bytes,
                                           int64_t* out_bytes) {
    Engine* g = E(e);
    return g ? g->debug_read_field(id, field, out, bytes, out_bytes) : PFSF_ERROR_INVALID_ARG;
}

PFSF_API void* pfsf_get_stream(pfsf_engine e) {
    Engine* g = E(e);
    return g ? (void*)g->stream() : nullptr;
}

PFSF_API int64_t pfsf_kernel_launch_count(pfsf_engine e) {
    Engine* g = E(e);
    return g ? g->launches() : 0;
}

}  // extern "C"
