// PFSF B200 engine: island registry, device buffers and the reference tick
// schedule driven from the host over CUDA kernel launches.
//
// The schedule restates L1-native/libpfsf/src/pfsf_engine.cpp:424-600
// (tickImpl) and L1-native/libpfsf/src/solver/dispatcher*.cpp (recordSolveSteps,
// tryRecordVCycleAt, recordVCycle, recordPCGInitialResidual, recordPCGStep)
// with the Vulkan command recording replaced by launches on one CUDA stream.
// The per-island host<->device round trips of the reference (upload submit,
// solve submit, three readbacks) become asynchronous copies with one stream
// synchronisation per tick for all islands plus one for failure tuples.
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "arena.h"
#include "tick_batch.h"
#include "compat.h"
#include "kappa.h"

namespace pfsf_b200 {

#define CU_OK(expr) (cudaSuccess == (expr))

Island::Island() = default;
Island::~Island() = default;

Engine::Engine(const pfsf_config& cfg) : cfg_(cfg) {
    if (const char* f = std::getenv("PFSF_FAULT_ALLOC_AFTER")) fault_alloc_after_ = std::atoll(f);
    if (const char* f = std::getenv("PFSF_SMOOTHER")) smoother_ = std::atoi(f);
}

Engine::~Engine() { shutdown(); }

pfsf_result Engine::init() {
    if (available_) return PFSF_OK;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return PFSF_ERROR_NO_DEVICE;
    }
    int dev = 0;
    if (const char* e = std::getenv("PFSF_CUDA_DEVICE")) dev = std::atoi(e);
    else cudaGetDevice(&dev);
    if (dev < 0 || dev >= count) return PFSF_ERROR_NO_DEVICE;
    if (!CU_OK(cudaSetDevice(dev))) return PFSF_ERROR_NO_DEVICE;
    device_ = dev;
    cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev);
    load_tuning();
    if (!CU_OK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking))) return PFSF_ERROR_VULKAN;
    // side stream of the batched solve (fills CTA slots clusters leave free);
    // without it the solve runs on stream_ alone
    if (!CU_OK(cudaStreamCreateWithFlags(&side_.stream, cudaStreamNonBlocking)) ||
        !CU_OK(cudaEventCreateWithFlags(&side_.fork, cudaEventDisableTiming)) ||
        !CU_OK(cudaEventCreateWithFlags(&side_.join, cudaEventDisableTiming))) {
        cudaGetLastError();
        destroy_side();
    }
    host_results_cap_ = 256;
    if (!CU_OK(cudaMallocHost((void**)&host_results_, sizeof(TickResult) * host_results_cap_))) {
        cudaStreamDestroy(stream_);
        stream_ = nullptr;
        return PFSF_ERROR_VULKAN;
    }
    available_ = true;
    return PFSF_OK;
}

void Engine::destroy_side() {
    if (side_.stream) cudaStreamDestroy(side_.stream);
    if (side_.fork) cudaEventDestroy(side_.fork);
    if (side_.join) cudaEventDestroy(side_.join);
    side_ = kappa::SideStream{nullptr, nullptr, nullptr};
}

void Engine::shutdown() {
    if (!available_) return;
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    free_arena();
    free_tick_batch();
    for (auto& kv : islands_) free_island(*kv.second);
    islands_.clear();
    if (host_results_) cudaFreeHost(host_results_);
    host_results_ = nullptr;
    destroy_side();
    cudaStreamDestroy(stream_);
    stream_ = nullptr;
    vram_used_ = 0;
    available_ = false;
}

pfsf_result Engine::get_stats(pfsf_stats* out) {
    if (!out) return PFSF_ERROR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(stats_mtx_);
    out->island_count = (int32_t)islands_.size();
    int64_t tv = 0;
    for (auto& kv : islands_) tv += kv.second->n;
    out->total_voxels = tv;
    out->vram_used_bytes = vram_used_;
    out->vram_budget_bytes = cfg_.vram_budget_bytes;
    out->last_tick_ms = last_tick_ms_;
    return PFSF_OK;
}

void* Engine::dalloc(Island& isl, size_t bytes) {
    if (bytes == 0) bytes = 4;
    if (fault_alloc_after_ >= 0 && alloc_count_ >= fault_alloc_after_) return nullptr;
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaMemsetAsync(p, 0, bytes, stream_);
    alloc_count_++;
    {
        std::lock_guard<std::mutex> lk(stats_mtx_);
        vram_used_ += (int64_t)bytes;
    }
    isl.allocations.emplace_back(p, bytes);
    return p;
}

void Engine::free_island(Island& isl) {
    cudaStreamSynchronize(stream_);
    for (void* h : isl.host_registered) cudaHostUnregister(h);
    isl.host_registered.clear();
    isl.host_pins.clear();
    int64_t freed = 0;
    for (auto& a : isl.allocations) { cudaFree(a.first); freed += (int64_t)a.second; }
    isl.allocations.clear();
    {
        std::lock_guard<std::mutex> lk(stats_mtx_);
        vram_used_ -= freed;
    }
    if (isl.sparse_host) cudaFreeHost(isl.sparse_host);
    isl.sparse_host = nullptr;
    isl.kappa.reset();
}

Island* Engine::find(int32_t id) {
    auto it = islands_.find(id);
    return it == islands_.end() ? nullptr : it->second.get();
}

pfsf_result Engine::add_island(const pfsf_island_desc* d) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!d) return PFSF_ERROR_INVALID_ARG;
    // pfsf_engine.cpp:156-173
    if (d->lx <= 0 || d->ly <= 0 || d->lz <= 0) return PFSF_ERROR_ISLAND_FULL;
    if ((int64_t)d->lx > cfg_.max_island_size || (int64_t)d->ly > cfg_.max_island_size ||
        (int64_t)d->lz > cfg_.max_island_size)
        return PFSF_ERROR_ISLAND_FULL;
    const int64_t n = (int64_t)d->lx * d->ly * d->lz;
    if (n > cfg_.max_island_size || n > INT32_MAX) return PFSF_ERROR_ISLAND_FULL;
    if (Island* existing = find(d->island_id)) {
        // getOrCreate semantics: same id returns the existing island
        (void)existing;
        return PFSF_OK;
    }
    auto isl = std::make_unique<Island>();
    isl->id = d->island_id;
    isl->origin = d->origin;
    isl->lx = d->lx;
    isl->ly = d->ly;
    isl->lz = d->lz;
    isl->n = n;
    isl->nmb = (int64_t)((d->lx + 7) / 8) * ((d->ly + 7) / 8) * ((d->lz + 7) / 8);
    // The reference allocates every per-island buffer here
    // (island_buffer.cpp:21-122).  Islands used only by the tolerance solve
    // never need the SoA-6 tick buffers, so those are allocated on first use
    // (ensure_compat); a failure there is reported (PFSF_ERROR_OUT_OF_VRAM)
    // by the call that needed them.
    islands_[d->island_id] = std::move(isl);
    return PFSF_OK;
}

bool Engine::ensure_compat(Island& s) {
    if (s.phi) return true;
    const int64_t n = s.n;
    const size_t first = s.allocations.size();
    bool ok = true;
    auto F = [&](int64_t cnt) { void* p = dalloc(s, (size_t)cnt * 4); ok &= p != nullptr; return (float*)p; };
    s.phi = F(n); s.src = F(n); s.sigma = F(6 * n); s.rcomp = F(n); s.rtens = F(n); s.maxphi = F(n);
    s.hyd = F(n); s.H = F(n); s.D = F(n); s.Dold = F(n);
    s.type = (uint8_t*)dalloc(s, (size_t)n); ok &= s.type != nullptr;
    s.fail = (uint8_t*)dalloc(s, (size_t)n); ok &= s.fail != nullptr;
    s.macro = (uint32_t*)dalloc(s, (size_t)std::max<int64_t>(s.nmb, 1) * 4); ok &= s.macro != nullptr;
    const int64_t nb = compat::pcg_blocks(n);  // failed voxels per 256-voxel block
    s.fcounts = (int32_t*)dalloc(s, (size_t)nb * 4); ok &= s.fcounts != nullptr;
    s.foffsets = (int32_t*)dalloc(s, (size_t)nb * 4); ok &= s.foffsets != nullptr;
    if (!ok) {
        int64_t freed = 0;
        for (size_t k = first; k < s.allocations.size(); k++) {
            cudaFree(s.allocations[k].first);
            freed += (int64_t)s.allocations[k].second;
        }
        s.allocations.resize(first);
        {
            std::lock_guard<std::mutex> lk(stats_mtx_);
            vram_used_ -= freed;
        }
        s.phi = nullptr;
        return false;
    }
    // hydration defaults to 1.0 (island_buffer.cpp vkCmdFillBuffer 0x3F800000)
    std::vector<float> ones((size_t)n, 1.0f);
    cudaMemcpyAsync(s.hyd, ones.data(), (size_t)n * 4, cudaMemcpyHostToDevice, stream_);
    cudaStreamSynchronize(stream_);
    return true;
}

void Engine::remove_island(int32_t id) {
    auto it = islands_.find(id);
    if (it == islands_.end()) return;
    free_island(*it->second);
    islands_.erase(it);
}

pfsf_result Engine::notify_block_change(int32_t id, const pfsf_voxel_update* u) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!u) return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    if (u->flat_index < 0 || (int64_t)u->flat_index >= s->n) return PFSF_ERROR_INVALID_ARG;
    s->dirty = true;
    return PFSF_OK;
}

void Engine::mark_full_rebuild(int32_t id) {
    if (Island* s = find(id)) s->dirty = true;
}

// Pins a caller-owned host array (mapped into the device address space) and
// returns its device-visible address, or nullptr when it cannot be pinned
// (the batched tick then copies it with cudaMemcpyAsync).  A range this
// island pinned earlier (the stress buffer aliasing phi, a re-registration)
// is looked up instead of pinned twice; ranges pinned by anyone else are not
// used, since nothing here can tell how far their mapping reaches.
const void* Engine::map_host(Island& s, void* p, int64_t bytes) {
    if (!p || bytes <= 0) return nullptr;
    const char* a = static_cast<const char*>(p);
    for (const Island::HostPin& h : s.host_pins) {
        const char* b = static_cast<const char*>(h.host);
        if (a >= b && a + bytes <= b + h.bytes) return static_cast<const char*>(h.dev) + (a - b);
    }
    if (cudaHostRegister(p, (size_t)bytes, cudaHostRegisterMapped) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    s.host_registered.push_back(p);
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess || !d) {
        cudaGetLastError();
        return nullptr;
    }
    s.host_pins.push_back(Island::HostPin{p, bytes, d});
    return d;
}

pfsf_result Engine::register_buffers(int32_t id, const pfsf_island_buffers* b) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!b) return PFSF_ERROR_INVALID_ARG;
    if (!b->phi_addr || !b->source_addr || !b->conductivity_addr || !b->voxel_type_addr || !b->rcomp_addr ||
        !b->rtens_addr || !b->max_phi_addr)
        return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    const int64_t n = s->n;
    if (b->phi_bytes < 4 * n || b->source_bytes < 4 * n || b->conductivity_bytes < 24 * n ||
        b->voxel_type_bytes < n || b->rcomp_bytes < 4 * n || b->rtens_bytes < 4 * n || b->max_phi_bytes < 4 * n)
        return PFSF_ERROR_INVALID_ARG;
    if (!ensure_compat(*s)) return PFSF_ERROR_OUT_OF_VRAM;
    HostBuffers& h = s->hosts;
    h.phi = b->phi_addr; h.phi_bytes = b->phi_bytes;
    h.source = b->source_addr; h.source_bytes = b->source_bytes;
    h.conductivity = b->conductivity_addr; h.conductivity_bytes = b->conductivity_bytes;
    h.voxel_type = b->voxel_type_addr; h.voxel_type_bytes = b->voxel_type_bytes;
    h.rcomp = b->rcomp_addr; h.rcomp_bytes = b->rcomp_bytes;
    h.rtens = b->rtens_addr; h.rtens_bytes = b->rtens_bytes;
    h.max_phi = b->max_phi_addr; h.max_phi_bytes = b->max_phi_bytes;
    h.registered = true;
    h.m_phi = map_host(*s, h.phi, 4 * n);
    h.m_source = map_host(*s, h.source, 4 * n);
    h.m_cond = map_host(*s, h.conductivity, 24 * n);
    h.m_type = map_host(*s, h.voxel_type, n);
    h.m_rcomp = map_host(*s, h.rcomp, 4 * n);
    h.m_rtens = map_host(*s, h.rtens, 4 * n);
    h.m_maxphi = map_host(*s, h.max_phi, 4 * n);
    if (!upload(*s)) return PFSF_ERROR_VULKAN;
    if (!CU_OK(cudaStreamSynchronize(stream_))) return PFSF_ERROR_VULKAN;
    s->dirty = true;
    return PFSF_OK;
}

pfsf_result Engine::register_lookups(int32_t id, const pfsf_island_lookups* l) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!l) return PFSF_ERROR_INVALID_ARG;
    if (!l->material_id_addr || !l->anchor_bitmap_addr || !l->fluid_pressure_addr || !l->curing_addr)
        return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    const int64_t n = s->n;
    if (l->material_id_bytes < 4 * n || l->anchor_bitmap_bytes < 8 * n || l->fluid_pressure_bytes < 4 * n ||
        l->curing_bytes < 4 * n)
        return PFSF_ERROR_INVALID_ARG;
    s->hosts.curing = l->curing_addr;
    s->hosts.curing_bytes = l->curing_bytes;
    s->hosts.lookups_registered = true;
    s->hosts.m_curing = map_host(*s, l->curing_addr, 4 * n);
    return PFSF_OK;
}

pfsf_result Engine::register_stress(int32_t id, void* addr, int64_t bytes) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!addr || bytes <= 0) return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    s->hosts.stress_out = addr;
    s->hosts.stress_bytes = bytes;
    s->hosts.m_stress = const_cast<void*>(map_host(*s, addr, std::min<int64_t>(bytes, 4 * s->n)));
    return PFSF_OK;
}

// island_buffer.cpp:427-598 uploadFromHosts: phi, source, conductivity, type,
// rcomp, rtens, max_phi and curing (hydration) from the registered host arrays.
bool Engine::upload(Island& s) {
    const HostBuffers& h = s.hosts;
    if (!h.registered) return false;
    const size_t n = (size_t)s.n;
    bool ok = true;
    ok &= CU_OK(cudaMemcpyAsync(s.phi, h.phi, n * 4, cudaMemcpyHostToDevice, stream_));
    ok &= CU_OK(cudaMemcpyAsync(s.src, h.source, n * 4, cudaMemcpyHostToDevice, stream_));
    ok &= CU_OK(cudaMemcpyAsync(s.sigma, h.conductivity, n * 24, cudaMemcpyHostToDevice, stream_));
    ok &= CU_OK(cudaMemcpyAsync(s.type, h.voxel_type, n, cudaMemcpyHostToDevice, stream_));
    ok &= CU_OK(cudaMemcpyAsync(s.rcomp, h.rcomp, n * 4, cudaMemcpyHostToDevice, stream_));
    ok &= CU_OK(cudaMemcpyAsync(s.rtens, h.rtens, n * 4, cudaMemcpyHostToDevice, stream_));
    ok &= CU_OK(cudaMemcpyAsync(s.maxphi, h.max_phi, n * 4, cudaMemcpyHostToDevice, stream_));
    if (h.lookups_registered && h.curing)
        ok &= CU_OK(cudaMemcpyAsync(s.hyd, h.curing, n * 4, cudaMemcpyHostToDevice, stream_));
    s.mg_dirty = true;
    s.amg_dirty = true;
    return ok;
}

// island_buffer.cpp:131-245 allocateMultigrid (L1 = ceil(L/2), L2 = ceil(L1/2))
bool Engine::ensure_mg(Island& s) {
    if (s.mg_alloc) return true;
    s.l1[0] = (s.lx + 1) / 2; s.l1[1] = (s.ly + 1) / 2; s.l1[2] = (s.lz + 1) / 2;
    s.l2[0] = (s.l1[0] + 1) / 2; s.l2[1] = (s.l1[1] + 1) / 2; s.l2[2] = (s.l1[2] + 1) / 2;
    s.n1 = (int64_t)s.l1[0] * s.l1[1] * s.l1[2];
    s.n2 = (int64_t)s.l2[0] * s.l2[1] * s.l2[2];
    bool ok = true;
    auto F = [&](int64_t c) { void* p = dalloc(s, (size_t)c * 4); ok &= p != nullptr; return (float*)p; };
    s.phi1[0] = F(s.n1); s.phi1[1] = F(s.n1); s.src1 = F(s.n1); s.sig1 = F(6 * s.n1);
    s.type1 = (uint8_t*)dalloc(s, (size_t)s.n1); ok &= s.type1 != nullptr;
    if (s.n2 > 0) {
        s.phi2[0] = F(s.n2); s.phi2[1] = F(s.n2); s.src2 = F(s.n2); s.sig2 = F(6 * s.n2);
        s.type2 = (uint8_t*)dalloc(s, (size_t)s.n2); ok &= s.type2 != nullptr;
    }
    if (!ok) return false;
    s.mg_alloc = true;
    s.cur1 = s.cur2 = 0;
    return true;
}

// island_buffer.cpp:67-128 allocatePCG
bool Engine::ensure_pcg(Island& s) {
    if (s.pcg_alloc) return true;
    bool ok = true;
    auto F = [&](int64_t c) { void* p = dalloc(s, (size_t)c * 4); ok &= p != nullptr; return (float*)p; };
    s.r[0] = F(s.n); s.r[1] = F(s.n); s.p = F(s.n); s.ap = F(s.n); s.invdiag = F(s.n);
    s.partial = F(compat::pcg_blocks(s.n)); s.red = F(4);
    if (!ok) return false;
    s.pcg_alloc = true;
    s.rcur = 0;
    return true;
}

// island_buffer.cpp:285-310 allocateAMG: aggregation (int32 per voxel),
// prolongation weights, coarse diagonal and coarse correction
bool Engine::ensure_amg(Island& s) {
    if (s.amg_alloc) return true;
    s.amg_nc = (int64_t)((s.lx + 1) / 2) * ((s.ly + 1) / 2) * ((s.lz + 1) / 2);
    bool ok = true;
    auto F = [&](int64_t c) { void* p = dalloc(s, (size_t)std::max<int64_t>(c, 1) * 4); ok &= p != nullptr; return p; };
    s.agg = (int32_t*)F(s.n);
    s.aw = (float*)F(s.n);
    s.adc = (float*)F(s.amg_nc);
    s.aec = (float*)F(s.amg_nc);
    if (!ok) return false;
    s.amg_alloc = true;
    s.amg_dirty = true;
    return true;
}







// pfsf_engine.cpp:424-600
pfsf_result Engine::tick(const int32_t* ids, int32_t count, pfsf_tick_result* result, void* fail_addr,
                         int64_t fail_bytes) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (count > 0 && !ids) return PFSF_ERROR_INVALID_ARG;
    const auto t0 = std::chrono::steady_clock::now();
    if (result) result->count = 0;
    const bool drain = fail_addr != nullptr && fail_bytes >= 20;

    // capacity (tuples) still free in the caller's failure buffer
    int32_t dbb_count = drain ? *static_cast<int32_t*>(fail_addr) : 0;
    const int32_t dbb_cap = drain ? (int32_t)((fail_bytes - 4) / 16) : 0;
    const int32_t legacy_cap = (result && result->events) ? result->capacity : 0;
    const int32_t want_cap = std::max(dbb_cap, legacy_cap);

    // the dirty islands of the call, each once, in call order (the order of
    // their failure tuples); the budget is checked while they are collected
    std::vector<Island*> dispatched;
    for (int32_t k = 0; k < count; k++) {
        Island* s = find(ids[k]);
        if (!s || !s->dirty) continue;
        if (std::find(dispatched.begin(), dispatched.end(), s) != dispatched.end()) continue;
        if (!ensure_compat(*s)) return PFSF_ERROR_OUT_OF_VRAM;
        const auto el = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0);
        if (el.count() >= cfg_.tick_budget_ms) break;
        dispatched.push_back(s);
    }
    if (pfsf_result rc = tick_batched(dispatched, want_cap); rc != PFSF_OK) return rc;
    if (pfsf_result rc = finish_dispatch(dispatched, drain, fail_addr, dbb_count, dbb_cap, result, legacy_cap);
        rc != PFSF_OK)
        return rc;
    const auto t1 = std::chrono::steady_clock::now();
    {
        std::lock_guard<std::mutex> lk(stats_mtx_);
        last_tick_ms_ = std::chrono::duration<float, std::milli>(t1 - t0).count();
    }
    return PFSF_OK;
}


// After tick_batched queued the dispatched islands' tick results into
// host_results_ (dispatch order): reads them and appends their failure
// tuples to the caller's buffers in island order, voxel order
// (island_buffer.cpp:864-966).
pfsf_result Engine::finish_dispatch(const std::vector<Island*>& dispatched, bool drain, void* fail_addr,
                                    int32_t dbb_count, int32_t dbb_cap, pfsf_tick_result* result,
                                    int32_t legacy_cap) {
    if (!dispatched.empty()) {
        if (!CU_OK(cudaStreamSynchronize(stream_))) return PFSF_ERROR_VULKAN;
        // failure tuples in island order, voxel order (island_buffer.cpp:864-966)
        int32_t legacy_count = 0;
        bool any_copy = false;
        for (size_t k = 0; k < dispatched.size(); k++) {
            Island* s = dispatched[k];
            s->prev_macro = s->last_macro;
            s->last_macro = host_results_[k].macro_max;
            const uint32_t key = host_results_[k].phi_max_key;
            if (key != 0u) {
                const uint32_t b = (key & 0x80000000u) ? (key & 0x7fffffffu) : ~key;
                std::memcpy(&s->phi_max, &b, 4);
            }
            const int32_t total = host_results_[k].fail_total;
            if (drain && total > 0 && dbb_count < dbb_cap) {
                const int32_t take = std::min(total, dbb_cap - dbb_count);
                cudaMemcpyAsync(static_cast<int32_t*>(fail_addr) + 1 + 4 * (int64_t)dbb_count, s->tuples,
                                (size_t)take * 16, cudaMemcpyDeviceToHost, stream_);
                dbb_count += take;
                any_copy = true;
            }
            if (result && result->events && total > 0 && legacy_count < legacy_cap) {
                const int32_t take = std::min(total, legacy_cap - legacy_count);
                cudaMemcpyAsync(result->events + legacy_count, s->tuples, (size_t)take * 16, cudaMemcpyDeviceToHost,
                                stream_);
                legacy_count += take;
                any_copy = true;
            }
            s->dirty = false;
        }
        if (any_copy && !CU_OK(cudaStreamSynchronize(stream_))) return PFSF_ERROR_VULKAN;
        if (drain) *static_cast<int32_t*>(fail_addr) = dbb_count;
        if (result) result->count = legacy_count;
    }
    return PFSF_OK;
}

pfsf_result Engine::island_phi_max(int32_t id, float* out) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    Island* s = find(id);
    if (!out || !s) return PFSF_ERROR_INVALID_ARG;
    *out = s->phi_max;
    return PFSF_OK;
}

pfsf_result Engine::read_stress(int32_t id, float* out, int32_t cap, int32_t* count) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!out || !count) return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    *count = 0;
    if (cap <= 0) return PFSF_ERROR_VULKAN;
    if (!ensure_compat(*s)) return PFSF_ERROR_OUT_OF_VRAM;
    const int64_t nf = std::min<int64_t>(s->n, cap);
    if (!CU_OK(cudaMemcpyAsync(out, s->phi, (size_t)nf * 4, cudaMemcpyDeviceToHost, stream_)) ||
        !CU_OK(cudaStreamSynchronize(stream_)))
        return PFSF_ERROR_VULKAN;
    *count = (int32_t)nf;
    return PFSF_OK;
}

pfsf_result Engine::debug_read_field(int32_t id, int32_t field, void* out, int64_t bytes, int64_t* out_bytes) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!out || !out_bytes || bytes < 0) return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    if (!ensure_compat(*s)) return PFSF_ERROR_OUT_OF_VRAM;
    if (field == 5) {
        struct {
            int32_t cheb, pcg, mg;
            float prev, last;
        } st{s->chebyshev_iter, s->pcg_alloc ? 1 : 0, s->mg_alloc ? 1 : 0, s->prev_macro, s->last_macro};
        *out_bytes = (int64_t)sizeof(st);
        std::memcpy(out, &st, (size_t)std::min<int64_t>(bytes, sizeof(st)));
        return PFSF_OK;
    }
    const void* src = nullptr;
    int64_t size = 0;
    switch (field) {
        case 0: src = s->phi; size = s->n * 4; break;
        case 1: src = s->H; size = s->n * 4; break;
        case 2: src = s->D; size = s->n * 4; break;
        case 3: src = s->fail; size = s->n; break;
        case 4: src = s->macro; size = s->nmb * 4; break;
        case 6: src = s->src; size = s->n * 4; break;
        case 7: src = s->sigma; size = s->n * 24; break;
        case 8: src = s->type; size = s->n; break;
        case 9: src = s->maxphi; size = s->n * 4; break;
        case 10: src = s->rcomp; size = s->n * 4; break;
        case 11: src = s->rtens; size = s->n * 4; break;
        case 12: src = s->agg; size = s->amg_alloc ? s->n * 4 : 0; break;
        case 13: src = s->aw; size = s->amg_alloc ? s->n * 4 : 0; break;
        case 14: src = s->adc; size = s->amg_alloc ? s->amg_nc * 4 : 0; break;
        default: return PFSF_ERROR_INVALID_ARG;
    }
    *out_bytes = size;
    const int64_t c = std::min(size, bytes);
    if (c > 0 && (!CU_OK(cudaMemcpyAsync(out, src, (size_t)c, cudaMemcpyDeviceToHost, stream_)) ||
                  !CU_OK(cudaStreamSynchronize(stream_))))
        return PFSF_ERROR_VULKAN;
    return PFSF_OK;
}

pfsf_result Engine::get_sparse_buffer(int32_t id, void** addr, int64_t* bytes) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!addr || !bytes) return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    if (!ensure_compat(*s)) return PFSF_ERROR_OUT_OF_VRAM;
    if (!s->sparse_host) {
        if (!CU_OK(cudaMallocHost(&s->sparse_host, (size_t)kSparseCapacity * kSparseRecordBytes)))
            return PFSF_ERROR_VULKAN;
        std::memset(s->sparse_host, 0, (size_t)kSparseCapacity * kSparseRecordBytes);
        s->sparse_dev = dalloc(*s, (size_t)kSparseCapacity * kSparseRecordBytes);
        if (!s->sparse_dev) return PFSF_ERROR_VULKAN;
    }
    *addr = s->sparse_host;
    *bytes = (int64_t)kSparseCapacity * kSparseRecordBytes;
    return PFSF_OK;
}

// pfsf_engine.cpp:332-402
pfsf_result Engine::notify_sparse(int32_t id, int32_t count) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (count <= 0) return PFSF_OK;
    Island* s = find(id);
    if (!s || !s->sparse_host) return PFSF_ERROR_INVALID_ARG;
    const int c = std::min(count, kSparseCapacity);
    bool ok = CU_OK(cudaMemcpyAsync(s->sparse_dev, s->sparse_host, (size_t)c * kSparseRecordBytes,
                                    cudaMemcpyHostToDevice, stream_));
    compat::sparse_scatter(stream_, s->sparse_dev, c, s->n, s->src, s->sigma, s->type, s->maxphi, s->rcomp, s->rtens);
    launches_++;
    ok &= CU_OK(cudaStreamSynchronize(stream_));
    s->dirty = true;
    if (!ok) return PFSF_ERROR_VULKAN;
    s->mg_dirty = true;
    s->amg_dirty = true;
    return PFSF_OK;
}

}  // namespace pfsf_b200
