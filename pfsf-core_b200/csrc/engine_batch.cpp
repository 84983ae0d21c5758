// The reference tick for many islands at once (pfsf_tick_dbb / pfsf_tick),
// and the tail of the tolerance tick (pfsf_tick_tolerance).
//
// The reference records and submits each dirty island's tick separately
// (L1-native/libpfsf/src/pfsf_engine.cpp:439-494: recordSolveSteps +
// recordPhaseFieldEvolve + recordFailureDetection, then submitAndWait), so a
// tick of many small islands is hundreds of tiny dispatches per island.
// Here the schedule of every island is decided on the host first (the
// adaptive RBGS -> PCG switch from the previous tick's macro residuals,
// dispatcher.cpp:106-186; the V-cycle cadence from the aspect ratio,
// :55-66, :188-238), islands with the same schedule form a group, and each
// step of a group's schedule is ONE launch over all the group's islands
// (compat::batch).  Per-island state that changes from tick to tick --
// chebyshev_iter (warm-up damping), the coarse ping-pong slots, the PCG
// residual slot, the array pointers -- lives in a device table written once
// per tick, so the launch sequence depends only on the group structure: it
// is captured once as a CUDA graph and replayed on every later tick with the
// same structure.  The upload from the caller's pinned arrays and the stress
// readback into its stress buffer are kernels over the device-visible
// mappings of those arrays, inside the graph.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "compat.h"
#include "engine.h"
#include "tick_batch.h"

namespace pfsf_b200 {

#define CU_OK(expr) (cudaSuccess == (expr))

namespace {

// The schedule one island runs this tick (dispatcher.cpp:106-186).
struct Plan {
    int pcg;       // 1: RBGS then PCG steps (rb, pc), 0: RBGS only
    int rb, pc;
    int interval;  // V-cycle every `interval` steps (aspect ratio, dispatcher.cpp:55-66)
    int extra;     // a second V-cycle when the aspect ratio is >= 8 (dispatcher.cpp:233)
    int mg;        // V-cycles this tick (multigrid available and the cadence reached)
    int mg_dirty;  // coarse conductivity / type rebuilt at the first V-cycle
    int amg;       // aggregation correction at the PCG start (dispatcher_amg.cpp:83)
    int amg_build; // aggregates rebuilt from sigma / type first
    bool operator<(const Plan& o) const { return std::memcmp(this, &o, sizeof(Plan)) < 0; }
    bool operator==(const Plan& o) const { return std::memcmp(this, &o, sizeof(Plan)) == 0; }
};

// Device-memory bytes of one island's tick: every array a pass touches
// counted once per pass, per fine voxel (n) or coarse cell (n1, n2).  An RBGS
// colour sweep or coarse Jacobi pass moves the SoA-6 conductivity (24 B),
// phi in and out (8), the source (4), the type (1) and H read and written
// (8): 45 B per cell.
double tick_bytes(const Island& s, const Plan& p, bool tail_only, bool phase, bool compact, bool uploaded,
                  bool stress) {
    const double n = (double)s.n, n1 = (double)s.n1, n2 = (double)s.n2;
    const double sweep = 45.0;
    double b = 0.0;
    if (tail_only) {
        b += 8.0 * n + 37.0 * n;  // phi taken from the solve; history update
    } else {
        const double vc = 2.0 * sweep * n + 33.0 * n + 8.0 * n1 +
                          2.0 * (4.0 * sweep * n1 + 33.0 * n1 + 8.0 * n2 + 4.0 * sweep * n2 + 8.0 * n1 + 4.0 * n2) +
                          8.0 * n + 4.0 * n1;
        int vcycles = 0, sweeps = 0;
        for (int k = 0; k < p.rb; k++) {
            if (p.mg && k > 0 && (k % p.interval) == 0) vcycles += p.extra ? 2 : 1;
            else sweeps++;
        }
        b += sweeps * sweep * n + vcycles * vc;
        if (p.mg_dirty) b += 25.0 * n + 50.0 * n1 + 25.0 * n2;
        if (p.pcg) b += (28.0 + 33.0 + 41.0) * n + p.pc * (33.0 + 53.0 + 37.0) * n;
        // aggregation correction: build (sigma, type; agg, w), coarse (agg, w, r),
        // prolong (agg, w, phi rw), then the PCG start again (matvec, update)
        if (p.amg_build) b += 33.0 * n;
        if (p.amg) b += 12.0 * n + 16.0 * n + (33.0 + 41.0) * n;
    }
    if (phase) b += 8.0 * n + 47.0 * n;
    b += 42.0 * n;               // failure pass (codes, residual and phi maxima, block counts)
    if (compact) b += 1.0 * n;   // the tuple write reads the codes once
    if (uploaded) b += 45.0 * n; // the uploaded arrays written into HBM
    if (stress) b += 4.0 * n;    // phi read for the stress readback
    return b;
}

inline int imax3(int a, int b, int c) { return std::max(a, std::max(b, c)); }
inline int imin3(int a, int b, int c) { return std::min(a, std::min(b, c)); }

}  // namespace

pfsf_result Engine::last_tick_report(pfsf_tick_report* out) const {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!out || !tbatch_ || !tbatch_->have_tick) return PFSF_ERROR_INVALID_ARG;
    pfsf_tick_report r = tbatch_->last;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, tbatch_->ev0, tbatch_->ev1) != cudaSuccess) {
        cudaGetLastError();
        ms = -1.0f;
    }
    r.device_ms = ms;
    *out = r;
    return PFSF_OK;
}

void Engine::free_tick_batch() {
    if (!tbatch_) return;
    TickBatch& B = *tbatch_;
    cudaStreamSynchronize(stream_);
    if (B.ev0) cudaEventDestroy(B.ev0);
    if (B.ev1) cudaEventDestroy(B.ev1);
    if (B.exec) cudaGraphExecDestroy(B.exec);
    for (cudaStream_t ls : B.lanes) cudaStreamDestroy(ls);
    for (cudaEvent_t le : B.lane_done) cudaEventDestroy(le);
    if (B.fork) cudaEventDestroy(B.fork);
    if (B.d_tab) cudaFree(B.d_tab);
    if (B.d_bs) cudaFree(B.d_bs);
    if (B.d_res) cudaFree(B.d_res);
    if (B.h_tab) cudaFreeHost(B.h_tab);
    if (B.h_bs) cudaFreeHost(B.h_bs);
    tbatch_.reset();
}

pfsf_result Engine::tick_batched(const std::vector<Island*>& set, int32_t want_cap,
                                 const std::vector<const float*>* phi_in) {
    if (set.empty()) return PFSF_OK;
    const auto host_t0 = std::chrono::steady_clock::now();
    if (!tbatch_) tbatch_.reset(new TickBatch());
    TickBatch& B = *tbatch_;
    const int nisl = (int)set.size();
    const bool tail_only = phi_in != nullptr;
    // the reference tick uploads every dispatched (dirty) island; the
    // tolerance tick only the dirty ones
    auto uploads = [&](const Island& s) { return s.hosts.registered && (!tail_only || s.dirty); };

    // ---- per-island plans (and the allocations they need), in call order
    std::vector<Plan> plan(nisl);
    for (int k = 0; k < nisl; k++) {
        Island& s = *set[k];
        Plan p{};
        // an island cannot fail more voxels than it has
        const int32_t need = (int32_t)std::min<int64_t>(want_cap, s.n);
        if (need > 0 && s.tuple_cap < need) {
            s.tuples = (int32_t*)dalloc(s, (size_t)need * 16);
            if (!s.tuples) return PFSF_ERROR_OUT_OF_VRAM;
            s.tuple_cap = need;
        }
        if (tail_only) {
            if (uploads(s)) s.mg_dirty = s.amg_dirty = true;
            plan[k] = p;
            continue;
        }
        const int maxd = imax3(s.lx, s.ly, s.lz), mind = imin3(s.lx, s.ly, s.lz);
        p.interval = kMgInterval;
        if (mind > 0) {
            const int ratio = maxd / mind;
            if (ratio >= 8) p.interval = std::max(1, kMgInterval / 4);
            else if (ratio >= 4) p.interval = std::max(1, kMgInterval / 2);
        }
        p.extra = (mind > 0 && maxd >= 8 * mind) ? 1 : 0;
        const float prev = s.prev_macro, curr = s.last_macro;
        const bool stalled = ((prev > 1e-10f) ? (curr / prev) : 0.0f) > 0.95f;
        if (stalled && pcg_enabled_ && !s.pcg_alloc && !ensure_pcg(s)) return PFSF_ERROR_OUT_OF_VRAM;
        if (pcg_enabled_ && s.n <= kPcgMaxN && s.pcg_alloc) {
            p.pcg = 1;
            p.rb = stalled ? kPcgMinRbgs : std::max(kPcgMinRbgs, kStepsMajor - kPcgMinSteps);
            p.pc = kStepsMajor - p.rb;
        } else {
            p.rb = kStepsMajor;
        }
        bool any_v = false;
        for (int q = 1; q < p.rb; q++) any_v |= (q % p.interval) == 0;
        p.mg = (cfg_.enable_multigrid && maxd > 4 && any_v) ? 1 : 0;
        if (p.mg && !s.mg_alloc) {
            if (!ensure_mg(s)) return PFSF_ERROR_OUT_OF_VRAM;
            s.mg_dirty = true;
        }
        if (s.hosts.registered) s.mg_dirty = s.amg_dirty = true;  // the upload below refreshes the fine inputs
        p.mg_dirty = (p.mg && s.mg_dirty) ? 1 : 0;
        if (p.pcg && amg_enabled_) {
            if (!ensure_amg(s)) return PFSF_ERROR_OUT_OF_VRAM;
            p.amg = 1;
            p.amg_build = s.amg_dirty ? 1 : 0;
        }
        plan[k] = p;
    }

    // ---- groups: islands of equal plans, contiguous in the table
    std::vector<int> order(nisl);
    for (int k = 0; k < nisl; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return plan[a] < plan[b]; });
    std::vector<std::pair<int, int>> groups;  // [begin, end) in table order
    for (int k = 0; k < nisl;) {
        int e = k + 1;
        while (e < nisl && plan[order[e]] == plan[order[k]]) e++;
        groups.emplace_back(k, e);
        k = e;
    }
    const int ng = (int)groups.size();

    // ---- capacity of the device table / prefixes / results
    const int need_bs = (nisl + ng + ng + 1) * compat::kbKinds + compat::kbKinds * (nisl + 1);
    if (nisl > B.cap_isl || need_bs > B.cap_bs) {
        cudaStreamSynchronize(stream_);
        if (B.exec) cudaGraphExecDestroy(B.exec);
        B.exec = nullptr;
        B.key.clear();
        if (B.d_tab) cudaFree(B.d_tab);
        if (B.d_res) cudaFree(B.d_res);
        if (B.h_tab) cudaFreeHost(B.h_tab);
        if (B.d_bs) cudaFree(B.d_bs);
        if (B.h_bs) cudaFreeHost(B.h_bs);
        B.d_tab = nullptr; B.d_res = nullptr; B.h_tab = nullptr; B.d_bs = nullptr; B.h_bs = nullptr;
        B.cap_isl = std::max(nisl, 2 * B.cap_isl);
        B.cap_bs = std::max(need_bs, 2 * B.cap_bs);
        if (!CU_OK(cudaMalloc(&B.d_tab, sizeof(compat::CIsl) * B.cap_isl)) ||
            !CU_OK(cudaMalloc(&B.d_res, sizeof(TickResult) * B.cap_isl)) ||
            !CU_OK(cudaMallocHost(&B.h_tab, sizeof(compat::CIsl) * B.cap_isl)) ||
            !CU_OK(cudaMalloc(&B.d_bs, sizeof(int) * B.cap_bs)) ||
            !CU_OK(cudaMallocHost(&B.h_bs, sizeof(int) * B.cap_bs))) {
            cudaGetLastError();
            free_tick_batch();
            return PFSF_ERROR_OUT_OF_VRAM;
        }
    }
    if (nisl > host_results_cap_) {
        cudaStreamSynchronize(stream_);
        cudaFreeHost(host_results_);
        host_results_cap_ = nisl * 2;
        if (!CU_OK(cudaMallocHost((void**)&host_results_, sizeof(TickResult) * host_results_cap_)))
            return PFSF_ERROR_VULKAN;
    }

    // ---- the table (every tick: pointers and schedule state may change)
    for (int j = 0; j < nisl; j++) {
        const int k = order[j];
        Island& s = *set[k];
        compat::CIsl& c = B.h_tab[j];
        std::memset(&c, 0, sizeof(c));
        c.lx = s.lx; c.ly = s.ly; c.lz = s.lz;
        c.ox = s.origin.x; c.oy = s.origin.y; c.oz = s.origin.z;
        c.n = s.n; c.nmb = s.nmb;
        c.phi = s.phi; c.src = s.src; c.sigma = s.sigma; c.rcomp = s.rcomp; c.rtens = s.rtens; c.maxphi = s.maxphi;
        c.hyd = s.hyd; c.H = s.H; c.D = s.D; c.Dold = s.Dold; c.type = s.type; c.fail = s.fail; c.macro = s.macro;
        c.res_macro = &B.d_res[k].macro_max;
        c.res_fail = &B.d_res[k].fail_total;
        c.res_phimax = &B.d_res[k].phi_max_key;
        c.fcounts = s.fcounts; c.foffsets = s.foffsets;
        c.tuples = want_cap > 0 ? s.tuples : nullptr;
        c.tuple_cap = (int32_t)std::min<int64_t>(want_cap, s.n);
        c.iter0 = s.chebyshev_iter;
        c.cur1 = s.cur1; c.cur2 = s.cur2; c.rcur = s.rcur;
        if (plan[k].mg) {
            c.l1x = s.l1[0]; c.l1y = s.l1[1]; c.l1z = s.l1[2];
            c.l2x = s.l2[0]; c.l2y = s.l2[1]; c.l2z = s.l2[2];
            c.n1 = s.n1; c.n2 = s.n2;
            c.phi1[0] = s.phi1[0]; c.phi1[1] = s.phi1[1]; c.src1 = s.src1; c.sig1 = s.sig1; c.type1 = s.type1;
            c.phi2[0] = s.phi2[0]; c.phi2[1] = s.phi2[1]; c.src2 = s.src2; c.sig2 = s.sig2; c.type2 = s.type2;
        }
        if (plan[k].pcg) {
            c.r[0] = s.r[0]; c.r[1] = s.r[1]; c.p = s.p; c.ap = s.ap; c.invdiag = s.invdiag; c.partial = s.partial;
            c.red = s.red;
        }
        if (plan[k].amg) {
            c.agg = s.agg; c.aw = s.aw; c.adc = s.adc; c.aec = s.aec;
            c.anc = s.amg_nc;
        }
        const HostBuffers& h = s.hosts;
        const bool mapped = uploads(s) && h.m_phi && h.m_source && h.m_cond && h.m_type && h.m_rcomp && h.m_rtens &&
                            h.m_maxphi && (!(h.lookups_registered && h.curing) || h.m_curing);
        if (mapped) {
            c.h_phi = static_cast<const float*>(h.m_phi);
            c.h_src = static_cast<const float*>(h.m_source);
            c.h_sigma = static_cast<const float*>(h.m_cond);
            c.h_type = static_cast<const uint8_t*>(h.m_type);
            c.h_rcomp = static_cast<const float*>(h.m_rcomp);
            c.h_rtens = static_cast<const float*>(h.m_rtens);
            c.h_maxphi = static_cast<const float*>(h.m_maxphi);
            c.h_curing = (h.lookups_registered && h.curing) ? static_cast<const float*>(h.m_curing) : nullptr;
        }
        if (h.stress_out && h.stress_bytes > 0 && h.m_stress) {
            c.h_stress = static_cast<float*>(h.m_stress);
            c.stress_n = std::min<int64_t>(s.n, h.stress_bytes / 4);
        }
        c.phi_in = tail_only ? (*phi_in)[k] : nullptr;
    }

    // ---- block prefixes: per group, then the whole set (for the shared steps)
    std::vector<compat::BGroup> G(ng + 1);
    int bo = 0;
    auto fill_group = [&](compat::BGroup& g, int b, int e) {
        g.nisl = e - b;
        g.tab = B.d_tab + b;
        g.bstart = B.d_bs + bo;
        for (int kind = 0; kind < compat::kbKinds; kind++) {
            int acc = 0;
            int* row = B.h_bs + bo + kind * (g.nisl + 1);
            for (int j = b; j < e; j++) {
                row[j - b] = acc;
                acc += (int)compat::batch_blocks(B.h_tab[j], kind);
            }
            row[g.nisl] = acc;
            g.blocks[kind] = acc;
        }
        bo += compat::kbKinds * (g.nisl + 1);
    };
    for (int q = 0; q < ng; q++) fill_group(G[q], groups[q].first, groups[q].second);
    compat::BGroup& ALL = G[ng];
    fill_group(ALL, 0, nisl);

    // ---- the structure key of the launch sequence
    std::vector<int64_t> key;
    key.reserve(8 + (size_t)nisl * 5 + (size_t)ng * 8);
    key.push_back(nisl);
    key.push_back(want_cap > 0 ? 1 : 0);
    key.push_back(cfg_.enable_phase_field ? 1 : 0);
    key.push_back(tail_only ? 1 : 0);
    for (int q = 0; q < ng; q++) {
        const Plan& p = plan[order[groups[q].first]];
        key.push_back(groups[q].second - groups[q].first);
        key.insert(key.end(), {p.pcg, p.rb, p.pc, p.interval, p.extra, p.mg, p.mg_dirty, p.amg, p.amg_build});
    }
    for (int j = 0; j < nisl; j++) {
        const compat::CIsl& c = B.h_tab[j];
        key.insert(key.end(), {(int64_t)c.lx, (int64_t)c.ly, (int64_t)c.lz, c.h_phi ? 1 : 0, c.h_stress ? 1 : 0});
    }

    if (!B.ev0 && (!CU_OK(cudaEventCreate(&B.ev0)) || !CU_OK(cudaEventCreate(&B.ev1)))) return PFSF_ERROR_VULKAN;
    cudaEventRecord(B.ev0, stream_);
    bool ok = CU_OK(cudaMemcpyAsync(B.d_tab, B.h_tab, sizeof(compat::CIsl) * nisl, cudaMemcpyHostToDevice, stream_));
    ok &= CU_OK(cudaMemcpyAsync(B.d_bs, B.h_bs, sizeof(int) * bo, cudaMemcpyHostToDevice, stream_));
    // islands whose arrays could not be pinned: uploaded by copies
    for (int j = 0; j < nisl; j++) {
        Island& s = *set[order[j]];
        if (uploads(s) && !B.h_tab[j].h_phi) ok &= upload(s);
    }
    if (!ok) return PFSF_ERROR_VULKAN;

    // a tick of another structure is captured again; its graph then updates
    // the instantiated one in place when the topology is the same (only
    // launch shapes and arguments differ), else it is instantiated anew
    const bool replayed = B.exec != nullptr && B.key == key;
    bool updated = false;
    if (!replayed) {
        // ---- record the tick once, under capture
        B.effects.assign(ng, TickEffect{});
        int64_t nl = 0;
        cudaGraph_t graph = nullptr;
        // groups touch disjoint islands: each group's chain (its upload, macro
        // seeding, schedule) is a branch of its own, on one of up to kLanes
        // capture streams, so small groups run beside big ones and a group's
        // sweeps start as soon as its own arrays are in; the tail over all
        // islands joins them.
        const int lanes = tail_only ? 0 : std::min(ng, kLanes);
        for (int l = (int)B.lanes.size(); l < lanes; l++) {
            cudaStream_t ls = nullptr;
            cudaEvent_t le = nullptr;
            if (!CU_OK(cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking)) ||
                !CU_OK(cudaEventCreateWithFlags(&le, cudaEventDisableTiming)))
                return PFSF_ERROR_VULKAN;
            B.lanes.push_back(ls);
            B.lane_done.push_back(le);
        }
        if (lanes > 0 && !B.fork &&
            !CU_OK(cudaEventCreateWithFlags(&B.fork, cudaEventDisableTiming)))
            return PFSF_ERROR_VULKAN;
        if (!CU_OK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal))) return PFSF_ERROR_VULKAN;
        cudaStream_t st = stream_;
        bool fork_ok = true;
        if (lanes > 0) {
            fork_ok &= CU_OK(cudaEventRecord(B.fork, stream_));
            for (int l = 0; l < lanes; l++) fork_ok &= CU_OK(cudaStreamWaitEvent(B.lanes[l], B.fork, 0));
        }
        if (tail_only) {
            compat::batch::upload(st, ALL);
            // the solved phi (the history update below is the one the
            // reference performs inside its sweeps, rbgs_smooth.comp.glsl:177-191)
            compat::batch::take_phi(st, ALL);
            compat::batch::macro_fill(st, ALL);
            compat::batch::history(st, ALL);
            nl += 4;
        }
        for (int q = 0; q < ng && !tail_only; q++) {
            const compat::BGroup& g = G[q];
            st = B.lanes[q % lanes];
            compat::batch::upload(st, g);
            compat::batch::macro_fill(st, g);
            nl += 2;
            const Plan& p = plan[order[groups[q].first]];
            TickEffect& ef = B.effects[q];
            auto rbgs_step = [&](int sidx_damp) {
                for (int c = 0; c < 8; c++)
                    compat::batch::rbgs_color(st, g, c, sidx_damp, kWarmupSteps, kDampingFactor);
                nl += 8;
                ef.steps++;
            };
            auto coarse = [&](int level, int sd) {
                compat::batch::jacobi(st, g, level, level == 1 ? ef.f1 : ef.f2, sd, kWarmupSteps, kDampingFactor);
                (level == 1 ? ef.f1 : ef.f2)++;
                nl++;
            };
            // dispatcher_vcycle.cpp:342-392 with the W-cycle legs (:315-340)
            auto vcycle = [&]() {
                const int sd = ef.steps;  // damping of the whole cycle: chebyshev_iter at its start
                rbgs_step(sd);
                compat::batch::restrict_to(st, g, 1, ef.f1, ef.f2);
                nl++;
                for (int leg = 0; leg < 2; leg++) {
                    coarse(1, sd);
                    coarse(1, sd);
                    compat::batch::restrict_to(st, g, 2, ef.f1, ef.f2);
                    nl++;
                    for (int k = 0; k < 4; k++) coarse(2, sd);
                    compat::batch::prolong_from(st, g, 2, ef.f1, ef.f2);
                    nl++;
                    coarse(1, sd);
                    coarse(1, sd);
                }
                compat::batch::prolong_from(st, g, 1, ef.f1, ef.f2);
                nl++;
                rbgs_step(sd);
            };
            bool mg_dirty = p.mg_dirty != 0;
            auto try_vcycle = [&](int k) {
                if (!(k > 0 && (k % p.interval) == 0 && p.mg)) return false;
                if (mg_dirty) {  // uploadMultigridData (island_buffer.cpp:600-776), on the device
                    compat::batch::downsample(st, g, 1);
                    compat::batch::downsample(st, g, 2);
                    nl += 2;
                    mg_dirty = false;
                    ef.downsampled = 1;
                }
                vcycle();
                if (p.extra) vcycle();
                return true;
            };
            for (int k = 0; k < p.rb; k++) {
                if (try_vcycle(k)) continue;
                rbgs_step(ef.steps);
            }
            if (p.pcg) {
                // dispatcher_pcg.cpp:254-298
                compat::batch::pcg_precompute(st, g);
                compat::batch::pcg_matvec(st, g, 0);
                compat::batch::pcg_update(st, g, 1, ef.fr);
                nl += 3;
                if (p.amg) {
                    // dispatcher_amg.cpp:83-161 from the start's residual, then
                    // the start again from the corrected phi
                    if (p.amg_build) {
                        compat::batch::amg_build(st, g);
                        nl++;
                    }
                    compat::batch::amg_coarse(st, g, ef.fr);
                    compat::batch::amg_prolong(st, g);
                    compat::batch::pcg_matvec(st, g, 0);
                    compat::batch::pcg_update(st, g, 1, ef.fr);
                    nl += 4;
                }
                compat::batch::finalize(st, g, 0, 0);
                nl++;
                for (int k = 0; k < p.pc; k++) {
                    compat::batch::pcg_matvec(st, g, 1);
                    compat::batch::finalize(st, g, 1, k == 0 ? 0 : 1);
                    compat::batch::pcg_update(st, g, 0, ef.fr);
                    ef.fr++;
                    compat::batch::finalize(st, g, 2, 0);
                    compat::batch::pcg_direction(st, g, ef.fr);
                    nl += 5;
                }
            }
        }
        st = stream_;
        for (int l = 0; l < lanes; l++) {
            fork_ok &= CU_OK(cudaEventRecord(B.lane_done[l], B.lanes[l]));
            fork_ok &= CU_OK(cudaStreamWaitEvent(stream_, B.lane_done[l], 0));
        }
        // the tick's tail over every island (pfsf_engine.cpp:513-560)
        if (cfg_.enable_phase_field) {
            compat::batch::copy_damage(st, ALL);
            compat::batch::phase_field(st, ALL, kPfL0, kPfGc, kPfRelax, 1);
            nl += 2;
        }
        compat::batch::failure_scan(st, ALL);
        nl++;
        if (want_cap > 0) {
            compat::batch::fail_compact(st, ALL);
            nl += 2;
        }
        compat::batch::stress_out(st, ALL);
        nl++;
        const cudaError_t ce = cudaStreamEndCapture(stream_, &graph);
        if (ce != cudaSuccess || !graph || !fork_ok) {
            if (graph) cudaGraphDestroy(graph);
            std::fprintf(stderr, "[libpfsf] tick capture failed: %s\n", cudaGetErrorString(ce));
            cudaGetLastError();
            return PFSF_ERROR_VULKAN;
        }
        if (B.exec) {
            cudaGraphExecUpdateResultInfo info{};
            if (cudaGraphExecUpdate(B.exec, graph, &info) == cudaSuccess) {
                updated = true;
            } else {
                cudaGetLastError();
                cudaGraphExecDestroy(B.exec);
                B.exec = nullptr;
            }
        }
        const cudaError_t ie = updated ? cudaSuccess : cudaGraphInstantiate(&B.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            std::fprintf(stderr, "[libpfsf] tick graph instantiation failed: %s\n", cudaGetErrorString(ie));
            cudaGetLastError();
            B.exec = nullptr;
            return PFSF_ERROR_VULKAN;
        }
        B.key = key;
        B.graph_launches = nl;
    }
    const auto host_t1 = std::chrono::steady_clock::now();
    if (!CU_OK(cudaGraphLaunch(B.exec, stream_))) return PFSF_ERROR_VULKAN;
    launches_ += B.graph_launches;
    // stress buffers that could not be mapped: copied
    for (Island* s : set) {
        if (s->hosts.stress_out && s->hosts.stress_bytes > 0 && !s->hosts.m_stress) {
            const int64_t nf = std::min<int64_t>(s->n, s->hosts.stress_bytes / 4);
            if (!CU_OK(cudaMemcpyAsync(s->hosts.stress_out, s->phi, (size_t)nf * 4, cudaMemcpyDeviceToHost, stream_)))
                return PFSF_ERROR_VULKAN;
        }
    }
    // results (call order) in one copy; finish_dispatch reads them after its sync
    if (!CU_OK(cudaMemcpyAsync(host_results_, B.d_res, sizeof(TickResult) * nisl, cudaMemcpyDeviceToHost, stream_)))
        return PFSF_ERROR_VULKAN;
    cudaEventRecord(B.ev1, stream_);
    pfsf_tick_report& R = B.last;
    R = pfsf_tick_report{};
    R.struct_bytes = (int32_t)sizeof(R);
    R.islands = nisl;
    R.groups = tail_only ? 1 : ng;
    R.graph_replayed = replayed ? 1 : (updated ? 2 : 0);
    R.kernel_launches = B.graph_launches;
    R.host_us = (int32_t)std::min<int64_t>(
        INT32_MAX, std::chrono::duration_cast<std::chrono::microseconds>(host_t1 - host_t0).count());
    for (int j = 0; j < nisl; j++) {
        const Island& s = *set[order[j]];
        R.algorithmic_bytes += tick_bytes(s, plan[order[j]], tail_only, cfg_.enable_phase_field, want_cap > 0,
                                          B.h_tab[j].h_phi != nullptr, B.h_tab[j].h_stress != nullptr);
        R.grid_voxels += (double)s.n;
    }
    B.have_tick = true;

    // ---- per-island schedule state after the tick
    for (int q = 0; q < ng; q++) {
        const TickEffect& ef = B.effects[q];
        for (int j = groups[q].first; j < groups[q].second; j++) {
            Island& s = *set[order[j]];
            s.chebyshev_iter += ef.steps;
            s.cur1 = (s.cur1 + ef.f1) & 1;
            s.cur2 = (s.cur2 + ef.f2) & 1;
            s.rcur = (s.rcur + ef.fr) & 1;
            if (ef.downsampled) s.mg_dirty = false;
            if (plan[order[j]].amg_build) s.amg_dirty = false;
        }
    }
    return PFSF_OK;
}

}  // namespace pfsf_b200
