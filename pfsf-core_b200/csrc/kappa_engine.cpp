// Engine side of the tolerance solve: kappa-form registration, the packed
// device arena for a set of islands, upload / solve / readback.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "arena.h"
#include "compat.h"

namespace pfsf_b200 {

#define CU_OK(expr) (cudaSuccess == (expr))

namespace {
constexpr int64_t kAlignElems = 32;
inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }
inline int64_t ceil_div64(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Device-visible address of a caller's kappa-form host array for the arena's
// gather / scatter: the island's own earlier mapping when one covers the
// range (the reference-layout phi can be the same array), else a new mapped
// registration owned by the arena (unregistered with it); nullptr when the
// range cannot be mapped (already registered by someone else), and the
// island is then copied with cudaMemcpyAsync.
const void* map_arena_host(Island& s, void* p, int64_t bytes, std::vector<void*>& owned) {
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
    owned.push_back(p);
    void* d = nullptr;
    if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess || !d) {
        cudaGetLastError();
        return nullptr;
    }
    return d;
}

// Compulsory bytes of the passes one island's solve made: every array a pass
// reads or writes counted once per pass (what a perfectly cached streaming
// implementation must move), per grid voxel / coarse cell.
double solve_bytes(const KDesc& d, int prec, int nu, int coarse_sweeps, int smoother, int cheb_k, int wcycle) {
    const double kb = prec > 0 ? 2.0 : 4.0;   // preconditioner kappa
    const double cb = prec > 0 ? 2.0 : 4.0;   // coarse coefficient
    const double wf = 4.0;                    // fine-level weights: the 1/kappa array of the solve
    const double n0 = (double)d.n;
    const double cell = 26.0 * cb + 4.0;      // coefficients + diagonal
    double setup = n0 * (kb + 4.0 + 8.0);     // the two 1/kappa arrays (op_rk)
    double vc = 0.0;
    if (d.nlev > 1) {
        setup += n0 * (kb + 1.0) + (double)d.lev[1].n * cell;
        for (int l = 1; l < d.nlev - 1; l++) setup += (double)d.lev[l].n * cell + (double)d.lev[l + 1].n * cell;
        if (smoother == 1) {
            // Chebyshev: first step (r, dinv -> d, z), then per step a stencil
            // pass (weights, type, z, r, dinv, d rw) and an update pass (d, z rw, type)
            const double step = (wf + 1.0 + 4.0 + 4.0 + 4.0 + 8.0) + (4.0 + 8.0 + 1.0);
            vc += n0 * 16.0 + (2.0 * cheb_k - 1.0) * n0 * step;
            setup += n0 * (kb + 1.0 + 4.0);  // inverse diagonal
        } else {
            vc += 2.0 * nu * n0 * (wf + 1.0 + 8.0 + 4.0);      // fine GS sweeps: weights, type, z rw, r
        }
        vc += n0 * (wf + 1.0 + 4.0 + 4.0) + (double)d.lev[1].n * 8.0;  // residual + restriction
        vc += n0 * (1.0 + 8.0) + (double)d.lev[1].n * 4.0;    // prolongation
        double coarse = 0.0;
        for (int l = 1; l < d.nlev - 1; l++) {
            const double nl = (double)d.lev[l].n;
            coarse += (smoother == 1 ? (2.0 * cheb_k) * (cell + 4.0 + 8.0 + 8.0) : 2.0 * nu * (cell + 4.0 + 8.0)) * nl;
            coarse += nl * (cell + 8.0) + (double)d.lev[l + 1].n * 8.0;
            coarse += nl * (4.0 + 8.0) + (double)d.lev[l + 1].n * 4.0;
        }
        coarse += 2.0 * coarse_sweeps * (double)d.lev[d.nlev - 1].n * (cell + 4.0 + 8.0);
        // a W-cycle visits everything below the fine level twice
        vc += (wcycle && d.nlev > 2 ? 2.0 : 1.0) * coarse;
    } else {
        vc += 2.0 * coarse_sweeps * n0 * (wf + 1.0 + 8.0 + 4.0);
    }
    const double outer_res = n0 * (4.0 + 8.0 + 4.0 + 1.0 + 12.0);  // kappa, x64, b, type; r, e, z
    const double accumulate = n0 * (16.0 + 4.0);
    const double matvec = n0 * 13.0, update = n0 * 24.0, dot = n0 * 8.0, pupd = n0 * 16.0;
    const int outer = d.outer_iters + 1;                // residual evaluations
    const int corrections = d.outer_iters;              // inner solves
    // each correction: V-cycle + r.z + p-update before its first iteration and
    // after every iteration but the last, i.e. once per inner iteration overall
    double b = setup + outer * outer_res + corrections * accumulate;
    b += (double)d.inner_iters * (matvec + update + vc + dot + pupd);
    return b;
}
}  // namespace

pfsf_result Engine::register_kappa(int32_t id, const pfsf_island_kappa_buffers* b) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!b || !b->phi_addr || !b->source_addr || !b->kappa_addr || !b->voxel_type_addr)
        return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    const int64_t n = s->n;
    if (b->phi_bytes < 4 * n || b->source_bytes < 4 * n || b->kappa_bytes < 4 * n || b->voxel_type_bytes < n)
        return PFSF_ERROR_INVALID_ARG;
    HostBuffers& h = s->hosts;
    h.k_phi = b->phi_addr;
    h.k_source = b->source_addr;
    h.k_kappa = b->kappa_addr;
    h.k_type = b->voxel_type_addr;
    h.kappa_registered = true;
    if (!s->kappa) s->kappa.reset(new KappaState());
    s->kappa->registered = true;
    // the arena is rebuilt (and re-uploaded) when its island set changes
    if (arena_) {
        auto& ids = arena_->ids;
        if (std::find(ids.begin(), ids.end(), id) != ids.end()) arena_->prec = -2;  // force re-upload
    }
    return PFSF_OK;
}

void Engine::free_arena() {
    if (!arena_) return;
    cudaStreamSynchronize(stream_);
    for (void* h : arena_->pinned) cudaHostUnregister(h);
    if (arena_->solve_exec) cudaGraphExecDestroy(arena_->solve_exec);
    kappa::free_plain_graphs(arena_->plain);
    if (arena_->hdesc) cudaFreeHost(arena_->hdesc);
    if (arena_->base) cudaFree(arena_->base);
    if (arena_->hscratch) cudaFreeHost(arena_->hscratch);
    if (arena_->xf) cudaFree(arena_->xf);
    {
        std::lock_guard<std::mutex> lk(stats_mtx_);
        vram_used_ -= (int64_t)arena_->bytes + (arena_->xf ? arena_->nfine * 8 : 0);
    }
    arena_.reset();
}

bool Engine::build_arena(const std::vector<Island*>& set) {
    free_arena();
    auto A = std::make_unique<Arena>();
    A->prec = (int)precision_;
    int64_t fine = 0, coarse = 0, starts = 0;
    for (Island* s : set) {
        KDesc d{};
        d.lx = s->lx; d.ly = s->ly; d.lz = s->lz;
        d.n = s->n;
        d.off = fine;
        fine = align_up(fine + s->n, kAlignElems);
        d.nlev = kappa::plan_levels(s->lx, s->ly, s->lz, d.lev);
        for (int l = 1; l < d.nlev; l++) {
            d.lev[l].off = coarse;
            coarse = align_up(coarse + d.lev[l].n, kAlignElems);
        }
        d.soff = starts;
        starts = align_up(starts + flat_starts(s->lx, s->ly, s->lz), kAlignElems);
        A->desc.push_back(d);
        A->ids.push_back(s->id);
        const uint8_t* t = static_cast<const uint8_t*>(s->hosts.k_type);
        int64_t act = 0;
        for (int64_t i = 0; i < s->n; i++) act += t[i] == 1;
        A->active.push_back(act);
    }
    if (coarse == 0) coarse = kAlignElems;
    A->nfine = fine;
    A->ncoarse = coarse;
    const int nisl = (int)set.size();
    const size_t cbytes = A->prec > 0 ? 2 : 4;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off = (off + b + 255) / 256 * 256; return o; };
    const size_t o_type = take(fine), o_k32 = take(fine * 4), o_k16 = take(fine * 2), o_b = take(fine * 4),
                 o_x64 = take(fine * 8), o_r = take(fine * 4), o_e = take(fine * 4), o_z = take(fine * 4),
                 o_p = take(fine * 4), o_q = take(fine * 4), o_cd = take(coarse * 4), o_cf = take(coarse * 26 * cbytes),
                 o_cx = take(coarse * 4), o_cb = take(coarse * 4), o_desc = take(sizeof(KDesc) * nisl),
                 o_order = take(sizeof(int) * nisl), o_queue = take(256),
                 o_scr = take(sizeof(float) * kappa::plain_scratch_floats()), o_dinv = take(fine * 4),
                 o_d0 = take(fine * 4), o_rkp = take(fine * 4), o_rk32 = take(fine * 4), o_cdd = take(coarse * 4),
                 o_cx2 = take(coarse * 4),
                 o_flist = take(fine * 4), o_fstart = take((size_t)std::max<int64_t>(starts, 1) * 4),
                 o_io = take(sizeof(kappa::IslandIO) * nisl);
    A->bytes = off;
    if (fault_alloc_after_ >= 0 && alloc_count_ >= fault_alloc_after_) return false;
    if (cudaMalloc(&A->base, A->bytes) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    alloc_count_++;
    {
        std::lock_guard<std::mutex> lk(stats_mtx_);
        vram_used_ += (int64_t)A->bytes;
    }
    cudaMemsetAsync(A->base, 0, A->bytes, stream_);
    char* b = static_cast<char*>(A->base);
    KArena& k = A->dev;
    k.type = reinterpret_cast<uint8_t*>(b + o_type);
    k.k32 = reinterpret_cast<float*>(b + o_k32);
    k.k16 = reinterpret_cast<uint16_t*>(b + o_k16);
    k.b = reinterpret_cast<float*>(b + o_b);
    k.x64 = reinterpret_cast<double*>(b + o_x64);
    k.r = reinterpret_cast<float*>(b + o_r);
    k.e = reinterpret_cast<float*>(b + o_e);
    k.z = reinterpret_cast<float*>(b + o_z);
    k.p = reinterpret_cast<float*>(b + o_p);
    k.q = reinterpret_cast<float*>(b + o_q);
    k.cdiag = reinterpret_cast<float*>(b + o_cd);
    k.coef16 = reinterpret_cast<uint16_t*>(b + o_cf);
    k.coef32 = reinterpret_cast<float*>(b + o_cf);
    k.cx = reinterpret_cast<float*>(b + o_cx);
    k.cb = reinterpret_cast<float*>(b + o_cb);
    k.desc = reinterpret_cast<KDesc*>(b + o_desc);
    k.order = reinterpret_cast<int*>(b + o_order);
    k.queue = reinterpret_cast<int*>(b + o_queue);
    k.scratch = reinterpret_cast<float*>(b + o_scr);
    k.dinv0 = reinterpret_cast<float*>(b + o_dinv);
    k.d0 = reinterpret_cast<float*>(b + o_d0);
    k.rkp = reinterpret_cast<float*>(b + o_rkp);
    k.rk32 = reinterpret_cast<float*>(b + o_rk32);
    k.cd = reinterpret_cast<float*>(b + o_cdd);
    k.cx2 = reinterpret_cast<float*>(b + o_cx2);
    k.flist = reinterpret_cast<uint32_t*>(b + o_flist);
    k.fstart = reinterpret_cast<int*>(b + o_fstart);
    k.nisl = nisl;
    k.prec = A->prec;
    if (!CU_OK(cudaMallocHost((void**)&A->hscratch, 256))) return false;
    if (!CU_OK(cudaMallocHost((void**)&A->hdesc, sizeof(KDesc) * std::max(nisl, 1)))) return false;
    // largest island first (load balance of the persistent queue)
    std::vector<int> order(nisl);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return A->desc[a].n > A->desc[c].n; });
    cudaMemcpyAsync(const_cast<int*>(k.order), order.data(), sizeof(int) * nisl, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(k.desc, A->desc.data(), sizeof(KDesc) * nisl, cudaMemcpyHostToDevice, stream_);
    A->io.assign(nisl, kappa::IslandIO{});
    int64_t io_blocks = 0;
    for (int q = 0; q < nisl; q++) {
        Island* s = set[q];
        const HostBuffers& h = s->hosts;
        void* ptrs[4] = {h.k_type, h.k_kappa, h.k_source, h.k_phi};
        const int64_t sz[4] = {s->n, s->n * 4, s->n * 4, s->n * 4};
        const void* dev[4];
        bool all = true;
        for (int t = 0; t < 4; t++) all &= (dev[t] = map_arena_host(*s, ptrs[t], sz[t], A->pinned)) != nullptr;
        kappa::IslandIO& o = A->io[q];
        if (all) {
            o.h_type = static_cast<const uint8_t*>(dev[0]);
            o.h_kappa = static_cast<const float*>(dev[1]);
            o.h_source = static_cast<const float*>(dev[2]);
            o.h_phi = static_cast<const float*>(dev[3]);
            o.h_phi_out = static_cast<float*>(const_cast<void*>(dev[3]));
            A->io_any = true;
        }
        o.off = A->desc[q].off;
        o.n = s->n;
        o.b0 = (int32_t)io_blocks;
        io_blocks += ceil_div64(s->n, kappa::kArenaIoBlock);
    }
    if (io_blocks > INT32_MAX) return false;
    A->io_blocks = (int)io_blocks;
    A->d_io = reinterpret_cast<kappa::IslandIO*>(b + o_io);
    cudaMemcpyAsync(A->d_io, A->io.data(), sizeof(kappa::IslandIO) * nisl, cudaMemcpyHostToDevice, stream_);
    if (!CU_OK(cudaStreamSynchronize(stream_))) return false;
    arena_ = std::move(A);
    return true;
}

bool Engine::collect_kappa_set(const int32_t* ids, int32_t count, std::vector<Island*>& set) {
    set.clear();
    for (int32_t k = 0; k < count; k++) {
        Island* s = find(ids[k]);
        if (!s || !s->hosts.kappa_registered) return false;
        if (std::find(set.begin(), set.end(), s) == set.end()) set.push_back(s);
    }
    return true;
}

KArena Engine::solve_params(double tol, int32_t max_iter) const {
    KArena k = arena_->dev;
    k.tol = tol;
    k.eta_min = (double)inner_eta_;
    k.max_outer = 8;
    k.max_inner = max_iter > 0 ? max_iter : 500;
    k.omega_c = coarse_weight_;
    k.nu = 2;
    k.coarse_sweeps = coarse_sweeps_;
    const bool batched = solve_mode_ == PFSF_SOLVE_BATCHED;
    k.fp64_dots = batched ? 1 : 0;
    // batched: Chebyshev smoothing (one stencil pass per step, few barriers);
    // plain: symmetric 8-colour Gauss-Seidel (the RBGS of the reference)
    k.smoother = smoother_ >= 0 ? smoother_ : (batched ? 1 : 0);
    k.wcycle = (batched && mg_cycle_ == 1) ? 1 : 0;
    k.cheb_k = std::max(1, std::min(4, cheb_k_));
    k.tail_cells = tail_cells_;
    k.io = arena_->d_io;
    k.ingest = k.cold = k.emit = 0;
    {
        const double lmax = 2.0, lmin = lmax * (double)cheb_lower_;
        const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
        double rho = 1.0 / sigma;
        k.cheb_c1[0] = 0.0f;
        k.cheb_c2[0] = (float)(1.0 / theta);
        for (int j = 1; j < 4; j++) {
            const double rn = 1.0 / (2.0 * sigma - rho);
            k.cheb_c1[j] = (float)(rn * rho);
            k.cheb_c2[j] = (float)(2.0 * rn / delta);
            rho = rn;
        }
    }
    return k;
}

// Launches the solve of every island in the arena (x64 is the starting
// guess, b the right-hand side) and queues the copy of the per-island
// results into the arena's pinned result records (collect_results reads
// them after the stream is synchronised).
pfsf_result Engine::run_solve(const KArena& k, int64_t& nl) {
    Arena& A = *arena_;
    const size_t nisl = A.desc.size();
    nl = 0;
    if (solve_mode_ != PFSF_SOLVE_BATCHED) {
        for (size_t q = 0; q < nisl; q++) {
            const int64_t l = kappa::solve_plain(stream_, k, (int)q, A.desc[q], A.plain);
            if (l <= 0) return PFSF_ERROR_VULKAN;
            nl += l;
        }
        launches_ += nl;
        cudaMemcpyAsync(A.hdesc, k.desc, sizeof(KDesc) * nisl, cudaMemcpyDeviceToHost, stream_);
        return PFSF_OK;
    }
    // islands at or above the grid threshold are solved by the whole GPU
    // (one at a time), those at or above the cluster threshold by whole
    // thread-block clusters (largest first), islands below the warp
    // threshold by single warps, the rest by single CTAs
    int ngiant = 0, nbig = 0, nsmall = 0;
    for (const KDesc& d : A.desc) {
        ngiant += d.n >= grid_min_voxels_ ? 1 : 0;
        nbig += (d.n >= cluster_min_voxels_ && d.n < grid_min_voxels_) ? 1 : 0;
        nsmall += d.n < warp_max_voxels_ ? 1 : 0;
    }
    int* flag = reinterpret_cast<int*>(A.hscratch) + 48;
    auto enqueue = [&](int& launches) {
        cudaMemsetAsync(k.queue, 0, 16 * sizeof(int), stream_);
        const int ctas = kappa::launch_batched(stream_, side_, k, ngiant, nbig, nsmall, cluster_size_, num_sms_,
                                               &launches);
        cudaMemcpyAsync(flag, k.queue + 10, sizeof(int), cudaMemcpyDeviceToHost, stream_);
        cudaMemcpyAsync(A.hdesc, k.desc, sizeof(KDesc) * nisl, cudaMemcpyDeviceToHost, stream_);
        return ctas;
    };
    // The whole-GPU tier's cooperative launch stays outside graphs; the rest
    // is captured once the arena has run one direct solve (kernel attributes
    // set, occupancy known) and replayed while the parameters stay the same.
    const std::vector<double> key = {k.tol, k.eta_min, (double)k.max_inner, (double)k.max_outer, (double)k.omega_c,
                                     (double)k.nu, (double)k.coarse_sweeps, (double)k.fp64_dots, (double)k.smoother,
                                     (double)k.cheb_k, (double)k.wcycle, (double)k.prec, (double)nbig, (double)nsmall,
                                     (double)cluster_size_, (double)num_sms_, (double)nisl, (double)k.cheb_c2[0],
                                     (double)k.cheb_c1[1], (double)k.tail_cells, (double)k.ingest, (double)k.cold,
                                     (double)k.emit};
    *flag = 0;
    if (ngiant == 0 && A.launched && !A.graph_off) {
        if (A.solve_exec && A.solve_key != key) {
            cudaGraphExecDestroy(A.solve_exec);
            A.solve_exec = nullptr;
        }
        if (!A.solve_exec) {
            cudaGraph_t graph = nullptr;
            int launches = 0, ctas = -1;
            if (CU_OK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed))) {
                ctas = enqueue(launches);
                const cudaError_t ce = cudaStreamEndCapture(stream_, &graph);
                if (ce == cudaSuccess && graph && ctas >= 0 &&
                    CU_OK(cudaGraphInstantiate(&A.solve_exec, graph, 0))) {
                    A.solve_key = key;
                    A.graph_launches = launches;
                    A.graph_ctas = ctas;
                } else {
                    A.solve_exec = nullptr;
                }
                if (graph) cudaGraphDestroy(graph);
            }
            if (!A.solve_exec) {
                std::fprintf(stderr, "[libpfsf] batched solve capture failed (%s); launching directly\n",
                             cudaGetErrorString(cudaGetLastError()));
                A.graph_off = true;
            }
        }
        if (A.solve_exec) {
            if (!CU_OK(cudaGraphLaunch(A.solve_exec, stream_))) return PFSF_ERROR_VULKAN;
            A.persistent_ctas = A.graph_ctas;
            nl = A.graph_launches;
            launches_ += nl;
            return PFSF_OK;
        }
    }
    int launches = 0;
    const int ctas = enqueue(launches);
    if (ctas < 0) return PFSF_ERROR_VULKAN;
    A.persistent_ctas = ctas;
    A.launched = true;
    nl = launches;
    launches_ += nl;
    return PFSF_OK;
}

void Engine::collect_results(std::vector<KDesc>& res) const {
    res.assign(arena_->hdesc, arena_->hdesc + arena_->desc.size());
}

// After the stream is synchronised: did a whole-GPU barrier time out?
bool Engine::grid_barrier_failed() const {
    return solve_mode_ == PFSF_SOLVE_BATCHED && arena_ && reinterpret_cast<const int*>(arena_->hscratch)[48] != 0;
}

void Engine::fill_stats(const KArena& k, const std::vector<KDesc>& res, pfsf_solve_stats& st) const {
    const Arena& A = *arena_;
    st.islands_solved = (int32_t)res.size();
    for (size_t q = 0; q < res.size(); q++) {
        const KDesc& d = res[q];
        st.islands_converged += d.converged ? 1 : 0;
        st.max_iterations = std::max(st.max_iterations, d.inner_iters);
        st.max_rel_residual = std::max(st.max_rel_residual, d.relres);
        st.inner_iterations_total += d.inner_iters;
        st.algorithmic_bytes += solve_bytes(d, k.prec, k.nu, k.coarse_sweeps, k.smoother, k.cheb_k, k.wcycle);
        st.active_voxels += A.active[q];
    }
    if (solve_mode_ == PFSF_SOLVE_BATCHED) {
        unsigned long long t0 = ~0ull, t1 = 0;
        for (const KDesc& d : res) {
            t0 = std::min(t0, d.t_start);
            t1 = std::max(t1, d.t_end);
            const double ms = (double)(d.t_end - d.t_start) * 1e-6;
            st.island_ms_sum += ms;
            st.island_ms_max = std::max(st.island_ms_max, ms);
            st.setup_ms_sum += (double)d.t_setup * 1e-6;
            st.precond_ms_sum += (double)d.t_precond * 1e-6;
            st.vcycle_fine_ms_sum += (double)d.t_vfine * 1e-6;
            st.vcycle_coarse_ms_sum += (double)d.t_vcoarse * 1e-6;
            st.vcycle_tail_ms_sum += (double)d.t_vtail * 1e-6;
        }
        st.span_ms = t1 > t0 ? (double)(t1 - t0) * 1e-6 : 0.0;
        st.persistent_ctas = A.persistent_ctas;
    }
}

pfsf_result Engine::solve_to_tolerance(const int32_t* ids, int32_t count, double tol, int32_t max_iter,
                                       uint32_t flags, pfsf_solve_stats* out) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (count < 0 || (count > 0 && !ids) || !(tol > 0.0)) return PFSF_ERROR_INVALID_ARG;
    std::vector<Island*> set;
    if (!collect_kappa_set(ids, count, set)) return PFSF_ERROR_INVALID_ARG;
    pfsf_solve_stats st{};
    st.struct_bytes = (int32_t)sizeof(pfsf_solve_stats);
    if (set.empty()) {
        if (out) *out = st;
        return PFSF_OK;
    }
    bool same = arena_ && arena_->prec == (int)precision_ && arena_->ids.size() == set.size();
    if (same)
        for (size_t k = 0; k < set.size(); k++) same &= arena_->ids[k] == set[k]->id;
    bool do_upload = !(flags & PFSF_SOLVE_NO_UPLOAD);
    if (!same) {
        if (!build_arena(set)) return PFSF_ERROR_OUT_OF_VRAM;
        do_upload = true;
    }
    Arena& A = *arena_;
    if (A.b_stale) do_upload = true;  // an adjoint solve replaced the sources
    KArena k = solve_params(tol, max_iter);
    // batched: every team reads its mapped island's inputs before its solve and
    // writes its solution back after it, inside the persistent launch, so the
    // host-link traffic overlaps the other teams' solves
    const bool fuse = solve_mode_ == PFSF_SOLVE_BATCHED && A.io_any;

    cudaEvent_t ev[4];
    for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], stream_);
    if (do_upload) {
        // mapped islands in one gather launch (or by their teams), the others by copies
        if (A.io_any && !fuse) {
            kappa::launch_arena_upload(stream_, A.d_io, (int)set.size(), A.io_blocks, const_cast<uint8_t*>(k.type),
                                       const_cast<float*>(k.k32), const_cast<float*>(k.b), k.e);
            launches_++;
        }
        for (size_t q = 0; q < set.size(); q++) {
            if (A.io[q].h_type) continue;
            const Island* s = set[q];
            const KDesc& d = A.desc[q];
            const size_t n = (size_t)s->n;
            bool ok = true;
            ok &= CU_OK(cudaMemcpyAsync(const_cast<uint8_t*>(k.type) + d.off, s->hosts.k_type, n,
                                        cudaMemcpyHostToDevice, stream_));
            ok &= CU_OK(cudaMemcpyAsync(const_cast<float*>(k.k32) + d.off, s->hosts.k_kappa, n * 4,
                                        cudaMemcpyHostToDevice, stream_));
            ok &= CU_OK(cudaMemcpyAsync(const_cast<float*>(k.b) + d.off, s->hosts.k_source, n * 4,
                                        cudaMemcpyHostToDevice, stream_));
            ok &= CU_OK(cudaMemcpyAsync(k.e + d.off, s->hosts.k_phi, n * 4, cudaMemcpyHostToDevice, stream_));
            if (!ok) return PFSF_ERROR_VULKAN;
        }
        kappa::launch_prepare(stream_, k, A.nfine, nullptr);
        launches_++;
        A.b_stale = false;
    }
    cudaEventRecord(ev[1], stream_);
    if (flags & PFSF_SOLVE_COLD_START) cudaMemsetAsync(k.x64, 0, (size_t)A.nfine * 8, stream_);
    const bool readback = !(flags & PFSF_SOLVE_NO_READBACK);
    k.ingest = (fuse && do_upload) ? 1 : 0;
    k.cold = (flags & PFSF_SOLVE_COLD_START) ? 1 : 0;
    k.emit = (fuse && readback) ? 1 : 0;
    std::vector<KDesc> res;
    int64_t nl = 0;
    if (pfsf_result rc = run_solve(k, nl); rc != PFSF_OK) return rc;
    cudaEventRecord(ev[2], stream_);
    if (readback) {
        // e = (float)x64 for every island (by the teams when fused), written to
        // mapped callers' phi in the same launch; the others copied from e
        if (!fuse) {
            kappa::launch_arena_readback(stream_, A.d_io, (int)set.size(), A.io_blocks, k.x64, k.e);
            launches_++;
            nl++;
        }
        for (size_t q = 0; q < set.size(); q++) {
            if (A.io[q].h_phi_out) continue;
            const Island* s = set[q];
            if (!CU_OK(cudaMemcpyAsync(s->hosts.k_phi, k.e + A.desc[q].off, (size_t)s->n * 4, cudaMemcpyDeviceToHost,
                                       stream_)))
                return PFSF_ERROR_VULKAN;
        }
    }
    cudaEventRecord(ev[3], stream_);
    if (!CU_OK(cudaStreamSynchronize(stream_)) || grid_barrier_failed()) return PFSF_ERROR_VULKAN;
    collect_results(res);
    float t_up = 0, t_solve = 0, t_rb = 0;
    cudaEventElapsedTime(&t_up, ev[0], ev[1]);
    cudaEventElapsedTime(&t_solve, ev[1], ev[2]);
    cudaEventElapsedTime(&t_rb, ev[2], ev[3]);
    for (auto& e : ev) cudaEventDestroy(e);
    fill_stats(k, res, st);
    st.device_ms = t_solve;
    st.upload_ms = t_up;
    st.readback_ms = t_rb;
    st.kernel_launches = (int32_t)std::min<int64_t>(nl, INT32_MAX);
    A.desc = res;
    A.solved = true;
    if (out) *out = st;
    return PFSF_OK;
}

pfsf_result Engine::register_adjoint(int32_t id, const pfsf_island_adjoint_buffers* b) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!b || !b->grad_phi_addr || !b->grad_source_addr || !b->grad_kappa_addr) return PFSF_ERROR_INVALID_ARG;
    Island* s = find(id);
    if (!s) return PFSF_ERROR_INVALID_ARG;
    const int64_t bytes = 4 * s->n;
    if (b->grad_phi_bytes < bytes || b->grad_source_bytes < bytes || b->grad_kappa_bytes < bytes)
        return PFSF_ERROR_INVALID_ARG;
    HostBuffers& h = s->hosts;
    h.a_grad_phi = b->grad_phi_addr;
    h.a_grad_source = b->grad_source_addr;
    h.a_grad_kappa = b->grad_kappa_addr;
    h.adjoint_registered = true;
    return PFSF_OK;
}

pfsf_result Engine::adjoint_to_tolerance(const int32_t* ids, int32_t count, double tol, int32_t max_iter,
                                         uint32_t flags, pfsf_solve_stats* out) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (count <= 0 || !ids || !(tol > 0.0)) return PFSF_ERROR_INVALID_ARG;
    std::vector<Island*> set;
    if (!collect_kappa_set(ids, count, set)) return PFSF_ERROR_INVALID_ARG;
    for (const Island* s : set)
        if (!s->hosts.adjoint_registered) return PFSF_ERROR_INVALID_ARG;
    // the arena must hold the forward solution of exactly this island set
    if (!arena_ || !arena_->solved || arena_->prec != (int)precision_ || arena_->ids.size() != set.size())
        return PFSF_ERROR_INVALID_ARG;
    for (size_t q = 0; q < set.size(); q++)
        if (arena_->ids[q] != set[q]->id) return PFSF_ERROR_INVALID_ARG;
    Arena& A = *arena_;
    if (!A.xf) {
        if (!CU_OK(cudaMalloc(&A.xf, (size_t)A.nfine * 8))) {
            cudaGetLastError();
            A.xf = nullptr;
            return PFSF_ERROR_OUT_OF_VRAM;
        }
        std::lock_guard<std::mutex> lk(stats_mtx_);
        vram_used_ += A.nfine * 8;
    }
    const KArena k = solve_params(tol, max_iter);
    pfsf_solve_stats st{};
    st.struct_bytes = (int32_t)sizeof(pfsf_solve_stats);
    cudaEvent_t ev[4];
    for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], stream_);
    // keep the forward solution; load dL/dphi as the right-hand side
    bool ok = CU_OK(cudaMemcpyAsync(A.xf, k.x64, (size_t)A.nfine * 8, cudaMemcpyDeviceToDevice, stream_));
    for (size_t q = 0; q < set.size() && ok; q++)
        ok &= CU_OK(cudaMemcpyAsync(const_cast<float*>(k.b) + A.desc[q].off, set[q]->hosts.a_grad_phi,
                                    (size_t)set[q]->n * 4, cudaMemcpyHostToDevice, stream_));
    if (!ok) return PFSF_ERROR_VULKAN;
    A.b_stale = true;
    kappa::launch_adjoint_prepare(stream_, k, A.nfine);
    launches_++;
    cudaEventRecord(ev[1], stream_);
    std::vector<KDesc> res;
    int64_t nl = 0;
    if (pfsf_result rc = run_solve(k, nl); rc != PFSF_OK) return rc;
    // gradients into the (now free) r / z work vectors, then restore x64
    kappa::launch_edge_product(stream_, k, A.xf, A.nfine, k.r, k.z, num_sms_);
    launches_++;
    nl++;
    cudaEventRecord(ev[2], stream_);
    if (!(flags & PFSF_SOLVE_NO_READBACK)) {
        for (size_t q = 0; q < set.size() && ok; q++) {
            const Island* s = set[q];
            const int64_t o = A.desc[q].off;
            ok &= CU_OK(cudaMemcpyAsync(s->hosts.a_grad_kappa, k.r + o, (size_t)s->n * 4, cudaMemcpyDeviceToHost,
                                        stream_));
            ok &= CU_OK(cudaMemcpyAsync(s->hosts.a_grad_source, k.z + o, (size_t)s->n * 4, cudaMemcpyDeviceToHost,
                                        stream_));
        }
    }
    ok &= CU_OK(cudaMemcpyAsync(k.x64, A.xf, (size_t)A.nfine * 8, cudaMemcpyDeviceToDevice, stream_));
    cudaEventRecord(ev[3], stream_);
    if (!ok || !CU_OK(cudaStreamSynchronize(stream_)) || grid_barrier_failed()) return PFSF_ERROR_VULKAN;
    collect_results(res);
    float t_up = 0, t_solve = 0, t_rb = 0;
    cudaEventElapsedTime(&t_up, ev[0], ev[1]);
    cudaEventElapsedTime(&t_solve, ev[1], ev[2]);
    cudaEventElapsedTime(&t_rb, ev[2], ev[3]);
    for (auto& e : ev) cudaEventDestroy(e);
    // the per-island results of the forward solve stay the arena's record
    fill_stats(k, res, st);
    st.device_ms = t_solve;
    st.upload_ms = t_up;
    st.readback_ms = t_rb;
    st.kernel_launches = (int32_t)std::min<int64_t>(nl, INT32_MAX);
    if (out) *out = st;
    return PFSF_OK;
}

pfsf_result Engine::island_report(int32_t id, pfsf_island_report* out) const {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!out || !arena_ || !arena_->solved) return PFSF_ERROR_INVALID_ARG;
    auto it = std::find(arena_->ids.begin(), arena_->ids.end(), id);
    if (it == arena_->ids.end()) return PFSF_ERROR_INVALID_ARG;
    const KDesc& d = arena_->desc[it - arena_->ids.begin()];
    pfsf_island_report r{};
    r.struct_bytes = (int32_t)sizeof(r);
    r.lx = d.lx; r.ly = d.ly; r.lz = d.lz;
    r.levels = d.nlev;
    r.inner_iterations = d.inner_iters;
    r.outer_iterations = d.outer_iters;
    r.converged = d.converged;
    r.team = d.team;
    r.team_ctas = d.team_ctas;
    r.rel_residual = d.relres;
    if (d.team != PFSF_TEAM_PLAIN) {
        r.solve_ms = (double)(d.t_end - d.t_start) * 1e-6;
        r.setup_ms = (double)d.t_setup * 1e-6;
        r.precond_ms = (double)d.t_precond * 1e-6;
        unsigned long long t0 = d.t_start;
        for (const KDesc& o : arena_->desc)
            if (o.team != PFSF_TEAM_PLAIN && o.t_start > 0) t0 = std::min(t0, o.t_start);
        r.start_ms = (double)(d.t_start - t0) * 1e-6;
    }
    *out = r;
    return PFSF_OK;
}

pfsf_result Engine::debug_time_pass(int32_t id, int32_t pass, int32_t reps, float* ms, double* bytes) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!ms || !bytes || (pass != 0 && pass != 1) || reps <= 0 || !arena_ || !arena_->solved) return PFSF_ERROR_INVALID_ARG;
    auto it = std::find(arena_->ids.begin(), arena_->ids.end(), id);
    if (it == arena_->ids.end()) return PFSF_ERROR_INVALID_ARG;
    const int q = (int)(it - arena_->ids.begin());
    const KArena k = solve_params(1e-6, 0);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemsetAsync(k.queue, 0, 16 * sizeof(int), stream_);
    cudaEventRecord(e0, stream_);
    const int rc = kappa::launch_pass(stream_, k, q, pass, reps, num_sms_);
    cudaEventRecord(e1, stream_);
    int err = 0;
    cudaMemcpyAsync(&err, k.queue + 10, sizeof(int), cudaMemcpyDeviceToHost, stream_);
    const bool ok = rc == 0 && CU_OK(cudaStreamSynchronize(stream_)) && err == 0;
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    launches_++;
    if (!ok) return PFSF_ERROR_VULKAN;
    // algorithmic bytes: the march stages the input vector and 1/kappa of
    // every cell of the island's box; the solid voxels read and write the rest
    const double n = (double)arena_->desc[q].n, na = (double)arena_->active[q];
    const double per = pass == 0 ? (4.0 + 4.0) * n + (4.0 + 4.0 + 8.0 + 4.0 + 4.0) * na  // r, dinv, d rw, zout, list
                                 : (4.0 + 4.0) * n + (4.0 + 4.0) * na;                     // p, 1/k32; q, list
    *ms = t / (float)reps;
    *bytes = per;
    return PFSF_OK;
}

pfsf_result Engine::read_solution64(int32_t id, double* out, int64_t cap, int64_t* count) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (!out || !count) return PFSF_ERROR_INVALID_ARG;
    *count = 0;
    if (!arena_) return PFSF_ERROR_INVALID_ARG;
    auto it = std::find(arena_->ids.begin(), arena_->ids.end(), id);
    if (it == arena_->ids.end()) return PFSF_ERROR_INVALID_ARG;
    const KDesc& d = arena_->desc[it - arena_->ids.begin()];
    const int64_t n = std::min<int64_t>(d.n, cap);
    if (n <= 0) return PFSF_OK;
    if (!CU_OK(cudaMemcpyAsync(out, arena_->dev.x64 + d.off, (size_t)n * 8, cudaMemcpyDeviceToHost, stream_)) ||
        !CU_OK(cudaStreamSynchronize(stream_)))
        return PFSF_ERROR_VULKAN;
    *count = n;
    return PFSF_OK;
}

// The reference tick with its fixed 16-step schedule replaced by the
// tolerance solve: solve every listed island to rel. tolerance (one batched
// launch), put the FP32 phi into the island's reference-layout buffers, apply
// the history update H = max(H, psi_e(phi)) the reference performs inside its
// sweeps, then the reference tick's tail (phase field, failure scan, failure
// compaction, stress readback) and append failures to the caller's buffer.
pfsf_result Engine::tick_tolerance(const int32_t* ids, int32_t count, void* fail_addr, int64_t fail_bytes, double tol,
                                   int32_t max_iter, pfsf_solve_stats* out) {
    if (!available_) return PFSF_ERROR_NOT_INIT;
    if (count < 0 || (count > 0 && !ids) || !(tol > 0.0)) return PFSF_ERROR_INVALID_ARG;
    const bool drain = fail_addr != nullptr && fail_bytes >= 20;
    if (fail_addr && fail_bytes >= 4) *static_cast<int32_t*>(fail_addr) = 0;
    const int32_t dbb_cap = drain ? (int32_t)((fail_bytes - 4) / 16) : 0;
    std::vector<Island*> set;
    if (!collect_kappa_set(ids, count, set)) return PFSF_ERROR_INVALID_ARG;
    std::vector<int32_t> sids;
    for (Island* s : set) {
        if (!s->hosts.registered) return PFSF_ERROR_INVALID_ARG;
        if (!ensure_compat(*s)) return PFSF_ERROR_OUT_OF_VRAM;
        sids.push_back(s->id);
    }
    pfsf_solve_stats st{};
    st.struct_bytes = (int32_t)sizeof(st);
    if (set.empty()) {
        if (out) *out = st;
        return PFSF_OK;
    }
    if (pfsf_result rc = solve_to_tolerance(sids.data(), (int32_t)sids.size(), tol, max_iter, 0, &st); rc != PFSF_OK)
        return rc;
    // the tail over all islands in one batched pass: dirty islands' reference
    // buffers uploaded (as pfsf_tick_dbb does), phi taken from the arena,
    // H = max(H, psi_e(phi)), phase field, failure scan and compaction
    std::vector<const float*> phi_in;
    for (size_t q = 0; q < set.size(); q++) phi_in.push_back(arena_->dev.e + arena_->desc[q].off);
    if (pfsf_result rc = tick_batched(set, dbb_cap, &phi_in); rc != PFSF_OK) return rc;
    if (pfsf_result rc = finish_dispatch(set, drain, fail_addr, 0, dbb_cap, nullptr, 0); rc != PFSF_OK) return rc;
    if (out) *out = st;
    return PFSF_OK;
}

}  // namespace pfsf_b200
