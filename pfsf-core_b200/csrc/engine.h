// PFSF B200 engine: island registry, device buffers, per-tick schedule.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include "kappa.h"
#include "pfsf/pfsf.h"

namespace pfsf_b200 {

// Reference constants (L1-native/libpfsf/src/core/constants.h).
constexpr int kWarmupSteps = 8;
constexpr float kDampingFactor = 0.995f;
constexpr int kMgInterval = 4;
constexpr int kStepsMajor = 16;
constexpr int kPcgMinRbgs = 2;
constexpr int kPcgMinSteps = 1;
constexpr int64_t kPcgMaxN = 512LL * 512LL;
constexpr float kPfL0 = 2.0f;  // max(PHASE_FIELD_L0 = 1.5, 2)
constexpr float kPfGc = 100.0f;
constexpr float kPfRelax = 0.3f;
constexpr int kSparseCapacity = 512;
constexpr int kSparseRecordBytes = 48;

struct HostBuffers {
    bool registered = false;
    void* phi = nullptr;
    int64_t phi_bytes = 0;
    void* source = nullptr;
    int64_t source_bytes = 0;
    void* conductivity = nullptr;
    int64_t conductivity_bytes = 0;
    void* voxel_type = nullptr;
    int64_t voxel_type_bytes = 0;
    void* rcomp = nullptr;
    int64_t rcomp_bytes = 0;
    void* rtens = nullptr;
    int64_t rtens_bytes = 0;
    void* max_phi = nullptr;
    int64_t max_phi_bytes = 0;
    bool lookups_registered = false;
    void* curing = nullptr;
    int64_t curing_bytes = 0;
    void* stress_out = nullptr;
    int64_t stress_bytes = 0;
    // kappa-form inputs (pfsf_register_island_kappa)
    bool kappa_registered = false;
    void* k_phi = nullptr;
    void* k_source = nullptr;
    void* k_kappa = nullptr;
    void* k_type = nullptr;
    // device-visible mappings of the pinned reference-layout arrays (nullptr:
    // the array could not be pinned and is copied with cudaMemcpyAsync)
    const void *m_phi = nullptr, *m_source = nullptr, *m_cond = nullptr, *m_type = nullptr, *m_rcomp = nullptr,
               *m_rtens = nullptr, *m_maxphi = nullptr, *m_curing = nullptr;
    void* m_stress = nullptr;
    // adjoint buffers (pfsf_register_island_adjoint)
    bool adjoint_registered = false;
    const void* a_grad_phi = nullptr;
    void* a_grad_source = nullptr;
    void* a_grad_kappa = nullptr;
};

// Per-island tick result (device records of the batched tick, read back in
// one copy).
struct TickResult {
    float macro_max;
    int32_t fail_total;
    uint32_t phi_max_key;  // order-preserving key of the max phi (0: none)
    int32_t pad;
};

struct KappaState;  // tolerance-solve state (kappa_solver.cu)

struct Island {
    int32_t id = 0;
    pfsf_pos origin{0, 0, 0};
    int lx = 0, ly = 0, lz = 0;
    int64_t n = 0, nmb = 0;
    bool dirty = true;
    HostBuffers hosts;

    // fine level (device)
    float *phi = nullptr, *src = nullptr, *sigma = nullptr, *rcomp = nullptr, *rtens = nullptr,
          *maxphi = nullptr, *hyd = nullptr, *H = nullptr, *D = nullptr, *Dold = nullptr;
    uint8_t *type = nullptr, *fail = nullptr;
    uint32_t* macro = nullptr;
    int32_t *fcounts = nullptr, *foffsets = nullptr, *tuples = nullptr;
    int32_t tuple_cap = 0;

    // multigrid (two coarse levels, reference island_buffer.cpp:179-188)
    bool mg_alloc = false, mg_dirty = true;
    int l1[3] = {0, 0, 0}, l2[3] = {0, 0, 0};
    int64_t n1 = 0, n2 = 0;
    float *phi1[2] = {nullptr, nullptr}, *src1 = nullptr, *sig1 = nullptr;
    float *phi2[2] = {nullptr, nullptr}, *src2 = nullptr, *sig2 = nullptr;
    uint8_t *type1 = nullptr, *type2 = nullptr;
    int cur1 = 0, cur2 = 0;

    // PCG (allocated on the first stalled tick, dispatcher.cpp:133)
    bool pcg_alloc = false;
    float *r[2] = {nullptr, nullptr}, *p = nullptr, *ap = nullptr, *invdiag = nullptr, *partial = nullptr,
          *red = nullptr;
    int rcur = 0;

    // aggregation coarse correction at the PCG start (reference
    // island_buffer.h:96-103, built from sigma and type on the device)
    bool amg_alloc = false, amg_dirty = true;
    int64_t amg_nc = 0;
    int32_t* agg = nullptr;
    float *aw = nullptr, *adc = nullptr, *aec = nullptr;

    // sparse upload region (pinned host) + device staging
    void* sparse_host = nullptr;
    void* sparse_dev = nullptr;

    // max phi at the end of the last tick (the divergence check's input)
    float phi_max = 0.0f;

    // schedule state
    int chebyshev_iter = 0;
    float prev_macro = 0.0f, last_macro = 0.0f;

    std::unique_ptr<KappaState> kappa;

    std::vector<std::pair<void*, size_t>> allocations;  // device allocations owned by this island
    std::vector<void*> host_registered;
    struct HostPin {
        const void* host;
        int64_t bytes;
        const void* dev;
    };
    std::vector<HostPin> host_pins;  // ranges pinned by map_host and their device addresses
    Island();
    ~Island();
};

class Engine {
public:
    explicit Engine(const pfsf_config& cfg);
    ~Engine();

    pfsf_result init();
    void shutdown();
    bool available() const { return available_; }
    pfsf_result get_stats(pfsf_stats* out);

    pfsf_result add_island(const pfsf_island_desc* d);
    void remove_island(int32_t id);
    pfsf_result notify_block_change(int32_t id, const pfsf_voxel_update* u);
    void mark_full_rebuild(int32_t id);
    pfsf_result register_buffers(int32_t id, const pfsf_island_buffers* b);
    pfsf_result register_lookups(int32_t id, const pfsf_island_lookups* l);
    pfsf_result register_stress(int32_t id, void* addr, int64_t bytes);
    pfsf_result tick(const int32_t* ids, int32_t count, pfsf_tick_result* result, void* fail_addr,
                     int64_t fail_bytes);
    pfsf_result read_stress(int32_t id, float* out, int32_t cap, int32_t* count);
    pfsf_result get_sparse_buffer(int32_t id, void** addr, int64_t* bytes);
    pfsf_result notify_sparse(int32_t id, int32_t count);

    void set_pcg_enabled(bool on) { pcg_enabled_ = on; }
    void set_wind(const pfsf_vec3* w) { wind_ = w ? *w : pfsf_vec3{0, 0, 0}; }
    void set_precision(pfsf_precision p) { precision_ = p; }
    void set_solve_mode(pfsf_solve_mode m) { solve_mode_ = m; }
    void set_mg_cycle(int c) { mg_cycle_ = c == 1 ? 1 : 0; }
    void set_amg(bool on) { amg_enabled_ = on; }
    pfsf_result get_tuning(pfsf_tuning* out) const;
    pfsf_result set_tuning(const pfsf_tuning* in);

    pfsf_result register_kappa(int32_t id, const pfsf_island_kappa_buffers* b);
    pfsf_result solve_to_tolerance(const int32_t* ids, int32_t count, double tol, int32_t max_iter, uint32_t flags,
                                   pfsf_solve_stats* out);
    pfsf_result read_solution64(int32_t id, double* out, int64_t cap, int64_t* count);
    pfsf_result debug_time_pass(int32_t id, int32_t pass, int32_t reps, float* ms, double* bytes);
    pfsf_result island_report(int32_t id, pfsf_island_report* out) const;
    pfsf_result tick_tolerance(const int32_t* ids, int32_t count, void* fail_addr, int64_t fail_bytes, double tol,
                               int32_t max_iter, pfsf_solve_stats* out);
    pfsf_result register_adjoint(int32_t id, const pfsf_island_adjoint_buffers* b);
    pfsf_result adjoint_to_tolerance(const int32_t* ids, int32_t count, double tol, int32_t max_iter,
                                     uint32_t flags, pfsf_solve_stats* out);
    pfsf_result debug_read_field(int32_t id, int32_t field, void* out, int64_t bytes, int64_t* out_bytes);
    pfsf_result last_tick_report(pfsf_tick_report* out) const;
    pfsf_result island_phi_max(int32_t id, float* out);

    cudaStream_t stream() const { return stream_; }
    int num_sms() const { return num_sms_; }
    int64_t launches() const { return launches_.load(); }
    void count_launches(int64_t k) { launches_ += k; }

    // device allocation with budget accounting and an optional injected failure
    // (for host-side fault-injection tests: PFSF_FAULT_ALLOC_AFTER=<k> fails
    // the (k+1)-th allocation).
    void* dalloc(Island& isl, size_t bytes);
    Island* find(int32_t id);

private:
    struct TickBatch;
    // One tick of the reference schedule for every island in `set` (all
    // dirty, compat buffers allocated): islands grouped by schedule, each
    // schedule step one launch per group, the whole tick replayed from a
    // CUDA graph while the group structure stays the same (engine_batch.cpp).
    // With phi_in (one device pointer per island of `set`) it runs the
    // tolerance tick's tail instead: phi taken from phi_in, the history
    // update, then the same tail; islands not dirty are not re-uploaded.
    pfsf_result tick_batched(const std::vector<Island*>& set, int32_t want_cap,
                             const std::vector<const float*>* phi_in = nullptr);
    void free_tick_batch();
    const void* map_host(Island& s, void* p, int64_t bytes);
    bool ensure_compat(Island& isl);
    bool build_arena(const std::vector<Island*>& set);
    void free_arena();
    bool collect_kappa_set(const int32_t* ids, int32_t count, std::vector<Island*>& set);
    KArena solve_params(double tol, int32_t max_iter) const;
    pfsf_result run_solve(const KArena& k, int64_t& launches);
    void collect_results(std::vector<KDesc>& res) const;
    bool grid_barrier_failed() const;
    void destroy_side();
    void fill_stats(const KArena& k, const std::vector<KDesc>& res, pfsf_solve_stats& st) const;
    pfsf_result finish_dispatch(const std::vector<Island*>& dispatched, bool drain, void* fail_addr, int32_t dbb_count,
                                int32_t dbb_cap, pfsf_tick_result* result, int32_t legacy_cap);
    bool upload(Island& isl);
    bool ensure_mg(Island& isl);
    bool ensure_pcg(Island& isl);
    bool ensure_amg(Island& isl);
    void free_island(Island& isl);

    pfsf_config cfg_;
    bool available_ = false;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    kappa::SideStream side_{nullptr, nullptr, nullptr};
    std::map<int32_t, std::unique_ptr<Island>> islands_;
    bool pcg_enabled_ = true;
    bool amg_enabled_ = false;            // aggregation correction at the PCG start
    pfsf_vec3 wind_{0, 0, 0};
    pfsf_precision precision_ = PFSF_PREC_FP32;
    pfsf_solve_mode solve_mode_ = PFSF_SOLVE_PER_ISLAND;
    std::atomic<int64_t> launches_{0};
    int64_t vram_used_ = 0;
    int64_t alloc_count_ = 0;
    int64_t fault_alloc_after_ = -1;
    mutable std::mutex stats_mtx_;
    float last_tick_ms_ = 0.0f;
    TickResult* host_results_ = nullptr;  // pinned
    int host_results_cap_ = 0;

    std::unique_ptr<TickBatch> tbatch_;

    // tolerance-solve arena (one packed allocation for a set of islands)
    struct Arena;
    std::unique_ptr<Arena> arena_;
    int num_sms_ = 148;
    int64_t grid_min_voxels_ = 1 << 21;    // PFSF_GRID_MIN_VOXELS: whole-GPU tier
    int64_t cluster_min_voxels_ = 262144;  // PFSF_CLUSTER_MIN_VOXELS
    int cluster_size_ = 4;                // PFSF_CLUSTER (8, 4 or 1)
    int64_t warp_max_voxels_ = 0;         // PFSF_WARP_MAX_VOXELS (0: no warp tier)
    int smoother_ = -1;                   // PFSF_SMOOTHER (-1: mode default)
    int cheb_k_ = 3;                      // PFSF_CHEB_K
    float cheb_lower_ = 0.1f;             // PFSF_CHEB_LOWER: Chebyshev interval [lower * lmax, lmax]
    float coarse_weight_ = 1.8f;          // PFSF_COARSE_WEIGHT: V-cycle coarse-correction weight
    int tail_cells_ = 512;                // PFSF_TAIL_CELLS: coarse levels this small run on one warp
    int coarse_sweeps_ = 4;               // PFSF_COARSE_SWEEPS: smoothing steps on the coarsest level
    float inner_eta_ = 1e-4f;             // PFSF_INNER_ETA: floor of the inner PCG's relative stop
    int tuning_source_ = PFSF_TUNING_DEFAULT;
    int mg_cycle_ = 0;                    // 0 V-cycle, 1 W-cycle (batched tolerance solve)
    void load_tuning();                   // tuning file, then environment overrides (init)
};

}  // namespace pfsf_b200
