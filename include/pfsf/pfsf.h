/*
 * pfsf.h -- libpfsf public C ABI, B200 (CUDA sm_100a) implementation.
 *
 * Every function below keeps the name, signature, argument meaning and
 * error behaviour of the reference declaration it replaces
 * (L1-native/libpfsf/include/pfsf/pfsf.h, cited per function).  The
 * implementation runs the per-tick structural solve as CUDA kernels instead
 * of Vulkan compute shaders.
 *
 * Threading (pfsf.h:4-7): one "physics thread" makes every call except
 * pfsf_get_stats, which is safe from any thread.  A tick has finished its
 * device work and written all caller buffers before it returns.
 */
#ifndef PFSF_H
#define PFSF_H

#include "pfsf_types.h"
#include "pfsf_version.h"
#include "pfsf_compute.h"
#include "pfsf_diagnostics.h"
#include "pfsf_extension.h"
#include "pfsf_plan.h"
#include "pfsf_trace.h"
#include "pfsf_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- lifecycle ---- */

/* pfsf.h:38.  NULL config selects defaults {50000 voxels, 8 ms, 512 MiB,
 * phase field on, multigrid on}.  Does not touch the GPU. */
PFSF_API pfsf_engine pfsf_create(const pfsf_config* config);

/* pfsf.h:48-62.  Vulkan handle hand-over.  There is no Vulkan device in
 * this build, so this returns NULL and the caller falls back to
 * pfsf_create (NativePFSFRuntime.java:155-170 does exactly that). */
typedef struct pfsf_vulkan_handles {
    uint64_t vk_instance;
    uint64_t vk_physical_device;
    uint64_t vk_device;
    uint32_t compute_queue_family;
    uint64_t vk_compute_queue;
} pfsf_vulkan_handles;
PFSF_API pfsf_engine pfsf_create_with_vulkan(const pfsf_config* config, const pfsf_vulkan_handles* handles);

/* pfsf.h:70.  Selects the CUDA device (PFSF_CUDA_DEVICE env, default the
 * current device), creates the stream.  PFSF_ERROR_NO_DEVICE without a GPU. */
PFSF_API pfsf_result pfsf_init(pfsf_engine engine);

/* pfsf.h:77.  Frees all device memory; safe to call repeatedly. */
PFSF_API void pfsf_shutdown(pfsf_engine engine);

/* pfsf.h:85.  NULL is a no-op. */
PFSF_API void pfsf_destroy(pfsf_engine engine);

/* pfsf.h:90 */
PFSF_API bool pfsf_is_available(pfsf_engine engine);

/* pfsf.h:95, thread-safe. */
PFSF_API pfsf_result pfsf_get_stats(pfsf_engine engine, pfsf_stats* out);

/* ---- configuration (pfsf.h:104-139) ---- */
PFSF_API void pfsf_set_material_lookup(pfsf_engine engine, pfsf_material_fn fn, void* user_data);
PFSF_API void pfsf_set_anchor_lookup(pfsf_engine engine, pfsf_anchor_fn fn, void* user_data);
PFSF_API void pfsf_set_fill_ratio_lookup(pfsf_engine engine, pfsf_fill_ratio_fn fn, void* user_data);
PFSF_API void pfsf_set_curing_lookup(pfsf_engine engine, pfsf_curing_fn fn, void* user_data);
PFSF_API void pfsf_set_wind(pfsf_engine engine, const pfsf_vec3* wind);
/* pfsf.h:152: gate the RBGS -> PCG tail (default enabled). */
PFSF_API void pfsf_set_pcg_enabled(pfsf_engine engine, int enabled);

/* ---- islands (pfsf.h:160-190) ---- */
/* OK, ISLAND_FULL (N > max_island_size or a non-positive side),
 * OUT_OF_VRAM (device allocation failed), NOT_INIT. */
PFSF_API pfsf_result pfsf_add_island(pfsf_engine engine, const pfsf_island_desc* desc);
PFSF_API void pfsf_remove_island(pfsf_engine engine, int32_t island_id);
/* Validates flat_index against N and marks the island dirty. */
PFSF_API pfsf_result pfsf_notify_block_change(pfsf_engine engine, int32_t island_id,
                                              const pfsf_voxel_update* update);
PFSF_API void pfsf_mark_full_rebuild(pfsf_engine engine, int32_t island_id);

/* ---- tick (pfsf.h:205-210) ---- */
/* Legacy result form; events are {x,y,z,type} in world coordinates. */
PFSF_API pfsf_result pfsf_tick(pfsf_engine engine, const int32_t* dirty_island_ids, int32_t dirty_count,
                               int64_t current_epoch, pfsf_tick_result* result);

/* pfsf.h:225.  Writes raw phi (count = min(N, capacity)). */
PFSF_API pfsf_result pfsf_read_stress(pfsf_engine engine, int32_t island_id, float* out_stress, int32_t capacity,
                                      int32_t* out_count);

/* ---- zero-copy host buffers (pfsf.h:232-287) ---- */
typedef struct pfsf_island_buffers {
    void* phi_addr; /* float32 x N */
    int64_t phi_bytes;
    void* source_addr; /* float32 x N */
    int64_t source_bytes;
    void* conductivity_addr; /* float32 x 6N, SoA sigma[d*N + i] */
    int64_t conductivity_bytes;
    void* voxel_type_addr; /* uint8 x N */
    int64_t voxel_type_bytes;
    void* rcomp_addr; /* float32 x N */
    int64_t rcomp_bytes;
    void* rtens_addr; /* float32 x N */
    int64_t rtens_bytes;
    void* max_phi_addr; /* float32 x N */
    int64_t max_phi_bytes;
} pfsf_island_buffers;

typedef struct pfsf_island_lookups {
    void* material_id_addr; /* int32 x N */
    int64_t material_id_bytes;
    void* anchor_bitmap_addr; /* int64 x N */
    int64_t anchor_bitmap_bytes;
    void* fluid_pressure_addr; /* float32 x N */
    int64_t fluid_pressure_bytes;
    void* curing_addr; /* float32 x N, hydration for the phase field */
    int64_t curing_bytes;
} pfsf_island_lookups;

/* Registers caller-owned buffers that stay valid for the island lifetime,
 * uploads them and marks the island dirty.  Any NULL pointer or undersized
 * buffer -> PFSF_ERROR_INVALID_ARG (pfsf_engine.cpp:205-259). */
PFSF_API pfsf_result pfsf_register_island_buffers(pfsf_engine engine, int32_t island_id,
                                                  const pfsf_island_buffers* bufs);
PFSF_API pfsf_result pfsf_register_island_lookups(pfsf_engine engine, int32_t island_id,
                                                  const pfsf_island_lookups* lookups);
/* After every dispatched tick the engine writes raw phi here. */
PFSF_API pfsf_result pfsf_register_stress_readback(pfsf_engine engine, int32_t island_id, void* addr,
                                                   int64_t bytes);

/* pfsf.h:282.  Ticks the listed dirty islands from the registered buffers.
 * failure_addr (optional, >= 20 bytes) receives {int32 count}{int32 x,y,z,type}*k;
 * the count is zeroed on entry and failures of every dispatched island are
 * appended in island order and voxel-index order until the buffer is full. */
PFSF_API pfsf_result pfsf_tick_dbb(pfsf_engine engine, const int32_t* dirty_island_ids, int32_t dirty_count,
                                   int64_t current_epoch, void* failure_addr, int64_t failure_bytes);

/* pfsf.h:296: no native->Java callbacks are queued; returns 0. */
PFSF_API int32_t pfsf_drain_callbacks(pfsf_engine engine, int32_t* out_events, int32_t capacity);

/* ---- sparse voxel re-upload (pfsf.h:319-339) ---- */
/* Engine-owned pinned host region of 512 records x 48 bytes. */
PFSF_API pfsf_result pfsf_get_sparse_upload_buffer(pfsf_engine engine, int32_t island_id, void** out_addr,
                                                   int64_t* out_bytes);
/* Scatters update_count (clamped to 512) records into the island's device
 * arrays and marks it dirty. */
PFSF_API pfsf_result pfsf_notify_sparse_updates(pfsf_engine engine, int32_t island_id, int32_t update_count);

/* pfsf.h:348 */
PFSF_API const char* pfsf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PFSF_H */
