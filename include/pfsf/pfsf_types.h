/*
 * pfsf_types.h -- public types of the libpfsf C ABI (B200 build).
 *
 * Binary layout, names and enum values are those of the reference ABI
 * (L1-native/libpfsf/include/pfsf/pfsf_types.h, frozen by
 * L1-native/libpfsf/abi/pfsf_v1.abi.json v1.5.0) so an existing caller -- the
 * Java JNI bridge -- loads this library without recompiling.  Nothing here
 * depends on CUDA or C++.
 */
#ifndef PFSF_TYPES_H
#define PFSF_TYPES_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#if defined(PFSF_EXPORT)
#define PFSF_API __declspec(dllexport)
#else
#define PFSF_API __declspec(dllimport)
#endif
#else
#define PFSF_API __attribute__((visibility("default")))
#endif

/* Opaque engine handle (pfsf_types.h:30). */
typedef struct pfsf_engine_t* pfsf_engine;

/* Result codes (pfsf_types.h:33-41).  Device failures keep the historical
 * PFSF_ERROR_VULKAN value so callers need no change. */
typedef enum {
    PFSF_OK = 0,
    PFSF_ERROR_VULKAN = -1,
    PFSF_ERROR_NO_DEVICE = -2,
    PFSF_ERROR_OUT_OF_VRAM = -3,
    PFSF_ERROR_INVALID_ARG = -4,
    PFSF_ERROR_NOT_INIT = -5,
    PFSF_ERROR_ISLAND_FULL = -6,
} pfsf_result;

/* Voxel classes stored per voxel (uint8 in the island buffers). */
typedef enum {
    PFSF_VOXEL_AIR = 0,
    PFSF_VOXEL_SOLID = 1,
    PFSF_VOXEL_ANCHOR = 2,
} pfsf_voxel_type;

/* Failure codes written by the tick. */
typedef enum {
    PFSF_FAIL_OK = 0,
    PFSF_FAIL_CANTILEVER = 1,
    PFSF_FAIL_CRUSHING = 2,
    PFSF_FAIL_NO_SUPPORT = 3,
    PFSF_FAIL_TENSION = 4,
} pfsf_failure_type;

/* Face order of the SoA-6 conductivity array: sigma[d * N + i]. */
typedef enum {
    PFSF_DIR_NEG_X = 0,
    PFSF_DIR_POS_X = 1,
    PFSF_DIR_NEG_Y = 2,
    PFSF_DIR_POS_Y = 3,
    PFSF_DIR_NEG_Z = 4,
    PFSF_DIR_POS_Z = 5,
} pfsf_direction;

typedef struct {
    int32_t x, y, z;
} pfsf_pos;

typedef struct {
    float x, y, z;
} pfsf_vec3;

/* Island grid: flat voxel index i = x + lx * (y + ly * z). */
typedef struct {
    int32_t island_id;
    pfsf_pos origin; /* world coordinates of local (0,0,0) */
    int32_t lx, ly, lz;
} pfsf_island_desc;

typedef struct {
    float density;
    float rcomp;
    float rtens;
    float youngs_gpa;
    float poisson;
    float gc;
    bool is_anchor;
} pfsf_material;

typedef struct {
    int32_t flat_index;
    float source;
    pfsf_voxel_type type;
    float max_phi;
    float rcomp;
    float cond[6];
} pfsf_voxel_update;

typedef struct {
    pfsf_pos pos;
    pfsf_failure_type type;
} pfsf_failure_event;

typedef struct {
    int32_t max_island_size;   /* default 50000 */
    int32_t tick_budget_ms;    /* default 8 */
    int64_t vram_budget_bytes; /* default 512 MiB */
    bool enable_phase_field;   /* default true */
    bool enable_multigrid;     /* default true */
} pfsf_config;

typedef struct {
    int32_t island_count;
    int64_t total_voxels;
    int64_t vram_used_bytes;
    int64_t vram_budget_bytes;
    float last_tick_ms;
} pfsf_stats;

typedef struct {
    pfsf_failure_event* events; /* caller-owned */
    int32_t capacity;
    int32_t count; /* out */
} pfsf_tick_result;

typedef pfsf_material (*pfsf_material_fn)(pfsf_pos pos, void* user_data);
typedef bool (*pfsf_anchor_fn)(pfsf_pos pos, void* user_data);
typedef float (*pfsf_fill_ratio_fn)(pfsf_pos pos, void* user_data);
typedef float (*pfsf_curing_fn)(pfsf_pos pos, void* user_data);

#ifdef __cplusplus
}
#endif

#endif /* PFSF_TYPES_H */
