/*
 * pfsf_extension.h -- per-island augmentation slots and hook table
 * (reference: L1-native/libpfsf/include/pfsf/pfsf_extension.h).  Host code.
 */
#ifndef PFSF_EXTENSION_H
#define PFSF_EXTENSION_H
#include "pfsf_types.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PFSF_AUG_THERMAL_FIELD = 1,
    PFSF_AUG_TENSION_OVERRIDE = 2,
    PFSF_AUG_FLUID_PRESSURE = 3,
    PFSF_AUG_EM_FIELD = 4,
    PFSF_AUG_FUSION_MASK = 5,
    PFSF_AUG_WIND_FIELD_3D = 6,
    PFSF_AUG_MATERIAL_OVR = 7,
    PFSF_AUG_CURING_FIELD = 8,
    PFSF_AUG_LOADPATH_HINT = 9,
} pfsf_augmentation_kind;

typedef struct {
    int32_t struct_bytes;
    pfsf_augmentation_kind kind;
    void* dbb_addr;
    int64_t dbb_bytes;
    int32_t stride_bytes;
    int32_t version;
} pfsf_aug_slot;

PFSF_API pfsf_result pfsf_register_augmentation(pfsf_engine e, int32_t island_id, const pfsf_aug_slot* slot);
PFSF_API void pfsf_clear_augmentation(pfsf_engine e, int32_t island_id, pfsf_augmentation_kind kind);

typedef enum {
    PFSF_HOOK_PRE_SOURCE = 0,
    PFSF_HOOK_POST_SOURCE = 1,
    PFSF_HOOK_PRE_SOLVE = 2,
    PFSF_HOOK_POST_SOLVE = 3,
    PFSF_HOOK_PRE_SCAN = 4,
    PFSF_HOOK_POST_SCAN = 5,
} pfsf_hook_point;
#define PFSF_HOOK_POINT_COUNT 6

typedef void (*pfsf_hook_fn)(int32_t island_id, int64_t epoch, void* user_data);
PFSF_API void pfsf_set_hook(pfsf_engine e, pfsf_hook_point pt, pfsf_hook_fn fn, void* user_data);

/* Process-global registries (thread-safe). */
PFSF_API pfsf_result pfsf_aug_register(int32_t island_id, const pfsf_aug_slot* slot);
PFSF_API void pfsf_aug_clear(int32_t island_id, pfsf_augmentation_kind kind);
PFSF_API void pfsf_aug_clear_island(int32_t island_id);
PFSF_API int32_t pfsf_aug_query(int32_t island_id, pfsf_augmentation_kind kind, pfsf_aug_slot* out);
PFSF_API int32_t pfsf_aug_island_count(int32_t island_id);
PFSF_API void pfsf_hook_set(int32_t island_id, pfsf_hook_point pt, pfsf_hook_fn fn, void* user_data);
PFSF_API int32_t pfsf_hook_fire(int32_t island_id, pfsf_hook_point pt, int64_t epoch);
PFSF_API void pfsf_hook_clear(int32_t island_id, pfsf_hook_point pt);
PFSF_API void pfsf_hook_clear_island(int32_t island_id);

#ifdef __cplusplus
}
#endif
#endif
