/*
 * pfsf_plan.h -- length-prefixed opcode stream over the host primitives
 * (reference: L1-native/libpfsf/include/pfsf/pfsf_plan.h).  Host code.
 */
#ifndef PFSF_PLAN_H
#define PFSF_PLAN_H
#include "pfsf_types.h"
#ifdef __cplusplus
extern "C" {
#endif

#define PFSF_PLAN_MAGIC 0x46534650u /* "PFSF" little-endian */
#define PFSF_PLAN_VERSION 1u
#define PFSF_PLAN_HEADER_BYTES 16
#define PFSF_PLAN_OP_HEADER_BYTES 4

typedef enum {
    PFSF_OP_NO_OP = 0,
    PFSF_OP_INCR_COUNTER = 1,
    PFSF_OP_CLEAR_AUG = 2,
    PFSF_OP_CLEAR_AUG_ISLAND = 3,
    PFSF_OP_FIRE_HOOK = 4,
    PFSF_OP_NORMALIZE_SOA6 = 5,
    PFSF_OP_APPLY_WIND_BIAS = 6,
    PFSF_OP_COMPUTE_CONDUCTIVITY = 7,
    PFSF_OP_ARM_MAP = 8,
    PFSF_OP_ARCH_FACTOR = 9,
    PFSF_OP_PHANTOM_EDGES = 10,
    PFSF_OP_DOWNSAMPLE_2TO1 = 11,
    PFSF_OP_TILED_LAYOUT = 12,
    PFSF_OP_CHEBYSHEV = 13,
    PFSF_OP_CHECK_DIVERGENCE = 14,
    PFSF_OP_EXTRACT_FEATURES = 15,
    PFSF_OP_WIND_PRESSURE = 16,
    PFSF_OP_TIMOSHENKO = 17,
    PFSF_OP_AUG_SOURCE_ADD = 18,
    PFSF_OP_AUG_COND_MUL = 19,
    PFSF_OP_AUG_RCOMP_MUL = 20,
    PFSF_OP_AUG_WIND_3D_BIAS = 21,
} pfsf_plan_opcode;

typedef struct {
    int32_t struct_bytes;
    int32_t executed_count;
    int32_t failed_index;
    int32_t error_code;
    int32_t hook_fire_count;
} pfsf_plan_result;

PFSF_API pfsf_result pfsf_plan_execute(const void* plan, int64_t plan_bytes, pfsf_plan_result* out);
PFSF_API int64_t pfsf_plan_test_counter_read_reset(void);
PFSF_API void pfsf_plan_test_hook_install(int32_t island_id, int32_t point);
PFSF_API int64_t pfsf_plan_test_hook_count_read_reset(int32_t island_id, int32_t point);

#ifdef __cplusplus
}
#endif
#endif
