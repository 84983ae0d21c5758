/*
 * pfsf_trace.h -- process-global trace ring and crash dump
 * (reference: L1-native/libpfsf/include/pfsf/pfsf_trace.h).  Host code.
 */
#ifndef PFSF_TRACE_H
#define PFSF_TRACE_H
#include "pfsf_types.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PFSF_TRACE_OFF = 0,
    PFSF_TRACE_ERROR = 1,
    PFSF_TRACE_WARN = 2,
    PFSF_TRACE_INFO = 3,
    PFSF_TRACE_VERBOSE = 4,
} pfsf_trace_level;

/* 64-byte event record. */
typedef struct {
    int64_t epoch;
    int32_t stage;
    int32_t island_id;
    int32_t voxel_index;
    int32_t errno_val;
    int16_t level;
    int16_t _pad;
    char msg[36];
} pfsf_trace_event;

#define PFSF_TRACE_RING_CAPACITY 4096

PFSF_API void pfsf_trace_emit(int16_t level, int64_t epoch, int32_t stage, int32_t island_id, int32_t voxel_index,
                              int32_t errno_val, const char* msg);
PFSF_API int32_t pfsf_drain_trace_dbb(void* out_addr, int64_t out_bytes, int32_t capacity);
PFSF_API int32_t pfsf_drain_trace(pfsf_engine e, pfsf_trace_event* out, int32_t capacity);
PFSF_API void pfsf_set_trace_level_global(pfsf_trace_level level);
PFSF_API int32_t pfsf_get_trace_level_global(void);
PFSF_API void pfsf_set_trace_level(pfsf_engine e, pfsf_trace_level level);
PFSF_API int32_t pfsf_trace_size(void);
PFSF_API void pfsf_trace_clear(void);

#define PFSF_CRASH_MAX_EVENTS 100
PFSF_API pfsf_result pfsf_install_crash_handler(void);
PFSF_API void pfsf_uninstall_crash_handler(void);
PFSF_API int32_t pfsf_dump_now_for_test(const char* path, int32_t signo, uintptr_t fault_addr);

#ifdef __cplusplus
}
#endif
#endif
