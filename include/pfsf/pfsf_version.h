/*
 * pfsf_version.h -- ABI / feature discovery (reference:
 * L1-native/libpfsf/include/pfsf/pfsf_version.h).
 */
#ifndef PFSF_VERSION_H
#define PFSF_VERSION_H
#include "pfsf_types.h"
#ifdef __cplusplus
extern "C" {
#endif

/* (major << 16) | (minor << 8) | patch of the libpfsf ABI this library implements. */
PFSF_API uint32_t pfsf_abi_version(void);
/* true for every feature flag the frozen ABI requires (compute.v1..v8,
 * diagnostics.v1, extension.v1, plan.v1, plan.v1.1, plan_buffer, trace.ring,
 * abi.v1, crash.handler.test) plus the B200 additions (cuda.sm100,
 * solve.tolerance, solve.batched, precision.bf16, precision.fp16). */
PFSF_API bool pfsf_has_feature(const char* name);
PFSF_API const char* pfsf_build_info(void);
/* Contract string checked by the Java bridge against its manifest ("1.5.0"). */
PFSF_API const char* pfsf_abi_contract_version(void);

#ifdef __cplusplus
}
#endif
#endif
