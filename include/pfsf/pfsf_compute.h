/*
 * pfsf_compute.h -- stateless host primitives used by the caller's data
 * assembly (reference: L1-native/libpfsf/include/pfsf/pfsf_compute.h,
 * implementations L1-native/libpfsf/src/compute/*.cpp).  Host code, no GPU.
 */
#ifndef PFSF_COMPUTE_H
#define PFSF_COMPUTE_H
#include "pfsf_types.h"
#ifdef __cplusplus
extern "C" {
#endif

/* Divide source, rcomp, rtens and the 6N conductivity by sigma_max =
 * max(1, max conductivity) when it exceeds 1; reports sigma_max. */
PFSF_API void pfsf_normalize_soa6(float* source, float* rcomp, float* rtens, float* conductivity,
                                  const float* hydration, int32_t n, float* out_sigma_max);
/* No-op kept for the ABI: the reference disabled the upwind face bias because
 * it made the operator non-symmetric (wind enters through the source term). */
PFSF_API void pfsf_apply_wind_bias(float* conductivity, int32_t n, pfsf_vec3 wind, float upwind_factor);
PFSF_API float pfsf_timoshenko_moment_factor(float b, float h, int32_t arm, float youngs_gpa, float nu);
PFSF_API float pfsf_wind_pressure_source(float wind_speed, float density_kg_m3, bool exposed);
/* Horizontal Manhattan distance to the nearest anchor-supported column. */
PFSF_API pfsf_result pfsf_compute_arm_map(const uint8_t* members, const uint8_t* anchors, int32_t lx, int32_t ly,
                                          int32_t lz, int32_t* out_arm);
PFSF_API pfsf_result pfsf_compute_arch_factor_map(const uint8_t* members, const uint8_t* anchors, int32_t lx,
                                                  int32_t ly, int32_t lz, float* out_arch);
PFSF_API int32_t pfsf_inject_phantom_edges(const uint8_t* members, float* conductivity, const float* rcomp,
                                           int32_t lx, int32_t ly, int32_t lz, float edge_penalty,
                                           float corner_penalty);
/* SoA-6 face conductivity from rcomp/rtens/type (vertical: min rcomp;
 * horizontal: tension-limited, wind-biased). */
PFSF_API void pfsf_compute_conductivity(float* conductivity, const float* rcomp, const float* rtens,
                                        const uint8_t* type, int32_t lx, int32_t ly, int32_t lz, pfsf_vec3 wind,
                                        float upwind_factor);
PFSF_API void pfsf_downsample_2to1(const float* fine, const uint8_t* fine_type, int32_t lxf, int32_t lyf,
                                   int32_t lzf, float* coarse, uint8_t* coarse_type);
PFSF_API uint32_t pfsf_morton_encode(uint32_t x, uint32_t y, uint32_t z);
PFSF_API void pfsf_morton_decode(uint32_t code, uint32_t* x, uint32_t* y, uint32_t* z);
PFSF_API void pfsf_tiled_layout_build(const float* linear, int32_t lx, int32_t ly, int32_t lz, int32_t tile,
                                      float* out);

#ifdef __cplusplus
}
#endif
#endif
