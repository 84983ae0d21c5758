/*
 * pfsf_diagnostics.h -- scheduler heuristics and divergence checks
 * (reference: L1-native/libpfsf/include/pfsf/pfsf_diagnostics.h).  Host code.
 */
#ifndef PFSF_DIAGNOSTICS_H
#define PFSF_DIAGNOSTICS_H
#include "pfsf_types.h"
#ifdef __cplusplus
extern "C" {
#endif

#define PFSF_OMEGA_TABLE_SIZE 64
#define PFSF_OMEGA_DENOM_EPSILON 0.01f
#define PFSF_MAX_OMEGA 1.98f
#define PFSF_MACRO_ACTIVATE_THRESHOLD 1.5e-4f
#define PFSF_MACRO_DEACTIVATE_THRESHOLD 0.8e-4f

/* Chebyshev semi-iteration weight: w0 = 1, w1 = 2/(2 - r^2),
 * wk = 4/(4 - r^2 w(k-1)), capped at PFSF_MAX_OMEGA. */
PFSF_API float pfsf_chebyshev_omega(int32_t iter, float rho_spec);
PFSF_API int32_t pfsf_precompute_omega_table(float rho_spec, float* out, int32_t capacity);
/* rho = cos(pi / l_max) * safety_margin */
PFSF_API float pfsf_estimate_spectral_radius(int32_t l_max, float safety_margin);

typedef struct {
    int32_t struct_bytes;
    float prev_max_phi;
    float prev_prev_max_phi;
    int32_t oscillation_count;
    int32_t damping_active;
    int32_t chebyshev_iter;
    float prev_max_macro_residual;
} pfsf_divergence_state;

typedef enum {
    PFSF_DIV_NONE = 0,
    PFSF_DIV_NAN_INF = 1,
    PFSF_DIV_RAPID_GROWTH = 2,
    PFSF_DIV_OSCILLATION = 3,
    PFSF_DIV_PERSISTENT_OSC = 4,
    PFSF_DIV_MACRO_REGION = 5,
} pfsf_divergence_kind;

PFSF_API int32_t pfsf_check_divergence(pfsf_divergence_state* st, float max_phi_now, const float* macro_residuals,
                                       int32_t macro_count, float divergence_ratio,
                                       float damping_settle_threshold);
PFSF_API int32_t pfsf_recommend_steps(int32_t ly, int32_t cheby_iter, int32_t is_dirty, int32_t has_collapse,
                                      int32_t steps_minor, int32_t steps_major, int32_t steps_collapse);
PFSF_API int32_t pfsf_macro_block_active(float residual, int32_t was_active);
PFSF_API float pfsf_macro_active_ratio(const float* residuals, int32_t n, const uint8_t* was_active);
PFSF_API void pfsf_extract_island_features(int32_t lx, int32_t ly, int32_t lz, int32_t chebyshev_iter,
                                           float rho_spec_override, float prev_max_macro_residual,
                                           int32_t oscillation_count, int32_t damping_active,
                                           int32_t stable_tick_count, int32_t lod_level, int32_t lod_dormant,
                                           int32_t pcg_allocated, const float* macro_residuals,
                                           int32_t macro_count, float* out12);

#ifdef __cplusplus
}
#endif
#endif
