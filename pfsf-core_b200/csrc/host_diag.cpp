// Scheduler heuristics of the frozen ABI (pfsf_diagnostics.h): Chebyshev
// weights, spectral-radius estimate, step recommendation, macro-block
// hysteresis, the divergence state machine and the 12-float island feature
// vector.  Host code with the reference's float/double arithmetic order so
// the Java golden-parity values carry over unchanged.
//
// Reference semantics followed (project-relative paths):
//   chebyshev_omega / precompute_omega_table / estimate_spectral_radius /
//   recommend_steps / macro_block_active / macro_active_ratio
//                          L1-native/libpfsf/src/compute/chebyshev.cpp:30-142
//   check_divergence       L1-native/libpfsf/src/compute/divergence.cpp:20-116
//   extract_island_features L1-native/libpfsf/src/compute/features.cpp:48-129
#include <cmath>
#include <cstdint>

#include "pfsf/pfsf_diagnostics.h"

extern "C" {

// w0 = 1, w1 = 2/(2 - r^2), wk = 4/(4 - r^2 w(k-1)).  The recurrence stops
// at the last good weight when its denominator nears zero or a weight leaves
// (0, 2]; the result is capped at PFSF_MAX_OMEGA.
PFSF_API float pfsf_chebyshev_omega(int32_t iter, float rho_spec) {
    if (iter <= 0) return 1.0f;
    const float r2 = rho_spec * rho_spec;
    if (r2 >= 1.0f) return 1.0f;
    float w = 2.0f / (2.0f - r2);
    if (iter == 1) return w;
    float w_prev = 1.0f;
    for (int32_t k = 2; k <= iter; ++k) {
        const float den = 4.0f - r2 * w;
        if (den < PFSF_OMEGA_DENOM_EPSILON) {
            w = w_prev;
            break;
        }
        const float nw = 4.0f / den;
        if (nw > 2.0f || std::isnan(nw)) {
            w = w_prev;
            break;
        }
        w_prev = w;
        w = nw;
    }
    return PFSF_MAX_OMEGA < w ? PFSF_MAX_OMEGA : w;
}

// Table form: each entry is clamped to PFSF_MAX_OMEGA and the recurrence
// continues from the clamped value (a NaN entry becomes 1).
PFSF_API int32_t pfsf_precompute_omega_table(float rho_spec, float* out, int32_t capacity) {
    if (!out || capacity <= 0) return PFSF_ERROR_INVALID_ARG;
    const float r2 = rho_spec * rho_spec;
    out[0] = 1.0f;
    if (capacity > 1) out[1] = r2 < 1.0f ? 2.0f / (2.0f - r2) : 1.0f;
    for (int32_t k = 2; k < capacity; ++k) {
        const float den = 4.0f - r2 * out[k - 1];
        if (den < PFSF_OMEGA_DENOM_EPSILON) {
            out[k] = out[k - 1];
            continue;
        }
        float w = 4.0f / den;
        if (w > PFSF_MAX_OMEGA) w = PFSF_MAX_OMEGA;
        if (std::isnan(w)) w = 1.0f;
        out[k] = w;
    }
    return capacity;
}

// Jacobi spectral radius of a box of longest side l_max, times a margin.
PFSF_API float pfsf_estimate_spectral_radius(int32_t l_max, float safety_margin) {
    if (l_max <= 1) return 0.5f;
    const double pi = 3.14159265358979323846;
    return float(std::cos(pi / double(l_max)) * double(safety_margin));
}

PFSF_API int32_t pfsf_recommend_steps(int32_t ly, int32_t cheby_iter, int32_t is_dirty, int32_t has_collapse,
                                      int32_t steps_minor, int32_t steps_major, int32_t steps_collapse) {
    if (!is_dirty && cheby_iter > PFSF_OMEGA_TABLE_SIZE) return 0;  // converged and clean: skip
    if (has_collapse) {
        int32_t s = int32_t(float(ly) * 1.5f);  // Java (int)(height * 1.5f)
        if (s < steps_collapse) s = steps_collapse;
        return s > 128 ? 128 : s;
    }
    return is_dirty ? steps_major : steps_minor;
}

// Hysteresis: an active block stays active above the lower threshold, an
// idle one wakes above the upper threshold.
PFSF_API int32_t pfsf_macro_block_active(float residual, int32_t was_active) {
    const float thr = was_active ? PFSF_MACRO_DEACTIVATE_THRESHOLD : PFSF_MACRO_ACTIVATE_THRESHOLD;
    return residual > thr ? 1 : 0;
}

PFSF_API float pfsf_macro_active_ratio(const float* residuals, int32_t n, const uint8_t* was_active) {
    if (!residuals || n <= 0) return 1.0f;
    int32_t on = 0;
    for (int32_t i = 0; i < n; ++i) on += pfsf_macro_block_active(residuals[i], was_active ? was_active[i] != 0 : 1);
    return float(on) / float(n);
}

// State machine over the per-tick max |phi| (and optionally the macro-block
// residuals).  Checks in order: NaN/Inf, rapid growth, direction flips
// (short and persistent), macro-region blow-up, then damping release.
PFSF_API int32_t pfsf_check_divergence(pfsf_divergence_state* st, float now, const float* macro, int32_t macro_count,
                                       float divergence_ratio, float settle) {
    if (!st) return PFSF_DIV_NONE;
    const float prev = st->prev_max_phi;
    const float prev2 = st->prev_prev_max_phi;
    auto shift = [&]() {
        st->prev_prev_max_phi = prev;
        st->prev_max_phi = now;
    };
    if (std::isnan(now) || std::isinf(now)) {
        st->chebyshev_iter = 0;
        st->damping_active = 1;
        st->prev_prev_max_phi = prev;
        st->prev_max_phi = -1.0f;  // marks "no usable history" for the next call
        return PFSF_DIV_NAN_INF;
    }
    if (prev < 0.0f) {
        st->prev_prev_max_phi = 0.0f;
        st->prev_max_phi = now;
        return PFSF_DIV_NONE;
    }
    if (prev > 0.0f && now > prev * divergence_ratio) {
        st->chebyshev_iter = 0;
        shift();
        return PFSF_DIV_RAPID_GROWTH;
    }
    if (prev2 > 0.0f && prev > 0.0f && now > 0.0f) {
        const bool flip = (prev > prev2) != (now > prev);
        st->oscillation_count = flip ? st->oscillation_count + 1 : 0;
        const float amp = std::fabs(now - prev) / prev;
        if (flip && amp > 0.10f) {
            st->chebyshev_iter = 0;
            st->damping_active = 1;
            shift();
            return PFSF_DIV_OSCILLATION;
        }
        if (st->oscillation_count >= 5 && amp > 0.02f) {
            st->chebyshev_iter = 0;
            st->damping_active = 1;
            st->oscillation_count = 0;
            shift();
            return PFSF_DIV_PERSISTENT_OSC;
        }
    }
    if (macro && macro_count > 0) {
        float m = 0.0f;
        for (int32_t i = 0; i < macro_count; ++i) m = macro[i] > m ? macro[i] : m;
        const bool blew_up = st->prev_max_macro_residual > 0.0f && m > st->prev_max_macro_residual * 2.0f;
        st->prev_max_macro_residual = m;
        if (blew_up) {
            st->chebyshev_iter = 0;
            shift();
            return PFSF_DIV_MACRO_REGION;
        }
    }
    if (st->damping_active && prev > 0.0f && std::fabs(now - prev) / prev < settle) st->damping_active = 0;
    shift();
    return PFSF_DIV_NONE;
}

// [0] log2 N, [1] aspect max/min side, [2] chebyshev_iter/64, [3] rho override,
// [4] log10 prev macro residual, [5] residual drop ratio, [6] oscillation/10,
// [7] damping flag, [8] stable ticks/100, [9] macro residual coefficient of
// variation, [10] lod level / dormant level, [11] PCG flag.
PFSF_API void pfsf_extract_island_features(int32_t lx, int32_t ly, int32_t lz, int32_t chebyshev_iter,
                                           float rho_spec_override, float prev_max_macro_residual,
                                           int32_t oscillation_count, int32_t damping_active,
                                           int32_t stable_tick_count, int32_t lod_level, int32_t lod_dormant,
                                           int32_t pcg_allocated, const float* macro_residuals, int32_t macro_count,
                                           float* out12) {
    if (!out12) return;
    constexpr float kTiny = 1e-20f;
    auto pos = [](int32_t v) { return int64_t(v > 0 ? v : 0); };
    int64_t n = pos(lx) * pos(ly) * pos(lz);
    if (n <= 0) n = 1;
    out12[0] = float(std::log(double(n)) / std::log(2.0));
    const int32_t lo = lx < ly ? (lx < lz ? lx : lz) : (ly < lz ? ly : lz);
    const int32_t hi = lx > ly ? (lx > lz ? lx : lz) : (ly > lz ? ly : lz);
    out12[1] = lo > 0 ? float(hi) / float(lo) : 1.0f;
    out12[2] = float(chebyshev_iter) / float(PFSF_OMEGA_TABLE_SIZE);
    out12[3] = rho_spec_override;
    const bool have_prev = prev_max_macro_residual > kTiny;
    out12[4] = float(std::log10(double(have_prev ? prev_max_macro_residual : kTiny)));
    float cur = 0.0f;
    if (macro_residuals && macro_count > 0) {
        cur = macro_residuals[0];
        for (int32_t i = 1; i < macro_count; ++i) cur = macro_residuals[i] > cur ? macro_residuals[i] : cur;
    }
    out12[5] = have_prev ? cur / prev_max_macro_residual : 1.0f;
    auto unit = [](float v) { return v > 1.0f ? 1.0f : (v < 0.0f ? 0.0f : v); };
    out12[6] = unit(float(oscillation_count) / 10.0f);
    out12[7] = damping_active ? 1.0f : 0.0f;
    out12[8] = unit(float(stable_tick_count) / 100.0f);
    float cv = 0.0f;
    if (macro_residuals && macro_count >= 2) {
        double s1 = 0.0, s2 = 0.0;
        for (int32_t i = 0; i < macro_count; ++i) {
            const double v = macro_residuals[i];
            s1 += v;
            s2 += v * v;
        }
        const double mean = s1 / double(macro_count);
        if (!(mean < double(kTiny))) {
            const double var = s2 / double(macro_count) - mean * mean;
            cv = float(std::sqrt(var > 0.0 ? var : 0.0) / mean);
        }
    }
    out12[9] = cv;
    out12[10] = float(lod_level) / float(lod_dormant > 1 ? lod_dormant : 1);
    out12[11] = pcg_allocated ? 1.0f : 0.0f;
}

}  // extern "C"
