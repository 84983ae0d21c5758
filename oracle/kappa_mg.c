/*
 * CPU multigrid-preconditioned CG on the symmetric harmonic-mean 26-point
 * operator -- TEST INFRASTRUCTURE (the checker and the timed CPU baseline),
 * never part of the product path.
 *
 *   (A phi)_i = sum_j w_ij (phi_i - phi_j),  w_ij = g_k k_i k_j / (k_i + k_j)
 *   g = 2 (face), 1 (edge), 1/3 (corner), i.e. {1, 0.5, 1/6} x the harmonic
 *   mean 2 k_i k_j / (k_i + k_j); unknowns are the solid voxels, anchors are
 *   Dirichlet (phi = 0), air and out-of-box links are dropped -- the operator
 *   of the benchmark configurations, with the structure of the reference's
 *   symmetric CPU solver (validation/VoxelPhysicsCpuReference.java:84-113).
 *
 * Hierarchy: 2x2x2 aggregation with Galerkin coarse operators (up to 5
 * levels, stopping at a side of 2 or 64 cells), symmetric 8-colour
 * Gauss-Seidel smoothing (the reference's RBGS colouring,
 * SH/rbgs_smooth.comp.glsl; 2 pre- and 2 post-sweeps, 4 symmetric sweeps on
 * the coarsest level), coarse correction weighted 1.8 -- the same V-cycle
 * the library's per-island FP32 solve runs on the GPU.  OpenMP over the
 * cells of a pass (the colours of a 26-point stencil are independent).
 *
 *   o_kappa_mgpcg64: everything FP64, for reference solutions (tol 1e-12).
 *   o_kappa_mgpcg32: FP32 hierarchy and inner PCG, FP64 outer residual and
 *                    solution -- the plain FP32 scheme, the timed baseline.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MG_MAX_LEVELS 5

/* the 26 neighbours in lexicographic (z, y, x) order, centre skipped: the
 * first 13 are "backward", the last 13 "forward" */
static int N26[26][3];
static double GS26[26];
static int FWD_OF[26], BWD_OF[26];

__attribute__((constructor)) static void mg_tables(void) {
    int k = 0;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                if (!dx && !dy && !dz) continue;
                N26[k][0] = dx; N26[k][1] = dy; N26[k][2] = dz;
                const int g = (dx != 0) + (dy != 0) + (dz != 0);
                GS26[k] = g == 1 ? 2.0 : (g == 2 ? 1.0 : 1.0 / 3.0);
                FWD_OF[k] = k >= 13 ? k - 13 : -1;  /* forward slot of this offset at i */
                BWD_OF[k] = k < 13 ? 12 - k : -1;   /* slot of the opposite offset at j */
                k++;
            }
}

static inline double mg_hm(double a, double b) { return (a + b) > 0.0 ? a * b / (a + b) : 0.0; }
static inline int mg_max3(int a, int b, int c) { return a > b ? (a > c ? a : c) : (b > c ? b : c); }

#define REAL double
#define SFX _f64
#include "kappa_mg_impl.h"
#undef REAL
#undef SFX

#define REAL float
#define SFX _f32
#include "kappa_mg_impl.h"
#undef REAL
#undef SFX

/* relative residual ||s - A x|| / ||s|| over solid rows with the FP64 fine
 * operator (r gets s - A x) */
static double mg_residual64(const level_t_f64 *L, const double *s, const double *x, double *r, int nt, double *bnorm) {
    apply_f64(L, x, r, nt);
    double rr = 0.0, bb = 0.0;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static) reduction(+ : rr, bb)
    for (int64_t i = 0; i < L->n; i++) {
        if (!(L->diag[i] > 0.0)) { r[i] = 0.0; continue; }
        r[i] = s[i] - r[i];
        rr += r[i] * r[i];
        bb += s[i] * s[i];
    }
    *bnorm = sqrt(bb);
    return bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
}

/* FP64 MG-PCG from x (in/out; zeroed off the solid voxels) to
 * ||s - A x|| <= tol ||s||, with up to 4 residual restarts.  Returns the
 * total PCG iterations; *relres the final FP64 relative residual. */
int o_kappa_mgpcg64(int lx, int ly, int lz, const double *kappa, const uint8_t *type, const double *s, double *x,
                    double tol, int maxit, int nthreads, double *relres) {
    const int nt = nthreads > 0 ? nthreads : 1;
    hier_t_f64 H;
    hier_build_f64(&H, lx, ly, lz, kappa, type, nt);
    const int64_t n = H.lev[0].n;
    double *r = malloc((size_t)n * 8), *e = malloc((size_t)n * 8), *p = malloc((size_t)n * 8),
           *q = malloc((size_t)n * 8), *w = malloc((size_t)n * 8);
    for (int64_t i = 0; i < n; i++)
        if (type[i] != 1) x[i] = 0.0;
    double bn = 0.0;
    double rel = mg_residual64(&H.lev[0], s, x, r, nt, &bn);
    int total = 0;
    for (int outer = 0; outer < 4 && rel > tol && total < maxit; outer++) {
        double inner_rel = 0.0;
        /* stop the inner solve a little below the target */
        const double stop = fmax(0.25 * tol / rel, 1e-15);
        total += pcg_f64(&H, r, e, p, q, w, stop, maxit - total, &inner_rel);
        for (int64_t i = 0; i < n; i++) x[i] += e[i];
        rel = mg_residual64(&H.lev[0], s, x, r, nt, &bn);
    }
    *relres = rel;
    free(r); free(e); free(p); free(q); free(w);
    hier_free_f64(&H);
    return total;
}

/* The plain FP32 scheme: FP32 hierarchy, FP32 inner PCG on A e = r stopping
 * at ||r_in|| <= max(1e-4, 0.3 tol / relres) ||r||, FP64 solution x and
 * FP64 outer residual, at most 8 refinements.  Returns total inner
 * iterations; *relres = final FP64 relative residual, *outer_out the
 * refinements. */
int o_kappa_mgpcg32(int lx, int ly, int lz, const double *kappa, const uint8_t *type, const double *s, double *x,
                    double tol, int maxit, int nthreads, double *relres, int *outer_out) {
    const int nt = nthreads > 0 ? nthreads : 1;
    level_t_f64 L64;
    level_alloc_f64(&L64, lx, ly, lz);
    build_fine_f64(&L64, kappa, type, nt);
    hier_t_f32 H;
    hier_build_f32(&H, lx, ly, lz, kappa, type, nt);
    const int64_t n = L64.n;
    double *r = malloc((size_t)n * 8);
    float *rf = malloc((size_t)n * 4), *e = malloc((size_t)n * 4), *p = malloc((size_t)n * 4),
          *q = malloc((size_t)n * 4), *w = malloc((size_t)n * 4);
    for (int64_t i = 0; i < n; i++)
        if (type[i] != 1) x[i] = 0.0;
    double bn = 0.0;
    double rel = mg_residual64(&L64, s, x, r, nt, &bn);
    int total = 0, outer = 0;
    for (outer = 0; outer < 8 && rel > tol && total < maxit; outer++) {
        for (int64_t i = 0; i < n; i++) rf[i] = (float)r[i];
        const double eta = fmax(1e-4, 0.3 * tol / rel);
        double inner_rel = 0.0;
        total += pcg_f32(&H, rf, e, p, q, w, eta, maxit - total, &inner_rel);
        for (int64_t i = 0; i < n; i++) x[i] += (double)e[i];
        rel = mg_residual64(&L64, s, x, r, nt, &bn);
    }
    *relres = rel;
    if (outer_out) *outer_out = outer;
    free(r); free(rf); free(e); free(p); free(q); free(w);
    free(L64.diag); free(L64.off); free(L64.x); free(L64.b); free(L64.r);
    hier_free_f32(&H);
    return total;
}
