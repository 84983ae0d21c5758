/* Template body of the CPU multigrid-preconditioned CG (kappa_mg.c): the
 * hierarchy, smoother and inner PCG in precision REAL, functions suffixed
 * SFX.  Included once per precision.  Test infrastructure only. */

#define MG_CAT2(a, b) a##b
#define MG_CAT(a, b) MG_CAT2(a, b)
#define F(name) MG_CAT(name, SFX)

typedef struct {
    int lx, ly, lz;
    int64_t n;
    REAL *diag; /* n: A_ii (0 on inactive cells) */
    REAL *off;  /* 13 * n: w_ij for the forward neighbour j = i + FO[k] (A_ij = -w) */
    REAL *x, *b, *r;
} F(level_t);

typedef struct {
    int nlev, nt;
    F(level_t) lev[MG_MAX_LEVELS];
} F(hier_t);

static void F(level_alloc)(F(level_t) * L, int lx, int ly, int lz) {
    L->lx = lx; L->ly = ly; L->lz = lz;
    L->n = (int64_t)lx * ly * lz;
    L->diag = calloc((size_t)L->n, sizeof(REAL));
    L->off = calloc((size_t)L->n * 13, sizeof(REAL));
    L->x = calloc((size_t)L->n, sizeof(REAL));
    L->b = calloc((size_t)L->n, sizeof(REAL));
    L->r = calloc((size_t)L->n, sizeof(REAL));
}

static void F(hier_free)(F(hier_t) * H) {
    for (int l = 0; l < H->nlev; l++) {
        free(H->lev[l].diag); free(H->lev[l].off); free(H->lev[l].x); free(H->lev[l].b); free(H->lev[l].r);
    }
    H->nlev = 0;
}

/* weight of link (i, j) for the 26 neighbours: forward slots at i, backward at j */
static inline REAL F(link_w)(const F(level_t) * L, int64_t i, int k26, int64_t j) {
    const int fk = FWD_OF[k26];
    return fk >= 0 ? L->off[(int64_t)fk * L->n + i] : L->off[(int64_t)BWD_OF[k26] * L->n + j];
}

/* sum_j w_ij v_j over the 26 neighbours of an interior cell i (no bounds
 * checks): forward weights stored at i, backward ones at the neighbour */
static inline REAL F(nbsum)(const F(level_t) * L, int64_t i, const REAL *v, int64_t sy, int64_t sz) {
    const int64_t n = L->n;
    const REAL *off = L->off;
    REAL s = 0;
    for (int k = 0; k < 13; k++) {
        const int64_t o = N26[k + 13][0] + sy * N26[k + 13][1] + sz * N26[k + 13][2];
        s += off[(int64_t)k * n + i] * v[i + o];
        s += off[(int64_t)k * n + i - o] * v[i - o];
    }
    return s;
}

/* fine level from kappa / type: unknowns are the solid voxels; anchors
 * (Dirichlet, phi = 0) and out-of-box / air links enter the diagonal only /
 * not at all. */
static void F(build_fine)(F(level_t) * L, const double *kappa, const uint8_t *type, int nt) {
    const int lx = L->lx, ly = L->ly, lz = L->lz;
    const int64_t n = L->n;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
    for (int z = 0; z < lz; z++)
        for (int y = 0; y < ly; y++)
            for (int x = 0; x < lx; x++) {
                const int64_t i = x + (int64_t)lx * (y + (int64_t)ly * z);
                double d = 0.0;
                if (type[i] == 1) {
                    for (int k = 0; k < 26; k++) {
                        const int nx = x + N26[k][0], ny = y + N26[k][1], nz = z + N26[k][2];
                        if (nx < 0 || ny < 0 || nz < 0 || nx >= lx || ny >= ly || nz >= lz) continue;
                        const int64_t j = nx + (int64_t)lx * (ny + (int64_t)ly * nz);
                        if (type[j] == 0) continue;
                        const double w = GS26[k] * mg_hm(kappa[i], kappa[j]);
                        d += w;
                        if (FWD_OF[k] >= 0 && type[j] == 1) L->off[(int64_t)FWD_OF[k] * n + i] = (REAL)w;
                    }
                }
                L->diag[i] = (REAL)d;
            }
}

/* Galerkin coarse level of 2x2x2 aggregates: A_c = P^T A P with P the
 * piecewise-constant prolongation.  Off-diagonals sum the links between two
 * aggregates, the diagonal sums the children's diagonals minus the links
 * inside the aggregate (so anchor couplings stay on the diagonal). */
static void F(build_coarse)(const F(level_t) * Fl, F(level_t) * C, int nt) {
    const int fx = Fl->lx, fy = Fl->ly, fz = Fl->lz;
    const int cx = C->lx, cy = C->ly, cz = C->lz;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
    for (int Z = 0; Z < cz; Z++)
        for (int Y = 0; Y < cy; Y++)
            for (int X = 0; X < cx; X++) {
                const int64_t c = X + (int64_t)cx * (Y + (int64_t)cy * Z);
                double diag = 0.0;
                double W[13] = {0};
                for (int a = 0; a < 8; a++) {
                    const int x = 2 * X + (a & 1), y = 2 * Y + ((a >> 1) & 1), z = 2 * Z + ((a >> 2) & 1);
                    if (x >= fx || y >= fy || z >= fz) continue;
                    const int64_t i = x + (int64_t)fx * (y + (int64_t)fy * z);
                    if (!(Fl->diag[i] > 0)) continue;
                    diag += (double)Fl->diag[i];
                    for (int k = 0; k < 26; k++) {
                        const int nx = x + N26[k][0], ny = y + N26[k][1], nz = z + N26[k][2];
                        if (nx < 0 || ny < 0 || nz < 0 || nx >= fx || ny >= fy || nz >= fz) continue;
                        const int64_t j = nx + (int64_t)fx * (ny + (int64_t)fy * nz);
                        const double w = (double)F(link_w)(Fl, i, k, j);
                        if (w == 0.0) continue;
                        const int dX = (nx >> 1) - X, dY = (ny >> 1) - Y, dZ = (nz >> 1) - Z;
                        if (!dX && !dY && !dZ) { diag -= w; continue; }
                        const int q = (dZ + 1) * 9 + (dY + 1) * 3 + (dX + 1);
                        if (q > 13) W[q - 14] += w;
                    }
                }
                C->diag[c] = (REAL)(diag > 0.0 ? diag : 0.0);
                for (int k = 0; k < 13; k++) C->off[(int64_t)k * C->n + c] = (REAL)W[k];
            }
}

static int F(hier_build)(F(hier_t) * H, int lx, int ly, int lz, const double *kappa, const uint8_t *type, int nt) {
    H->nt = nt;
    H->nlev = 1;
    F(level_alloc)(&H->lev[0], lx, ly, lz);
    F(build_fine)(&H->lev[0], kappa, type, nt);
    int x = lx, y = ly, z = lz;
    while (H->nlev < MG_MAX_LEVELS && mg_max3(x, y, z) > 2 && (int64_t)x * y * z > 64) {
        x = (x + 1) / 2; y = (y + 1) / 2; z = (z + 1) / 2;
        F(level_alloc)(&H->lev[H->nlev], x, y, z);
        F(build_coarse)(&H->lev[H->nlev - 1], &H->lev[H->nlev], nt);
        H->nlev++;
    }
    return H->nlev;
}

/* y = A v on level L (active rows; 0 elsewhere); returns nothing */
static void F(apply)(const F(level_t) * L, const REAL *v, REAL *y, int nt) {
    const int lx = L->lx, ly = L->ly, lz = L->lz;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
    for (int z = 0; z < lz; z++)
        for (int yy = 0; yy < ly; yy++)
            for (int x = 0; x < lx; x++) {
                const int64_t i = x + (int64_t)lx * (yy + (int64_t)ly * z);
                const REAL d = L->diag[i];
                if (!(d > 0)) { y[i] = 0; continue; }
                REAL s = 0;
                if (x > 0 && yy > 0 && z > 0 && x + 1 < lx && yy + 1 < ly && z + 1 < lz) {
                    s = F(nbsum)(L, i, v, lx, (int64_t)lx * ly);
                    y[i] = d * v[i] - s;
                    continue;
                }
                for (int k = 0; k < 26; k++) {
                    const int nx = x + N26[k][0], ny = yy + N26[k][1], nz = z + N26[k][2];
                    if (nx < 0 || ny < 0 || nz < 0 || nx >= lx || ny >= ly || nz >= lz) continue;
                    const int64_t j = nx + (int64_t)lx * (ny + (int64_t)ly * nz);
                    s += F(link_w)(L, i, k, j) * v[j];
                }
                y[i] = d * v[i] - s;
            }
}

/* one Gauss-Seidel pass over the cells of colour col (x, y, z parities) */
static void F(gs_color)(F(level_t) * L, int col, int nt) {
    const int lx = L->lx, ly = L->ly, lz = L->lz;
    const int px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
    const int nzc = (lz - pz + 1) / 2;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
    for (int zi = 0; zi < nzc; zi++) {
        const int z = pz + 2 * zi;
        for (int yy = py; yy < ly; yy += 2)
            for (int x = px; x < lx; x += 2) {
                const int64_t i = x + (int64_t)lx * (yy + (int64_t)ly * z);
                const REAL d = L->diag[i];
                if (!(d > 0)) continue;
                REAL s = L->b[i];
                if (x > 0 && yy > 0 && z > 0 && x + 1 < lx && yy + 1 < ly && z + 1 < lz) {
                    L->x[i] = (s + F(nbsum)(L, i, L->x, lx, (int64_t)lx * ly)) / d;
                    continue;
                }
                for (int k = 0; k < 26; k++) {
                    const int nx = x + N26[k][0], ny = yy + N26[k][1], nz = z + N26[k][2];
                    if (nx < 0 || ny < 0 || nz < 0 || nx >= lx || ny >= ly || nz >= lz) continue;
                    const int64_t j = nx + (int64_t)lx * (ny + (int64_t)ly * nz);
                    s += F(link_w)(L, i, k, j) * L->x[j];
                }
                L->x[i] = s / d;
            }
    }
}

static void F(sweep)(F(level_t) * L, int forward, int nt) {
    for (int c = 0; c < 8; c++) F(gs_color)(L, forward ? c : 7 - c, nt);
}

/* b_{l+1} = sum over each aggregate of (b - A x) on level l; x_{l+1} = 0 */
static void F(restrict_res)(F(level_t) * Fl, F(level_t) * C, int nt) {
    F(apply)(Fl, Fl->x, Fl->r, nt);
    const int fx = Fl->lx, fy = Fl->ly, fz = Fl->lz, cx = C->lx, cy = C->ly, cz = C->lz;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
    for (int Z = 0; Z < cz; Z++)
        for (int Y = 0; Y < cy; Y++)
            for (int X = 0; X < cx; X++) {
                const int64_t c = X + (int64_t)cx * (Y + (int64_t)cy * Z);
                REAL s = 0;
                for (int a = 0; a < 8; a++) {
                    const int x = 2 * X + (a & 1), y = 2 * Y + ((a >> 1) & 1), z = 2 * Z + ((a >> 2) & 1);
                    if (x >= fx || y >= fy || z >= fz) continue;
                    const int64_t i = x + (int64_t)fx * (y + (int64_t)fy * z);
                    if (Fl->diag[i] > 0) s += Fl->b[i] - Fl->r[i];
                }
                C->b[c] = s;
                C->x[c] = 0;
            }
}

static void F(prolong_add)(F(level_t) * Fl, const F(level_t) * C, REAL omega, int nt) {
    const int fx = Fl->lx, fy = Fl->ly, fz = Fl->lz, cx = C->lx, cy = C->ly;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
    for (int z = 0; z < fz; z++)
        for (int y = 0; y < fy; y++)
            for (int x = 0; x < fx; x++) {
                const int64_t i = x + (int64_t)fx * (y + (int64_t)fy * z);
                if (Fl->diag[i] > 0) Fl->x[i] += omega * C->x[(x >> 1) + (int64_t)cx * ((y >> 1) + (int64_t)cy * (z >> 1))];
            }
}

/* One symmetric V-cycle on A_l x = b_l from x = 0: nu forward-colour GS
 * sweeps, restriction, the next level, prolongation weighted by omega, nu
 * reverse-colour sweeps; coarse_sweeps symmetric sweeps on the coarsest. */
static void F(vcycle)(F(hier_t) * H, int l, int nu, int coarse_sweeps, REAL omega) {
    F(level_t) *L = &H->lev[l];
    const int nt = L->n >= 32768 ? H->nt : 1;
    memset(L->x, 0, (size_t)L->n * sizeof(REAL));
    if (l >= H->nlev - 1 || l >= MG_MAX_LEVELS - 1) {
        for (int s = 0; s < coarse_sweeps; s++) { F(sweep)(L, 1, nt); F(sweep)(L, 0, nt); }
        return;
    }
    for (int s = 0; s < nu; s++) F(sweep)(L, 1, nt);
    F(restrict_res)(L, &H->lev[l + 1], nt);
    F(vcycle)(H, l + 1, nu, coarse_sweeps, omega);
    F(prolong_add)(L, &H->lev[l + 1], omega, nt);
    for (int s = 0; s < nu; s++) F(sweep)(L, 0, nt);
}

static double F(dot)(const REAL *a, const REAL *b, int64_t n, int nt) {
    double s = 0.0;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static) reduction(+ : s)
    for (int64_t i = 0; i < n; i++) s += (double)a[i] * (double)b[i];
    return s;
}

/* PCG on A e = rhs (level 0 of H), e from 0, preconditioned by one V-cycle,
 * until ||r|| <= stop * ||rhs|| or maxit iterations.  Returns iterations;
 * work vectors p, q, rr of n entries; e out. */
static int F(pcg)(F(hier_t) * H, const REAL *rhs, REAL *e, REAL *p, REAL *q, REAL *rr, double stop, int maxit,
                  double *relres) {
    F(level_t) *L0 = &H->lev[0];
    const int64_t n = L0->n;
    const int nt = H->nt;
    const int nu = 2, csw = 4;
    const REAL omega = (REAL)1.8;
    memcpy(rr, rhs, (size_t)n * sizeof(REAL));
    memset(e, 0, (size_t)n * sizeof(REAL));
    const double r0 = sqrt(F(dot)(rr, rr, n, nt));
    if (r0 == 0.0) { *relres = 0.0; return 0; }
    memcpy(L0->b, rr, (size_t)n * sizeof(REAL));
    F(vcycle)(H, 0, nu, csw, omega);
    memcpy(p, L0->x, (size_t)n * sizeof(REAL));
    double rz = F(dot)(rr, L0->x, n, nt);
    int it = 0;
    double rn = r0;
    for (it = 0; it < maxit;) {
        F(apply)(L0, p, q, nt);
        const double pq = F(dot)(p, q, n, nt);
        if (!(pq > 0.0)) break;
        const REAL a = (REAL)(rz / pq);
        double s = 0.0;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static) reduction(+ : s)
        for (int64_t i = 0; i < n; i++) {
            e[i] += a * p[i];
            rr[i] -= a * q[i];
            s += (double)rr[i] * (double)rr[i];
        }
        it++;
        rn = sqrt(s);
        if (rn <= stop * r0) break;
        memcpy(L0->b, rr, (size_t)n * sizeof(REAL));
        F(vcycle)(H, 0, nu, csw, omega);
        const double rzn = F(dot)(rr, L0->x, n, nt);
        const REAL beta = (REAL)(rzn / rz);
        rz = rzn;
        const REAL *z = L0->x;
#pragma omp parallel for num_threads(nt) if (nt > 1) schedule(static)
        for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
    *relres = rn / r0;
    return it;
}

#undef F
#undef MG_CAT
#undef MG_CAT2
