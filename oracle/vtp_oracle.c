/*
 * CPU oracle (test infrastructure; see vtp_oracle.h).  Restates:
 *   neighbour search  UGNSCudaImpl.cu:28-203, UniformGridNeighborSearch.cpp:33-60
 *   SPH kernels       KernelFunctions.cuh:13-70
 *   PBF               PBFCudaImpl.cu:34-194 in the order of PBFSolver.cpp:326-362
 *   DFSPH             DFSPHCudaImpl.cu:38-611 in the order of DFSPHSolver.cpp:339-391
 *   IMM-CT / IMM      IMMCTCudaImpl.cu:52-821 in the order of IMMCTSolver.cpp:408-477 and
 *                     IMMCTCudaImpl.cu:849-1152; IMM the same without the conformation
 *                     terms and with a constant Cd (IMMSolver.cpp:400-466, IMMCudaImpl.cu)
 * Build: gcc -O2 -fopenmp -ffp-contract=off -fPIC -shared (oracle/build.py).
 */
#include "vtp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NBR_NONE 0xffffffffu

/* PI as the reference spells it: const float PI = 3.14159265 (KernelFunctions.cuh:16). */
static const double kPi = (double)3.14159265f;

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------ grid */

static void cell_of(const float *p, const or_grid *g, int *c) {
    for (int a = 0; a < 3; ++a) {
        float t = (p[a] - g->lb[a]) / g->cell; /* IEEE single sub + div */
        c[a] = (int)floorf(t);
    }
}

static int cell_available(const int *c, const or_grid *g) {
    return c[0] >= 0 && c[1] >= 0 && c[2] >= 0 && c[0] <= g->dims[0] && c[1] <= g->dims[1] && c[2] <= g->dims[2];
}

static uint32_t cell_key(const int *c, const or_grid *g) {
    return (uint32_t)c[2] * (uint32_t)(g->dims[1] * g->dims[0]) + (uint32_t)c[1] * (uint32_t)g->dims[0] +
           (uint32_t)c[0];
}

static float dist2_f32(const float *a, const float *b) {
    float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

uint32_t or_neighbors(uint32_t n, const float *pos, const or_grid *g, uint32_t *counts, uint32_t *nbrs,
                      uint32_t *sorted_ids, uint32_t *keys_out) {
    const uint64_t nkey = (uint64_t)g->dims[2] * g->dims[1] * g->dims[0] + (uint64_t)g->dims[1] * g->dims[0] +
                          (uint64_t)g->dims[0] + 1;
    uint32_t *key = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *start = (uint32_t *)calloc(nkey + 1, sizeof(uint32_t));
    uint32_t *order = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t alive = 0;
    for (uint32_t i = 0; i < n; ++i) {
        int c[3];
        cell_of(pos + 3 * (size_t)i, g, c);
        if (cell_available(c, g)) {
            key[i] = cell_key(c, g);
            start[key[i] + 1]++;
            ++alive;
        } else {
            key[i] = NBR_NONE;
        }
    }
    for (uint64_t k = 0; k < nkey; ++k) start[k + 1] += start[k];
    {
        uint32_t *fill = (uint32_t *)malloc(sizeof(uint32_t) * nkey);
        memcpy(fill, start, sizeof(uint32_t) * nkey);
        for (uint32_t i = 0; i < n; ++i) /* ascending id: stable */
            if (key[i] != NBR_NONE) order[fill[key[i]]++] = i;
        free(fill);
    }
    if (sorted_ids)
        for (uint32_t k = 0; k < alive; ++k) sorted_ids[k] = order[k];
    if (keys_out)
        for (uint32_t k = 0; k < alive; ++k) keys_out[k] = key[order[k]];
    const uint32_t M = g->maxnbr;
    const float cell = g->cell;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        uint32_t *lst = nbrs + (size_t)i * M;
        for (uint32_t t = 0; t < M; ++t) lst[t] = NBR_NONE;
        if (key[i] == NBR_NONE) {
            counts[i] = 0;
            continue;
        }
        uint32_t cnt = 1;
        lst[0] = i;
        int c[3];
        cell_of(pos + 3 * (size_t)i, g, c);
        for (int t = 0; t < 27; ++t) {
            int cc[3] = {c[0] + t / 9 - 1, c[1] + (t / 3) % 3 - 1, c[2] + t % 3 - 1};
            if (!cell_available(cc, g)) continue;
            uint32_t k = cell_key(cc, g);
            for (uint32_t s = start[k]; s < start[k + 1]; ++s) {
                uint32_t j = order[s];
                if (j == i) continue;
                float d2 = dist2_f32(pos + 3 * (size_t)i, pos + 3 * (size_t)j);
                float r = sqrtf(d2);
                if (r > 0.f && r <= cell) {
                    if (cnt < M) lst[cnt++] = j;
                }
            }
        }
        counts[i] = cnt;
    }
    free(key);
    free(start);
    free(order);
    return alive;
}

/* ------------------------------------------------------------------ kernels (FP64) */

typedef struct {
    double h, sigma;
} cubic_t;

static cubic_t cubic_make(double h) {
    cubic_t k;
    k.h = h;
    k.sigma = 8.0 / kPi / (h * h * h);
    return k;
}

static double cubic_w(const cubic_t *k, double r) {
    double q = r / k->h;
    if (q > 1.0) return 0.0;
    if (q <= 0.5) return k->sigma * (6.0 * q * q * q - 6.0 * q * q + 1.0);
    double t = 1.0 - q;
    return 2.0 * k->sigma * t * t * t;
}

/* gradient factor g with gradW = g * r_vec */
static double cubic_g(const cubic_t *k, double r) {
    double q = r / k->h;
    if (q < 1e-6 || q > 1.0) return 0.0;
    double f;
    if (q <= 0.5) f = 6.0 * (3.0 * q * q - 2.0 * q);
    else f = -6.0 * (1.0 - q) * (1.0 - q);
    return f * k->sigma / (r * k->h);
}

static double tension_c(double r, double h) {
    double cs = 32.0 / kPi / pow(h, 9.0);
    if (r * 2 > h && r <= h) return cs * pow(h - r, 3) * pow(r, 3);
    if (r > 0 && r * 2 <= h) return cs * (2 * pow(h - r, 3) * pow(r, 3) - pow(h, 6) / 64);
    return 0.0;
}

static void to_f32(uint32_t n, const double *p, float *f) {
    for (size_t i = 0; i < 3 * (size_t)n; ++i) f[i] = (float)p[i];
}

typedef struct {
    uint32_t *cnt, *nbr;
} lists_t;

static lists_t build_lists(uint32_t n, const double *pos, const or_grid *g) {
    lists_t L;
    float *pf = (float *)malloc(sizeof(float) * 3 * (n ? n : 1));
    to_f32(n, pos, pf);
    L.cnt = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    L.nbr = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1) * g->maxnbr);
    or_neighbors(n, pf, g, L.cnt, L.nbr, NULL, NULL);
    free(pf);
    return L;
}

static void free_lists(lists_t *L) {
    free(L->cnt);
    free(L->nbr);
}

#define FOR_NBR(L, g, i, j)                                                              \
    for (uint32_t t_ = 0, j = 0; t_ < (L).cnt[i] && ((j = (L).nbr[(size_t)(i) * (g)->maxnbr + t_]), 1); ++t_)

/* The entries of row i of lists in the layout of or_neighbors (self first). */
#define FOR_LIST(cnt, nbr, M, i, j) \
    for (uint32_t t_ = 0, j = 0; t_ < (cnt)[i] && ((j = (nbr)[(size_t)(i) * (M) + t_]), 1); ++t_)

static double rdiff(const double *pos, uint32_t i, uint32_t j, double *r) {
    r[0] = pos[3 * (size_t)i] - pos[3 * (size_t)j];
    r[1] = pos[3 * (size_t)i + 1] - pos[3 * (size_t)j + 1];
    r[2] = pos[3 * (size_t)i + 2] - pos[3 * (size_t)j + 2];
    return sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

/* ------------------------------------------------------------------ PBF */

/* Standard-PBF kernels (Mueller et al. poly6 density, Desbrun spiky gradient). */
static double poly6_w(double h, double r) {
    if (r > h) return 0.0;
    double d = h * h - r * r;
    return 315.0 / (64.0 * kPi * pow(h, 9.0)) * d * d * d;
}
static double spiky_g(double h, double r) {   /* gradW = g * r_vec */
    if (r > h || r < 1e-6 * h) return 0.0;
    double d = h - r;
    return -45.0 / (kPi * pow(h, 6.0)) * d * d / r;
}
static double pbf_w(const or_pbf_params *p, const cubic_t *k, double r) {
    return p->form == 1 ? poly6_w(p->h, r) : cubic_w(k, r);
}
static double pbf_g(const or_pbf_params *p, const cubic_t *k, double r) {
    return p->form == 1 ? spiky_g(p->h, r) : cubic_g(k, r);
}

void or_pbf_init(uint32_t n, const int32_t *mat, const double *pos, double *mass, double *vol, const or_grid *g,
                 const or_pbf_params *p) {
    /* init_cuda + compute_rigid_particle_volume_cuda (PBFCudaImpl.cu:34-68). */
    lists_t L = build_lists(n, pos, g);
    cubic_t k = cubic_make(p->h);
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 1) continue;
        double delta = 0, r[3];
        FOR_NBR(L, g, i, j) {
            if (mat[j] == mat[i]) delta += pbf_w(p, &k, rdiff(pos, i, j, r));
        }
        vol[i] = 1.0 / delta;
        mass[i] = p->rho_b * vol[i];
    }
    free_lists(&L);
}

/* Constraint iterations + XSPH of one substep on the lists L (positions
 * already advanced by the external force). */
/* PBF substep stages over given lists (layout of or_neighbors).  pbf_core (the
 * monolithic step) runs them over every particle; a slab-decomposed run runs them
 * over one rank's particles and replaces the ghosts' lambda after or_pbf_lambda
 * and their positions and velocities after or_pbf_dx. */
void or_pbf_lambda(uint32_t n, const int32_t *mat, const double *pos, const double *mass, const uint32_t *cnt,
                   const uint32_t *nbr, uint32_t maxnbr, const or_pbf_params *p, double *rho, double *lam) {
    /* compute_sph_density_and_error_cuda + update_lamb_cuda (PBFCudaImpl.cu:70-122). */
    cubic_t k = cubic_make(p->h);
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) {
            lam[i] = 0.0;   /* boundary lambda never set: 0 */
            continue;
        }
        double d = 0, gs[3] = {0, 0, 0}, s2 = 0, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            double rl = rdiff(pos, i, j, r);
            d += mass[j] * pbf_w(p, &k, rl);
            double gg = pbf_g(p, &k, rl) * (p->form == 1 ? mass[j] : 1.0);
            for (int a = 0; a < 3; ++a) {
                double e = gg * r[a];
                gs[a] += e;
                s2 += (e / p->rho0) * (e / p->rho0);
            }
        }
        if (d < p->rho0) d = p->rho0;
        double C = d / p->rho0 - 1.0;
        for (int a = 0; a < 3; ++a) {
            gs[a] /= p->rho0;
            s2 += gs[a] * gs[a];
        }
        rho[i] = d;
        lam[i] = -C / (s2 + p->eps);
    }
}

void or_pbf_dx(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *mass, const double *lam,
               const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr, const or_pbf_params *p, double *dx) {
    /* compute_dx_cuda + apply_dx_cuda (PBFCudaImpl.cu:124-170): Jacobi, all dx first. */
    cubic_t k = cubic_make(p->h);
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double s[3] = {0, 0, 0}, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            double gg = pbf_g(p, &k, rdiff(pos, i, j, r));
            double lj = mat[j] == 0 ? lam[j] : 0.0;
            double c = p->form == 1 ? lam[i] * mass[j] + lj * mass[i] : lam[i] + lj;
            for (int a = 0; a < 3; ++a) s[a] += c * gg * r[a];
        }
        for (int a = 0; a < 3; ++a) dx[3 * (size_t)i + a] = s[a] / p->rho0;
    }
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int a = 0; a < 3; ++a) {
            pos[3 * (size_t)i + a] += dx[3 * (size_t)i + a];
            vel[3 * (size_t)i + a] += dx[3 * (size_t)i + a] / p->dt;
        }
    }
}

void or_pbf_xsph(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *vol, const uint32_t *cnt,
                 const uint32_t *nbr, uint32_t maxnbr, const or_pbf_params *p, double *dx) {
    /* XSPH_cuda + apply_dx_cuda (PBFCudaImpl.cu:172-194). */
    cubic_t k = cubic_make(p->h);
    const double dt = p->dt;
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double dv[3] = {0, 0, 0}, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            double w = pbf_w(p, &k, rdiff(pos, i, j, r));
            for (int a = 0; a < 3; ++a) dv[a] += p->xsph_k * vol[j] * (vel[3 * (size_t)j + a] - vel[3 * (size_t)i + a]) * w;
        }
        for (int a = 0; a < 3; ++a) dx[3 * (size_t)i + a] = dv[a] * dt;
    }
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int a = 0; a < 3; ++a) {
            pos[3 * (size_t)i + a] += dx[3 * (size_t)i + a];
            vel[3 * (size_t)i + a] += dx[3 * (size_t)i + a] / dt;
        }
    }
}

static void pbf_core(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *mass,
                     const double *vol, const lists_t *Lp, const or_grid *g, const or_pbf_params *p,
                     double *density_out, double *lambda_out) {
    const lists_t L = *Lp;
    const uint32_t M = g->maxnbr;
    double *lam = (double *)calloc(n ? n : 1, sizeof(double));
    double *rho = (double *)calloc(n ? n : 1, sizeof(double));
    double *dx = (double *)calloc(3 * (size_t)(n ? n : 1), sizeof(double));
    for (int it = 0; it < p->iterations; ++it) {
        or_pbf_lambda(n, mat, pos, mass, L.cnt, L.nbr, M, p, rho, lam);
        or_pbf_dx(n, mat, pos, vel, mass, lam, L.cnt, L.nbr, M, p, dx);
    }
    or_pbf_xsph(n, mat, pos, vel, vol, L.cnt, L.nbr, M, p, dx);
    if (density_out) memcpy(density_out, rho, sizeof(double) * n);
    if (lambda_out) memcpy(lambda_out, lam, sizeof(double) * n);
    free(lam);
    free(rho);
    free(dx);
}

static void pbf_apply_force(uint32_t n, const int32_t *mat, double *pos, double *vel, const or_pbf_params *p) {
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int a = 0; a < 3; ++a) {
            vel[3 * (size_t)i + a] += p->g[a] * p->dt;
            pos[3 * (size_t)i + a] += vel[3 * (size_t)i + a] * p->dt;
        }
    }
}

void or_pbf_apply_force(uint32_t n, const int32_t *mat, double *pos, double *vel, const or_pbf_params *p) {
    pbf_apply_force(n, mat, pos, vel, p);
}

void or_pbf_step(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *mass, const double *vol,
                 const or_grid *g, const or_pbf_params *p, double *density_out, double *lambda_out) {
    pbf_apply_force(n, mat, pos, vel, p);
    lists_t L = build_lists(n, pos, g);
    pbf_core(n, mat, pos, vel, mass, vol, &L, g, p, density_out, lambda_out);
    free_lists(&L);
}

void or_pbf_step_frozen(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *mass,
                        const double *vol, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                        const or_pbf_params *p) {
    or_grid g;
    memset(&g, 0, sizeof(g));
    g.maxnbr = maxnbr;
    lists_t L = {(uint32_t *)cnt, (uint32_t *)nbr};
    pbf_apply_force(n, mat, pos, vel, p);
    pbf_core(n, mat, pos, vel, mass, vol, &L, &g, p, NULL, NULL);
}

/* g'(r) / r for gradW = g(r) r_vec: d(g r_vec)/d r_vec = g I + hh r_vec r_vec^T. */
static double cubic_hh(const cubic_t *k, double r) {
    double q = r / k->h;
    if (q < 1e-6 || q > 1.0) return 0.0;
    double h4 = k->h * k->h * k->h * k->h;
    if (q <= 0.5) return 18.0 * k->sigma / (h4 * q);
    return 6.0 * k->sigma * (1.0 - q * q) / (h4 * q * q * q);
}

void or_pbf_step_adjoint(uint32_t n, const int32_t *mat, const double *pos_in, const double *vel_in,
                         const double *mass, const double *vol, const uint32_t *cnt, const uint32_t *nbr,
                         uint32_t maxnbr, const or_pbf_params *p, double *xbar, double *vbar, double *kbar) {
    or_grid gg;
    memset(&gg, 0, sizeof(gg));
    gg.maxnbr = maxnbr;
    const or_grid *g = &gg;
    lists_t L = {(uint32_t *)cnt, (uint32_t *)nbr};
    const int I = p->iterations;
    const double dt = p->dt, rho0 = p->rho0, c = p->xsph_k;
    cubic_t k = cubic_make(p->h);
    const size_t n3 = 3 * (size_t)(n ? n : 1);
    /* ---- forward recompute with tape: X[it] positions before iteration it (X[I] = after), LAM, RHO */
    double *X = (double *)malloc(sizeof(double) * n3 * (I + 1));
    double *LAM = (double *)calloc((size_t)(n ? n : 1) * (I ? I : 1), sizeof(double));
    double *RHO = (double *)calloc((size_t)(n ? n : 1) * (I ? I : 1), sizeof(double));
    double *S2 = (double *)calloc((size_t)(n ? n : 1) * (I ? I : 1), sizeof(double));
    double *GS = (double *)calloc(n3 * (I ? I : 1), sizeof(double));
    double *v = (double *)malloc(sizeof(double) * n3);
    memcpy(X, pos_in, sizeof(double) * 3 * n);
    memcpy(v, vel_in, sizeof(double) * 3 * n);
    pbf_apply_force(n, mat, X, v, p);
    for (int it = 0; it < I; ++it) {
        double *x = X + n3 * it, *xn = X + n3 * (it + 1);
        double *lam = LAM + (size_t)n * it;
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            if (mat[i] != 0) continue;
            double d = 0, gs[3] = {0, 0, 0}, s2 = 0, r[3];
            FOR_NBR(L, g, i, j) {
                double rl = rdiff(x, i, j, r);
                d += mass[j] * cubic_w(&k, rl);
                double q = cubic_g(&k, rl);
                for (int a = 0; a < 3; ++a) {
                    double e = q * r[a] / rho0;
                    gs[a] += e;
                    s2 += e * e;
                }
            }
            RHO[(size_t)n * it + i] = d;
            if (d < rho0) d = rho0;
            double C = d / rho0 - 1.0;
            for (int a = 0; a < 3; ++a) s2 += gs[a] * gs[a];
            for (int a = 0; a < 3; ++a) GS[n3 * it + 3 * (size_t)i + a] = gs[a];
            S2[(size_t)n * it + i] = s2;
            lam[i] = -C / (s2 + p->eps);
        }
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            for (int a = 0; a < 3; ++a) xn[3 * (size_t)i + a] = x[3 * (size_t)i + a];
            if (mat[i] != 0) continue;
            double s[3] = {0, 0, 0}, r[3];
            FOR_NBR(L, g, i, j) {
                double q = cubic_g(&k, rdiff(x, i, j, r));
                double lj = mat[j] == 0 ? lam[j] : 0.0;
                for (int a = 0; a < 3; ++a) s[a] += (lam[i] + lj) * q * r[a] / rho0;
            }
            for (int a = 0; a < 3; ++a) {
                xn[3 * (size_t)i + a] += s[a];
                v[3 * (size_t)i + a] += s[a] / dt;
            }
        }
    }
    /* ---- XSPH adjoint: a_i = c sum_j V_j (v_j - v_i) W_ij; x_out = x + a dt; v_out = v + a */
    const double *xI = X + n3 * I;
    double *ab = (double *)calloc(n3, sizeof(double));
    double *xb = (double *)calloc(n3, sizeof(double));
    double *vb = (double *)calloc(n3, sizeof(double));
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int a = 0; a < 3; ++a) ab[3 * (size_t)i + a] = xbar[3 * (size_t)i + a] * dt + vbar[3 * (size_t)i + a];
    }
    double ksum = 0.0;
#pragma omp parallel for reduction(+ : ksum)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double r[3], xo[3], vo[3];
        for (int a = 0; a < 3; ++a) {
            xo[a] = xbar[3 * (size_t)i + a];
            vo[a] = vbar[3 * (size_t)i + a];
        }
        const double *ai = ab + 3 * (size_t)i;
        FOR_NBR(L, g, i, j) {
            if (j == i) continue;
            double rl = rdiff(xI, i, j, r);
            double w = cubic_w(&k, rl), q = cubic_g(&k, rl);
            const int fj = mat[j] == 0;
            const double *aj = ab + 3 * (size_t)j;
            double dvdot_i = 0, dvdot_j = 0;
            for (int a = 0; a < 3; ++a) {
                double dv = v[3 * (size_t)j + a] - v[3 * (size_t)i + a];
                dvdot_i += dv * ai[a];
                dvdot_j += dv * (fj ? aj[a] : 0.0);
                vo[a] += -c * vol[j] * w * ai[a] + (fj ? c * vol[i] * w * aj[a] : 0.0);
            }
            for (int a = 0; a < 3; ++a) xo[a] += c * q * r[a] * (vol[j] * dvdot_i - (fj ? vol[i] * dvdot_j : 0.0));
            ksum += vol[j] * w * dvdot_i;
        }
        for (int a = 0; a < 3; ++a) {
            xb[3 * (size_t)i + a] = xo[a];
            vb[3 * (size_t)i + a] = vo[a];
        }
    }
    *kbar += ksum;
    /* ---- constraint iterations, last to first */
    double *db = (double *)calloc(n3, sizeof(double));  /* Delta-bar */
    double *sb = (double *)calloc(n ? n : 1, sizeof(double));  /* s2-bar */
    double *rb = (double *)calloc(n ? n : 1, sizeof(double));  /* rho-bar */
    double *xn = (double *)calloc(n3, sizeof(double));
    for (int it = I - 1; it >= 0; --it) {
        const double *x = X + n3 * it, *lam = LAM + (size_t)n * it, *GSi = GS + n3 * it;
        for (uint32_t i = 0; i < n; ++i) {
            if (mat[i] != 0) continue;
            for (int a = 0; a < 3; ++a) db[3 * (size_t)i + a] = xb[3 * (size_t)i + a] + vb[3 * (size_t)i + a] / dt;
        }
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            sb[i] = rb[i] = 0.0;
            if (mat[i] != 0) continue;
            double lb = 0, r[3];
            FOR_NBR(L, g, i, j) {
                if (j == i) continue;
                double q = cubic_g(&k, rdiff(x, i, j, r));
                const int fj = mat[j] == 0;
                for (int a = 0; a < 3; ++a)
                    lb += q * r[a] / rho0 * (db[3 * (size_t)i + a] - (fj ? db[3 * (size_t)j + a] : 0.0));
            }
            double den = S2[(size_t)n * it + i] + p->eps;
            double rho = RHO[(size_t)n * it + i];
            double Cb = -lb / den;
            sb[i] = -lb * lam[i] / den;
            rb[i] = rho < rho0 ? 0.0 : Cb / rho0;
        }
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            for (int a = 0; a < 3; ++a) xn[3 * (size_t)i + a] = xb[3 * (size_t)i + a];
            if (mat[i] != 0) continue;
            double r[3], acc[3] = {0, 0, 0};
            FOR_NBR(L, g, i, j) {
                if (j == i) continue;
                double rl = rdiff(x, i, j, r);
                double q = cubic_g(&k, rl), hh = cubic_hh(&k, rl);
                const int fj = mat[j] == 0;
                double lj = fj ? lam[j] : 0.0;
                double e[3], ebar[3], rdot = 0;
                for (int a = 0; a < 3; ++a) e[a] = q * r[a] / rho0;
                for (int a = 0; a < 3; ++a) {
                    double eij = (lam[i] + lj) * db[3 * (size_t)i + a] + 2.0 * sb[i] * (e[a] + GSi[3 * (size_t)i + a]);
                    double eji = fj ? (lam[i] + lj) * db[3 * (size_t)j + a] + 2.0 * sb[j] * (-e[a] + GSi[3 * (size_t)j + a])
                                    : 0.0;
                    ebar[a] = eij - eji;
                    rdot += r[a] * ebar[a];
                }
                double dens = mass[j] * rb[i] + (fj ? mass[i] * rb[j] : 0.0);
                for (int a = 0; a < 3; ++a)
                    acc[a] += q * r[a] * dens + (q * ebar[a] + hh * r[a] * rdot) / rho0;
            }
            for (int a = 0; a < 3; ++a) xn[3 * (size_t)i + a] += acc[a];
        }
        memcpy(xb, xn, sizeof(double) * 3 * n);
    }
    /* ---- external force: x0 = x + dt (v + g dt), v0 = v + g dt */
    for (uint32_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            if (mat[i] != 0) {
                xbar[3 * (size_t)i + a] = 0.0;
                vbar[3 * (size_t)i + a] = 0.0;
                continue;
            }
            xbar[3 * (size_t)i + a] = xb[3 * (size_t)i + a];
            vbar[3 * (size_t)i + a] = vb[3 * (size_t)i + a] + dt * xb[3 * (size_t)i + a];
        }
    }
    free(X); free(LAM); free(RHO); free(S2); free(GS); free(v);
    free(ab); free(xb); free(vb); free(db); free(sb); free(rb); free(xn);
}

/* ------------------------------------------------------------------ DFSPH */

void or_dfsph_init(uint32_t n, const int32_t *mat, const double *pos, double *vol, double *rest_density,
                   const or_grid *g, const or_dfsph_params *p) {
    /* compute_rigid_volume_cuda (DFSPHCudaImpl.cu:63-83). */
    lists_t L = build_lists(n, pos, g);
    cubic_t k = cubic_make(p->h);
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 1) continue;
        double delta = 0, r[3];
        FOR_NBR(L, g, i, j) {
            if (mat[j] == mat[i]) delta += cubic_w(&k, rdiff(pos, i, j, r));
        }
        vol[i] = 1.0 / delta;
        rest_density[i] = vol[i] * p->rho_b;
    }
    free_lists(&L);
}

/* DFSPH substep stages.  or_dfsph_step runs them over every particle; a
 * slab-decomposed run runs them over one rank's particles (owned fluid, ghost
 * fluid, a band of the boundary) and exchanges the ghosts' values between them.
 * Lists are in the layout of or_neighbors: cnt[n], nbr[n * maxnbr]. */

void or_dfsph_ratio_alpha(uint32_t n, const int32_t *mat, const double *pos, const double *vol, const double *mass,
                          const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr, double h, double *ratio,
                          double *alpha) {
    /* compute_compression_ratio_cuda + compute_df_beta_cuda (DFSPHCudaImpl.cu:85-140). */
    cubic_t k = cubic_make(h);
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double rt = 0, a1[3] = {0, 0, 0}, a2 = 1e-6, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            double rl = rdiff(pos, i, j, r);
            rt += vol[j] * cubic_w(&k, rl);
            double gg = cubic_g(&k, rl);
            for (int a = 0; a < 3; ++a) a1[a] += vol[j] * gg * r[a];
            if (mat[j] == 0) a2 += gg * gg * (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) * vol[j] * vol[j] / mass[j];
        }
        double al = (a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]) / mass[i] + a2;
        if (al < 1e-6) al = 1e-6;
        ratio[i] = rt;
        alpha[i] = al;
    }
}

void or_dfsph_solve_a(uint32_t n, const int32_t *mat, const double *pos, const double *vol, const double *ratio,
                      const double *alpha, const double *vadv, const uint32_t *cnt, const uint32_t *nbr,
                      uint32_t maxnbr, double h, double dt, double *delta, double *kappa) {
    /* compute_delta_compression_ratio_cuda + update_delta_compression_ratio_from_vel_adv_cuda
     * (DFSPHCudaImpl.cu:142-196): the clamped compression error; compute_kappa_{div,incomp}
     * (:355-367): kappa = delta / alpha / dt^2 / V (0 for boundary particles). */
    cubic_t k = cubic_make(h);
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) {
            delta[i] = 0.0;
            kappa[i] = 0.0;
            continue;
        }
        double d = ratio[i] - 1.0, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            double gg = cubic_g(&k, rdiff(pos, i, j, r));
            double dot = 0;
            for (int a = 0; a < 3; ++a) dot += gg * r[a] * (vadv[3 * (size_t)i + a] - vadv[3 * (size_t)j + a]);
            d += dot * vol[j] * dt;
        }
        if (d < 0) d = 0;
        delta[i] = d;
        kappa[i] = d / alpha[i] / (dt * dt) / vol[i];
    }
}

void or_dfsph_solve_b(uint32_t n, const int32_t *mat, const double *pos, const double *vol, const double *mass,
                      const double *kappa, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr, double h,
                      double dt, double *vadv) {
    /* vf_update_vel_adv_from_kappa_{div,incomp}_cuda (DFSPHCudaImpl.cu:198-220, :369-391). */
    cubic_t k = cubic_make(h);
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            double gg = cubic_g(&k, rdiff(pos, i, j, r));
            double s = dt * vol[i] * vol[j] / mass[i] * (kappa[i] + kappa[j]) * gg;
            for (int a = 0; a < 3; ++a) vadv[3 * (size_t)i + a] -= s * r[a];
        }
    }
}

void or_dfsph_pressure_apply(uint32_t n, const int32_t *mat, double *vel, double *vadv, double dt) {
    /* apply_pressure_acc (DFSPHCudaImpl.cu:505-521): acc = (v* - v)/dt; v += acc dt; v* = v. */
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int a = 0; a < 3; ++a) {
            size_t q = 3 * (size_t)i + a;
            vel[q] += (vadv[q] - vel[q]) / dt * dt;
            vadv[q] = vel[q];
        }
    }
}

void or_dfsph_forces(uint32_t n, const int32_t *mat, const double *pos, const double *vel, const double *mass,
                     const double *rest_density, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                     const or_dfsph_params *p, double *acc, double *nrm) {
    /* dfsph_gravity_vis_surface (DFSPHCudaImpl.cu:523-554): gravity plus explicit Laplacian
     * viscosity into acc, surface normals into nrm (both 0 for boundary particles). */
    cubic_t k = cubic_make(p->h);
    const double h2_001 = 0.001 * p->h * p->h;
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) {
            for (int a = 0; a < 3; ++a) acc[3 * (size_t)i + a] = nrm[3 * (size_t)i + a] = 0.0;
            continue;
        }
        double av[3] = {0, 0, 0}, nn[3] = {0, 0, 0}, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            if (mat[j] != mat[i]) continue;
            double rl = rdiff(pos, i, j, r);
            double gg = cubic_g(&k, rl);
            double vij[3], dot = 0;
            for (int a = 0; a < 3; ++a) {
                vij[a] = vel[3 * (size_t)i + a] - vel[3 * (size_t)j + a];
                dot += vij[a] * r[a];
            }
            double pi = p->vis * mass[j] / rest_density[j] * dot / (rl * rl + h2_001);
            for (int a = 0; a < 3; ++a) {
                av[a] += 10.0 * pi * gg * r[a];
                nn[a] += p->h * mass[j] / rest_density[j] * gg * r[a];
            }
        }
        for (int a = 0; a < 3; ++a) {
            acc[3 * (size_t)i + a] = p->g[a] + av[a];
            nrm[3 * (size_t)i + a] = nn[a];
        }
    }
}

void or_dfsph_tension(uint32_t n, const int32_t *mat, const double *pos, const double *mass,
                      const double *rest_density, const double *nrm, const uint32_t *cnt, const uint32_t *nbr,
                      uint32_t maxnbr, const or_dfsph_params *p, double *acc) {
    /* add_acc_surface_tension_cuda (DFSPHCudaImpl.cu:298-353): cohesion and curvature terms. */
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double at[3] = {0, 0, 0}, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            if (mat[j] != mat[i] || j == i) continue;
            double rl = rdiff(pos, i, j, r);
            double kk = 2 * rest_density[i] / (rest_density[i] + rest_density[j]);
            double cc = tension_c(rl, p->h);
            for (int a = 0; a < 3; ++a) {
                double a1 = -p->gamma * mass[i] * mass[j] * cc * r[a] / rl;
                double a2 = -p->gamma * mass[i] * (nrm[3 * (size_t)i + a] - nrm[3 * (size_t)j + a]);
                at[a] += kk * (a1 + a2);
            }
        }
        for (int a = 0; a < 3; ++a) acc[3 * (size_t)i + a] += at[a];
    }
}

void or_dfsph_accelerate(uint32_t n, const int32_t *mat, double *vel, double *vadv, const double *acc, double dt) {
    /* acc_2_vel (DFSPHCudaImpl.cu:222-296): v += acc dt; v* = v. */
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int a = 0; a < 3; ++a) {
            size_t q = 3 * (size_t)i + a;
            vel[q] += acc[q] * dt;
            vadv[q] = vel[q];
        }
    }
}

void or_dfsph_advance(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *vadv, double dt) {
    /* apply_pressure_acc + update_pos_cuda (DFSPHSolver.cpp:393-404). */
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int a = 0; a < 3; ++a) {
            size_t q = 3 * (size_t)i + a;
            vel[q] += (vadv[q] - vel[q]) / dt * dt;
            pos[q] += vel[q] * dt;
        }
    }
}

typedef struct {
    uint32_t n;
    const int32_t *mat, *obj, *obj_is_fluid;
    int32_t nobj;
    const double *pos, *vol, *mass, *ratio, *alpha;
    const lists_t *L;
    const or_grid *g;
    double h, dt;
} dfctx;

static int pressure_solve(const dfctx *c, double *vadv, double *kappa, double thr, int force, int max_iters,
                          double *residual_out) {
    const uint32_t n = c->n, M = c->g->maxnbr;
    double *delta = (double *)calloc(n ? n : 1, sizeof(double));
    double *osum = (double *)calloc(c->nobj > 0 ? c->nobj : 1, sizeof(double));
    double *ocnt = (double *)calloc(c->nobj > 0 ? c->nobj : 1, sizeof(double));
    for (uint32_t i = 0; i < n; ++i) ocnt[c->obj[i]] += 1.0;
    int iter = 0;
    double residual = 0;
    for (;;) {
        ++iter;
        or_dfsph_solve_a(n, c->mat, c->pos, c->vol, c->ratio, c->alpha, vadv, c->L->cnt, c->L->nbr, M, c->h, c->dt,
                         delta, kappa);
        /* vfsph_div / vfsph_incomp residual: mean over fluid objects of the object's mean
         * clamped error (cal_mean, DFSPHCudaImpl.cu:449-503). */
        for (int o = 0; o < c->nobj; ++o) osum[o] = 0;
        for (uint32_t i = 0; i < n; ++i)
            if (c->obj_is_fluid[c->obj[i]]) osum[c->obj[i]] += delta[i];
        double acc = 0;
        int nf = 0;
        for (int o = 0; o < c->nobj; ++o)
            if (c->obj_is_fluid[o]) {
                acc += osum[o] / ocnt[o];
                ++nf;
            }
        residual = nf ? acc / nf : 0.0;
        or_dfsph_solve_b(n, c->mat, c->pos, c->vol, c->mass, kappa, c->L->cnt, c->L->nbr, M, c->h, c->dt, vadv);
        if (force > 0) {
            if (iter >= force) break;
        } else if (residual < thr || iter > max_iters - 1) {
            break;
        }
    }
    free(delta);
    free(osum);
    free(ocnt);
    *residual_out = residual;
    return iter;
}

void or_dfsph_step(uint32_t n, const int32_t *mat, const int32_t *obj, int32_t nobj, const int32_t *obj_is_fluid,
                   double *pos, double *vel, const double *vol, const double *rest_density, const or_grid *g,
                   const or_dfsph_params *p, or_solve_out *out, double *ratio_out, double *alpha_out) {
    /* DFSPHSolver::tick (DFSPHSolver.cpp:339-406). */
    const double dt = p->dt;
    const uint32_t M = g->maxnbr;
    lists_t L = build_lists(n, pos, g);
    double *mass = (double *)calloc(n ? n : 1, sizeof(double));
    double *ratio = (double *)calloc(n ? n : 1, sizeof(double));
    double *alpha = (double *)calloc(n ? n : 1, sizeof(double));
    double *vadv = (double *)malloc(sizeof(double) * 3 * (n ? n : 1));
    double *kappa = (double *)calloc(n ? n : 1, sizeof(double));
    double *acc = (double *)calloc(3 * (size_t)(n ? n : 1), sizeof(double));
    double *nrm = (double *)calloc(3 * (size_t)(n ? n : 1), sizeof(double));
    for (uint32_t i = 0; i < n; ++i) mass[i] = mat[i] == 0 ? rest_density[i] * vol[i] : 0.0;
    memcpy(vadv, vel, sizeof(double) * 3 * n);
    or_dfsph_ratio_alpha(n, mat, pos, vol, mass, L.cnt, L.nbr, M, p->h, ratio, alpha);
    dfctx c = {n, mat, obj, obj_is_fluid, nobj, pos, vol, mass, ratio, alpha, &L, g, p->h, dt};
    out->crashed = 0;
    out->div_iters = pressure_solve(&c, vadv, kappa, p->div_thr, p->force_div, p->max_iters, &out->div_residual);
    if (p->force_div <= 0 && out->div_iters > p->max_iters - 1) out->crashed = 1;
    or_dfsph_pressure_apply(n, mat, vel, vadv, dt);
    or_dfsph_forces(n, mat, pos, vel, mass, rest_density, L.cnt, L.nbr, M, p, acc, nrm);
    if (p->gamma != 0.0) or_dfsph_tension(n, mat, pos, mass, rest_density, nrm, L.cnt, L.nbr, M, p, acc);
    or_dfsph_accelerate(n, mat, vel, vadv, acc, dt);
    out->inc_iters = pressure_solve(&c, vadv, kappa, p->inc_thr, p->force_inc, p->max_iters, &out->inc_residual);
    if (p->force_inc <= 0 && out->inc_iters > p->max_iters - 1) out->crashed = 1;
    or_dfsph_advance(n, mat, pos, vel, vadv, dt);
    if (ratio_out) memcpy(ratio_out, ratio, sizeof(double) * n);
    if (alpha_out) memcpy(alpha_out, alpha, sizeof(double) * n);
    free(mass);
    free(ratio);
    free(alpha);
    free(vadv);
    free(kappa);
    free(acc);
    free(nrm);
    free_lists(&L);
}

/* ------------------------------------------------------------------ DFSPH pressure solve as an operator */

void or_dfsph_solve_op(uint32_t n, const int32_t *mat, const double *pos, const double *vol,
                       const double *rest_density, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                       double h, double dt, int iters, double *vadv, double *vbar) {
    or_grid gg;
    memset(&gg, 0, sizeof(gg));
    gg.maxnbr = maxnbr;
    const or_grid *g = &gg;
    lists_t L = {(uint32_t *)cnt, (uint32_t *)nbr};
    cubic_t k = cubic_make(h);
    const size_t nn = n ? n : 1;
    double *mass = (double *)calloc(nn, sizeof(double));
    double *ratio = (double *)calloc(nn, sizeof(double));
    double *alpha = (double *)calloc(nn, sizeof(double));
    double *kappa = (double *)calloc(nn, sizeof(double));
    unsigned char *mask = (unsigned char *)calloc(nn * (iters > 0 ? iters : 1), 1);
    for (uint32_t i = 0; i < n; ++i) mass[i] = mat[i] == 0 ? rest_density[i] * vol[i] : 0.0;
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double rt = 0, a1[3] = {0, 0, 0}, a2 = 1e-6, r[3];
        FOR_NBR(L, g, i, j) {
            double rl = rdiff(pos, i, j, r);
            rt += vol[j] * cubic_w(&k, rl);
            double q = cubic_g(&k, rl);
            for (int a = 0; a < 3; ++a) a1[a] += vol[j] * q * r[a];
            if (mat[j] == 0) a2 += q * q * (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) * vol[j] * vol[j] / mass[j];
        }
        double al = (a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]) / mass[i] + a2;
        if (al < 1e-6) al = 1e-6;
        ratio[i] = rt;
        alpha[i] = al;
    }
    for (int it = 0; it < iters; ++it) {
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            kappa[i] = 0.0;
            if (mat[i] != 0) continue;
            double d = ratio[i] - 1.0, r[3];
            FOR_NBR(L, g, i, j) {
                double q = cubic_g(&k, rdiff(pos, i, j, r));
                double dot = 0;
                for (int a = 0; a < 3; ++a) dot += q * r[a] * (vadv[3 * (size_t)i + a] - vadv[3 * (size_t)j + a]);
                d += dot * vol[j] * dt;
            }
            mask[(size_t)n * it + i] = d > 0;
            if (d < 0) d = 0;
            kappa[i] = d / alpha[i] / (dt * dt) / vol[i];
        }
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            if (mat[i] != 0) continue;
            double r[3];
            FOR_NBR(L, g, i, j) {
                double q = cubic_g(&k, rdiff(pos, i, j, r));
                double sc = dt * vol[i] * vol[j] / mass[i] * (kappa[i] + kappa[j]) * q;
                for (int a = 0; a < 3; ++a) vadv[3 * (size_t)i + a] -= sc * r[a];
            }
        }
    }
    if (vbar) {
        /* v' = v - B kappa(v), kappa = P mask (c + A v): vbar_in = vbar + A^T P mask (-B^T vbar) */
        double *kb = (double *)calloc(nn, sizeof(double));
        for (int it = iters - 1; it >= 0; --it) {
#pragma omp parallel for
            for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
                uint32_t i = (uint32_t)ii;
                kb[i] = 0.0;
                if (mat[i] != 0) continue;
                double s = 0, r[3];
                const double ci = dt * vol[i] / mass[i];
                FOR_NBR(L, g, i, j) {
                    if (j == i) continue;
                    double q = cubic_g(&k, rdiff(pos, i, j, r));
                    double di = 0, dj = 0;
                    for (int a = 0; a < 3; ++a) {
                        di += r[a] * vbar[3 * (size_t)i + a];
                        dj += r[a] * vbar[3 * (size_t)j + a];
                    }
                    s -= q * vol[j] * ci * di;
                    if (mat[j] == 0) s += q * (dt * vol[j] / mass[j]) * vol[i] * dj;
                }
                kb[i] = mask[(size_t)n * it + i] ? s / alpha[i] / (dt * dt) / vol[i] : 0.0;
            }
#pragma omp parallel for
            for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
                uint32_t i = (uint32_t)ii;
                if (mat[i] != 0) continue;
                double r[3], acc[3] = {0, 0, 0};
                FOR_NBR(L, g, i, j) {
                    if (j == i) continue;
                    double q = cubic_g(&k, rdiff(pos, i, j, r));
                    double c = dt * q * (vol[j] * kb[i] + (mat[j] == 0 ? vol[i] * kb[j] : 0.0));
                    for (int a = 0; a < 3; ++a) acc[a] += c * r[a];
                }
                for (int a = 0; a < 3; ++a) vbar[3 * (size_t)i + a] += acc[a];
            }
        }
        for (uint32_t i = 0; i < n; ++i)
            if (mat[i] != 0) vbar[3 * (size_t)i] = vbar[3 * (size_t)i + 1] = vbar[3 * (size_t)i + 2] = 0.0;
        free(kb);
    }
    free(mass); free(ratio); free(alpha); free(kappa); free(mask);
}

/* ------------------------------------------------------------------ differentiable DFSPH substep */

/* One DFSPH substep (DFSPHSolver::tick, DFSPHSolver.cpp:339-406, surface tension off) over
 * frozen lists with exactly div_iters / inc_iters iterations of the two pressure solves.
 * With a tape, every quantity the adjoint reads is recorded: VS*[it] = v* entering iteration
 * it, KA*[it] = its kappa, VP = the velocity after the divergence solve, ALPHA, A1 (the
 * unclamped alpha's gradient sum). */
typedef struct {
    double *VSd, *KAd, *VSi, *KAi, *VP, *ALPHA, *A1;
} df_tape;

static void dfsph_frozen(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *vol,
                         const double *mass, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                         const or_dfsph_params *p, int div_iters, int inc_iters, df_tape *T) {
    const double dt = p->dt;
    const size_t nn = n ? n : 1, n3 = 3 * nn;
    cubic_t k = cubic_make(p->h);
    double *ratio = (double *)calloc(nn, sizeof(double));
    double *alpha = (double *)calloc(nn, sizeof(double));
    double *vadv = (double *)malloc(sizeof(double) * n3);
    double *kappa = (double *)calloc(nn, sizeof(double));
    double *delta = (double *)calloc(nn, sizeof(double));
    double *acc = (double *)calloc(n3, sizeof(double));
    double *nrm = (double *)calloc(n3, sizeof(double));
    double *rest = (double *)calloc(nn, sizeof(double));
    for (uint32_t i = 0; i < n; ++i) rest[i] = vol[i] > 0 ? mass[i] / vol[i] : 0.0;
    or_dfsph_ratio_alpha(n, mat, pos, vol, mass, cnt, nbr, maxnbr, p->h, ratio, alpha);
    if (T) {
        memcpy(T->ALPHA, alpha, sizeof(double) * n);
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            double a1[3] = {0, 0, 0}, r[3];
            if (mat[i] == 0) {
                FOR_LIST(cnt, nbr, maxnbr, i, j) {
                    double gg = cubic_g(&k, rdiff(pos, i, j, r));
                    for (int a = 0; a < 3; ++a) a1[a] += vol[j] * gg * r[a];
                }
            }
            for (int a = 0; a < 3; ++a) T->A1[3 * (size_t)i + a] = a1[a];
        }
    }
    memcpy(vadv, vel, sizeof(double) * 3 * n);
    for (int s = 0; s < 2; ++s) {
        const int iters = s == 0 ? div_iters : inc_iters;
        for (int it = 0; it < iters; ++it) {
            if (T) memcpy((s == 0 ? T->VSd : T->VSi) + n3 * it, vadv, sizeof(double) * 3 * n);
            or_dfsph_solve_a(n, mat, pos, vol, ratio, alpha, vadv, cnt, nbr, maxnbr, p->h, dt, delta, kappa);
            if (T) memcpy((s == 0 ? T->KAd : T->KAi) + nn * it, kappa, sizeof(double) * n);
            or_dfsph_solve_b(n, mat, pos, vol, mass, kappa, cnt, nbr, maxnbr, p->h, dt, vadv);
        }
        if (s == 0) {
            or_dfsph_pressure_apply(n, mat, vel, vadv, dt);
            if (T) memcpy(T->VP, vel, sizeof(double) * 3 * n);
            or_dfsph_forces(n, mat, pos, vel, mass, rest, cnt, nbr, maxnbr, p, acc, nrm);
            or_dfsph_accelerate(n, mat, vel, vadv, acc, dt);
        }
    }
    or_dfsph_advance(n, mat, pos, vel, vadv, dt);
    free(ratio); free(alpha); free(vadv); free(kappa); free(delta); free(acc); free(nrm); free(rest);
}

void or_dfsph_step_frozen(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *vol,
                          const double *mass, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                          const or_dfsph_params *p, int div_iters, int inc_iters) {
    dfsph_frozen(n, mat, pos, vel, vol, mass, cnt, nbr, maxnbr, p, div_iters, inc_iters, NULL);
}

/* Adjoint of one pressure-solve iteration v' = v - B(x) kappa, kappa_i = P_i max(0, ratio_i - 1
 * + (A(x) v)_i) (DFSPHCudaImpl.cu:142-220): vb (adjoint of v') becomes the adjoint of v; the
 * position adjoint and the adjoints of ratio and alpha are accumulated.  J_ij = g I + hh r r^T
 * is the Jacobian of gradW_ij = g r with respect to r = x_i - x_j. */
static void dfsph_iter_adjoint(uint32_t n, const int32_t *mat, const double *pos, const double *vol,
                               const double *mass, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                               const cubic_t *k, double dt, const double *alpha, const double *vs,
                               const double *kap, double *vb, double *xb, double *rb, double *ab, double *db) {
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        db[i] = 0.0;
        if (mat[i] != 0) continue;
        const double ci = dt * vol[i] / mass[i];
        double kb = 0, xa[3] = {0, 0, 0}, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            if (j == i) continue;
            const double rl = rdiff(pos, i, j, r);
            const double g = cubic_g(k, rl), hh = cubic_hh(k, rl);
            const int fj = mat[j] == 0;
            const double kj = fj ? kap[j] : 0.0;
            double w[3], rw = 0;   /* w = c_j V_i vb_j - c_i V_j vb_i */
            for (int a = 0; a < 3; ++a) {
                w[a] = (fj ? dt * vol[j] / mass[j] * vol[i] * vb[3 * (size_t)j + a] : 0.0) -
                       ci * vol[j] * vb[3 * (size_t)i + a];
                rw += r[a] * w[a];
            }
            kb += g * rw;
            const double kk = kap[i] + kj;
            for (int a = 0; a < 3; ++a) xa[a] += kk * (g * w[a] + hh * r[a] * rw);
        }
        for (int a = 0; a < 3; ++a) xb[3 * (size_t)i + a] += xa[a];
        const double P = 1.0 / (alpha[i] * dt * dt * vol[i]);
        db[i] = kap[i] > 0 ? kb * P : 0.0;
        ab[i] -= kb * kap[i] / alpha[i];
        rb[i] += db[i];
    }
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double va[3] = {0, 0, 0}, xa[3] = {0, 0, 0}, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            if (j == i) continue;
            const double rl = rdiff(pos, i, j, r);
            const double g = cubic_g(k, rl), hh = cubic_hh(k, rl);
            const double c = dt * (vol[j] * db[i] + (mat[j] == 0 ? vol[i] * db[j] : 0.0));
            double u[3], ru = 0;
            for (int a = 0; a < 3; ++a) {
                u[a] = vs[3 * (size_t)i + a] - vs[3 * (size_t)j + a];
                ru += r[a] * u[a];
            }
            for (int a = 0; a < 3; ++a) {
                va[a] += c * g * r[a];
                xa[a] += c * (g * u[a] + hh * r[a] * ru);
            }
        }
        for (int a = 0; a < 3; ++a) {
            vb[3 * (size_t)i + a] += va[a];
            xb[3 * (size_t)i + a] += xa[a];
        }
    }
}

void or_dfsph_step_adjoint(uint32_t n, const int32_t *mat, const double *pos_in, const double *vel_in,
                           const double *vol, const double *mass, const uint32_t *cnt, const uint32_t *nbr,
                           uint32_t maxnbr, const or_dfsph_params *p, int div_iters, int inc_iters, double *xbar,
                           double *vbar, double *visbar) {
    const double dt = p->dt;
    const size_t nn = n ? n : 1, n3 = 3 * nn;
    cubic_t k = cubic_make(p->h);
    df_tape T;
    T.VSd = (double *)malloc(sizeof(double) * n3 * (div_iters > 0 ? div_iters : 1));
    T.VSi = (double *)malloc(sizeof(double) * n3 * (inc_iters > 0 ? inc_iters : 1));
    T.KAd = (double *)malloc(sizeof(double) * nn * (div_iters > 0 ? div_iters : 1));
    T.KAi = (double *)malloc(sizeof(double) * nn * (inc_iters > 0 ? inc_iters : 1));
    T.VP = (double *)malloc(sizeof(double) * n3);
    T.ALPHA = (double *)malloc(sizeof(double) * nn);
    T.A1 = (double *)malloc(sizeof(double) * n3);
    double *x = (double *)malloc(sizeof(double) * n3);
    double *v = (double *)malloc(sizeof(double) * n3);
    memcpy(x, pos_in, sizeof(double) * 3 * n);
    memcpy(v, vel_in, sizeof(double) * 3 * n);
    dfsph_frozen(n, mat, x, v, vol, mass, cnt, nbr, maxnbr, p, div_iters, inc_iters, &T);
    const double *pos = pos_in;
    double *xb = (double *)calloc(n3, sizeof(double));
    double *vb = (double *)calloc(n3, sizeof(double));
    double *vb2 = (double *)calloc(n3, sizeof(double));
    double *rb = (double *)calloc(nn, sizeof(double));
    double *ab = (double *)calloc(nn, sizeof(double));
    double *db = (double *)calloc(nn, sizeof(double));
    double *a1b = (double *)calloc(n3, sizeof(double));
    /* position update: x' = x + dt v', v' = v* of the density solve */
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int a = 0; a < 3; ++a) {
            xb[3 * (size_t)i + a] = xbar[3 * (size_t)i + a];
            vb[3 * (size_t)i + a] = vbar[3 * (size_t)i + a] + dt * xbar[3 * (size_t)i + a];
        }
    }
    for (int it = inc_iters - 1; it >= 0; --it)
        dfsph_iter_adjoint(n, mat, pos, vol, mass, cnt, nbr, maxnbr, &k, dt, T.ALPHA, T.VSi + n3 * it,
                           T.KAi + nn * it, vb, xb, rb, ab, db);
    /* gravity + viscosity (dfsph_gravity_vis_surface, DFSPHCudaImpl.cu:523-554):
     * v' = vp + dt (g + sum_j C (u.r) phi r), u = vp_i - vp_j, phi = g/(|r|^2 + 0.001 h^2),
     * C = 10 nu m_j / rho_j (fluid neighbours only) */
    const double eps = 0.001 * p->h * p->h;
    double vsum = 0.0;
#pragma omp parallel for reduction(+ : vsum)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        for (int a = 0; a < 3; ++a) vb2[3 * (size_t)i + a] = vb[3 * (size_t)i + a];
        if (mat[i] != 0) continue;
        double va[3] = {0, 0, 0}, xa[3] = {0, 0, 0}, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            if (j == i || mat[j] != 0) continue;
            const double rl = rdiff(pos, i, j, r);
            const double d2 = rl * rl;
            const double g = cubic_g(&k, rl), hh = cubic_hh(&k, rl);
            const double C = 10.0 * p->vis * mass[j] / (mass[j] / vol[j]);
            const double phi = g / (d2 + eps);
            const double psi = hh / (d2 + eps) - 2.0 * g / ((d2 + eps) * (d2 + eps));
            double u[3], w[3], ru = 0, rw = 0, uw = 0;
            for (int a = 0; a < 3; ++a) {
                u[a] = T.VP[3 * (size_t)i + a] - T.VP[3 * (size_t)j + a];
                w[a] = vb[3 * (size_t)i + a] - vb[3 * (size_t)j + a];
                ru += r[a] * u[a];
                rw += r[a] * w[a];
            }
            for (int a = 0; a < 3; ++a) {
                va[a] += dt * C * phi * r[a] * rw;
                xa[a] += dt * C * (phi * u[a] * rw + ru * (phi * w[a] + psi * r[a] * rw));
                uw += vb[3 * (size_t)i + a] * r[a];
            }
            vsum += dt * 10.0 * mass[j] / (mass[j] / vol[j]) * ru * phi * uw;
        }
        for (int a = 0; a < 3; ++a) {
            vb2[3 * (size_t)i + a] += va[a];
            xb[3 * (size_t)i + a] += xa[a];
        }
    }
    if (visbar) *visbar += vsum;
    for (int it = div_iters - 1; it >= 0; --it)
        dfsph_iter_adjoint(n, mat, pos, vol, mass, cnt, nbr, maxnbr, &k, dt, T.ALPHA, T.VSd + n3 * it,
                           T.KAd + nn * it, vb2, xb, rb, ab, db);
    /* compression ratio and alpha (DFSPHCudaImpl.cu:85-140): ratio_i = sum_j V_j W_ij,
     * alpha_i = max(|a1_i|^2 / m_i + 1e-6 + sum_{fluid j} V_j^2 |gradW_ij|^2 / m_j, 1e-6),
     * a1_i = sum_j V_j gradW_ij */
    for (uint32_t i = 0; i < n; ++i) {
        const int live = mat[i] == 0 && T.ALPHA[i] > 1e-6;
        if (!live) ab[i] = 0.0;
        for (int a = 0; a < 3; ++a) a1b[3 * (size_t)i + a] = live ? ab[i] * 2.0 * T.A1[3 * (size_t)i + a] / mass[i] : 0.0;
    }
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double xa[3] = {0, 0, 0}, r[3];
        FOR_LIST(cnt, nbr, maxnbr, i, j) {
            if (j == i) continue;
            const double rl = rdiff(pos, i, j, r);
            const double g = cubic_g(&k, rl), hh = cubic_hh(&k, rl);
            const int fj = mat[j] == 0;
            const double cr = rb[i] * vol[j] + (fj ? rb[j] * vol[i] : 0.0);
            double w[3], rw = 0;
            for (int a = 0; a < 3; ++a) {
                w[a] = vol[j] * a1b[3 * (size_t)i + a] - (fj ? vol[i] * a1b[3 * (size_t)j + a] : 0.0);
                rw += r[a] * w[a];
            }
            const double c2 = fj ? 2.0 * g * (g + hh * rl * rl) *
                                       (ab[i] * vol[j] * vol[j] / mass[j] + ab[j] * vol[i] * vol[i] / mass[i])
                                 : 0.0;
            for (int a = 0; a < 3; ++a) xa[a] += (cr * g + c2) * r[a] + g * w[a] + hh * r[a] * rw;
        }
        for (int a = 0; a < 3; ++a) xb[3 * (size_t)i + a] += xa[a];
    }
    for (uint32_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            xbar[3 * (size_t)i + a] = mat[i] == 0 ? xb[3 * (size_t)i + a] : 0.0;
            vbar[3 * (size_t)i + a] = mat[i] == 0 ? vb2[3 * (size_t)i + a] : 0.0;
        }
    }
    free(T.VSd); free(T.VSi); free(T.KAd); free(T.KAi); free(T.VP); free(T.ALPHA); free(T.A1);
    free(x); free(v); free(xb); free(vb); free(vb2); free(rb); free(ab); free(db); free(a1b);
}

/* ------------------------------------------------------------------ IMM / IMM-CT */

#define V3(a, i) (&(a)[3 * (size_t)(i)])
#define VPH(i, k) (&vph[3 * ((size_t)(i) * P + (k))])
#define FR(i, k) (frac[(size_t)(i) * P + (k)])

void or_imm_init(uint32_t n, const int32_t *mat, const double *pos, double *vol, const or_grid *g,
                 const or_imm_params *p) {
    /* init_data_cuda (IMMCTCudaImpl.cu:52-81): V = fPart_rest_volume; compute_rigid_volume_cuda
     * (:108-127): boundary V = 1 / sum over same-material neighbours of W (self included). */
    lists_t L = build_lists(n, pos, g);
    cubic_t k = cubic_make(p->h);
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] == 0) {
            vol[i] = p->vol0;
            continue;
        }
        double delta = 0, r[3];
        FOR_NBR(L, g, i, j) {
            if (mat[j] == mat[i]) delta += cubic_w(&k, rdiff(pos, i, j, r));
        }
        vol[i] = 1.0 / delta;
    }
    free_lists(&L);
}

/* update_rest_density_and_mass_cuda (:83-106): rest density = sum_k alpha_k rho_k.  A boundary
 * particle's value (the reference's racy max over fluid neighbours) enters no fluid term. */
static void imm_rest_density(uint32_t n, int P, const double *frac, const or_imm_params *p, const double *vol,
                             double *rd, double *mass) {
    for (uint32_t i = 0; i < n; ++i) {
        double s = 0;
        for (int k = 0; k < P; ++k) s += FR(i, k) * p->rho[k];
        rd[i] = s;
        mass[i] = s * vol[i];
    }
}

/* update_vel_from_phase_vel_cuda (:405-424): v = sum_k alpha_k v_k (drift u_k = v_k - v). */
static void imm_mix_velocity(uint32_t n, const int32_t *mat, int P, const double *frac, const double *vph,
                             double *vel) {
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        double v[3] = {0, 0, 0};
        for (int k = 0; k < P; ++k)
            for (int a = 0; a < 3; ++a) v[a] += VPH(i, k)[a] * FR(i, k);
        for (int a = 0; a < 3; ++a) V3(vel, i)[a] = v[a];
    }
}

/* phase_acc_2_phase_vel_cuda (:392-403) then update_vel_from_phase_vel_cuda. */
static void imm_apply_phase_acc(uint32_t n, const int32_t *mat, int P, const double *frac, double *vph,
                                const double *acc, double dt, double *vel) {
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        for (int k = 0; k < P; ++k)
            for (int a = 0; a < 3; ++a) VPH(i, k)[a] += acc[3 * ((size_t)i * P + k) + a] * dt;
    }
    imm_mix_velocity(n, mat, P, frac, vph, vel);
}

/* A mixture acceleration a_i shared out to the phases with the factor Cd + (1 - Cd) rho_i / rho_k
 * (distribute_acc_pressure_2_phase_cuda :426-440, add_phase_pct_acc_cuda :772-778). */
static void imm_share(uint32_t i, int P, const double *a, double cd, double rd, const or_imm_params *p,
                      double *acc) {
    for (int k = 0; k < P; ++k) {
        double f = cd + (1.0 - cd) * (rd / p->rho[k]);
        for (int a3 = 0; a3 < 3; ++a3) acc[3 * ((size_t)i * P + k) + a3] = a[a3] * f;
    }
}

/* apply_pressure_acc (:919-937): acc = (v* - v) / dt distributed to the phases. */
static void imm_apply_pressure(uint32_t n, const int32_t *mat, int P, const double *frac, double *vph,
                               const double *vadv, const double *cd, const double *rd, const or_imm_params *p,
                               double *acc, double *vel) {
    for (uint32_t i = 0; i < n; ++i) {
        if (mat[i] != 0) continue;
        double a[3];
        for (int a3 = 0; a3 < 3; ++a3) a[a3] = (V3(vadv, i)[a3] - V3(vel, i)[a3]) / p->dt;
        imm_share(i, P, a, cd[i], rd[i], p, acc);
    }
    imm_apply_phase_acc(n, mat, P, frac, vph, acc, p->dt, vel);
}

/* One pass of update_phase_change_from_drift_cuda + update_phase_change_from_diffuse_cuda
 * (:541-614) over the unflagged fluid particles; flagged ones get no change. */
static void imm_phase_pass(uint32_t n, const int32_t *mat, int P, const double *pos, const double *vel,
                           const double *vph, const double *frac, const double *vol, const int32_t *flag,
                           const lists_t *L, const or_grid *g, const cubic_t *kc, const or_imm_params *p,
                           double *fin, double *fout) {
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        for (int k = 0; k < P; ++k) fin[(size_t)i * P + k] = fout[(size_t)i * P + k] = 0.0;
        if (flag[i]) continue;
        double r[3];
        FOR_NBR(*L, g, i, j) {   /* drift */
            if (j == i || mat[j] != mat[i] || flag[j]) continue;
            double gg = cubic_g(kc, rdiff(pos, i, j, r));
            for (int k = 0; k < P; ++k) {
                double d = 0;
                for (int a = 0; a < 3; ++a) {
                    double ui = VPH(i, k)[a] - V3(vel, i)[a], uj = VPH(j, k)[a] - V3(vel, j)[a];
                    d += (FR(i, k) * ui + FR(j, k) * uj) * gg * r[a];
                }
                double ch = -p->dt * vol[j] * d;
                if (ch < 0) fout[(size_t)i * P + k] += ch;
                else fin[(size_t)i * P + k] += ch;
            }
        }
        FOR_NBR(*L, g, i, j) {   /* diffusion */
            if (j == i || mat[j] != mat[i] || flag[j]) continue;
            double rl = rdiff(pos, i, j, r);
            double gg = cubic_g(kc, rl);
            double factor = gg * rl * rl / (rl * rl);   /* (gradW . x_ij) / |x_ij|^2 */
            for (int k = 0; k < P; ++k) {
                double ch = p->dt * p->Cf * (FR(i, k) - FR(j, k)) * vol[j] * factor;
                if (ch < 0) fout[(size_t)i * P + k] += ch;
                else fin[(size_t)i * P + k] += ch;
            }
        }
    }
}

void or_imm_step(uint32_t n, const int32_t *mat, const int32_t *obj, int32_t nobj, const int32_t *obj_is_fluid,
                 double *pos, double *vel, double *vph, double *frac, double *Q, double *cd, const double *vol,
                 const or_grid *g, const or_imm_params *p, or_imm_out *out) {
    const int P = p->P;
    const double dt = p->dt;
    const size_t nn = n ? n : 1;
    lists_t L = build_lists(n, pos, g);
    cubic_t kc = cubic_make(p->h);
    double *rd = (double *)calloc(nn, sizeof(double)), *mass = (double *)calloc(nn, sizeof(double));
    double *ratio = (double *)calloc(nn, sizeof(double)), *alpha = (double *)calloc(nn, sizeof(double));
    double *kappa = (double *)calloc(nn, sizeof(double));
    double *vadv = (double *)malloc(sizeof(double) * 3 * nn);
    double *acc = (double *)calloc(3 * nn * P, sizeof(double));
    double *nrm = (double *)calloc(3 * nn, sizeof(double));
    double *tau = (double *)calloc(9 * nn, sizeof(double));
    double *fin = (double *)calloc(nn * P, sizeof(double)), *fout = (double *)calloc(nn * P, sizeof(double));
    int32_t *flag = (int32_t *)calloc(nn, sizeof(int32_t));
    imm_rest_density(n, P, frac, p, vol, rd, mass);

    /* sph_precompute (:849-864): compression ratio, alpha (as DFSPH, m_j = rest density_j V_j),
     * and for IMM-CT update_Cd_cuda (:782-804). */
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double rt = 0, a1[3] = {0, 0, 0}, a2 = 1e-6, blk = 0, r[3];
        FOR_NBR(L, g, i, j) {
            double rl = rdiff(pos, i, j, r);
            double w = cubic_w(&kc, rl);
            rt += vol[j] * w;
            double gg = cubic_g(&kc, rl);
            for (int a = 0; a < 3; ++a) a1[a] += vol[j] * gg * r[a];
            if (mat[j] == 0) a2 += gg * gg * (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) * vol[j] * vol[j] / mass[j];
            if (p->ct && mat[j] == mat[i] && j != i) blk += vol[j] * FR(j, 1) * w;
        }
        double al = (a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]) / mass[i] + a2;
        ratio[i] = rt;
        alpha[i] = al < 1e-6 ? 1e-6 : al;
        cd[i] = p->ct ? p->Cd0 + (1.0 - p->Cd0) * blk : p->Cd0;
    }
    memcpy(vadv, vel, sizeof(double) * 3 * n);
    dfctx c = {n, mat, obj, obj_is_fluid, nobj, pos, vol, mass, ratio, alpha, &L, g, p->h, dt};
    out->crashed = 0;
    out->div_iters = pressure_solve(&c, vadv, kappa, p->div_thr, p->force_div, p->max_iters, &out->div_residual);
    if (p->force_div <= 0 && out->div_iters > p->max_iters - 1) out->crashed = 1;
    imm_apply_pressure(n, mat, P, frac, vph, vadv, cd, rd, p, acc, vel);

    /* immct_gravity_vis_surface (:939-964): gravity, phase viscosity (:297-330), surface normal
     * (:332-355) and surface tension (:357-390) on every phase. */
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double nn3[3] = {0, 0, 0}, r[3];
        for (int k = 0; k < P; ++k)
            for (int a = 0; a < 3; ++a) acc[3 * ((size_t)i * P + k) + a] = p->g[a];
        FOR_NBR(L, g, i, j) {
            if (mat[j] != mat[i]) continue;
            double rl = rdiff(pos, i, j, r);
            double gg = cubic_g(&kc, rl);
            for (int a = 0; a < 3; ++a) nn3[a] += p->h * mass[j] / rd[j] * gg * r[a];
            if (j == i) continue;
            for (int k = 0; k < P; ++k) {
                double d = 0;
                for (int a = 0; a < 3; ++a) {
                    double vkmj = VPH(i, k)[a] - V3(vel, j)[a], vij = V3(vel, i)[a] - V3(vel, j)[a];
                    d += (p->mu[k] * (1.0 - cd[i]) * vkmj + p->mu[k] * cd[i] * vij) * r[a];
                }
                for (int a = 0; a < 3; ++a) acc[3 * ((size_t)i * P + k) + a] += 10.0 * vol[j] * d * gg * r[a] / (rl * rl);
            }
        }
        for (int a = 0; a < 3; ++a) V3(nrm, i)[a] = nn3[a];
    }
#pragma omp parallel for
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        uint32_t i = (uint32_t)ii;
        if (mat[i] != 0) continue;
        double at[3] = {0, 0, 0}, r[3];
        FOR_NBR(L, g, i, j) {
            if (mat[j] != mat[i] || j == i) continue;
            double rl = rdiff(pos, i, j, r);
            double kk = 2 * rd[i] / (rd[i] + rd[j]);
            double cc = tension_c(rl, p->h);
            for (int a = 0; a < 3; ++a) {
                double a1 = -p->gamma * mass[i] * mass[j] * cc * r[a] / rl;
                double a2 = -p->gamma * mass[i] * (V3(nrm, i)[a] - V3(nrm, j)[a]);
                at[a] += kk * (a1 + a2);
            }
        }
        for (int k = 0; k < P; ++k)
            for (int a = 0; a < 3; ++a) acc[3 * ((size_t)i * P + k) + a] += at[a];
    }
    imm_apply_phase_acc(n, mat, P, frac, vph, acc, dt, vel);

    if (p->ct) {
        /* immct_pct (:966-995): velocity gradient (:687-714), rheological factors (:806-821),
         * conformation update (:716-744), stress divergence (:746-780). */
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            if (mat[i] != 0) continue;
            double G[9] = {0}, r[3];
            FOR_NBR(L, g, i, j) {
                if (mat[j] != 0) continue;
                double gg = cubic_g(&kc, rdiff(pos, i, j, r));
                double vj = mass[j] / rd[j];
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) G[3 * a + b] += vj * (V3(vel, j)[a] - V3(vel, i)[a]) * gg * r[b];
            }
            const double a1f = FR(i, 1);
            const double thin = p->thin0 * fmax(0.0, p->theta - a1f) / (p->theta + 1e-6);
            const double vinc = pow(1.0 - a1f, -1.2);
            double *q = &Q[9 * (size_t)i], dq[9];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double qg = 0, gq = 0, qiq = 0;
                    for (int m = 0; m < 3; ++m) {
                        qg += q[3 * a + m] * G[3 * m + b];          /* Q gradv */
                        gq += G[3 * m + a] * q[3 * m + b];          /* gradv^T Q */
                        qiq += (q[3 * a + m] - (a == m)) * q[3 * m + b];   /* (Q - I) Q */
                    }
                    dq[3 * a + b] = (qg + gq - (q[3 * a + b] - (a == b)) / p->relax - thin * qiq) * dt;
                }
            for (int m = 0; m < 9; ++m) q[m] += dq[m];
            double trD = G[0] + G[4] + G[8];   /* trace of D = (gradv + gradv^T) / 2 */
            double shear = sqrt(0.5 * trD * trD);
            double vis = fmin(p->vis_base * vinc, p->vis_max);
            vis = p->vis_base + (vis - p->vis_base) / (1.0 + pow(10.0 * shear, 5.0)) * fmin(1.0, a1f / (p->theta + 1e-6));
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) tau[9 * (size_t)i + 3 * a + b] = vis * (q[3 * a + b] - (a == b));
        }
#pragma omp parallel for
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            if (mat[i] != 0) continue;
            double a[3] = {0, 0, 0}, r[3];
            FOR_NBR(L, g, i, j) {
                if (mat[j] != 0) continue;
                double gg = cubic_g(&kc, rdiff(pos, i, j, r));
                for (int x = 0; x < 3; ++x)
                    for (int y = 0; y < 3; ++y)
                        a[x] += (tau[9 * (size_t)i + 3 * x + y] / (rd[i] * rd[i]) +
                                 tau[9 * (size_t)j + 3 * x + y] / (rd[j] * rd[j])) * gg * r[y];
            }
            for (int x = 0; x < 3; ++x) a[x] *= FR(i, 1) * rd[i];
            imm_share(i, P, a, cd[i], rd[i], p, acc);
        }
        imm_apply_phase_acc(n, mat, P, frac, vph, acc, dt, vel);
    }
    memcpy(vadv, vel, sizeof(double) * 3 * n);
    out->inc_iters = pressure_solve(&c, vadv, kappa, p->inc_thr, p->force_inc, p->max_iters, &out->inc_residual);
    if (p->force_inc <= 0 && out->inc_iters > p->max_iters - 1) out->crashed = 1;
    imm_apply_pressure(n, mat, P, frac, vph, vadv, cd, rd, p, acc, vel);
    for (uint32_t i = 0; i < n; ++i)   /* update_pos_cuda (:480-491) */
        if (mat[i] == 0)
            for (int a = 0; a < 3; ++a) V3(pos, i)[a] += V3(vel, i)[a] * dt;

    /* phase_transfer (:1065-1137): exchange with the lists of the substep's start and the new
     * positions; particles whose fractions would turn negative are flagged and the exchange is
     * recomputed without them until no particle is newly flagged (at most 100 passes). */
    imm_phase_pass(n, mat, P, pos, vel, vph, frac, vol, flag, &L, g, &kc, p, fin, fout);
    int iter = 1;
    out->retries = 0;
    for (;;) {
        int newly = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (mat[i] != 0 || flag[i]) continue;
            for (int k = 0; k < P; ++k)
                if (FR(i, k) + fout[(size_t)i * P + k] + fin[(size_t)i * P + k] < 0) {
                    flag[i] = 1;
                    ++newly;
                    break;
                }
        }
        if (newly == 0 || iter > 100) break;
        imm_phase_pass(n, mat, P, pos, vel, vph, frac, vol, flag, &L, g, &kc, p, fin, fout);
        ++iter;
        ++out->retries;
    }
    if (iter > 100) out->crashed = 1;
    for (uint32_t i = 0; i < n; ++i) {   /* update_phase_change, release_unused_drift_vel, release_negative */
        if (mat[i] != 0) continue;
        for (int k = 0; k < P; ++k) FR(i, k) += fout[(size_t)i * P + k] + fin[(size_t)i * P + k];
        if (flag[i])
            for (int k = 0; k < P; ++k)
                for (int a = 0; a < 3; ++a) VPH(i, k)[a] = V3(vel, i)[a];
    }
    /* regularize_vol_frac_cuda (:493-510) + rest density + mixture velocity, then
     * update_mass_and_vel (:1139-1152) does the three again. */
    for (int pass = 0; pass < 2; ++pass) {
        for (uint32_t i = 0; i < n; ++i) {
            if (mat[i] != 0) continue;
            double s = 0;
            for (int k = 0; k < P; ++k) s += FR(i, k);
            for (int k = 0; k < P; ++k) FR(i, k) /= s;
        }
        imm_rest_density(n, P, frac, p, vol, rd, mass);
        imm_mix_velocity(n, mat, P, frac, vph, vel);
    }
    free(rd); free(mass); free(ratio); free(alpha); free(kappa); free(vadv); free(acc); free(nrm); free(tau);
    free(fin); free(fout); free(flag);
    free_lists(&L);
}
