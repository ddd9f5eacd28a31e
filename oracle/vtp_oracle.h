/*
 * CPU oracle (test infrastructure only): an FP64 OpenMP restatement of the
 * reference's uniform-grid neighbour search and PBF / DFSPH / IMM / IMM-CT
 * substeps, used
 * by tests/ to check the sm_100a library and by bench.py as the timed CPU
 * baseline.  Product code never links or calls it.
 *
 * Arrays are in attach order (the reference's original particle order).
 * Neighbour search runs in FP32 exactly as UGNSCudaImpl.cu:28-203 does
 * (cell keys with IEEE division, membership sqrtf(d2) <= cell with d2 =
 * fmaf(dz,dz,fmaf(dy,dy,dx*dx))); the physics runs in FP64.
 */
#ifndef VTP_ORACLE_H
#define VTP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_grid {
    float lb[3];
    float cell;        /* gridCellSize = h */
    int32_t dims[3];   /* ceil(simSpaceSize / cell) */
    uint32_t maxnbr;
} or_grid;

typedef struct or_pbf_params {
    double dt, h, rho0, rho_b, xsph_k, eps;
    double g[3];
    int32_t iterations;
    /* 0: the reference's formulation (cubic W and gradient, constraint gradients
     *    without the particle mass, PBFCudaImpl.cu:70-144);
     * 1: standard PBF (poly6 density, spiky gradient, mass-weighted constraint
     *    gradients, Delta x_i = (1/rho0) sum_j (lambda_i m_j + lambda_j m_i) gradW). */
    int32_t form;
} or_pbf_params;

typedef struct or_dfsph_params {
    double dt, h, rho0, rho_b, vis, div_thr, inc_thr, gamma;
    double g[3];
    int32_t force_div, force_inc;   /* >0: fixed iteration counts */
    int32_t max_iters;              /* the reference stops after iteration 101 */
} or_dfsph_params;

typedef struct or_solve_out {
    int32_t div_iters, inc_iters;
    double div_residual, inc_residual;
    int32_t crashed;
} or_solve_out;

/* Neighbour lists in the reference layout: counts[n] (self included, 0 when
 * outside the grid), nbrs[n * maxnbr] attach ids, self first, UINT32_MAX
 * padded.  sorted_ids/keys (may be NULL) receive the stable (cell, id)
 * order of the particles inside the grid; returns how many are inside. */
uint32_t or_neighbors(uint32_t n, const float *pos, const or_grid *g, uint32_t *counts, uint32_t *nbrs,
                      uint32_t *sorted_ids, uint32_t *keys);

/* PBF: initialize boundary volume / mass (PBFCudaImpl.cu:34-68), then substeps
 * (PBFSolver.cpp:326-376).  pos/vel are FP64 xyz, mass/vol FP64 per particle,
 * mat 0 = fluid, 1 = boundary.  density/lambda (may be NULL) receive the last
 * constraint iteration's values. */
void or_pbf_init(uint32_t n, const int32_t *mat, const double *pos, double *mass, double *vol,
                 const or_grid *g, const or_pbf_params *p);
void or_pbf_step(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *mass,
                 const double *vol, const or_grid *g, const or_pbf_params *p, double *density, double *lambda);

/* The stages of a PBF substep over given lists (cnt[n], nbr[n * maxnbr] in the layout of
 * or_neighbors): the external force (before the lists are built), then per constraint
 * iteration or_pbf_lambda and or_pbf_dx (dx[3n] scratch; positions and velocities updated
 * in place), then or_pbf_xsph.  A slab-decomposed run replaces the ghosts' lambda between
 * lambda and dx, and their positions and velocities after dx. */
void or_pbf_apply_force(uint32_t n, const int32_t *mat, double *pos, double *vel, const or_pbf_params *p);
void or_pbf_lambda(uint32_t n, const int32_t *mat, const double *pos, const double *mass, const uint32_t *cnt,
                   const uint32_t *nbr, uint32_t maxnbr, const or_pbf_params *p, double *rho, double *lam);
void or_pbf_dx(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *mass, const double *lam,
               const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr, const or_pbf_params *p, double *dx);
void or_pbf_xsph(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *vol, const uint32_t *cnt,
                 const uint32_t *nbr, uint32_t maxnbr, const or_pbf_params *p, double *dx);

/* Differentiable PBF (no counterpart in the reference).  A substep with the
 * neighbour lists given (frozen: reference layout, attach ids, self first),
 * and its FP64 adjoint: from the pre-step state (pos, vel) and the same lists,
 * maps (xbar, vbar) = dL/d(post-step pos, vel) to dL/d(pre-step pos, vel) in
 * place (boundary rows 0) and adds dL/dXSPH_k to *kbar. */
void or_pbf_step_frozen(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *mass,
                        const double *vol, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                        const or_pbf_params *p);
void or_pbf_step_adjoint(uint32_t n, const int32_t *mat, const double *pos, const double *vel, const double *mass,
                         const double *vol, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                         const or_pbf_params *p, double *xbar, double *vbar, double *kbar);

/* DFSPH pressure solve as an operator (no counterpart in the reference): with
 * the lists given and exactly `iters` iterations of the solve loop
 * (DFSPHCudaImpl.cu:142-220), maps vadv (v*, in place) as the solve does, the
 * compression ratio and alpha computed from pos / vol first; with vbar
 * non-NULL it then maps vbar = dL/d(v* out) to dL/d(v* in) in place, each
 * iteration's clamp pattern (delta > 0) frozen.  mass = rest_density * vol. */
void or_dfsph_solve_op(uint32_t n, const int32_t *mat, const double *pos, const double *vol,
                       const double *rest_density, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                       double h, double dt, int iters, double *vadv, double *vbar);

/* Differentiable DFSPH substep (no counterpart in the reference): one substep
 * (DFSPHSolver.cpp:339-406, surface tension off) over frozen lists (cnt[n],
 * nbr[n * maxnbr], layout of or_neighbors) with exactly div_iters / inc_iters
 * pressure-solve iterations; mass = rest_density * vol for fluid particles.
 * or_dfsph_step_adjoint recomputes that substep from (pos, vel) and maps the
 * adjoint of its output state (xbar, vbar, in place) to the adjoint of its input
 * state, the clamp patterns of the forward held fixed; *visbar accumulates
 * dL/d(fPartRestViscosity). */
void or_dfsph_step_frozen(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *vol,
                          const double *mass, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                          const or_dfsph_params *p, int div_iters, int inc_iters);
void or_dfsph_step_adjoint(uint32_t n, const int32_t *mat, const double *pos, const double *vel, const double *vol,
                           const double *mass, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                           const or_dfsph_params *p, int div_iters, int inc_iters, double *xbar, double *vbar,
                           double *visbar);

/* DFSPH (DFSPHSolver.cpp:339-406): obj[n] gives each particle's object index
 * and obj_is_fluid/obj_count describe the objects (residual = mean over fluid
 * objects of the object's mean clamped compression error). */
void or_dfsph_init(uint32_t n, const int32_t *mat, const double *pos, double *vol, double *rest_density,
                   const or_grid *g, const or_dfsph_params *p);
void or_dfsph_step(uint32_t n, const int32_t *mat, const int32_t *obj, int32_t nobj, const int32_t *obj_is_fluid,
                   double *pos, double *vel, const double *vol, const double *rest_density, const or_grid *g,
                   const or_dfsph_params *p, or_solve_out *out, double *ratio, double *alpha);

/* The stages or_dfsph_step is made of, over given lists (cnt[n], nbr[n * maxnbr]
 * in the layout of or_neighbors).  A slab-decomposed run calls them on one
 * rank's particles and exchanges the ghosts' values in between: kappa after
 * solve_a, v* after solve_b, velocities after forces / tension and normals
 * between the two.  mass = rest_density * vol for fluid particles. */
void or_dfsph_ratio_alpha(uint32_t n, const int32_t *mat, const double *pos, const double *vol, const double *mass,
                          const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr, double h, double *ratio,
                          double *alpha);
void or_dfsph_solve_a(uint32_t n, const int32_t *mat, const double *pos, const double *vol, const double *ratio,
                      const double *alpha, const double *vadv, const uint32_t *cnt, const uint32_t *nbr,
                      uint32_t maxnbr, double h, double dt, double *delta, double *kappa);
void or_dfsph_solve_b(uint32_t n, const int32_t *mat, const double *pos, const double *vol, const double *mass,
                      const double *kappa, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr, double h,
                      double dt, double *vadv);
void or_dfsph_pressure_apply(uint32_t n, const int32_t *mat, double *vel, double *vadv, double dt);
void or_dfsph_forces(uint32_t n, const int32_t *mat, const double *pos, const double *vel, const double *mass,
                     const double *rest_density, const uint32_t *cnt, const uint32_t *nbr, uint32_t maxnbr,
                     const or_dfsph_params *p, double *acc, double *nrm);
void or_dfsph_tension(uint32_t n, const int32_t *mat, const double *pos, const double *mass,
                      const double *rest_density, const double *nrm, const uint32_t *cnt, const uint32_t *nbr,
                      uint32_t maxnbr, const or_dfsph_params *p, double *acc);
void or_dfsph_accelerate(uint32_t n, const int32_t *mat, double *vel, double *vadv, const double *acc, double dt);
void or_dfsph_advance(uint32_t n, const int32_t *mat, double *pos, double *vel, const double *vadv, double dt);

/* IMM / IMM-CT mixtures (IMMCTSolver.cpp:408-477 with IMMCTCudaImpl.cu:52-1152;
 * IMMSolver.cpp:400-466 with IMMCudaImpl.cu).  P phases; per particle:
 * frac[n*P] volume fractions, vph[n*P*3] phase velocities, Q[n*9] conformation
 * tensor (row-major, IMM-CT), cd[n] momentum-exchange coefficient (IMM-CT:
 * recomputed every substep from the blocking factor; IMM: p->Cd0 throughout).
 * vol from or_imm_init (fluid vol0, boundary 1 / sum of same-material W). */
#define OR_MAX_PHASES 8
typedef struct or_imm_params {
    double dt, h, vol0, gamma, Cf, Cd0;
    double g[3];
    int32_t P, ct;                          /* phases; 1 = IMM-CT, 0 = IMM */
    double rho[OR_MAX_PHASES], mu[OR_MAX_PHASES];
    double vis_base, vis_max;               /* IMM-CT, after init_data_cuda's x1000 */
    double relax, thin0, theta;             /* relaxationTime, shearThinningBasicFactor, rheologicalThreshold */
    double div_thr, inc_thr;
    int32_t force_div, force_inc, max_iters;
} or_imm_params;
typedef struct or_imm_out {
    int32_t div_iters, inc_iters;
    double div_residual, inc_residual;
    int32_t retries;                        /* phase-transfer passes after the first */
    int32_t crashed;
} or_imm_out;
void or_imm_init(uint32_t n, const int32_t *mat, const double *pos, double *vol, const or_grid *g,
                 const or_imm_params *p);
void or_imm_step(uint32_t n, const int32_t *mat, const int32_t *obj, int32_t nobj, const int32_t *obj_is_fluid,
                 double *pos, double *vel, double *vph, double *frac, double *Q, double *cd, const double *vol,
                 const or_grid *g, const or_imm_params *p, or_imm_out *out);

int or_num_threads(void);
void or_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
