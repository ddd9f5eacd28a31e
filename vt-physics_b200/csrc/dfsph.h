// DFSPH pass launchers (dfsph.cu).
#pragma once

#include "internal.h"
#include "staged.h"
#include "halo.h"

namespace vtp {

// Device-side state of one pressure solve (divergence or density) of one scene.
struct SolveState {
    uint32_t iter;          // iterations done in the current solve
    uint32_t stopped;       // 1 once the current solve has stopped
    uint32_t last_iters;    // iterations of the previous completed solve
    uint32_t pad_;
    uint64_t total_iters;   // summed since the counters were cleared
    double residual;        // last FP64 residual
};

// State of the batched solve loop of one solve kind (all scenes of a solver
// iterate together; a scene that has stopped is skipped until all have).
struct LoopState {
    uint32_t done;          // solve_end blocks finished in the current iteration
    uint32_t active;        // scenes still iterating after the current iteration
    uint32_t running;       // 1 while any scene iterates (read by the host loop)
    uint32_t iters;         // loop iterations of the current solve
    uint64_t total;         // loop iterations since the counters were cleared
};

// Scene-offset tiles: tile t covers fluid rows [row0, row0 + rows) of one
// scene, so per-block residual partial sums never mix scenes and split each
// scene's rows exactly as a solver holding that scene alone would.
struct SceneTiles {
    uint32_t tile0, ntiles; // the scene's tiles
    uint32_t obj0, nobj;    // the scene's fluid objects (global slots)
};

struct DfsphArgs {
    uint32_t nf, nb;
    uint32_t ell_stride;
    Cubic k;
    float dt, inv_dt, inv_dt2;
    float rho0, rho_b, mass_f, vol_f;
    float vis_coef;         // (nu + nu) / 2 * m_f / rho0
    float h2_001;           // 0.001 h^2
    float gamma;            // surface tension coefficient
    float csigma, h6_64;    // tension spline constants
    const uint32_t *nbr, *ncnt;
    float4 *pos;            // w = volume
    float4 *vel, *vel_alt;
    float4 *vadv, *vadv_alt;
    float *ratio, *alpha, *kappa, *delta;
    float4 *acc_tmp, *normal;   // tension path only
    const uint32_t *orig;       // sorted row -> attach id
    const uint16_t *obj_of;     // attach id -> fluid object slot (multi-object scenes only)
    int nobj_max;               // most fluid objects in one scene (>= 1)
    double *partials;           // [tiles][nobj_max]
    const uint4 *tiles;         // {row0, rows, scene, 0}
    uint32_t ntiles;
    bool persistent;            // persistent grid over the tiles
    const SceneTiles *scene_tiles;  // [S]
    const SolveState *state;    // [S] states of the running solve (stopped scenes are skipped); null in
                                // solve_b: no scene has stopped (a one-scene loop ends when it stops)
    uint32_t *tile_ran;         // [tiles] or null: solve_a records whether it ran each tile and solve_b
                                // follows that record, not the stop flags, which the stop test of the
                                // same iteration may be writing beside solve_b
    Scenes sc;                  // per-scene gravity
    uint32_t *status;
    uint64_t *tick;             // substep counter, advanced by the finalize pass
    int unroll;                 // neighbours in flight per thread (1, 2, 4, 8)
    const float *rest_density;  // IMM / IMM-CT: per-row rest density (mass = rest_density * volume)
    // Packed gather rows of the pressure solve (filled by dfsph_solve_pack):
    float4 *pva;                // [2n] row j = {pos_j, v*_j} (32 B): one 256-bit load per pair in solve_a
    float4 *pk;                 // [n] {x, y, z, kappa_j} for fluid rows, {x, y, z, V_j} for boundary rows
    // Staged pressure solve (single scene, bricked order): one block per cell group gathers
    // its neighbours from a shared-memory copy of the group's neighbourhood through the slot
    // lists; the residual partials are then per group (ngroups + 1 entries, the last for the
    // rows outside the grid).
    int staged;
    Staging stg;
    const float *dtp;           // adaptive time step (CFL) on the device; null: the fixed dt above
    uint32_t *vmax_bits;        // adaptive step: the finalize pass folds max |v|^2 of the new velocities here
    const HaloPush *halo;       // peer-store halos (device struct; null: none)
    int halo_vadv, halo_vel;    // current buffer index of vadv / vel (the peers' parity equals ours)
};

struct SolveCtl {
    SolveState *state;          // [S]
    LoopState *loop;
    const double *inv_count;    // [fluid objects] 1 / object size
    const SceneTiles *scene_tiles;  // [S]
    int nscenes;
    int nobj_max;               // partials per tile
    float threshold;
    uint32_t force_iters;       // 0 = residual test
    const uint32_t *force_seq;  // optional per-substep [div, incomp] counts (device)
    uint32_t force_seq_len;     // substeps covered by force_seq
    const uint64_t *tick;       // device substep counter (advanced by dfsph_finalize)
    int which;                  // 0 divergence solve, 1 density solve
    uint32_t max_iters;         // reference: stop after iteration 101
    cudaGraphConditionalHandle cond;
    int use_cond;
};

void dfsph_rigid_volume(cudaStream_t st, const DfsphArgs &a, const uint32_t *bncnt, const uint32_t *bnbr,
                        float *rest_density_b);
void dfsph_ratio_alpha(cudaStream_t st, const DfsphArgs &a, int block);
void dfsph_solve_begin(cudaStream_t st, SolveState *s, LoopState *loop, int nscenes);
// Packs pva / pk for a pressure solve (after v* and positions are final for it).
void dfsph_solve_pack(cudaStream_t st, const DfsphArgs &a);
void dfsph_solve_a(cudaStream_t st, const DfsphArgs &a, int block);
void dfsph_solve_b(cudaStream_t st, const DfsphArgs &a, int block);
void dfsph_solve_end(cudaStream_t st, const SolveCtl &c, const double *partials, uint32_t *status);
// Packed rows {x, v after the pressure step} for the viscosity pass (after the
// divergence solve, before dfsph_viscosity / dfsph_vis_normal).
void dfsph_pressure_pack(cudaStream_t st, const DfsphArgs &a);
void dfsph_viscosity(cudaStream_t st, const DfsphArgs &a, int block);
// Adaptive time step: dt = min(dt_max, cfl * diameter / max |v_fluid|) (dt_max when at rest),
// written to *dtp and added to the FP32 simulated time *sim_time.  max |v|^2 comes from
// *vmax_bits, which the previous substep's finalize pass filled (and dfsph_cfl_refresh after
// initialize or a velocity write from the host); the step zeroes it for the next finalize.
void dfsph_cfl_step(cudaStream_t st, float cfl, float diameter, float dt_max, uint32_t *vmax_bits, float *dtp,
                    float *sim_time);
void dfsph_cfl_refresh(cudaStream_t st, const DfsphArgs &a, uint32_t *vmax_bits);
void dfsph_vis_normal(cudaStream_t st, const DfsphArgs &a, int block);
void dfsph_tension(cudaStream_t st, const DfsphArgs &a, int block);
void dfsph_finalize(cudaStream_t st, const DfsphArgs &a);
// Grid of the tile kernels: one block per tile, or (persistent) just enough
// blocks to fill the GPU, each looping over tiles.
unsigned dfsph_tile_grid(uint32_t ntiles, int block, bool persistent);

}  // namespace vtp
