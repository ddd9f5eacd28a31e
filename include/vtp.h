/*
 * vtp.h - C ABI of the B200 particle-fluid hot path (uniform-grid neighbour
 * search + PBF / DFSPH / IMM-CT solver steps).
 *
 * The entry points replace the reference's solver plugin interface, the
 * abstract class `VT_Physics::Solver` (Simulator/Runtime/Include/Framework/
 * Solver.hpp:27-62) and its factory `SolverManager::createSolver`
 * (Simulator/Runtime/Source/Manager/SolverManager.cpp:19-40).  Each function
 * below names the virtual it stands in for.  Plain pointers and sizes only;
 * configs travel as the reference's JSON text.
 *
 * Conventions
 *  - Every function returns a vtp_status (0 = VTP_OK) except destroy/strings.
 *  - Host pointers are borrowed for the duration of the call.
 *  - Per-particle fields are exchanged in ATTACH ORDER (the order in which
 *    objects were attached, then the object's own particle order), exactly
 *    as the reference stores them; internally particles are kept sorted by
 *    grid cell.
 *  - One handle must not be used from two host threads at once.  Each
 *    handle owns its own CUDA stream.
 */
#ifndef VTP_H
#define VTP_H

#include <stddef.h>
#include <stdint.h>

#if defined(VTP_BUILD)
#define VTP_API __attribute__((visibility("default")))
#else
#define VTP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum vtp_status {
    VTP_OK = 0,
    VTP_ERR_CONFIG = 1,      /* missing / invalid JSON key (reference: checkConfig() false) */
    VTP_ERR_CUDA = 2,        /* a CUDA call failed (reference: m_isCrashed after cudaGetLastError) */
    VTP_NOT_CONVERGED = 3,   /* a pressure solve exceeded 100 iterations (reference: "crash") */
    VTP_ERR_NAN = 4,         /* non-finite state detected */
    VTP_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    VTP_ERR_BOUNDS = 6,      /* size / index outside a documented limit */
    VTP_ERR_STATE = 7,       /* call out of order (e.g. tick before attach) */
    VTP_ERR_ARG = 8,         /* null pointer / wrong byte count */
    VTP_ERR_NOMEM = 9        /* device allocation failed */
} vtp_status;

/* Same numbering as the reference's eSolverType (Solver.hpp:17-22). */
typedef enum vtp_solver_type {
    VTP_SOLVER_PBF = 0,
    VTP_SOLVER_DFSPH = 1,
    VTP_SOLVER_IMM = 2,
    VTP_SOLVER_IMMCT = 3
} vtp_solver_type;

/* Per-particle fields for vtp_solver_get_field / vtp_solver_set_field. */
typedef enum vtp_field {
    VTP_FIELD_POS = 0,            /* float[3] */
    VTP_FIELD_VEL = 1,            /* float[3] */
    VTP_FIELD_COLOR = 2,          /* float[3] */
    VTP_FIELD_MAT = 3,            /* int32 */
    VTP_FIELD_MASS = 4,           /* float */
    VTP_FIELD_VOLUME = 5,         /* float */
    VTP_FIELD_DENSITY = 6,        /* float: PBF density_sph; DFSPH/IMM compression ratio */
    VTP_FIELD_LAMBDA = 7,         /* float: PBF lambda */
    VTP_FIELD_ALPHA = 8,          /* float: DFSPH/IMM df_alpha */
    VTP_FIELD_KAPPA = 9,          /* float: last pressure-solve kappa */
    VTP_FIELD_REST_DENSITY = 10,  /* float */
    VTP_FIELD_VOL_FRAC = 11,      /* float[P] (IMM / IMM-CT) */
    VTP_FIELD_PHASE_VEL = 12,     /* float[P][3] (IMM / IMM-CT) */
    VTP_FIELD_CONFORMATION = 13,  /* float[9] row-major Q (IMM-CT) */
    VTP_FIELD_VEL_GRAD = 14,      /* float[9] row-major (IMM-CT) */
    VTP_FIELD_STRESS = 15,        /* float[9] row-major viscoelastic stress (IMM-CT) */
    VTP_FIELD_CD = 16,            /* float: momentum-exchange coefficient (IMM-CT) */
    VTP_FIELD_DELTA = 17          /* float: last compression-ratio residual field */
} vtp_field;

/* Conservation and density-error sums of the fluid of one scene (or all),
 * FP64 on the device. */
typedef struct vtp_conservation {
    double fluid_mass;            /* sum of fluid masses (PBF m, DFSPH rho0 V, IMM rest density * V) */
    double momentum[3];           /* sum m v */
    double kinetic_energy;        /* sum m |v|^2 / 2 */
    double mean_density_error;    /* mean of rho / rho0 - 1 (PBF, its clamped density) or of the
                                     compression ratio - 1 (DFSPH, IMM) of the last substep */
    uint32_t fluid_particles;
    uint32_t phases;              /* IMM / IMM-CT: phases reported (at most 8); 0 otherwise */
    double phase_mass[8];         /* IMM / IMM-CT: sum V alpha_k rho_k per phase */
} vtp_conservation;

/* Statistics of the most recent vtp_solver_tick_n_steps call. */
typedef struct vtp_stats {
    uint64_t steps_done;          /* substeps completed since initialize */
    float sim_time;               /* accumulated like the reference: FP32 += dt */
    uint32_t last_div_iters;      /* DFSPH/IMM: iterations of the last divergence solve */
    uint32_t last_incomp_iters;   /* DFSPH/IMM: iterations of the last density solve */
    uint64_t total_div_iters;     /* summed over the last call */
    uint64_t total_incomp_iters;
    double last_div_residual;     /* FP64 mean clamped compression-ratio error */
    double last_incomp_residual;
    uint32_t neighbor_overflow;   /* particles whose list hit maxNeighborNum (last substep) */
    uint32_t dead_particles;      /* fluid particles outside the grid (last substep) */
    uint32_t phase_retries;       /* IMM-CT phase-transfer retries (last substep) */
    uint32_t status_bits;         /* device status word, bit (1<<vtp_status) per event */
    float last_dt;                /* time step of the last substep (the adaptive one with "cfl") */
} vtp_stats;

typedef struct vtp_solver vtp_solver;

/* Human-readable text for a vtp_status. */
VTP_API const char *vtp_status_string(int status);

/* Library build id, e.g. "vtp 0.1 sm_100a". */
VTP_API const char *vtp_version(void);

/* Last error message of this thread (empty string if none). */
VTP_API const char *vtp_last_error(void);

/* Replaces SolverManager::createSolver(eSolverType) (SolverManager.cpp:19-40);
 * the solver's CUDA stream is created on the current device. */
VTP_API int vtp_solver_create(int solver_type, vtp_solver **out);

/* Replaces Solver::setConfig(json) (PBFSolver.cpp:30-62, DFSPHSolver.cpp:30-64,
 * IMMCTSolver.cpp:31-99): `json_text` is the reference's solver config
 * (e.g. {"DFSPH":{"Required":{...},"Optional":{...}},"EXPORT":{...}}).  An
 * optional top-level "B200" object carries extensions:
 *   "forceDivIterations" / "forceIncompIterations": run exactly k solver
 *       iterations instead of testing the residual (parity runs);
 *   "deviceLoop": false drives the pressure-solve loops from the host;
 *   "useGraphs": false launches kernels one by one instead of a CUDA graph;
 *   "blockSize": threads per block of the neighbour passes (32..256);
 *   "unroll": neighbour-list entries in flight per thread (1, 2, 4, 8);
 *   "persistentTiles": true runs the pressure-solve passes as a persistent
 *       grid looping over the scene-offset tiles (default: one block per tile);
 *   "pbfFormulation": "reference" (default: the reference's PBF arithmetic,
 *       PBFCudaImpl.cu:70-194) or "standard" (poly6 density, spiky gradient,
 *       mass-weighted constraint gradients); "pbfEpsilon": the relaxation
 *       added to the lambda denominator (default 1e-6 / 100);
 *   "cfl": DFSPH, single scene: an adaptive time step per substep,
 *       dt = min(timeStep, cfl * 2 particleRadius / max |v_fluid|) (timeStep
 *       when the fluid is at rest), computed on the device; 0 (default) keeps
 *       the reference's fixed timeStep (DFSPHSolver.cpp:43-45);
 *   "cellOrder": "brick" (default) keeps rows in 4x4x4-cell bricks with
 *       Morton order inside (compact neighbourhoods for the gathers) or
 *       "linear" in the reference's linear cell order; lists, exported keys
 *       and sorted order are the reference's either way;
 *   "rowLanes": threads per row of the PBF neighbour passes (1 = the list
 *       walked in order by one thread, default; 4 or 8 = the row's entries
 *       split over lanes and their sums added by a shuffle butterfly, for
 *       small scenes);
 *   "listLanes": neighbour-list builder lanes per row (0 = by row count,
 *       default; 1 or 8); every setting writes the same lists;
 *   "cubicCube": "rounded" (default) takes the (1 - q)^3 of the cubic
 *       kernel's outer branch correctly rounded, at most one ulp from the
 *       reference's powf(1 - q, 3) (KernelFunctions.cuh:29); "powf" calls powf
 *       as the reference does, for bit-identical W at a higher cost;
 *   "phaseRetry": IMM / IMM-CT phase-transfer retries (IMMCTCudaImpl.cu:
 *       1065-1137): "nearFlagged" (default) recomputes only the particles
 *       that were just flagged negative or have such a fluid neighbour, the
 *       only ones whose changes a retry alters; "all" recomputes every
 *       particle as the reference does; both give the same results;
 *   "pdl": PBF: true (default) launches the substep's kernels, and those of
 *       the differentiable adjoint, with programmatic dependent launch (each
 *       starts as the previous one exits, results unchanged); false launches
 *       them plainly;
 *   "stageTimers": true records CUDA-event stage times. */
VTP_API int vtp_solver_set_config(vtp_solver *s, const char *json_text);

/* Replaces Solver::attachObject(Object*) (PBFSolver.cpp:169-221 and the
 * other solvers' attachObject): `pos` is the object's particle positions
 * (n x float[3], what Object::getObjectComponent()->getElements() returns);
 * `object_json` holds the two per-object configs the reference reads:
 *   {"name": "...",
 *    "ObjectComponentConfig": {"epmMaterial": 0|1, ...},
 *    "SolverObjectComponentConfig": {"solverType": k, "exportFlag": b,
 *        "velocityStart": [..], "colorStart": [..], "phaseFraction": [..]}}
 * `vel` may be NULL (velocityStart is used) or n x float[3] per-particle
 * initial velocities (an extension used by the differentiable scenes). */
VTP_API int vtp_solver_attach_object(vtp_solver *s, const float *pos, uint32_t n,
                             const float *vel, const char *object_json);

/* Scene batching (no counterpart in the reference, which runs one scene per
 * solver).  Adds scene k >= 1 to a PBF or DFSPH solver after set_config
 * (which defines scene 0) and before initialize.  `json_text` is a full
 * solver config; its domain (simSpaceLB / simSpaceSize) and gravity are the
 * new scene's own, every other parameter must equal scene 0's
 * (VTP_ERR_CONFIG otherwise).  Objects join a scene through the key
 * "scene": k at the top level of their object_json (default 0).  All scenes
 * advance together in the same kernel launches; each scene's results are
 * those a solver holding that scene alone produces (bit-identical, iteration
 * counts included).  set_config drops all added scenes. */
VTP_API int vtp_solver_add_scene(vtp_solver *s, const char *json_text, uint32_t *scene_index);

/* Statistics of one scene of the most recent tick_n_steps call (pressure-solve
 * iteration counts and residuals are per scene; the rest as get_stats). */
VTP_API int vtp_solver_get_scene_stats(vtp_solver *s, uint32_t scene, vtp_stats *out);

/* Replaces Solver::initialize() (PBFSolver.cpp:73-125, DFSPHSolver.cpp:75-137). */
VTP_API int vtp_solver_initialize(vtp_solver *s);

/* Replaces Solver::tickNsteps(n) (PBFSolver.cpp:148-167).  Runs n substeps
 * (initializing first if needed) and returns after they finished on the GPU. */
VTP_API int vtp_solver_tick_n_steps(vtp_solver *s, uint32_t n);

/* Replaces Solver::run() (PBFSolver.cpp:127-146): ticks until the FP32
 * simulated time reaches animationTime. */
VTP_API int vtp_solver_run(vtp_solver *s);

/* Replaces Solver::reset() (PBFSolver.cpp:233-236): back to the template config. */
VTP_API int vtp_solver_reset(vtp_solver *s);

/* Replaces Solver::destroy() (PBFSolver.cpp:238-246); frees the handle. */
VTP_API void vtp_solver_destroy(vtp_solver *s);

/* Copies the solver's config JSON (after defaults) into buf (NUL-terminated);
 * stands in for Solver::getSolverConfigTemplate() when called before set_config. */
VTP_API int vtp_solver_get_config(vtp_solver *s, char *buf, size_t buf_bytes, size_t *needed);

VTP_API int vtp_solver_get_stats(vtp_solver *s, vtp_stats *out);
VTP_API int vtp_solver_particle_counts(vtp_solver *s, uint32_t *n_total, uint32_t *n_fluid,
                               uint32_t *n_boundary, uint32_t *n_phases);

/* Field I/O in attach order.  `bytes` must equal n_total * element size. */
VTP_API int vtp_solver_get_field(vtp_solver *s, int field, void *host, size_t bytes);
VTP_API int vtp_solver_set_field(vtp_solver *s, int field, const void *host, size_t bytes);

/* Field I/O for the attach-order particle range [first, first + count), e.g. one
 * object (the reference's exportData reads per-object ranges the same way,
 * PBFSolver.cpp:262-273).  `bytes` = count * element size; set_field_range
 * takes pos / vel (boundary rows are static and keep their values). */
VTP_API int vtp_solver_get_field_range(vtp_solver *s, int field, uint32_t first, uint32_t count, void *host,
                                       size_t bytes);
VTP_API int vtp_solver_set_field_range(vtp_solver *s, int field, uint32_t first, uint32_t count, const void *host,
                                       size_t bytes);

/* Page-locked host memory for state I/O buffers (cudaHostAlloc): host <-> device
 * copies from it run at the full PCIe rate (measured on B200: 55 GB/s host to
 * device, against 29 GB/s from PyTorch's pinned-memory allocator). */
VTP_API int vtp_host_alloc(size_t bytes, void **ptr);
VTP_API void vtp_host_free(void *ptr);

/* Scene generation on the device, into caller-owned device memory: the
 * reference's particle generators (ModelHandler.cpp:43-67 lattice cube,
 * :124-154 hollow box), with the coordinates its host loops produce, bit for
 * bit (the cube's per-axis FP32 running sums, the box's lb + r + 2 r i in
 * double), as n x float[3] in the generators' order.  vtp_generate_cube can
 * add the SplitMix64 jitter the test scenes use: component c of particle p
 * draws u_(3p+c+1) from `seed` and moves by (2u - 1) * jitter_amp *
 * jitter_spacing (double, rounded once); jitter_amp = 0 means none.
 * *count receives the particle count even when it exceeds `capacity` (then
 * VTP_ERR_BOUNDS and nothing is written), so a first call with capacity 0
 * sizes the buffer.  Work is enqueued on `stream` (cudaStream_t; NULL =
 * default stream) and the call returns without waiting. */
VTP_API int vtp_generate_cube(float radius, const float lb[3], const float size[3], double jitter_amp,
                              double jitter_spacing, uint64_t seed, float *d_out, uint32_t capacity,
                              uint32_t *count, void *stream);
VTP_API int vtp_generate_box(float radius, const float lb[3], const float size[3], int32_t layers, float *d_out,
                             uint32_t capacity, uint32_t *count, void *stream);

/* Particle geometry on the host (no device work).
 *
 * vtp_generate_particles replaces ModelHandler::generateObjectElements
 * (Simulator/Library/Source/Model/ModelHandler.cpp:13-175): config_json is
 * the generator config an object component builds ("genType" 1 sphere
 * {particleRadius, volumeCenter, volumeRadius}, 2 cube {particleRadius, lb,
 * size}, 3 cylinder {particleRadius, center, bottomAreaRadius, height},
 * 4 plane {particleRadius, lb, size, layerNum}, 5 box {particleRadius, lb,
 * size, layerNum}); the positions are the reference's bit for bit, in its
 * order, as n x float[3] into `out` (host memory, `capacity` particles).
 * With out == NULL only *count is set.  Unknown genType: VTP_ERR_CONFIG.
 *
 * vtp_read_ply replaces ModelHandler::load_PLY_ParticleElements
 * (ModelHandler.cpp:207-228): every vertex of the PLY file at `path`
 * (ASCII or binary, float or double coordinates) is one particle, x y z in
 * file order.  With out == NULL only *count is set.
 *
 * vtp_write_ply replaces ExportUtil::exportAsPly (ExportUtil.cpp:28-88): the
 * ASCII PLY "x y z [r g b] [p1 .. pk]" with the default iostream float
 * format, written to dir + "/" + name + ".ply" (directories created; the
 * reference joins with a backslash).  color (n x 3) and phase (n x n_phase)
 * may be NULL. */
VTP_API int vtp_generate_particles(const char *config_json, float *out, uint64_t capacity, uint64_t *count);
VTP_API int vtp_read_ply(const char *path, float *out, uint64_t capacity, uint64_t *count);
VTP_API int vtp_write_ply(const char *dir, const char *name, const float *pos, uint64_t n, const float *color,
                          const float *phase, int32_t n_phase);

/* Trajectory statistics that long runs are compared by (no counterpart call in the
 * reference, which has no such diagnostics): the FP64 sums of
 * vtp_conservation over the fluid of scene `scene` (-1: every scene of the
 * solver), summed on the device in a fixed order, so repeated calls on the
 * same state agree bit for bit.  Synchronous. */
VTP_API int vtp_solver_get_conservation(vtp_solver *s, int scene, vtp_conservation *out);

/* Device self-test of the cubic kernel's outer branch: sph::cubic_value
 * (KernelFunctions.cuh:29) takes (1 - q)^3 by powf; the library takes it by a
 * correctly rounded compensated FP32 product unless the "B200" config key
 * "cubicCube" is "powf".  This compares the two bit for bit over every input
 * of that branch (t = 1 - q, q in (0.5, 1], i.e. t = k * 2^-24 for k in
 * [0, 2^23]) on the current device: *mismatches = inputs whose results
 * differ, *max_ulp = the largest difference in ulps. */
VTP_API int vtp_selftest_cube(uint32_t *mismatches, uint32_t *max_ulp);

/* Positions and velocities of the particle range [first, first + count)
 * together (pos and vel: count x float[3] host buffers each), one device pass
 * and one synchronisation per call: the state round trip of a host-side
 * driver loop. */
VTP_API int vtp_solver_get_state_range(vtp_solver *s, uint32_t first, uint32_t count, float *pos, float *vel);
VTP_API int vtp_solver_set_state_range(vtp_solver *s, uint32_t first, uint32_t count, const float *pos,
                                       const float *vel);

/* One host-driven frame in one call: set_state_range(first, count, pos_in,
 * vel_in), tickNsteps(n_steps), get_state_range(first, count, pos_out,
 * vel_out) (the reference's setter / Solver::tickNsteps / getter sequence,
 * Solver.hpp and PBFSolver.cpp:326-376), enqueued in stream order behind one
 * synchronisation.  The input buffers are read and the output buffers hold
 * the new state when it returns VTP_OK; on an error the outputs are
 * unspecified.  count = 0 only ticks. */
VTP_API int vtp_solver_step_state_range(vtp_solver *s, uint32_t first, uint32_t count, const float *pos_in,
                                        const float *vel_in, uint32_t n_steps, float *pos_out, float *vel_out);

/* The same frame for several attach-order ranges [firsts[k], firsts[k] + counts[k]),
 * ascending and disjoint (e.g. the fluid objects of a batched solver's scenes): the
 * host buffers hold the ranges' particles back to back (sum of counts x float[3]
 * each). */
VTP_API int vtp_solver_step_state_ranges(vtp_solver *s, uint32_t nranges, const uint32_t *firsts,
                                         const uint32_t *counts, const float *pos_in, const float *vel_in,
                                         uint32_t n_steps, float *pos_out, float *vel_out);

/* Neighbour lists in the reference's layout (UniformGridNeighborSearch.hpp:
 * 39-51): counts[n_total] (self included, 0 for particles outside the grid)
 * and nbrs[n_total * max_nbr] original indices, self first, UINT32_MAX padded. */
VTP_API int vtp_solver_get_neighbors(vtp_solver *s, uint32_t *counts, uint32_t *nbrs, uint32_t max_nbr);

/* Sorted order: sorted_ids[k] = attach-order index at sorted position k and
 * cell_ids[k] its linear cell id (z*gy*gx + y*gx + x), i.e. the reference's
 * particleIndices_cuData / cellIndices_cuData after sortByHashValue
 * (UGNSCudaImpl.cu:128-142). */
VTP_API int vtp_solver_get_sorted_order(vtp_solver *s, uint32_t *sorted_ids, uint32_t *cell_ids);

/* Device timing of the last tick_n_steps call, in milliseconds, per stage:
 * [0] neighbour search, [1] solver passes, [2] total.  Zero when timing
 * is disabled ("B200": {"stageTimers": false}). */
VTP_API int vtp_solver_get_stage_times(vtp_solver *s, float *ms3);

/* Per-kernel device time of vtp_solver_profile_kernels. */
typedef struct vtp_kernel_time {
    char name[32];
    float total_ms;       /* summed CUDA-event time of all launches */
    uint32_t launches;
} vtp_kernel_time;

/* Runs n substeps with direct launches (no graph) and a CUDA event pair
 * around every kernel on the solver's stream; writes one entry per kernel
 * name (at most cap) and their number to *count.  The substeps advance the
 * simulation like tick_n_steps. */
VTP_API int vtp_solver_profile_kernels(vtp_solver *s, uint32_t n, vtp_kernel_time *out, uint32_t cap,
                                       uint32_t *count);

/* Number of kernel launches (graph kernel nodes included) issued by the last
 * tick_n_steps call. */
VTP_API int vtp_solver_get_launch_count(vtp_solver *s, uint64_t *launches);

/* Differentiable rollouts (no counterpart in the reference; PBF or DFSPH
 * solver, one scene; DFSPH: fixed time step, surface tension 0).
 *
 * vtp_solver_diff_forward runs n_steps ordinary substeps from the current
 * state, saving the fluid state every `checkpoint_every` substeps (and at
 * the end).  With keep_lists != 0 every substep's neighbour lists are kept
 * for vtp_solver_diff_lists (finite-difference checks with frozen lists) and,
 * DFSPH, its pressure-solve iteration counts for vtp_solver_diff_iterations.
 *
 * vtp_solver_diff_backward takes dL/d(positions) and dL/d(velocities) of
 * the state after the recorded substeps (attach order, n_total x float[3];
 * NULL = zero) and returns dL/d(positions) and dL/d(velocities) of the state
 * before them and the derivative with respect to the solver's scalar
 * parameter (any output may be NULL): PBF dL/dXSPH_k, DFSPH
 * dL/dfPartRestViscosity.  Each checkpoint segment is recomputed with the
 * substep kernels into a tape (lists frozen per substep as the forward built
 * them; DFSPH: the pressure solves' iteration counts and clamp patterns too),
 * then the hand-written adjoint passes run in reverse.  The solver is left at
 * the forward's final state. */
VTP_API int vtp_solver_diff_forward(vtp_solver *s, uint32_t n_steps, uint32_t checkpoint_every, int keep_lists);
VTP_API int vtp_solver_diff_backward(vtp_solver *s, const float *dl_dpos, const float *dl_dvel, float *dl_dpos0,
                                     float *dl_dvel0, double *dl_dxsph_k);
/* Neighbour lists of recorded substep `step` in the layout of
 * vtp_solver_get_neighbors (PBF: built after the substep's external force;
 * DFSPH: built from the substep's starting positions). */
VTP_API int vtp_solver_diff_lists(vtp_solver *s, uint32_t step, uint32_t *counts, uint32_t *nbrs, uint32_t max_nbr);
/* DFSPH: divergence- and density-solve iteration counts of recorded substep
 * `step` (a rollout recorded with keep_lists). */
VTP_API int vtp_solver_diff_iterations(vtp_solver *s, uint32_t step, uint32_t *div_iters, uint32_t *inc_iters);

/* DFSPH pressure solve as a differentiable operator (no counterpart in the
 * reference; DFSPH solver, one scene).
 *
 * vtp_solver_dfsph_solve_forward runs one pressure solve (which = 0: the
 * divergence solve, 1: the density solve; DFSPHCudaImpl.cu:142-220) on the
 * solver's current positions: the neighbour search and compression-ratio /
 * alpha pass a substep starts with, then the solve loop on v* = v_in (attach
 * order, n_total x float[3], boundary rows ignored) until the residual test
 * stops it (or exactly force_iters iterations when > 0).  v_out (may be NULL)
 * receives v* after the solve, *iterations the iteration count.  The
 * solver's own state is left unchanged; the lists, the iteration count and
 * each iteration's clamp pattern (delta > 0) are kept.
 * vtp_solver_dfsph_solve_backward maps dL/d(v_out) to dL/d(v_in) through the
 * recorded solve (hand-written adjoint passes, two per iteration), valid
 * until the solver advances. */
VTP_API int vtp_solver_dfsph_solve_forward(vtp_solver *s, int which, const float *v_in, float *v_out,
                                           uint32_t force_iters, uint32_t *iterations);
VTP_API int vtp_solver_dfsph_solve_backward(vtp_solver *s, const float *vbar_out, float *vbar_in);

/* Allocation-free neighbour search (no counterpart in the reference).
 *
 * For callers that cannot call cudaMalloc when they need neighbour lists:
 * hosts that give this library a fixed memory budget managed by their own
 * allocator, and real-time loops that forbid allocation after start-up
 * (an allocation can block on the driver and fail under fragmentation at a
 * moment the caller cannot recover from).  Inputs and outputs are the
 * caller's device buffers: d_pos (n x float[3], any order), d_counts[n] and
 * d_nbrs[n * max_nbr] in the layout of vtp_solver_get_neighbors (self first,
 * then the 27 cells in the reference's order, ascending index inside a cell,
 * UINT32_MAX padded; count 0 for particles outside the grid).  The grid is
 * the reference's: cell size `cell`, lower corner lb, ceil(size / cell)
 * cells per axis.  All scratch lives in a fixed array inside the library
 * (VTP_NOALLOC_SCRATCH_BYTES on every GPU that loads it, held until exit),
 * which limits n to VTP_NOALLOC_MAX_PARTICLES and the grid to
 * VTP_NOALLOC_MAX_CELLS cell buckets; larger inputs return VTP_ERR_BOUNDS.
 * The work is enqueued on `stream` (a cudaStream_t; NULL = default stream)
 * and the call returns without waiting.  Every call looks up the array's
 * device address on the current device (a lookup, not an allocation), so a
 * device reset that reloads the library's device code is followed; the
 * first call on a device (and the first after a reset) also loads that code
 * and the array: make that first call before any stream capture.  Every
 * call on a device shares the array and it keeps the last call's contents,
 * so calls whose GPU work overlaps (other streams, unsynchronised threads)
 * race: order them on one stream. */
#define VTP_NOALLOC_MAX_PARTICLES 1048576u
#define VTP_NOALLOC_MAX_CELLS 2097152u
#define VTP_NOALLOC_SCRATCH_BYTES 50336512ull
VTP_API int vtp_ugns_neighbors_noalloc(const float *d_pos, uint32_t n, const float lb[3], const float size[3],
                                       float cell, uint32_t max_nbr, uint32_t *d_counts, uint32_t *d_nbrs,
                                       void *stream);

/* ---- Single-scene domain decomposition (no counterpart in the reference,
 * which runs a scene on one device, SolverManager.cpp:11-17).  One worker per
 * rank runs the DFSPH substep (DFSPHSolver.cpp:339-406) over the fluid rows
 * the rank owns, ghost copies of other ranks' fluid rows within the ghost
 * width of its slab, and a band of the scene's boundary; the host calls the
 * stages in order and replaces ghost values between them:
 *   load, prepare,
 *   per pressure solve (divergence, then density): solve_begin, then per
 *     iteration solve_a (+ kappa to ghosts, residual sums added over ranks),
 *     solve_b (+ v* to ghosts), the stop test on the summed residual;
 *   between the solves: forces, [normals to ghosts, tension], velocities to
 *     ghosts;
 *   finalize, read.
 * A PBF worker (PBFSolver::tick, PBFSolver.cpp:326-376) runs load, prepare
 * (the external force applied in the sort to owned and ghost rows alike),
 * then per constraint iteration pbf_lambda (+ lambda to ghosts) and pbf_dx
 * (+ positions and velocities to ghosts), then pbf_xsph and read.
 * Every row carries its scene-wide attach id, so an owned row's neighbour
 * list and arithmetic are those of a solver holding the whole scene.  Device
 * pointers throughout; the work is enqueued on the worker's stream (the
 * wrapped solver's, or the one set by vtp_domain_set_stream). */
typedef struct vtp_domain vtp_domain;
typedef enum vtp_domain_field {
    VTP_DOMAIN_KAPPA = 0,    /* float per row: kappa after solve_a */
    VTP_DOMAIN_VADV = 1,     /* float4 per row: v* after solve_b */
    VTP_DOMAIN_VEL = 2,      /* float4 per row: velocity after forces / tension */
    VTP_DOMAIN_NORMAL = 3,   /* float4 per row: surface normal after forces (tension on) */
    VTP_DOMAIN_LAMBDA = 4,   /* PBF, float per row: lambda after a lambda pass */
    VTP_DOMAIN_POSVEL = 5    /* PBF, 2 float4 per row {position, velocity}: after a correction pass */
} vtp_domain_field;
/* config_json: the scene's DFSPH or PBF config (a DFSPH "cfl" step is set per substep by
 * the host: vtp_domain_owned_vmax2 after load, the maximum over ranks, vtp_domain_set_dt).
 * fluid_pos: the worker's initial fluid rows (owned and ghost, host xyz,
 * ascending scene-wide id), used for the boundary volumes at create;
 * boundary_pos / boundary_ids: the boundary band (host, ids ascending);
 * boundary_first: 1 when the scene's boundary ids are all below its fluid ids
 * (0: all above); capacity: most owned + ghost rows a substep may load
 * (<= 2^24); n_objects: the scene's fluid objects (<= 16, residual means are
 * per object). */
VTP_API int vtp_domain_create(const char *config_json, const float *fluid_pos, uint32_t n_fluid,
                              const float *boundary_pos, const uint32_t *boundary_ids, uint32_t nb,
                              int boundary_first, uint32_t capacity, uint32_t n_objects, vtp_domain **out);
VTP_API void vtp_domain_destroy(vtp_domain *d);
/* stream: a cudaStream_t the stages are enqueued on from now on (cudaStreamLegacy for the
 * legacy default stream); NULL returns to the worker's own stream. */
VTP_API int vtp_domain_set_stream(vtp_domain *d, void *stream);
VTP_API int vtp_domain_capacity(vtp_domain *d, uint32_t *capacity, uint32_t *n_boundary);
/* Rows [0, n_own) are owned, [n_own, n_own + n_ghost) ghosts (load slots);
 * d_pos / d_vel float[3] per row, d_ids scene-wide ids, d_obj the fluid object
 * of each owned row (may be NULL: object 0). */
VTP_API int vtp_domain_load(vtp_domain *d, uint32_t n_own, uint32_t n_ghost, const float *d_pos,
                            const float *d_vel, const uint32_t *d_ids, const uint32_t *d_obj);
VTP_API int vtp_domain_prepare(vtp_domain *d);
/* DFSPH adaptive step: max |v|^2 of the owned rows (between load and prepare; waits), and the
 * step the stages use from now on (dt = min(timeStep, cfl 2r / sqrt(max over ranks)), as the
 * solver's own adaptive step forms it). */
VTP_API int vtp_domain_owned_vmax2(vtp_domain *d, float *out);
VTP_API int vtp_domain_set_dt(vtp_domain *d, float dt);
VTP_API int vtp_domain_solve_begin(vtp_domain *d, int which);
/* d_sums: double[n_objects], the owned rows' clamped compression errors summed per object. */
VTP_API int vtp_domain_solve_a(vtp_domain *d, double *d_sums);
VTP_API int vtp_domain_solve_b(vtp_domain *d);
VTP_API int vtp_domain_forces(vtp_domain *d);
VTP_API int vtp_domain_tension(vtp_domain *d);
VTP_API int vtp_domain_finalize(vtp_domain *d);
VTP_API int vtp_domain_pbf_lambda(vtp_domain *d);
VTP_API int vtp_domain_pbf_dx(vtp_domain *d);
VTP_API int vtp_domain_pbf_xsph(vtp_domain *d);
/* Gathers `field` of the rows at load slots d_slots[count] into d_out
 * (count values of the field's size); unpack writes count values into the ghost
 * rows at load slots [first_slot, first_slot + count). */
VTP_API int vtp_domain_pack(vtp_domain *d, int field, const uint32_t *d_slots, uint32_t count, float *d_out);
VTP_API int vtp_domain_unpack(vtp_domain *d, int field, uint32_t first_slot, uint32_t count, const float *d_in);
/* Peer-store halos: instead of pack / exchange / unpack, the stage kernels of the owner
 * write each value a ghost needs (DFSPH: kappa and its packed row in solve_a, v* and its
 * packed row in solve_b, velocities in forces / tension, normals in the normal pass; PBF:
 * lambda in pbf_lambda, the corrected position and velocity in pbf_dx) straight into the
 * ghost rows of the peer workers, whose buffers this worker maps: a
 * worker of the same process (vtp_domain_link_peer) or of another process through CUDA IPC
 * (vtp_domain_export_ipc on the peer, vtp_domain_link_peer_ipc here).  Ghost rows then skip
 * their own writes.  Per substep, after prepare: for each peer the owned load slots that
 * are its ghosts and their rows there (vtp_domain_rows on the peer) go to
 * vtp_domain_halo_targets.  The caller orders each peer's next stage after the stores (a
 * collective on the stream, or a barrier); both sides must have the same buffer parity
 * (vtp_domain_buffer_parity: v*, velocity, position), which the same stage sequence gives. */
#define VTP_DOMAIN_IPC_BUFFERS 8
typedef struct vtp_domain_ipc {
    unsigned char handle[VTP_DOMAIN_IPC_BUFFERS][64];   /* cudaIpcMemHandle_t of each buffer */
    uint32_t capacity;                                   /* the worker's fluid rows */
    uint32_t count;                                      /* handles used (DFSPH 8, PBF 5) */
    uint32_t solver_type;
} vtp_domain_ipc;
VTP_API int vtp_domain_export_ipc(vtp_domain *d, vtp_domain_ipc *out);
VTP_API int vtp_domain_link_peer(vtp_domain *d, int peer, vtp_domain *local_peer);
VTP_API int vtp_domain_link_peer_ipc(vtp_domain *d, int peer, const vtp_domain_ipc *h);
VTP_API int vtp_domain_set_halo(vtp_domain *d, int on);
VTP_API int vtp_domain_buffer_parity(vtp_domain *d, int32_t *out3);
VTP_API int vtp_domain_rows(vtp_domain *d, uint32_t first_slot, uint32_t count, uint32_t *d_rows);
VTP_API int vtp_domain_halo_targets(vtp_domain *d, int peer, const uint32_t *d_slots, const uint32_t *d_dst_rows,
                                    uint32_t count, uint32_t peer_capacity);
/* Owned rows' positions and velocities in load-slot order (float[3] each);
 * waits for the worker's stream and reports a device-side status. */
VTP_API int vtp_domain_read(vtp_domain *d, float *d_pos, float *d_vel);

#ifdef __cplusplus
}
#endif

#endif /* VTP_H */
