// The solver object behind the C ABI handle (shared by capi.cu and immct.cu).
#pragma once

#include <functional>
#include <memory>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

#include "../../include/vtp.h"
#include "dfsph.h"
#include "staged.h"
#include "internal.h"
#include "pbf.h"

namespace vtp {
struct ImmState;
int fail(int code, const std::string &msg);
extern thread_local std::string g_last_error;
}  // namespace vtp

template <class T>
struct DB {
    T *b[2] = {nullptr, nullptr};
    int cur = 0;
    T *c() const { return b[cur]; }
    T *n() const { return b[cur ^ 1]; }
    void swap() { cur ^= 1; }
};

struct ObjRec {
    std::string name;
    int mat = 0;
    uint32_t scene = 0;
    uint32_t start = 0, end = 0;
    bool export_flag = false;
    float vel0[3] = {0, 0, 0};
    float color[3] = {0, 0, 0};
    std::vector<float> phase;
};

// One scene of a solver: its own domain and gravity (everything else is shared).
struct SceneRec {
    float lb[3] = {0, 0, 0}, size[3] = {0, 0, 0};
    float3 gravity = make_float3(0.f, -9.8f, 0.f);
    // filled at initialize
    uint32_t nf = 0, nb = 0;       // fluid / boundary particles
    uint32_t fbase = 0, bbase = 0; // first fluid row, first boundary row (absolute)
    uint32_t attach_lo = 0;        // smallest attach id of the scene's particles
    vtp::SceneGrid grid{};
};

// Recording targets of one PBF substep in differentiable mode: the substep's
// lists are built into the tape and its intermediate states copied out.
struct PbfTapeSlot {
    uint32_t *orig = nullptr;            // [nf] sorted fluid row -> attach id
    uint32_t *nbr = nullptr, *ncnt = nullptr;
    std::vector<float4 *> x;             // [iterations + 1] positions (n rows; fluid rows recorded)
    std::vector<float *> lam, rho;       // [iterations] lambda, clamped density
    float4 *v = nullptr;                 // velocity before XSPH (n rows; fluid rows recorded)
};

namespace vtp {
struct DiffState;
struct DfDiffState;
}

struct vtp_solver {
    int type = 0;
    nlohmann::json cfg;
    bool configured = false;
    bool initialized = false;
    bool crashed = false;

    // attach-order host data
    std::vector<ObjRec> objs;
    std::vector<float> hpos, hvel, hcolor, hphase;
    std::vector<int> hmat;

    // parsed parameters (same derivations as the reference's setConfig)
    float dt = 0, inv_dt = 0, inv_dt2 = 0, radius = 0, h = 0, rho_f = 0, rho_b = 0, vol0 = 0;
    // DFSPH adaptive time step (extension "cfl"): dt = min(timeStep, cfl * 2r / max |v|) per
    // substep on the device; d_cfl = {dt, FP32 simulated time}, d_vmax = scratch word.
    double *d_cons = nullptr;       // conservation sums: totals + per-block partials
    uint32_t cons_blocks = 0;
    float cfl = 0.f;
    float last_dt = 0.f;         // step of the last substep (adaptive or fixed)
    float *d_cfl = nullptr;
    uint32_t *d_vmax = nullptr;
    float xsph_k = 0, viscosity = 0, div_thr = 0, incomp_thr = 0, gamma = 0, anim_time = 0;
    float lbx = 0, lby = 0, lbz = 0, sx = 0, sy = 0, sz = 0;
    float3 gravity = make_float3(0.f, -9.8f, 0.f);
    uint32_t maxnbr = 60;
    int iterations = 1;
    float sim_time = 0.f;

    // extensions ("B200" block)
    uint32_t force_div = 0, force_inc = 0;
    std::vector<uint32_t> force_seq;    // per-substep [div, incomp] iteration counts
    uint32_t *d_force_seq = nullptr;
    uint64_t *d_tick = nullptr;
    bool device_loop = true, use_graphs = true, stage_timers = false, stop_on_crash = true;
    int block = 128;
    int unroll = 4;
    bool persistent_tiles = false;
    bool cell_order_brick = true;   // bucket order: bricked (4^3 cells, Morton inside) or linear
    bool pdl = true;                // programmatic dependent launch between the substep's kernels
    int row_lanes = 1;        // threads per row of the PBF neighbour passes (1, 4, 8)
    int list_lanes = 0;       // neighbour-list builder lanes per row (0 = by row count)
    bool cell_cull = false;   // list builder skips neighbour cells beyond h (same lists)
    bool staged_solve = false;      // DFSPH pressure solve gathers from shared-memory cell-group copies
    uint32_t tape_budget_mb = 8192;  // differentiable PBF / DFSPH: device memory for resident segment tapes
    int adj_lanes = 1;              // differentiable PBF: lanes per row of the adjoint's neighbour passes
    int stage_rows = 2048;          // staged rows per brick at most
    bool cube_powf = false;   // cubic W outer branch: powf (reference rounding) or cube_rn
    bool phase_retry_all = false;   // IMM phase-transfer retries: every row, or rows near new flags
    int pbf_form = 0;                   // 0: the reference's PBF formulation, 1: standard PBF
    float pbf_eps = 1e-6f;

    // device state
    cudaStream_t st = nullptr, side = nullptr;
    cudaStream_t side2 = nullptr;       // second branch of the one-scene solve-loop body (the stop test)
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::vector<SceneRec> scenes;       // scene 0 comes from setConfig, the rest from add_scene
    vtp::SceneGrid *d_sg = nullptr;     // [S]
    uint16_t *row_scene = nullptr;      // [n]
    uint32_t nbuckets = 0;              // cell buckets of all scenes incl. their outside buckets
    float d2max = 0.f;
    uint4 *d_tiles = nullptr;           // scene-offset tiles of the fluid rows
    uint32_t *d_tile_ran = nullptr;     // batched solve-loop graph: tiles solve_a ran this iteration
    uint32_t ntiles = 0;
    vtp::SceneTiles *d_scene_tiles = nullptr;
    bool staged = false;                // staged solve in use (DFSPH, one scene, bricked order, merge mode 0 / 1)
    vtp::Staging stg{};
    vtp::SceneTiles *d_scene_groups = nullptr;   // residual partials of the staged solve: one per cell group
    int nobj_max = 1;
    vtp::LoopState *loop = nullptr;     // [2]: divergence, density
    vtp::Layout L{};
    vtp::Cubic kc{};
    DB<float4> pos, vel, vadv;
    DB<uint32_t> orig;
    float *vol = nullptr, *density = nullptr, *lambda = nullptr;
    float *ratio = nullptr, *alpha = nullptr, *kappa = nullptr, *delta = nullptr, *rest_b = nullptr;
    float4 *acc_tmp = nullptr, *normal = nullptr;
    float4 *pva = nullptr, *pk = nullptr;   // packed gather rows of the pressure solve
    double *partials = nullptr, *inv_count = nullptr;
    uint16_t *obj_of = nullptr;
    vtp::SolveState *solve = nullptr;   // [2][S]: divergence, density per scene
    vtp::UgnsBuffers u{};
    uint32_t *d_status = nullptr, *d_overflow = nullptr;
    uint32_t *h_pinned = nullptr;       // [8] status, overflow, iter, spare
    uint8_t *h_tick = nullptr;          // end-of-tick readback: status, overflow, CFL step, solve + loop states
    size_t h_tick_bytes = 0;
    std::shared_ptr<vtp::ImmState> imm;
    std::shared_ptr<vtp::DiffState> diff;
    std::shared_ptr<vtp::DfDiffState> dfdiff;   // differentiable DFSPH rollout

    // graphs: two parities (double-buffer swaps alternate between substeps)
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int gstate[2][4] = {{0}};
    int parity = 0;
    bool graphs_ready = false;
    uint64_t launches_per_tick = 0, last_launches = 0;

    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    vtp::Profiler *prof = nullptr;      // set only while vtp_solver_profile_kernels runs
    float *stage = nullptr;             // device staging buffer for field I/O
    size_t stage_bytes = 0;
    uint32_t *d_ranges = nullptr;       // {first, count, first slot} per range of a multi-range state frame
    uint32_t ranges_cap = 0;
    float stage_ms[3] = {0, 0, 0};

    uint64_t steps_done = 0;
    // PLY export (EXPORT block of the config)
    bool export_enabled = false;
    float export_gap = 0.f;
    uint32_t out_frames = 0, frames_written = 0;
    vtp_stats stats{};
    std::vector<vtp_stats> scene_stats;

    std::vector<void *> allocs;

    ~vtp_solver() { release(); }

    int ensure_stage(size_t bytes) {
        if (bytes <= stage_bytes) return 0;
        if (stage) cudaFree(stage), stage = nullptr, stage_bytes = 0;
        if (cudaMalloc((void **)&stage, bytes) != cudaSuccess) return vtp::fail(VTP_ERR_NOMEM, "staging buffer");
        stage_bytes = bytes;
        return 0;
    }

    int ensure_ranges(uint32_t nr) {
        if (nr <= ranges_cap) return 0;
        if (d_ranges) cudaFree(d_ranges), d_ranges = nullptr, ranges_cap = 0;
        if (cudaMalloc((void **)&d_ranges, 3 * (size_t)nr * sizeof(uint32_t)) != cudaSuccess)
            return vtp::fail(VTP_ERR_NOMEM, "range table");
        ranges_cap = nr;
        return 0;
    }

    void release() {
        for (int p = 0; p < 2; ++p)
            if (gexec[p]) cudaGraphExecDestroy(gexec[p]), gexec[p] = nullptr;
        for (void *a : allocs) cudaFree(a);
        allocs.clear();
        if (stage) cudaFree(stage), stage = nullptr, stage_bytes = 0;
        if (d_ranges) cudaFree(d_ranges), d_ranges = nullptr, ranges_cap = 0;
        if (d_cons) cudaFree(d_cons), d_cons = nullptr, cons_blocks = 0;
        if (h_pinned) cudaFreeHost(h_pinned), h_pinned = nullptr;
        if (h_tick) cudaFreeHost(h_tick), h_tick = nullptr, h_tick_bytes = 0;
        for (auto &e : ev)
            if (e) cudaEventDestroy(e), e = nullptr;
        if (st) cudaStreamDestroy(st), st = nullptr;
        if (side) cudaStreamDestroy(side), side = nullptr;
        if (side2) cudaStreamDestroy(side2), side2 = nullptr;
        if (ev_fork) cudaEventDestroy(ev_fork), ev_fork = nullptr;
        if (ev_join) cudaEventDestroy(ev_join), ev_join = nullptr;
        imm.reset();
        diff.reset();
        dfdiff.reset();
        graphs_ready = false;
        initialized = false;
    }

    template <class T>
    int alloc(T **p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
        if (e != cudaSuccess) return vtp::fail(VTP_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        allocs.push_back(*p);
        return VTP_OK;
    }

    int parse_config(const nlohmann::json &c);
    int add_scene(const nlohmann::json &c, uint32_t *index);
    int nscenes() const { return (int)scenes.size(); }
    vtp::Scenes scn() const { return vtp::Scenes{d_sg, row_scene, h, d2max, maxnbr}; }
    int attach(const float *p, uint32_t n, const float *v, const nlohmann::json &o);
    int initialize();
    // `tail` enqueues work after the substeps and before the end-of-tick readback, so that the
    // readback's single synchronisation covers it.
    int tick_n(uint32_t n, const std::function<int()> &tail = nullptr);
    int enqueue_tick(cudaStream_t s, bool capture);
    int enqueue_pbf_substep(cudaStream_t s, const PbfTapeSlot *tape);
    int enqueue_solve(cudaStream_t s, int which, bool capture);
    int build_graphs();
    int sort_boundary_and_lists();
    int get_field(int f, void *host, size_t bytes);
    int set_field(int f, const void *host, size_t bytes);
    vtp::PbfArgs pbf_args();
    vtp::DfsphArgs dfsph_args(int which = 0);
    vtp::SolveCtl solve_ctl(int which, cudaGraphConditionalHandle h, int use_cond);
    int check_status();
    int apply_status(uint32_t status_bits, uint32_t overflow);
    void fill_solve_stats(const vtp::SolveState *hs);
    int export_frame();
    int maybe_export();
    int conservation(int scene, vtp_conservation *out);   // conserve.cu
    int sync_parity();
};

