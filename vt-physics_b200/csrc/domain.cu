// Single-scene domain decomposition: the worker one rank runs for its slab of
// a DFSPH or PBF scene (no counterpart in the reference, which runs a scene on
// one device: SolverManager.cpp:11-17).
//
// A rank holds the fluid particles it owns, copies ("ghosts") of the fluid
// particles other ranks own within the ghost width of its slab, and the
// boundary particles of a band around the slab.  Every substep the host
// loads owned and ghost rows, and the worker runs the DFSPH substep of
// DFSPHSolver::tick (DFSPHSolver.cpp:339-406) as separate stages with the
// library's own kernels; between the stages the host replaces the ghosts'
// values with their owners' (kappa after solve_a, v* after solve_b, the
// velocities after the viscosity / tension pass and the surface normals
// between the two) and adds the ranks' FP64 residual sums.  A PBF worker runs
// PBFSolver::tick (PBFSolver.cpp:326-376) the same way: the external force is
// applied in the sort to every loaded row (owned and ghost alike), and the host
// replaces the ghosts' lambda after each lambda pass and their positions and
// velocities after each position-correction pass.
//
// Rows carry their scene-wide attach ids, so the sort by (cell, attach id)
// and the lists of an owned row are those of a solver holding the whole
// scene: the per-row FP32 arithmetic of owned rows is the same, bit for bit,
// given the same pressure-solve iteration counts.
//
// Layout inside the wrapped solver: fluid rows [0, n_act) (owned and ghost,
// re-sorted every substep), rows [n_act, capacity) unused, boundary rows
// [capacity, capacity + nb) sorted once.  A neighbour index j < n_act is a
// fluid row and j >= capacity a boundary row, as the DFSPH kernels test
// (j < nf).  Load slots (the order the host loads rows in: owned first, then
// each peer's ghosts) travel through the sort so that the exchanges address
// rows by load slot.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

#include "../../include/vtp.h"
#include "dfsph.h"
#include "solver.h"

using json = nlohmann::json;
using vtp::fail;

namespace {

#define CU(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(VTP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
    } while (0)

constexpr uint32_t kMaxCapacity = 1u << 24;   // load slots travel as exact FP32 integers
constexpr uint32_t kMaxObjects = 16;          // fluid objects whose residual sums are kept apart
constexpr int kSumBlocks = 296;               // 2 x 148 SMs
constexpr int kSumThreads = 256;

inline unsigned nblk(uint32_t n, int b) { return (unsigned)((n + (uint32_t)b - 1) / (uint32_t)b); }

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum (result valid in thread 0).
__device__ double block_sum_d(double v) {
    __shared__ double sm[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum_d(v);
    __syncthreads();
    if (lane == 0) sm[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        s = lane < (int)(blockDim.x >> 5) ? sm[lane] : 0.0;
        s = warp_sum_d(s);
    }
    return s;
}

__global__ void k_dd_load(uint32_t n, const float *__restrict__ pos3, const float *__restrict__ vel3,
                          const uint32_t *__restrict__ ids, const uint32_t *__restrict__ obj, float w,
                          float4 *__restrict__ pos, float4 *__restrict__ vel, float4 *__restrict__ vadv,
                          uint32_t *__restrict__ orig, float *__restrict__ slot, float *__restrict__ objf) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    // w: the volume (DFSPH) or the mass (PBF) every fluid row carries
    pos[r] = make_float4(pos3[3 * (size_t)r], pos3[3 * (size_t)r + 1], pos3[3 * (size_t)r + 2], w);
    const float4 v = make_float4(vel3[3 * (size_t)r], vel3[3 * (size_t)r + 1], vel3[3 * (size_t)r + 2], 0.f);
    vel[r] = v;
    if (vadv) vadv[r] = v;   // DFSPH: v* = v at the start of the substep
    orig[r] = ids[r];
    slot[r] = (float)r;
    objf[r] = obj ? (float)obj[r] : 0.f;
}

// Boundary rows: local attach ids -> scene-wide ids (ascending with the local ones, so the
// rows stay sorted by (cell, id)), in both buffers.
__global__ void k_dd_band_ids(uint32_t nb, uint32_t row0, uint32_t local0, const uint32_t *__restrict__ gid,
                              uint32_t *orig_a, uint32_t *orig_b, uint32_t *status) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nb) return;
    const uint32_t local = orig_a[row0 + r] - local0;
    if (local >= nb) {
        atomicOr(status, vtp::ST_BOUNDS);
        return;
    }
    const uint32_t g = gid[local];
    orig_a[row0 + r] = g;
    orig_b[row0 + r] = g;
}

__global__ void k_dd_tiles(uint4 *tiles, uint32_t n, uint32_t block) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nt = (n + block - 1) / block;
    if (t >= nt) return;
    tiles[t] = make_uint4(t * block, min(block, n - t * block), 0u, 0u);
}

__global__ void k_dd_row_of_slot(uint32_t n, const float *__restrict__ slot, uint32_t *__restrict__ row_of_slot,
                                 uint32_t *status) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t s = (uint32_t)slot[r];
    if (s >= n) {
        atomicOr(status, vtp::ST_BOUNDS);
        return;
    }
    row_of_slot[s] = r;
}

// Per-object sums of the clamped compression error over the owned rows (load slots below
// n_own), in FP64: block partials in a fixed order, then one block adds them.  NOBJ bounds
// the objects at compile time so the accumulators stay in registers.
template <int NOBJ>
__global__ void __launch_bounds__(kSumThreads) k_dd_sums(uint32_t n, uint32_t n_own, const float *__restrict__ delta,
                                                         const float *__restrict__ slot,
                                                         const float *__restrict__ objf, int nobj,
                                                         double *__restrict__ part) {
    double acc[NOBJ];
#pragma unroll
    for (int o = 0; o < NOBJ; ++o) acc[o] = 0.0;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        if ((uint32_t)slot[r] >= n_own) continue;
        const double d = (double)delta[r];
        if (NOBJ == 1) {
            acc[0] += d;
        } else {
            const int o = (int)objf[r];
#pragma unroll
            for (int k = 0; k < NOBJ; ++k)
                if (k == o) acc[k] += d;
        }
    }
#pragma unroll
    for (int o = 0; o < NOBJ; ++o) {
        if (o >= nobj) break;   // block-uniform
        const double s = block_sum_d(acc[o]);
        if (threadIdx.x == 0) part[(size_t)blockIdx.x * nobj + o] = s;
    }
}

__global__ void __launch_bounds__(kSumThreads) k_dd_sums_final(int nblocks, int nobj, const double *__restrict__ part,
                                                               double *__restrict__ out) {
    for (int o = 0; o < nobj; ++o) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += part[(size_t)b * nobj + o];
        s = block_sum_d(s);
        if (threadIdx.x == 0) out[o] = s;
    }
}

__global__ void k_dd_ghost_flags(uint32_t n, uint32_t n_own, const float *__restrict__ slot, uint8_t *__restrict__ ghost) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    ghost[r] = (uint32_t)slot[r] >= n_own ? 1 : 0;
}

__device__ __forceinline__ bool slot_row(uint32_t s, uint32_t n, const uint32_t *row_of_slot, uint32_t *status,
                                         uint32_t &row) {
    if (s >= n) {
        atomicOr(status, vtp::ST_BOUNDS);
        return false;
    }
    row = row_of_slot[s];
    return true;
}

__global__ void k_dd_pack1(uint32_t count, uint32_t n, const uint32_t *__restrict__ slots,
                           const uint32_t *__restrict__ row_of_slot, const float *__restrict__ src,
                           float *__restrict__ out, uint32_t *status) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r;
    if (k >= count || !slot_row(slots[k], n, row_of_slot, status, r)) return;
    out[k] = src[r];
}

__global__ void k_dd_pack_posvel(uint32_t count, uint32_t n, const uint32_t *__restrict__ slots,
                                 const uint32_t *__restrict__ row_of_slot, const float4 *__restrict__ pos,
                                 const float4 *__restrict__ vel, float4 *__restrict__ out, uint32_t *status) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r;
    if (k >= count || !slot_row(slots[k], n, row_of_slot, status, r)) return;
    out[2 * (size_t)k] = pos[r];
    out[2 * (size_t)k + 1] = vel[r];
}

__global__ void k_dd_unpack_pbf(int field, uint32_t count, uint32_t first, uint32_t n,
                                const uint32_t *__restrict__ row_of_slot, const float *__restrict__ in1,
                                const float4 *__restrict__ in4, float *__restrict__ lambda, float4 *__restrict__ pos,
                                float4 *__restrict__ vel, uint32_t *status) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r;
    if (k >= count || !slot_row(first + k, n, row_of_slot, status, r)) return;
    if (field == VTP_DOMAIN_LAMBDA) {
        lambda[r] = in1[k];
    } else {
        pos[r] = in4[2 * (size_t)k];
        vel[r] = in4[2 * (size_t)k + 1];
    }
}

__global__ void k_dd_pack4(uint32_t count, uint32_t n, const uint32_t *__restrict__ slots,
                           const uint32_t *__restrict__ row_of_slot, const float4 *__restrict__ src,
                           float4 *__restrict__ out, uint32_t *status) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r;
    if (k >= count || !slot_row(slots[k], n, row_of_slot, status, r)) return;
    out[k] = src[r];
}

// Ghost values in: kappa goes to kappa[] and to the packed {x, kappa} rows solve_b gathers;
// v* to vadv[] and the packed {x, v*} rows solve_a gathers; velocities after the
// viscosity / tension pass to vel[] and vadv[] (v* = v); normals to normal[].
__global__ void k_dd_unpack(int field, uint32_t count, uint32_t first, uint32_t n,
                            const uint32_t *__restrict__ row_of_slot, const float *__restrict__ in1,
                            const float4 *__restrict__ in4, vtp::DfsphArgs a, uint32_t *status) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r;
    if (k >= count || !slot_row(first + k, n, row_of_slot, status, r)) return;
    switch (field) {
        case VTP_DOMAIN_KAPPA: {
            const float v = in1[k];
            a.kappa[r] = v;
            a.pk[r].w = v;
            break;
        }
        case VTP_DOMAIN_VADV: {
            const float4 v = in4[k];
            a.vadv[r] = v;
            a.pva[2 * (size_t)r + 1] = v;
            break;
        }
        case VTP_DOMAIN_VEL: {
            const float4 v = in4[k];
            a.vel[r] = v;
            a.vadv[r] = v;
            break;
        }
        default:
            a.normal[r] = in4[k];
            break;
    }
}

// Targets of peer `peer`: the owned rows at load slots slots[k] are ghosts there at rows
// dst[k] (below dst_limit, the peer's loaded rows).
__global__ void k_dd_targets(uint32_t count, uint32_t n, uint32_t n_own, uint32_t peer,
                             const uint32_t *__restrict__ slots, const uint32_t *__restrict__ dst, uint32_t dst_limit,
                             const uint32_t *__restrict__ row_of_slot, uint32_t *__restrict__ ntarget,
                             uint2 *__restrict__ target, uint32_t *status) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r;
    if (k >= count) return;
    if (slots[k] >= n_own || dst[k] >= dst_limit || !slot_row(slots[k], n, row_of_slot, status, r)) {
        atomicOr(status, vtp::ST_BOUNDS);
        return;
    }
    const uint32_t e = atomicAdd(&ntarget[r], 1u);
    if (e >= (uint32_t)vtp::kMaxHaloTargets) {
        atomicOr(status, vtp::ST_BOUNDS);
        return;
    }
    target[(size_t)r * vtp::kMaxHaloTargets + e] = make_uint2(peer, dst[k]);
}

__global__ void k_dd_rows(uint32_t count, uint32_t first, uint32_t n, const uint32_t *__restrict__ row_of_slot,
                          uint32_t *__restrict__ out, uint32_t *status) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r;
    if (k >= count || !slot_row(first + k, n, row_of_slot, status, r)) return;
    out[k] = r;
}

// Largest |v|^2 of the owned rows (load order, before the sort), with the arithmetic of the
// adaptive step's own reduction (k_cfl_max): fmax over dist2, folded by unsigned atomicMax.
__global__ void k_dd_vmax2(uint32_t n_own, const float4 *__restrict__ vel, uint32_t *__restrict__ out_bits) {
    float m = 0.f;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_own; r += gridDim.x * blockDim.x) {
        const float4 v = vel[r];
        m = fmaxf(m, vtp::dist2(v.x, v.y, v.z));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31u) == 0 && m > 0.f) atomicMax(out_bits, __float_as_uint(m));
}

__global__ void k_dd_read(uint32_t n_own, uint32_t n, const uint32_t *__restrict__ row_of_slot,
                          const float4 *__restrict__ pos, const float4 *__restrict__ vel, float *__restrict__ pos3,
                          float *__restrict__ vel3, uint32_t *status) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t r;
    if (s >= n_own || !slot_row(s, n, row_of_slot, status, r)) return;
    const float4 p = pos[r], v = vel[r];
    pos3[3 * (size_t)s] = p.x;
    pos3[3 * (size_t)s + 1] = p.y;
    pos3[3 * (size_t)s + 2] = p.z;
    vel3[3 * (size_t)s] = v.x;
    vel3[3 * (size_t)s + 1] = v.y;
    vel3[3 * (size_t)s + 2] = v.z;
}

std::string object_json(int material, int type) {
    json o = {{"name", material == 0 ? "domain fluid" : "domain boundary"},
              {"ObjectComponentConfig", {{"epmMaterial", material}}},
              {"SolverObjectComponentConfig",
               {{"solverType", type}, {"exportFlag", false}, {"velocityStart", {0, 0, 0}},
                {"colorStart", {0, 0, 0}}}}};
    return o.dump();
}

}  // namespace

struct vtp_domain {
    vtp_solver *s = nullptr;
    int type = VTP_SOLVER_DFSPH;   // VTP_SOLVER_DFSPH or VTP_SOLVER_PBF
    uint32_t cap = 0, nb = 0, nobj = 1;
    uint32_t n_own = 0, n_act = 0;
    int which = 0;
    bool loaded = false, prepared = false;
    cudaStream_t st = nullptr;
    DB<float> slot, objf;
    uint32_t *row_of_slot = nullptr;
    double *part = nullptr;
    uint32_t *status = nullptr;     // the domain kernels' own status word (ST_BOUNDS: a bad slot)
    uint32_t *h_status = nullptr;   // [2]: the domain word, the wrapped solver's word
    // Peer-store halos (DFSPH): per sorted row its ghost flag and its targets on peer workers
    bool dt_set = false;            // adaptive step: this substep's dt from the host
    float dt_now = 0.f;
    uint32_t *vmax_bits = nullptr;
    bool halo_on = false;
    uint8_t *ghost = nullptr;
    uint32_t *ntarget = nullptr;
    uint2 *target = nullptr;
    vtp::HaloPush h_halo{};
    vtp::HaloPush *d_halo = nullptr;
    std::vector<void *> ipc_opened;   // peer buffers mapped through CUDA IPC
    std::vector<void *> allocs;

    ~vtp_domain() {
        for (void *p : ipc_opened) cudaIpcCloseMemHandle(p);
        for (void *p : allocs) cudaFree(p);
        if (h_status) cudaFreeHost(h_status);
        if (s) vtp_solver_destroy(s);
    }
    template <class T>
    int alloc(T **p, size_t count) {
        *p = nullptr;
        cudaError_t e = cudaMalloc((void **)p, (count ? count : 1) * sizeof(T));
        if (e != cudaSuccess) return fail(VTP_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        allocs.push_back(*p);
        return VTP_OK;
    }
    vtp::DfsphArgs args() const {
        vtp::DfsphArgs a = s->dfsph_args(which);
        a.nf = n_act;
        a.ntiles = nblk(n_act, s->block);
        a.nobj_max = 1;     // per-tile partials of solve_a are not used; k_dd_sums keeps the objects apart
        a.staged = 0;
        a.dtp = nullptr;
        a.vmax_bits = nullptr;
        a.tick = nullptr;
        if (dt_set) {   // the adaptive step, 1/dt and 1/dt^2 formed as the device forms them
            const float inv = 1.f / dt_now;
            a.dt = dt_now;
            a.inv_dt = inv;
            a.inv_dt2 = inv * inv;
        }
        if (halo_on) {
            a.halo = d_halo;
            a.halo_vadv = s->vadv.cur;
            a.halo_vel = s->vel.cur;
        }
        return a;
    }
    vtp::PbfArgs pbf() const {
        vtp::PbfArgs a = s->pbf_args();
        a.nf = n_act;
        if (halo_on) {
            a.halo = d_halo;
            a.halo_pos = s->pos.cur;
            a.halo_vel = s->vel.cur;
        }
        return a;
    }
    vtp::Layout layout() const {
        vtp::Layout L = s->L;
        L.nf = n_act;
        return L;
    }
};

namespace {

int need_prepared(vtp_domain *d) {
    if (!d) return fail(VTP_ERR_ARG, "null domain");
    if (!d->prepared) return fail(VTP_ERR_STATE, "domain stage before vtp_domain_prepare");
    return VTP_OK;
}

int need_type(vtp_domain *d, int type) {
    int rc;
    if ((rc = need_prepared(d))) return rc;
    if (d->type != type)
        return fail(VTP_ERR_STATE, type == VTP_SOLVER_PBF ? "a PBF stage on a DFSPH domain worker"
                                                          : "a DFSPH stage on a PBF domain worker");
    return VTP_OK;
}

}  // namespace

int vtp_domain_create(const char *config_json, const float *fluid_pos, uint32_t n_fluid, const float *boundary_pos,
                      const uint32_t *boundary_ids, uint32_t nb, int boundary_first, uint32_t capacity,
                      uint32_t n_objects, vtp_domain **out) {
    if (!out || !config_json) return fail(VTP_ERR_ARG, "null argument");
    *out = nullptr;
    if (capacity == 0 || capacity > kMaxCapacity) return fail(VTP_ERR_BOUNDS, "capacity outside 1..2^24");
    if (n_fluid > capacity) return fail(VTP_ERR_BOUNDS, "more initial fluid rows than the capacity");
    if (n_objects == 0 || n_objects > kMaxObjects) return fail(VTP_ERR_BOUNDS, "fluid objects outside 1..16");
    if ((n_fluid && !fluid_pos) || (nb && (!boundary_pos || !boundary_ids))) return fail(VTP_ERR_ARG, "null array");
    for (uint32_t k = 1; k < nb; ++k)
        if (boundary_ids[k] <= boundary_ids[k - 1]) return fail(VTP_ERR_ARG, "boundary ids not ascending");
    try {
        json cfg = json::parse(config_json);
        const bool pbf = cfg.contains("PBF");
        if (!pbf && !cfg.contains("DFSPH")) return fail(VTP_ERR_CONFIG, "domain workers run DFSPH or PBF scenes");
        const char *key = pbf ? "PBF" : "DFSPH";
        json ext = cfg.contains("B200") ? cfg["B200"] : json::object();
        ext.erase("cfl");   // the host sets an adaptive step per substep (vtp_domain_set_dt)
        const int mode = boundary_first ? 1 : 0;
        ext["useGraphs"] = false;
        ext["deviceLoop"] = false;
        ext["stagedSolve"] = false;
        cfg["B200"] = ext;
        const json &req = cfg[key]["Required"];
        const float r = req.at("particleRadius").get<float>();
        const float h = r * 4.f;
        float park[3];
        for (int a = 0; a < 3; ++a) park[a] = req.at("simSpaceLB")[a].get<float>() - 8.f * h;   // outside the grid

        auto d = std::make_unique<vtp_domain>();
        d->type = pbf ? VTP_SOLVER_PBF : VTP_SOLVER_DFSPH;
        d->cap = capacity;
        d->nb = nb;
        d->nobj = n_objects;
        int rc;
        if ((rc = vtp_solver_create(d->type, &d->s))) return rc;
        if ((rc = vtp_solver_set_config(d->s, cfg.dump().c_str()))) return rc;
        // Fluid rows: the initial owned and ghost particles (ascending scene-wide id, so that
        // the boundary rows' lists at initialize, and with them the boundary volumes, are those
        // of the whole scene near the slab), then unused rows parked outside the grid.
        std::vector<float> fl((size_t)capacity * 3);
        for (uint32_t i = 0; i < capacity; ++i)
            for (int a = 0; a < 3; ++a) fl[3 * (size_t)i + a] = i < n_fluid ? fluid_pos[3 * (size_t)i + a] : park[a];
        const std::string fj = object_json(0, d->type), bj = object_json(1, d->type);
        if (mode == 1 && nb && (rc = vtp_solver_attach_object(d->s, boundary_pos, nb, nullptr, bj.c_str()))) return rc;
        if ((rc = vtp_solver_attach_object(d->s, fl.data(), capacity, nullptr, fj.c_str()))) return rc;
        if (mode == 0 && nb && (rc = vtp_solver_attach_object(d->s, boundary_pos, nb, nullptr, bj.c_str()))) return rc;
        if ((rc = vtp_solver_initialize(d->s))) return rc;
        vtp_solver *s = d->s;
        if (s->L.nf != capacity || s->L.nb != nb) return fail(VTP_ERR_STATE, "domain worker layout");
        d->st = s->st;
        CU(cudaMallocHost((void **)&d->h_status, 2 * sizeof(uint32_t)));
        if ((rc = d->alloc(&d->status, 1))) return rc;
        CU(cudaMemsetAsync(d->status, 0, sizeof(uint32_t), d->st));
        for (int k = 0; k < 2; ++k) {
            if ((rc = d->alloc(&d->slot.b[k], capacity))) return rc;
            if ((rc = d->alloc(&d->objf.b[k], capacity))) return rc;
        }
        if ((rc = d->alloc(&d->row_of_slot, capacity))) return rc;
        if ((rc = d->alloc(&d->vmax_bits, 1))) return rc;
        if ((rc = d->alloc(&d->part, (size_t)kSumBlocks * n_objects))) return rc;
        {
            if ((rc = d->alloc(&d->ghost, capacity))) return rc;
            if ((rc = d->alloc(&d->ntarget, capacity))) return rc;
            if ((rc = d->alloc(&d->target, (size_t)capacity * vtp::kMaxHaloTargets))) return rc;
            if ((rc = d->alloc(&d->d_halo, 1))) return rc;
            d->h_halo.ghost = d->ghost;
            d->h_halo.ntarget = d->ntarget;
            d->h_halo.target = d->target;
            CU(cudaMemsetAsync(d->ntarget, 0, capacity * sizeof(uint32_t), d->st));
            CU(cudaMemcpyAsync(d->d_halo, &d->h_halo, sizeof(vtp::HaloPush), cudaMemcpyHostToDevice, d->st));
        }
        if (nb) {
            uint32_t *gid = nullptr;
            if ((rc = d->alloc(&gid, nb))) return rc;
            CU(cudaMemcpyAsync(gid, boundary_ids, nb * sizeof(uint32_t), cudaMemcpyHostToDevice, d->st));
            const uint32_t local0 = mode == 0 ? capacity : 0u;
            k_dd_band_ids<<<nblk(nb, 256), 256, 0, d->st>>>(nb, capacity, local0, gid, s->orig.b[0], s->orig.b[1],
                                                            d->status);
            CU(cudaGetLastError());
        }
        // DFSPH: the boundary rows' packed gather rows ({x, V_b}, {x, v*}) never change: pack them once.
        if (!pbf) vtp::dfsph_solve_pack(d->st, s->dfsph_args());
        CU(cudaGetLastError());
        CU(cudaStreamSynchronize(d->st));
        *out = d.release();
        return VTP_OK;
    } catch (const std::exception &e) {
        return fail(VTP_ERR_CONFIG, e.what());
    }
}

void vtp_domain_destroy(vtp_domain *d) {
    if (d) cudaStreamSynchronize(d->st);
    delete d;
}

int vtp_domain_set_stream(vtp_domain *d, void *stream) {
    if (!d) return fail(VTP_ERR_ARG, "null domain");
    d->st = stream ? (cudaStream_t)stream : d->s->st;
    return VTP_OK;
}

int vtp_domain_capacity(vtp_domain *d, uint32_t *capacity, uint32_t *n_boundary) {
    if (!d) return fail(VTP_ERR_ARG, "null domain");
    if (capacity) *capacity = d->cap;
    if (n_boundary) *n_boundary = d->nb;
    return VTP_OK;
}

int vtp_domain_load(vtp_domain *d, uint32_t n_own, uint32_t n_ghost, const float *d_pos, const float *d_vel,
                    const uint32_t *d_ids, const uint32_t *d_obj) {
    if (!d) return fail(VTP_ERR_ARG, "null domain");
    const uint64_t n = (uint64_t)n_own + n_ghost;
    if (n > d->cap) return fail(VTP_ERR_BOUNDS, "owned plus ghost rows exceed the capacity");
    if (n && (!d_pos || !d_vel || !d_ids)) return fail(VTP_ERR_ARG, "null array");
    vtp_solver *s = d->s;
    d->n_own = n_own;
    d->n_act = (uint32_t)n;
    if (n)
        k_dd_load<<<nblk((uint32_t)n, 256), 256, 0, d->st>>>(
            (uint32_t)n, d_pos, d_vel, d_ids, d_obj, d->type == VTP_SOLVER_PBF ? s->rho_f * s->vol0 : s->vol0,
            s->pos.c(), s->vel.c(), d->type == VTP_SOLVER_PBF ? nullptr : s->vadv.c(), s->orig.c(), d->slot.c(),
            d->objf.c());
    CU(cudaGetLastError());
    d->loaded = true;
    d->prepared = false;
    return VTP_OK;
}

int vtp_domain_prepare(vtp_domain *d) {
    if (!d) return fail(VTP_ERR_ARG, "null domain");
    if (!d->loaded) return fail(VTP_ERR_STATE, "vtp_domain_prepare before vtp_domain_load");
    vtp_solver *s = d->s;
    const vtp::NvtxRange r("vtp domain neighbour search");
    // The UGNS sort of the loaded rows (load slot and object carried along; DFSPH: v* too;
    // PBF: the external force applied on the way, PBFCudaImpl.cu:146-157), the lists, then
    // (DFSPH) compression ratio and alpha.
    const bool pbf = d->type == VTP_SOLVER_PBF;
    vtp::Carry carry{};
    if (!pbf) {
        carry.nf4 = 1;
        carry.src4[0] = s->vadv.c();
        carry.dst4[0] = s->vadv.n();
    }
    carry.nf1 = 2;
    carry.src1[0] = d->slot.c();
    carry.dst1[0] = d->slot.n();
    carry.src1[1] = d->objf.c();
    carry.dst1[1] = d->objf.n();
    vtp::ugns_sort(d->st, s->scn(), s->nbuckets, 0, d->n_act, s->pos.c(), s->pos.n(), s->vel.c(), s->vel.n(),
                   s->orig.c(), s->orig.n(), carry, pbf ? s->dt : 0.f, s->u, s->u.fstart);
    s->pos.swap(); s->vel.swap(); s->orig.swap();
    if (!pbf) s->vadv.swap();
    d->slot.swap(); d->objf.swap();
    const vtp::Layout L = d->layout();
    vtp::ugns_build_lists(d->st, s->scn(), L, 0, d->n_act, s->pos.c(), s->orig.c(), s->u, s->u.nbr, s->u.ncnt,
                          s->d_status, s->d_overflow, s->block);
    if (d->n_act) {
        k_dd_row_of_slot<<<nblk(d->n_act, 256), 256, 0, d->st>>>(d->n_act, d->slot.c(), d->row_of_slot, d->status);
        if (d->halo_on) {
            k_dd_ghost_flags<<<nblk(d->n_act, 256), 256, 0, d->st>>>(d->n_act, d->n_own, d->slot.c(), d->ghost);
            CU(cudaMemsetAsync(d->ntarget, 0, d->n_act * sizeof(uint32_t), d->st));
        }
        if (!pbf)
            k_dd_tiles<<<nblk(nblk(d->n_act, s->block), 256), 256, 0, d->st>>>(s->d_tiles, d->n_act,
                                                                             (uint32_t)s->block);
    }
    d->which = 0;
    if (!pbf) vtp::dfsph_ratio_alpha(d->st, d->args(), s->block);
    CU(cudaGetLastError());
    d->prepared = true;
    return VTP_OK;
}

int vtp_domain_pbf_lambda(vtp_domain *d) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_PBF))) return rc;
    vtp::pbf_lambda(d->st, d->pbf(), d->s->block);
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_pbf_dx(vtp_domain *d) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_PBF))) return rc;
    vtp::pbf_dx(d->st, d->pbf(), d->s->block);   // positions into the second buffer, velocities in place
    d->s->pos.swap();
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_pbf_xsph(vtp_domain *d) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_PBF))) return rc;
    vtp::pbf_xsph(d->st, d->pbf(), d->s->block);
    d->s->pos.swap(); d->s->vel.swap();
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_solve_begin(vtp_domain *d, int which) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_DFSPH))) return rc;
    if (which != 0 && which != 1) return fail(VTP_ERR_ARG, "which: 0 divergence, 1 density");
    d->which = which;
    vtp_solver *s = d->s;
    vtp::dfsph_solve_begin(d->st, s->solve + which, s->loop + which, 1);
    vtp::DfsphArgs a = d->args();
    a.nb = 0;   // the boundary rows were packed at create
    vtp::dfsph_solve_pack(d->st, a);
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_solve_a(vtp_domain *d, double *d_sums) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_DFSPH))) return rc;
    if (!d_sums) return fail(VTP_ERR_ARG, "null sums");
    const vtp::DfsphArgs a = d->args();
    vtp::dfsph_solve_a(d->st, a, d->s->block);
    if (d->nobj == 1)
        k_dd_sums<1><<<kSumBlocks, kSumThreads, 0, d->st>>>(d->n_act, d->n_own, a.delta, d->slot.c(), d->objf.c(), 1,
                                                            d->part);
    else if (d->nobj <= 4)
        k_dd_sums<4><<<kSumBlocks, kSumThreads, 0, d->st>>>(d->n_act, d->n_own, a.delta, d->slot.c(), d->objf.c(),
                                                            (int)d->nobj, d->part);
    else
        k_dd_sums<kMaxObjects><<<kSumBlocks, kSumThreads, 0, d->st>>>(d->n_act, d->n_own, a.delta, d->slot.c(),
                                                                      d->objf.c(), (int)d->nobj, d->part);
    k_dd_sums_final<<<1, kSumThreads, 0, d->st>>>(kSumBlocks, (int)d->nobj, d->part, d_sums);
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_solve_b(vtp_domain *d) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_DFSPH))) return rc;
    vtp::dfsph_solve_b(d->st, d->args(), d->s->block);
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_forces(vtp_domain *d) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_DFSPH))) return rc;
    vtp_solver *s = d->s;
    const vtp::DfsphArgs a = d->args();
    vtp::dfsph_pressure_pack(d->st, a);
    if (s->gamma == 0.f) {
        vtp::dfsph_viscosity(d->st, a, s->block);
        s->vel.swap(); s->vadv.swap();
    } else {
        vtp::dfsph_vis_normal(d->st, a, s->block);
    }
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_tension(vtp_domain *d) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_DFSPH))) return rc;
    vtp_solver *s = d->s;
    if (s->gamma == 0.f) return fail(VTP_ERR_STATE, "surface tension pass with surfaceTensionCoefficient 0");
    vtp::dfsph_tension(d->st, d->args(), s->block);
    s->vel.swap(); s->vadv.swap();
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_finalize(vtp_domain *d) {
    int rc;
    if ((rc = need_type(d, VTP_SOLVER_DFSPH))) return rc;
    vtp::dfsph_finalize(d->st, d->args());
    CU(cudaGetLastError());
    return VTP_OK;
}

namespace {

int need_halo(vtp_domain *d) {
    if (!d) return fail(VTP_ERR_ARG, "null domain");
    if (!d->d_halo) return fail(VTP_ERR_STATE, "domain worker without halo state");
    return VTP_OK;
}

// The buffers a peer stores ghost values into, in vtp_domain_ipc order: DFSPH kappa, packed
// {x, kappa} and {x, v*} rows, normals, both v* and both velocity buffers; PBF lambda, both
// position and both velocity buffers.  Returns how many.
int halo_buffers(vtp_domain *d, void *out[VTP_DOMAIN_IPC_BUFFERS]) {
    vtp_solver *s = d->s;
    if (d->type == VTP_SOLVER_PBF) {
        void *b[5] = {s->lambda, s->pos.b[0], s->pos.b[1], s->vel.b[0], s->vel.b[1]};
        for (int k = 0; k < 5; ++k) out[k] = b[k];
        return 5;
    }
    void *b[VTP_DOMAIN_IPC_BUFFERS] = {s->kappa, s->pk, s->pva, s->normal, s->vadv.b[0], s->vadv.b[1],
                                       s->vel.b[0], s->vel.b[1]};
    for (int k = 0; k < VTP_DOMAIN_IPC_BUFFERS; ++k) out[k] = b[k];
    return VTP_DOMAIN_IPC_BUFFERS;
}

vtp::PeerRows peer_rows(int type, void *const b[VTP_DOMAIN_IPC_BUFFERS]) {
    vtp::PeerRows r{};
    if (type == VTP_SOLVER_PBF) {
        r.lambda = (float *)b[0];
        r.pos[0] = (float4 *)b[1];
        r.pos[1] = (float4 *)b[2];
        r.vel[0] = (float4 *)b[3];
        r.vel[1] = (float4 *)b[4];
        return r;
    }
    r.kappa = (float *)b[0];
    r.pk = (float4 *)b[1];
    r.pva = (float4 *)b[2];
    r.normal = (float4 *)b[3];
    r.vadv[0] = (float4 *)b[4];
    r.vadv[1] = (float4 *)b[5];
    r.vel[0] = (float4 *)b[6];
    r.vel[1] = (float4 *)b[7];
    return r;
}

bool linked(const vtp::PeerRows &r) { return r.kappa || r.lambda; }

}  // namespace

int vtp_domain_export_ipc(vtp_domain *d, vtp_domain_ipc *out) {
    int rc;
    if ((rc = need_halo(d))) return rc;
    if (!out) return fail(VTP_ERR_ARG, "null output");
    std::memset(out, 0, sizeof(*out));
    void *b[VTP_DOMAIN_IPC_BUFFERS];
    const int nbuf = halo_buffers(d, b);
    for (int k = 0; k < nbuf; ++k) {
        cudaIpcMemHandle_t h;
        CU(cudaIpcGetMemHandle(&h, b[k]));
        static_assert(sizeof(h) <= sizeof(out->handle[0]), "IPC handle size");
        std::memcpy(out->handle[k], &h, sizeof(h));
    }
    out->capacity = d->cap;
    out->count = (uint32_t)nbuf;
    out->solver_type = (uint32_t)d->type;
    return VTP_OK;
}

int vtp_domain_link_peer(vtp_domain *d, int peer, vtp_domain *local_peer) {
    int rc;
    if ((rc = need_halo(d)) || (rc = need_halo(local_peer))) return rc;
    if (peer < 0 || peer >= vtp::kMaxPeers) return fail(VTP_ERR_BOUNDS, "peer index outside 0..7");
    if (local_peer->type != d->type) return fail(VTP_ERR_STATE, "peer worker of another solver type");
    void *b[VTP_DOMAIN_IPC_BUFFERS] = {};
    halo_buffers(local_peer, b);
    d->h_halo.peer[peer] = peer_rows(d->type, b);
    CU(cudaMemcpyAsync(d->d_halo, &d->h_halo, sizeof(vtp::HaloPush), cudaMemcpyHostToDevice, d->st));
    CU(cudaStreamSynchronize(d->st));
    return VTP_OK;
}

int vtp_domain_link_peer_ipc(vtp_domain *d, int peer, const vtp_domain_ipc *h) {
    int rc;
    if ((rc = need_halo(d))) return rc;
    if (!h) return fail(VTP_ERR_ARG, "null handles");
    if (peer < 0 || peer >= vtp::kMaxPeers) return fail(VTP_ERR_BOUNDS, "peer index outside 0..7");
    if (h->solver_type != (uint32_t)d->type || h->count > VTP_DOMAIN_IPC_BUFFERS)
        return fail(VTP_ERR_STATE, "peer handles of another solver type");
    void *b[VTP_DOMAIN_IPC_BUFFERS] = {};
    for (uint32_t k = 0; k < h->count; ++k) {
        cudaIpcMemHandle_t hk;
        std::memcpy(&hk, h->handle[k], sizeof(hk));
        CU(cudaIpcOpenMemHandle(&b[k], hk, cudaIpcMemLazyEnablePeerAccess));
        d->ipc_opened.push_back(b[k]);
    }
    d->h_halo.peer[peer] = peer_rows(d->type, b);
    CU(cudaMemcpyAsync(d->d_halo, &d->h_halo, sizeof(vtp::HaloPush), cudaMemcpyHostToDevice, d->st));
    CU(cudaStreamSynchronize(d->st));
    return VTP_OK;
}

int vtp_domain_set_halo(vtp_domain *d, int on) {
    int rc;
    if ((rc = need_halo(d))) return rc;
    d->halo_on = on != 0;
    d->prepared = false;   // the next prepare sets the ghost flags
    return VTP_OK;
}

int vtp_domain_buffer_parity(vtp_domain *d, int32_t *out3) {
    if (!d || !out3) return fail(VTP_ERR_ARG, "null argument");
    out3[0] = d->s->vadv.cur;
    out3[1] = d->s->vel.cur;
    out3[2] = d->s->pos.cur;
    return VTP_OK;
}

int vtp_domain_rows(vtp_domain *d, uint32_t first_slot, uint32_t count, uint32_t *d_rows) {
    int rc;
    if ((rc = need_prepared(d))) return rc;
    if (count == 0) return VTP_OK;
    if (!d_rows) return fail(VTP_ERR_ARG, "null array");
    if ((uint64_t)first_slot + count > d->n_act) return fail(VTP_ERR_BOUNDS, "rows outside the loaded rows");
    k_dd_rows<<<nblk(count, 256), 256, 0, d->st>>>(count, first_slot, d->n_act, d->row_of_slot, d_rows, d->status);
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_halo_targets(vtp_domain *d, int peer, const uint32_t *d_slots, const uint32_t *d_dst_rows,
                            uint32_t count, uint32_t peer_capacity) {
    int rc;
    if ((rc = need_halo(d)) || (rc = need_prepared(d))) return rc;
    if (!d->halo_on) return fail(VTP_ERR_STATE, "halo targets with peer-store halos off");
    if (peer < 0 || peer >= vtp::kMaxPeers || !linked(d->h_halo.peer[peer]))
        return fail(VTP_ERR_STATE, "halo targets on a peer that is not linked");
    if (count == 0) return VTP_OK;
    if (!d_slots || !d_dst_rows) return fail(VTP_ERR_ARG, "null array");
    k_dd_targets<<<nblk(count, 256), 256, 0, d->st>>>(count, d->n_act, d->n_own, (uint32_t)peer, d_slots, d_dst_rows,
                                                     peer_capacity, d->row_of_slot, d->ntarget, d->target,
                                                     d->status);
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_owned_vmax2(vtp_domain *d, float *out) {
    if (!d || !out) return fail(VTP_ERR_ARG, "null argument");
    if (!d->loaded) return fail(VTP_ERR_STATE, "vtp_domain_owned_vmax2 before vtp_domain_load");
    if (d->prepared) return fail(VTP_ERR_STATE, "vtp_domain_owned_vmax2 between load and prepare");
    CU(cudaMemsetAsync(d->vmax_bits, 0, sizeof(uint32_t), d->st));
    if (d->n_own) {
        const unsigned g = std::min<unsigned>(nblk(d->n_own, 256), 148u * 8u);
        k_dd_vmax2<<<g, 256, 0, d->st>>>(d->n_own, d->s->vel.c(), d->vmax_bits);
    }
    CU(cudaGetLastError());
    uint32_t bits = 0;
    CU(cudaMemcpyAsync(d->h_status, d->vmax_bits, sizeof(uint32_t), cudaMemcpyDeviceToHost, d->st));
    CU(cudaStreamSynchronize(d->st));
    bits = d->h_status[0];
    std::memcpy(out, &bits, sizeof(float));
    return VTP_OK;
}

int vtp_domain_set_dt(vtp_domain *d, float dt) {
    if (!d) return fail(VTP_ERR_ARG, "null domain");
    if (!(dt > 0.f) || !std::isfinite(dt)) return fail(VTP_ERR_ARG, "time step must be finite and positive");
    d->dt_set = true;
    d->dt_now = dt;
    return VTP_OK;
}

int vtp_domain_pack(vtp_domain *d, int field, const uint32_t *d_slots, uint32_t count, float *d_out) {
    int rc;
    if ((rc = need_prepared(d))) return rc;
    if (count == 0) return VTP_OK;
    if (!d_slots || !d_out) return fail(VTP_ERR_ARG, "null array");
    uint32_t *status = d->status;
    if (d->type == VTP_SOLVER_PBF) {
        vtp_solver *s = d->s;
        if (field == VTP_DOMAIN_LAMBDA)
            k_dd_pack1<<<nblk(count, 256), 256, 0, d->st>>>(count, d->n_act, d_slots, d->row_of_slot, s->lambda,
                                                           d_out, status);
        else if (field == VTP_DOMAIN_POSVEL)
            k_dd_pack_posvel<<<nblk(count, 256), 256, 0, d->st>>>(count, d->n_act, d_slots, d->row_of_slot,
                                                                 s->pos.c(), s->vel.c(), (float4 *)d_out, status);
        else
            return fail(VTP_ERR_ARG, "not a PBF domain field");
        CU(cudaGetLastError());
        return VTP_OK;
    }
    const vtp::DfsphArgs a = d->args();
    switch (field) {
        case VTP_DOMAIN_KAPPA:
            k_dd_pack1<<<nblk(count, 256), 256, 0, d->st>>>(count, d->n_act, d_slots, d->row_of_slot, a.kappa, d_out,
                                                           status);
            break;
        case VTP_DOMAIN_VADV:
        case VTP_DOMAIN_VEL:   // after the viscosity / tension pass vel[] and vadv[] hold the same velocity
            k_dd_pack4<<<nblk(count, 256), 256, 0, d->st>>>(count, d->n_act, d_slots, d->row_of_slot, a.vadv,
                                                           (float4 *)d_out, status);
            break;
        case VTP_DOMAIN_NORMAL:
            k_dd_pack4<<<nblk(count, 256), 256, 0, d->st>>>(count, d->n_act, d_slots, d->row_of_slot, a.normal,
                                                           (float4 *)d_out, status);
            break;
        default:
            return fail(VTP_ERR_ARG, "unknown domain field");
    }
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_unpack(vtp_domain *d, int field, uint32_t first_slot, uint32_t count, const float *d_in) {
    int rc;
    if ((rc = need_prepared(d))) return rc;
    const bool pbf = d->type == VTP_SOLVER_PBF;
    if (pbf ? (field != VTP_DOMAIN_LAMBDA && field != VTP_DOMAIN_POSVEL)
            : (field < VTP_DOMAIN_KAPPA || field > VTP_DOMAIN_NORMAL))
        return fail(VTP_ERR_ARG, "not a domain field of this solver");
    if (count == 0) return VTP_OK;
    if (!d_in) return fail(VTP_ERR_ARG, "null array");
    if ((uint64_t)first_slot + count > d->n_act || first_slot < d->n_own)
        return fail(VTP_ERR_BOUNDS, "unpack outside the ghost rows");
    if (pbf)
        k_dd_unpack_pbf<<<nblk(count, 256), 256, 0, d->st>>>(field, count, first_slot, d->n_act, d->row_of_slot, d_in,
                                                            (const float4 *)d_in, d->s->lambda, d->s->pos.c(),
                                                            d->s->vel.c(), d->status);
    else
        k_dd_unpack<<<nblk(count, 256), 256, 0, d->st>>>(field, count, first_slot, d->n_act, d->row_of_slot, d_in,
                                                        (const float4 *)d_in, d->args(), d->status);
    CU(cudaGetLastError());
    return VTP_OK;
}

int vtp_domain_read(vtp_domain *d, float *d_pos, float *d_vel) {
    int rc;
    if ((rc = need_prepared(d))) return rc;
    vtp_solver *s = d->s;
    if (d->n_own) {
        if (!d_pos || !d_vel) return fail(VTP_ERR_ARG, "null array");
        k_dd_read<<<nblk(d->n_own, 256), 256, 0, d->st>>>(d->n_own, d->n_act, d->row_of_slot, s->pos.c(), s->vel.c(),
                                                         d_pos, d_vel, d->status);
    }
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(d->h_status, d->status, sizeof(uint32_t), cudaMemcpyDeviceToHost, d->st));
    CU(cudaMemcpyAsync(d->h_status + 1, s->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, d->st));
    CU(cudaStreamSynchronize(d->st));
    // A list longer than maxNeighborNum is truncated as the reference truncates it (the
    // solver's word records it, not an error); the checked build's bounds reports are.
    if (d->h_status[0] & vtp::ST_BOUNDS)
        return fail(VTP_ERR_BOUNDS, "a domain stage addressed a row outside the loaded rows");
#ifdef VTP_CHECKED
    if (d->h_status[1] & vtp::ST_BOUNDS) return fail(VTP_ERR_BOUNDS, "a list entry or cell slot out of range");
#endif
    if (d->h_status[1] & vtp::ST_NAN) return fail(VTP_ERR_NAN, "non-finite state in a domain worker");
    return VTP_OK;
}
