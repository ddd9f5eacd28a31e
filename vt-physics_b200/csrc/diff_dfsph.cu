// Differentiable DFSPH rollout: a recorded forward with checkpoints and the
// hand-written adjoint of the DFSPH substep (no counterpart in the reference).
//
// One substep (DFSPHSolver::tick, DFSPHSolver.cpp:339-406, as the library runs
// it; surface tension off, fixed time step):
//   lists from x;  ratio_i = V_i W0 + sum_j V_j W_ij,  a1_i = sum_j V_j gradW_ij,
//   alpha_i = max(|a1_i|^2 / m + 1e-6 + sum_{fluid j} V_j^2 |gradW_ij|^2 / m, 1e-6)
//   divergence solve, density solve: from v* = v, each iteration
//     kappa_i = max(0, ratio_i - 1 + dt sum_j V_j gradW_ij.(v*_i - v*_j)) / (alpha_i dt^2 V_i)
//     v*_i -= (dt V_i / m) sum_j V_j (kappa_i + kappa_j) gradW_ij      (kappa_j = 0 for boundary j)
//   between them: v' = v* + dt (g + sum_{fluid j} C (u.r) gradW_ij / (|r|^2 + 0.001 h^2)),
//     u = v*_i - v*_j, C = 10 nu V_j
//   v_new = v*, x_new = x + dt v_new
// with gradW_ij = g r (r = x_i - x_j) and d(g r)/dr = J = g I + hh r r^T.
//
// Forward (vtp_solver_diff_forward on a DFSPH solver): the ordinary substeps, with
// the fluid state saved every k substeps; the last segments (as many as fit the tape
// budget) run recording substeps: the substep's lists, positions, alpha, the velocity
// after the divergence solve and, per pressure-solve iteration, {v* entering it, its
// kappa}.  A segment of an even checkpoint interval replays a CUDA graph captured once
// per tape, its solve loops WHILE nodes whose iterations address their records on the
// device (one readback per segment); other segments run host-driven solve loops that
// read the stop flag once per chunk of iterations.
// Backward: the segments last to first, each recomputed from its checkpoint into a
// tape unless the forward recorded it, then the adjoint substeps in reverse.  Every
// adjoint neighbour sum is in gather form over the same symmetric lists, so no pass
// uses atomics; the clamps (kappa > 0, alpha > 1e-6) of the forward are held fixed.
#include "solver.h"
#include "diff_dfsph.h"

#include <algorithm>
#include <string>
#include <vector>

namespace vtp {

struct DfTapeSlot {
    uint32_t *orig = nullptr, *nbr = nullptr, *ncnt = nullptr;
    float4 *x = nullptr;        // [n] positions, w = volume (boundary rows static)
    float4 *vp = nullptr;       // [nf] velocity after the divergence solve
    float *alpha = nullptr;     // [nf]
    uint32_t iters[2] = {0, 0}; // divergence / density solve iterations
    uint32_t first[2] = {0, 0}; // their first record in the tape's record pool
};

// Record pointers a tape's graph-recorded segment can address (the device table's size).
constexpr uint32_t kRecTable = 8192;

struct DfTape {
    std::vector<DfTapeSlot> slots;
    std::vector<float4 *> recs;   // [n] {v* entering the iteration, its kappa}; boundary rows {v_b, 0}
    // Graph-recorded segments: the segment's substeps captured once into `exec` (buffer parity
    // `par` at its start), the solve loops as WHILE nodes; each iteration's record is recs[pool +
    // iteration], pool = ctl[0] (advanced by each solve's iteration count), up to cap[0] records.
    float4 **d_recs = nullptr;    // [kRecTable] device copy of recs
    uint32_t *d_cap = nullptr;    // [1] records d_recs holds
    uint32_t *d_ctl = nullptr;    // [2] pool counter, overflow flag
    uint32_t *d_info = nullptr;   // [slots][4] first record and iterations of each slot's two solves
    uint32_t uploaded = 0;        // recs entries copied to d_recs
    cudaGraphExec_t exec = nullptr;
    int par[4] = {-1, -1, -1, -1};
};

struct DfDiffState {
    uint32_t steps = 0, every = 0, nf = 0, n = 0;
    bool keep_lists = false;
    std::vector<void *> mem;
    std::vector<float4 *> ck_pos, ck_vel;
    std::vector<uint32_t *> ck_orig;
    std::vector<DfTape> tapes;
    std::vector<int> taped;
    float4 *bstat = nullptr;      // [n] boundary rows {v_b, 0}, copied into every record
    uint32_t hint[2] = {2, 2};    // iterations of the last recorded divergence / density solve
    // adjoint work arrays
    float4 *xbar_a = nullptr, *vbar_a = nullptr;    // attach order [n]
    float4 *xbar = nullptr, *vb[2] = {nullptr, nullptr}, *a1b = nullptr;
    float *db = nullptr, *rbar = nullptr, *abar = nullptr;
    double *vpart = nullptr, *vacc = nullptr;
    uint32_t blocks = 0;

    uint32_t *h_info = nullptr;   // page-locked: one tape's d_info and d_ctl after a graph-recorded segment

    ~DfDiffState() {
        for (auto &t : tapes)
            if (t.exec) cudaGraphExecDestroy(t.exec);
        for (void *p : mem) cudaFree(p);
        if (h_info) cudaFreeHost(h_info);
    }
    template <class T>
    int alloc(T **p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
        if (e != cudaSuccess)
            return fail(VTP_ERR_NOMEM, std::string("differentiable DFSPH: ") + cudaGetErrorString(e));
        mem.push_back(*p);
        return VTP_OK;
    }
};

namespace {

inline unsigned nblk(uint32_t n, int b) { return (unsigned)((n + b - 1) / b); }

// g'(r) / r of the cubic spline's gradient factor (gradW = g r).
__device__ __forceinline__ float cubic_hh(float d2, const Cubic &k) {
    if (!(d2 > 0.f)) return 0.f;
    const float r = sqrtf(d2);
    const float q = r * k.invh;
    if (q < 1e-6f || q > 1.f) return 0.f;
    const float ih2 = k.invh * k.invh, ih4 = ih2 * ih2;
    if (q <= 0.5f) return 18.f * k.sigma * ih4 / q;
    return 6.f * k.sigma * ih4 * (1.f - q * q) / (q * q * q);
}

__device__ __forceinline__ double block_sum_d(double v) {
    __shared__ double sm[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sm[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    double s = 0.0;
    if (wid == 0) {
        s = lane < nw ? sm[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    return s;
}

struct DfdArgs {
    uint32_t nf, ell_stride;
    Cubic k;
    float dt, mass_f, vis10;   // vis10 = 10 nu V_f (the viscosity pair factor C)
    float eps;                 // 0.001 h^2
    const uint32_t *nbr, *ncnt, *orig;
    const float4 *x;           // [n] w = volume
    const float4 *rec;         // [n] {v*, kappa} of the iteration
    const float4 *vp;          // [nf]
    const float *alpha;        // [nf]
    float4 *xbar, *vb, *vb_out, *a1b;
    float *db, *rbar, *abar;
    float4 *xbar_a, *vbar_a;
    double *vpart;
};

// Recording: {v* entering the iteration, kappa} of every fluid row.
__global__ void k_dfd_record(uint32_t nf, const float4 *__restrict__ vadv, const float *__restrict__ kappa,
                             float4 *__restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nf) return;
    const float4 v = vadv[r];
    out[r] = make_float4(v.x, v.y, v.z, kappa[r]);
}

// Graph-recorded solves: the record of the running iteration is recs[ctl[0] + st->iter] (the
// solve's iterations so far); past the table's valid records the overflow flag is set and the
// record skipped (the host grows the table and replays the segment).
__global__ void k_dfd_record_dev(uint32_t nf, const float4 *__restrict__ vadv, const float *__restrict__ kappa,
                                 const SolveState *st, float4 *const *recs, const uint32_t *cap, uint32_t *ctl) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t idx = ctl[0] + st->iter;
    if (idx >= *cap) {
        if (r == 0) ctl[1] = 1u;
        return;
    }
    if (r >= nf) return;
    const float4 v = vadv[r];
    recs[idx][r] = make_float4(v.x, v.y, v.z, kappa[r]);
}

// After a graph-recorded solve: its first record and iteration count, and the pool advanced.
__global__ void k_dfd_solve_done(const SolveState *st, uint32_t *ctl, uint32_t *info) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t it = st->iter;
    info[0] = ctl[0];
    info[1] = it;
    ctl[0] += it;
}

__global__ void k_dfd_tick_add(uint64_t *tick, uint32_t k) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *tick += k;
}

// Recording: the velocity after the divergence solve (second half of the packed rows).
__global__ void k_dfd_vp(uint32_t nf, const float4 *__restrict__ pva, float4 *__restrict__ out) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nf) return;
    out[r] = pva[2 * (size_t)r + 1];
}

// Attach order -> this substep's rows; the position update's adjoint (v-bar of the density
// solve's output = v-bar + dt x-bar); the ratio / alpha adjoints start at zero.
__global__ void k_dfd_gather(DfdArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const uint32_t id = a.orig[r];
    const float4 xo = a.xbar_a[id], vo = a.vbar_a[id];
    a.xbar[r] = xo;
    a.vb[r] = make_float4(vo.x + a.dt * xo.x, vo.y + a.dt * xo.y, vo.z + a.dt * xo.z, 0.f);
    a.rbar[r] = 0.f;
    a.abar[r] = 0.f;
}

// The neighbour passes of the adjoint split each row's list over L lanes (consecutive
// threads; lane l takes entries l, l + L, ...) and sum the lanes' partials with a shuffle
// butterfly: at the tens of thousands of rows a differentiable scene has, one thread per
// row leaves most warp slots of the GPU empty and every gather's latency exposed.
template <int L>
__device__ __forceinline__ float lanes_sum(float v) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Pressure-solve iteration adjoint, pass A: kappa-bar_i = sum_j gradW_ij.w_ij with
// w_ij = c_j V_i vb_j - c_i V_j vb_i (c = dt V / m; the j term only for fluid j), then
// delta-bar (clamp of the forward), ratio-bar and alpha-bar, and the position adjoint of
// the velocity update: x-bar_i += sum_j (kappa_i + kappa_j) J_ij w_ij.
template <int L>
__global__ void __launch_bounds__(256) k_dfd_iter_a(DfdArgs a) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = g / L, lane = g % L;
    const bool live = r < a.nf;
    float kb = 0.f, xx = 0.f, xy = 0.f, xz = 0.f, ki = 0.f;
    float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
    if (live) {
        p = a.x[r];
        const float4 vi = a.vb[r];
        ki = a.rec[r].w;
        const float ci = a.dt * p.w / a.mass_f;
        const uint32_t n = a.ncnt[r];
        const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
        for (uint32_t t = lane; t + 1 < n; t += L) {
            const uint32_t j = lst[(size_t)t * 32u];
            const float4 q = __ldg(a.x + j);
            const bool fj = j < a.nf;
            const float kj = __ldg(&a.rec[j].w);   // 0 for boundary rows
            const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
            const float d2 = dist2(rx, ry, rz);
            const float gg = cubic_g(d2, a.k), hh = cubic_hh(d2, a.k);
            float wx = -ci * q.w * vi.x, wy = -ci * q.w * vi.y, wz = -ci * q.w * vi.z;
            if (fj) {
                const float4 vj = __ldg(a.vb + j);
                const float cj = a.dt * q.w / a.mass_f * p.w;
                wx += cj * vj.x;
                wy += cj * vj.y;
                wz += cj * vj.z;
            }
            const float rw = rx * wx + ry * wy + rz * wz;
            kb += gg * rw;
            const float kk = ki + kj;
            xx += kk * (gg * wx + hh * rx * rw);
            xy += kk * (gg * wy + hh * ry * rw);
            xz += kk * (gg * wz + hh * rz * rw);
        }
    }
    kb = lanes_sum<L>(kb);
    xx = lanes_sum<L>(xx);
    xy = lanes_sum<L>(xy);
    xz = lanes_sum<L>(xz);
    if (!live || lane != 0) return;
    float4 xb = a.xbar[r];
    xb.x += xx; xb.y += xy; xb.z += xz;
    a.xbar[r] = xb;
    const float al = a.alpha[r];
    const float d = ki > 0.f ? kb / (al * a.dt * a.dt * p.w) : 0.f;
    a.db[r] = d;
    a.rbar[r] += d;
    a.abar[r] -= kb * ki / al;
}

// Pressure-solve iteration adjoint, pass B: the delta term's adjoints,
// vb_i += dt sum_j (V_j db_i + V_i db_j) gradW_ij and
// x-bar_i += dt sum_j (V_j db_i + V_i db_j) J_ij (v*_i - v*_j) (db_j only for fluid j).
template <int L>
__global__ void __launch_bounds__(256) k_dfd_iter_b(DfdArgs a) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = g / L, lane = g % L;
    const bool live = r < a.nf;
    float vx = 0.f, vy = 0.f, vz = 0.f, xx = 0.f, xy = 0.f, xz = 0.f;
    if (live) {
        const float4 p = a.x[r], si = a.rec[r];
        const float di = a.db[r];
        const uint32_t n = a.ncnt[r];
        const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
        for (uint32_t t = lane; t + 1 < n; t += L) {
            const uint32_t j = lst[(size_t)t * 32u];
            const float4 q = __ldg(a.x + j), sj = __ldg(a.rec + j);
            const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
            const float d2 = dist2(rx, ry, rz);
            const float gg = cubic_g(d2, a.k), hh = cubic_hh(d2, a.k);
            const float c = a.dt * (q.w * di + (j < a.nf ? p.w * __ldg(a.db + j) : 0.f));
            const float ux = si.x - sj.x, uy = si.y - sj.y, uz = si.z - sj.z;
            const float ru = rx * ux + ry * uy + rz * uz;
            vx += c * gg * rx;
            vy += c * gg * ry;
            vz += c * gg * rz;
            xx += c * (gg * ux + hh * rx * ru);
            xy += c * (gg * uy + hh * ry * ru);
            xz += c * (gg * uz + hh * rz * ru);
        }
    }
    vx = lanes_sum<L>(vx);
    vy = lanes_sum<L>(vy);
    vz = lanes_sum<L>(vz);
    xx = lanes_sum<L>(xx);
    xy = lanes_sum<L>(xy);
    xz = lanes_sum<L>(xz);
    if (!live || lane != 0) return;
    float4 v = a.vb[r];
    v.x += vx; v.y += vy; v.z += vz;
    a.vb[r] = v;
    float4 xb = a.xbar[r];
    xb.x += xx; xb.y += xy; xb.z += xz;
    a.xbar[r] = xb;
}

// Gravity + viscosity adjoint: vb_out_i = vb_i + dt C sum_{fluid j} phi r (r.(vb_i - vb_j)),
// x-bar_i += dt C sum_j [phi u (r.w) + (u.r)(phi w + psi r (r.w))] with u = vp_i - vp_j,
// w = vb_i - vb_j, phi = g / (|r|^2 + eps), psi = 2 dphi/d|r|^2; block partials of
// dL/dnu / V_f = sum_i dt vb_i . sum_j 10 (u.r) phi r.
template <int L>
__global__ void __launch_bounds__(256) k_dfd_visc(DfdArgs a) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = g / L, lane = g % L;
    const bool live = r < a.nf;
    float vx = 0.f, vy = 0.f, vz = 0.f, xx = 0.f, xy = 0.f, xz = 0.f, ps = 0.f;
    float4 wi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (live) {
        const float4 p = a.x[r], ui = a.vp[r];
        wi = a.vb[r];
        const uint32_t n = a.ncnt[r];
        const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
        for (uint32_t t = lane; t + 1 < n; t += L) {
            const uint32_t j = lst[(size_t)t * 32u];
            if (j >= a.nf) continue;   // same-material neighbours only
            const float4 q = __ldg(a.x + j), uj = __ldg(a.vp + j), wj = __ldg(a.vb + j);
            const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
            const float d2 = dist2(rx, ry, rz);
            const float gg = cubic_g(d2, a.k), hh = cubic_hh(d2, a.k);
            const float den = d2 + a.eps;
            const float phi = gg / den;
            const float psi = hh / den - 2.f * gg / (den * den);
            const float ux = ui.x - uj.x, uy = ui.y - uj.y, uz = ui.z - uj.z;
            const float wx = wi.x - wj.x, wy = wi.y - wj.y, wz = wi.z - wj.z;
            const float ru = rx * ux + ry * uy + rz * uz, rw = rx * wx + ry * wy + rz * wz;
            const float cv = a.dt * a.vis10 * phi * rw;
            vx += cv * rx;
            vy += cv * ry;
            vz += cv * rz;
            const float cx = a.dt * a.vis10;
            xx += cx * (phi * ux * rw + ru * (phi * wx + psi * rx * rw));
            xy += cx * (phi * uy * rw + ru * (phi * wy + psi * ry * rw));
            xz += cx * (phi * uz * rw + ru * (phi * wz + psi * rz * rw));
            ps += ru * phi * (rx * wi.x + ry * wi.y + rz * wi.z);
        }
    }
    vx = lanes_sum<L>(vx);
    vy = lanes_sum<L>(vy);
    vz = lanes_sum<L>(vz);
    xx = lanes_sum<L>(xx);
    xy = lanes_sum<L>(xy);
    xz = lanes_sum<L>(xz);
    ps = lanes_sum<L>(ps);
    double part = 0.0;
    if (live && lane == 0) {
        a.vb_out[r] = make_float4(wi.x + vx, wi.y + vy, wi.z + vz, 0.f);
        float4 xb = a.xbar[r];
        xb.x += xx; xb.y += xy; xb.z += xz;
        a.xbar[r] = xb;
        part = (double)a.dt * 10.0 * (double)ps;
    }
    const double s = block_sum_d(part);
    if (threadIdx.x == 0) a.vpart[blockIdx.x] = s;
}

__global__ void k_dfd_vreduce(const double *part, uint32_t nb, double vol_f, double *acc) {
    double s = 0.0;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) s += part[b];
    s = block_sum_d(s);
    if (threadIdx.x == 0) *acc += s * vol_f;
}

// alpha adjoint, pass 1: a1-bar_i = alpha-bar_i 2 a1_i / m (a1 recomputed), with
// alpha-bar zeroed where the forward clamped alpha; stored {a1-bar, alpha-bar}.
template <int L>
__global__ void __launch_bounds__(256) k_dfd_a1(DfdArgs a) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = g / L, lane = g % L;
    const bool live = r < a.nf && a.alpha[r] > 1e-6f;
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (live) {
        const float4 p = a.x[r];
        const uint32_t n = a.ncnt[r];
        const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
        for (uint32_t t = lane; t + 1 < n; t += L) {
            const uint32_t j = lst[(size_t)t * 32u];
            const float4 q = __ldg(a.x + j);
            const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
            const float gg = cubic_g(dist2(rx, ry, rz), a.k) * q.w;
            ax += gg * rx;
            ay += gg * ry;
            az += gg * rz;
        }
    }
    ax = lanes_sum<L>(ax);
    ay = lanes_sum<L>(ay);
    az = lanes_sum<L>(az);
    if (r >= a.nf || lane != 0) return;
    const float ab = live ? a.abar[r] : 0.f;
    const float c = 2.f * ab / a.mass_f;
    a.a1b[r] = make_float4(c * ax, c * ay, c * az, ab);
}

// ratio / alpha adjoint, pass 2: x-bar_i += sum_j (ratio-bar_i V_j + ratio-bar_j V_i) g r
// + J (V_j a1-bar_i - V_i a1-bar_j) + 2 g (g + hh |r|^2) (alpha-bar_i V_j^2 + alpha-bar_j V_i^2) / m r
// (the j terms only for fluid j); then this substep's rows -> attach order.
template <int L>
__global__ void __launch_bounds__(256) k_dfd_ratio_x(DfdArgs a) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = g / L, lane = g % L;
    const bool live = r < a.nf;
    float xx = 0.f, xy = 0.f, xz = 0.f;
    if (live) {
        const float4 p = a.x[r], Ai = a.a1b[r];
        const float rbi = a.rbar[r];
        const uint32_t n = a.ncnt[r];
        const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
        const float im = 1.f / a.mass_f;
        for (uint32_t t = lane; t + 1 < n; t += L) {
            const uint32_t j = lst[(size_t)t * 32u];
            const float4 q = __ldg(a.x + j);
            const bool fj = j < a.nf;
            const float4 Aj = fj ? __ldg(a.a1b + j) : make_float4(0.f, 0.f, 0.f, 0.f);
            const float rbj = fj ? __ldg(a.rbar + j) : 0.f;
            const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
            const float d2 = dist2(rx, ry, rz);
            const float gg = cubic_g(d2, a.k), hh = cubic_hh(d2, a.k);
            const float cr = rbi * q.w + rbj * p.w;
            const float c2 = fj ? 2.f * gg * (gg + hh * d2) * (Ai.w * q.w * q.w + Aj.w * p.w * p.w) * im : 0.f;
            const float wx = q.w * Ai.x - p.w * Aj.x, wy = q.w * Ai.y - p.w * Aj.y, wz = q.w * Ai.z - p.w * Aj.z;
            const float rw = rx * wx + ry * wy + rz * wz;
            const float s = cr * gg + c2;
            xx += s * rx + gg * wx + hh * rx * rw;
            xy += s * ry + gg * wy + hh * ry * rw;
            xz += s * rz + gg * wz + hh * rz * rw;
        }
    }
    xx = lanes_sum<L>(xx);
    xy = lanes_sum<L>(xy);
    xz = lanes_sum<L>(xz);
    if (!live || lane != 0) return;
    float4 xb = a.xbar[r];
    xb.x += xx; xb.y += xy; xb.z += xz;
    const uint32_t id = a.orig[r];
    a.xbar_a[id] = xb;
    a.vbar_a[id] = a.vb[r];
}

__global__ void k_f3_to_f4(uint32_t n, const float *src, float4 *dst) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = src ? make_float4(src[3 * (size_t)i], src[3 * (size_t)i + 1], src[3 * (size_t)i + 2], 0.f)
                 : make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void k_f4_to_f3(uint32_t n, const float4 *src, float *dst) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = src[i];
    dst[3 * (size_t)i] = v.x;
    dst[3 * (size_t)i + 1] = v.y;
    dst[3 * (size_t)i + 2] = v.z;
}

__global__ void k_bstat(uint32_t nf, uint32_t n, const float4 *__restrict__ vadv, float4 *__restrict__ out) {
    const uint32_t i = nf + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = vadv[i];
    out[i] = make_float4(v.x, v.y, v.z, 0.f);
}

}  // namespace
}  // namespace vtp

using vtp::fail;

#define CU(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return fail(VTP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

using vtp::DfDiffState;
using vtp::DfTape;
using vtp::DfTapeSlot;

int df_save(vtp_solver &s, float4 *p, float4 *v, uint32_t *o) {
    const size_t nf = s.L.nf;
    if (!nf) return VTP_OK;
    CU(cudaMemcpyAsync(p, s.pos.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(v, s.vel.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(o, s.orig.c(), nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s.st));
    return VTP_OK;
}

// A substep starts from v* = v (the finalize pass leaves them equal).
int df_restore(vtp_solver &s, const float4 *p, const float4 *v, const uint32_t *o) {
    const size_t nf = s.L.nf;
    if (!nf) return VTP_OK;
    CU(cudaMemcpyAsync(s.pos.c(), p, nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(s.vel.c(), v, nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(s.vadv.c(), v, nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(s.orig.c(), o, nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s.st));
    return VTP_OK;
}

// The record of iteration `k` of the tape's pool, allocated (with its static boundary rows) on
// first use.
int df_record_slot(vtp_solver &s, DfDiffState &d, DfTape &tape, uint32_t k, float4 **out) {
    while (tape.recs.size() <= k) {
        float4 *p = nullptr;
        int rc = d.alloc(&p, d.n);
        if (rc) return rc;
        if (d.n > d.nf)
            CU(cudaMemcpyAsync(p + d.nf, d.bstat + d.nf, (size_t)(d.n - d.nf) * sizeof(float4),
                               cudaMemcpyDeviceToDevice, s.st));
        tape.recs.push_back(p);
    }
    *out = tape.recs[k];
    return VTP_OK;
}

// One pressure solve of a recording substep, host-driven, each iteration's {v*, kappa}
// recorded.  The stop test is the solver's (its constant forced counts included; a
// per-substep forced sequence is not followed).
int df_record_solve(vtp_solver &s, DfDiffState &d, DfTape &tape, DfTapeSlot &slot, int which, uint32_t &pool) {
    const vtp::NvtxRange nvtx_range(which == 0 ? "vtp divergence solve (recorded)" : "vtp density solve (recorded)");
    vtp::DfsphArgs a = s.dfsph_args(which);
    a.nbr = slot.nbr;
    a.ncnt = slot.ncnt;
    a.staged = 0;
    vtp::SolveCtl c = s.solve_ctl(which, cudaGraphConditionalHandle{}, 0);
    c.force_iters = which == 0 ? s.force_div : s.force_inc;
    c.force_seq = nullptr;
    c.scene_tiles = s.d_scene_tiles;   // the unstaged passes write one residual partial per tile
    vtp::dfsph_solve_begin(s.st, s.solve + (size_t)which * s.scenes.size(), s.loop + which, 1);
    vtp::dfsph_solve_pack(s.st, a);
    slot.first[which] = pool;
    const uint32_t nf = s.L.nf;
    // Iterations are enqueued in chunks and the stop flag read once per chunk: an iteration
    // enqueued after the stop test has stopped the solve is a no-op (solve_a and solve_b skip a
    // stopped scene's tiles, solve_end leaves its state alone), and its record lands in a slot
    // past the solve's last, which the next solve overwrites.  The first chunk is as long as
    // the previous substep's solve of this kind was.
    const vtp::SolveState *state = s.solve + (size_t)which * s.scenes.size();
    uint32_t issued = 0, iters = 0;
    uint32_t chunk = std::max<uint32_t>(d.hint[which], 1u);
    for (;;) {
        for (uint32_t c2 = 0; c2 < chunk; ++c2, ++issued) {
            float4 *rec = nullptr;
            int rc = df_record_slot(s, d, tape, pool + issued, &rec);
            if (rc) return rc;
            vtp::dfsph_solve_a(s.st, a, s.block);
            if (nf) vtp::k_dfd_record<<<vtp::nblk(nf, 256), 256, 0, s.st>>>(nf, a.vadv, a.kappa, rec);
            vtp::dfsph_solve_b(s.st, a, s.block);
            vtp::dfsph_solve_end(s.st, c, s.partials, s.d_status);
        }
        CU(cudaMemcpyAsync(s.h_pinned + 2, state, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s.st));
        CU(cudaStreamSynchronize(s.st));
        iters = s.h_pinned[2];
        if (s.h_pinned[3] || issued >= 101) break;   // stopped (the stop test ends every solve by 101)
        chunk = 2;
    }
    iters = std::min<uint32_t>(std::max<uint32_t>(iters, 1u), 101u);
    pool += iters;
    slot.iters[which] = iters;
    d.hint[which] = iters;
    return VTP_OK;
}

// One DFSPH substep recording into `slot` (the buffer swaps of enqueue_tick, so the substep
// graphs' parities stay valid).  recompute: leave the device substep counter alone (the
// iteration counts come from the stop test, which sees the forward's bits again).
int df_record_substep(vtp_solver &s, DfDiffState &d, DfTape &tape, DfTapeSlot &slot, uint32_t &pool,
                      bool recompute) {
    const vtp::NvtxRange nvtx_range("vtp DFSPH substep (recorded)");
    const uint32_t nf = s.L.nf;
    cudaStream_t st = s.st;
    vtp::Carry carry{};
    carry.nf4 = 1;
    carry.src4[0] = s.vadv.c();
    carry.dst4[0] = s.vadv.n();
    vtp::ugns_sort(st, s.scn(), s.nbuckets, 0, nf, s.pos.c(), s.pos.n(), s.vel.c(), s.vel.n(), s.orig.c(),
                   s.orig.n(), carry, 0.f, s.u, s.u.fstart);
    s.pos.swap(); s.vel.swap(); s.orig.swap(); s.vadv.swap();
    vtp::ugns_build_lists(st, s.scn(), s.L, 0, nf, s.pos.c(), s.orig.c(), s.u, slot.nbr, slot.ncnt, s.d_status,
                          s.d_overflow, s.block);
    if (nf) {
        CU(cudaMemcpyAsync(slot.orig, s.orig.c(), nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        CU(cudaMemcpyAsync(slot.x, s.pos.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    }
    vtp::DfsphArgs a = s.dfsph_args();
    a.nbr = slot.nbr;
    a.ncnt = slot.ncnt;
    a.staged = 0;
    vtp::dfsph_ratio_alpha(st, a, s.block);
    if (nf) CU(cudaMemcpyAsync(slot.alpha, s.alpha, nf * sizeof(float), cudaMemcpyDeviceToDevice, st));
    int rc;
    if ((rc = df_record_solve(s, d, tape, slot, 0, pool))) return rc;
    a = s.dfsph_args();
    a.nbr = slot.nbr;
    a.ncnt = slot.ncnt;
    a.staged = 0;
    vtp::dfsph_pressure_pack(st, a);
    if (nf) vtp::k_dfd_vp<<<vtp::nblk(nf, 256), 256, 0, st>>>(nf, s.pva, slot.vp);
    vtp::dfsph_viscosity(st, a, s.block);
    s.vel.swap(); s.vadv.swap();
    if ((rc = df_record_solve(s, d, tape, slot, 1, pool))) return rc;
    a = s.dfsph_args();
    a.nbr = slot.nbr;
    a.ncnt = slot.ncnt;
    if (recompute) a.tick = nullptr;
    vtp::dfsph_finalize(st, a);
    return VTP_OK;
}

// A segment recorded with host-driven solve loops.
int df_record_segment_host(vtp_solver &s, DfDiffState &d, uint32_t k, int tp, bool recompute) {
    DfTape &tape = d.tapes[tp];
    uint32_t pool = 0;
    for (uint32_t t = 0; t < k; ++t) {
        int rc = df_record_substep(s, d, tape, tape.slots[t], pool, recompute);
        if (rc) return rc;
    }
    CU(cudaStreamSynchronize(s.st));
    return s.check_status();
}

// Copies the record pointers the host-side pool has gained to the tape's device table (rare:
// only when the pool grows; synchronous).
int df_upload_recs(vtp_solver &s, DfTape &tape) {
    const uint32_t n = (uint32_t)std::min<size_t>(tape.recs.size(), vtp::kRecTable);
    if (n == tape.uploaded) return VTP_OK;
    CU(cudaStreamSynchronize(s.st));
    CU(cudaMemcpy(tape.d_recs + tape.uploaded, tape.recs.data() + tape.uploaded,
                  (size_t)(n - tape.uploaded) * sizeof(float4 *), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(tape.d_cap, &n, sizeof(uint32_t), cudaMemcpyHostToDevice));
    tape.uploaded = n;
    return VTP_OK;
}

// One pressure solve of a graph-recorded substep (being captured on s.st): the solve loop as a
// WHILE node whose body is solve_a, the record, solve_b and the stop test, then the solve's
// first record and iteration count into `info`.
int df_capture_solve(vtp_solver &s, DfTape &tape, DfTapeSlot &slot, int which, uint32_t *info) {
    vtp::DfsphArgs a = s.dfsph_args(which);
    a.nbr = slot.nbr;
    a.ncnt = slot.ncnt;
    a.staged = 0;
    vtp::SolveState *state = s.solve + (size_t)which * s.scenes.size();
    vtp::dfsph_solve_begin(s.st, state, s.loop + which, 1);
    vtp::dfsph_solve_pack(s.st, a);
    cudaStreamCaptureStatus cs;
    cudaGraph_t g;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CU(cudaStreamGetCaptureInfo(s.st, &cs, nullptr, &g, &deps, &ndeps));
    cudaGraphConditionalHandle hnd;
    CU(cudaGraphConditionalHandleCreate(&hnd, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hnd;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CU(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CU(cudaStreamUpdateCaptureDependencies(s.st, &node, 1, cudaStreamSetCaptureDependencies));
    CU(cudaStreamBeginCaptureToGraph(s.side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    vtp::SolveCtl c = s.solve_ctl(which, hnd, 1);
    c.force_iters = which == 0 ? s.force_div : s.force_inc;
    c.force_seq = nullptr;
    c.scene_tiles = s.d_scene_tiles;   // the unstaged passes write one residual partial per tile
    const uint32_t nf = s.L.nf;
    vtp::dfsph_solve_a(s.side, a, s.block);
    if (nf)
        vtp::k_dfd_record_dev<<<vtp::nblk(nf, 256), 256, 0, s.side>>>(nf, a.vadv, a.kappa, state, tape.d_recs,
                                                                      tape.d_cap, tape.d_ctl);
    vtp::dfsph_solve_b(s.side, a, s.block);
    vtp::dfsph_solve_end(s.side, c, s.partials, s.d_status);
    cudaGraph_t out;
    CU(cudaStreamEndCapture(s.side, &out));
    vtp::k_dfd_solve_done<<<1, 32, 0, s.st>>>(state, tape.d_ctl, info);
    return VTP_OK;
}

// One substep of a graph-recorded segment (being captured): df_record_substep with the solve
// loops as WHILE nodes and the device substep counter left alone.
int df_capture_substep(vtp_solver &s, DfTape &tape, DfTapeSlot &slot, uint32_t *info) {
    const uint32_t nf = s.L.nf;
    cudaStream_t st = s.st;
    vtp::Carry carry{};
    carry.nf4 = 1;
    carry.src4[0] = s.vadv.c();
    carry.dst4[0] = s.vadv.n();
    vtp::ugns_sort(st, s.scn(), s.nbuckets, 0, nf, s.pos.c(), s.pos.n(), s.vel.c(), s.vel.n(), s.orig.c(),
                   s.orig.n(), carry, 0.f, s.u, s.u.fstart);
    s.pos.swap(); s.vel.swap(); s.orig.swap(); s.vadv.swap();
    vtp::ugns_build_lists(st, s.scn(), s.L, 0, nf, s.pos.c(), s.orig.c(), s.u, slot.nbr, slot.ncnt, s.d_status,
                          s.d_overflow, s.block);
    if (nf) {
        CU(cudaMemcpyAsync(slot.orig, s.orig.c(), nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        CU(cudaMemcpyAsync(slot.x, s.pos.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, st));
    }
    vtp::DfsphArgs a = s.dfsph_args();
    a.nbr = slot.nbr;
    a.ncnt = slot.ncnt;
    a.staged = 0;
    vtp::dfsph_ratio_alpha(st, a, s.block);
    if (nf) CU(cudaMemcpyAsync(slot.alpha, s.alpha, nf * sizeof(float), cudaMemcpyDeviceToDevice, st));
    int rc;
    if ((rc = df_capture_solve(s, tape, slot, 0, info))) return rc;
    a = s.dfsph_args();
    a.nbr = slot.nbr;
    a.ncnt = slot.ncnt;
    a.staged = 0;
    vtp::dfsph_pressure_pack(st, a);
    if (nf) vtp::k_dfd_vp<<<vtp::nblk(nf, 256), 256, 0, st>>>(nf, s.pva, slot.vp);
    vtp::dfsph_viscosity(st, a, s.block);
    s.vel.swap(); s.vadv.swap();
    if ((rc = df_capture_solve(s, tape, slot, 1, info + 2))) return rc;
    a = s.dfsph_args();
    a.nbr = slot.nbr;
    a.ncnt = slot.ncnt;
    a.tick = nullptr;
    vtp::dfsph_finalize(st, a);
    return VTP_OK;
}

// A segment of `every` substeps (an even number, so it ends at the buffer parity it started
// from) replayed from the tape's captured graph: no readback until its end, where the solves'
// records and iteration counts come back.  If the record table ran out, it is grown to the
// segment's iteration total and the segment replayed from its checkpoint (ck_*), which the
// solver's state equals on entry.  Returns 1 (nothing done) when the graph path does not apply.
int df_record_segment_graph(vtp_solver &s, DfDiffState &d, uint32_t k, int tp, const float4 *ck_p,
                            const float4 *ck_v, const uint32_t *ck_o) {
    DfTape &tape = d.tapes[tp];
    if (!s.use_graphs || k != d.every || k % 2 != 0 || !d.nf || !tape.d_recs) return 1;
    const int par[4] = {s.pos.cur, s.vel.cur, s.orig.cur, s.vadv.cur};
    int rc;
    if (!tape.exec) {
        // records for one iteration of each solve to start with; the table grows on overflow
        float4 *rec = nullptr;
        if ((rc = df_record_slot(s, d, tape, 2 * k - 1, &rec)) || (rc = df_upload_recs(s, tape))) return rc;
        CU(cudaStreamBeginCapture(s.st, cudaStreamCaptureModeRelaxed));
        cudaMemsetAsync(tape.d_ctl, 0, 2 * sizeof(uint32_t), s.st);
        rc = VTP_OK;
        for (uint32_t t = 0; t < k && !rc; ++t) rc = df_capture_substep(s, tape, tape.slots[t], tape.d_info + 4 * (size_t)t);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(s.st, &g);
        const bool same = s.pos.cur == par[0] && s.vel.cur == par[1] && s.orig.cur == par[2] && s.vadv.cur == par[3];
        s.pos.cur = par[0]; s.vel.cur = par[1]; s.orig.cur = par[2]; s.vadv.cur = par[3];
        cudaError_t e = !rc && ec == cudaSuccess && same ? cudaGraphInstantiate(&tape.exec, g, 0) : cudaErrorInvalidValue;
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {   // record this tape's segments with host-driven solves instead
            cudaGetLastError();
            tape.exec = nullptr;
            tape.d_recs = nullptr;
            return 1;
        }
        std::copy(par, par + 4, tape.par);
    }
    if (!std::equal(par, par + 4, tape.par)) return 1;
    for (int attempt = 0; attempt < 2; ++attempt) {
        CU(cudaMemcpyAsync(s.h_pinned + 4, s.d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s.st));
        CU(cudaMemcpyAsync(s.h_pinned + 5, s.d_overflow, sizeof(uint32_t), cudaMemcpyDeviceToHost, s.st));
        CU(cudaGraphLaunch(tape.exec, s.st));
        CU(cudaMemcpyAsync(d.h_info, tape.d_info, 4 * (size_t)k * sizeof(uint32_t), cudaMemcpyDeviceToHost, s.st));
        CU(cudaMemcpyAsync(d.h_info + 4 * (size_t)k, tape.d_ctl, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s.st));
        CU(cudaStreamSynchronize(s.st));
        if (!d.h_info[4 * (size_t)k + 1]) break;   // every record fitted
        // Grow the table to the segment's iteration total (the counts are right: only
        // records were skipped) and replay from the checkpoint, status words restored.
        const uint32_t total = d.h_info[4 * (size_t)k];
        if (attempt == 1 || total > vtp::kRecTable) return 2;
        float4 *rec = nullptr;
        if ((rc = df_record_slot(s, d, tape, total - 1, &rec)) || (rc = df_upload_recs(s, tape))) return rc;
        if ((rc = df_restore(s, ck_p, ck_v, ck_o))) return rc;
        CU(cudaMemcpyAsync(s.d_status, s.h_pinned + 4, sizeof(uint32_t), cudaMemcpyHostToDevice, s.st));
        CU(cudaMemcpyAsync(s.d_overflow, s.h_pinned + 5, sizeof(uint32_t), cudaMemcpyHostToDevice, s.st));
    }
    for (uint32_t t = 0; t < k; ++t)
        for (int w = 0; w < 2; ++w) {
            tape.slots[t].first[w] = d.h_info[4 * t + 2 * w];
            tape.slots[t].iters[w] = std::min<uint32_t>(std::max<uint32_t>(d.h_info[4 * t + 2 * w + 1], 1u), 101u);
        }
    return VTP_OK;
}

// The k substeps of a checkpoint segment recorded into tape `tp`, from checkpoint (ck_*),
// which the solver's state equals on entry: replayed from the tape's graph where that applies,
// else with host-driven solve loops.  forward: the device substep counter advances by k.
int df_record_segment(vtp_solver &s, DfDiffState &d, uint32_t k, int tp, bool forward, const float4 *ck_p,
                      const float4 *ck_v, const uint32_t *ck_o) {
    int rc = df_record_segment_graph(s, d, k, tp, ck_p, ck_v, ck_o);
    if (rc == VTP_OK) {
        if (forward && s.d_tick) vtp::k_dfd_tick_add<<<1, 32, 0, s.st>>>(s.d_tick, k);
        CU(cudaStreamSynchronize(s.st));
        return s.check_status();
    }
    if (rc == 2) {   // the record table cannot hold the segment: host-driven from the checkpoint
        if ((rc = df_restore(s, ck_p, ck_v, ck_o))) return rc;
        CU(cudaMemcpyAsync(s.d_status, s.h_pinned + 4, sizeof(uint32_t), cudaMemcpyHostToDevice, s.st));
        CU(cudaMemcpyAsync(s.d_overflow, s.h_pinned + 5, sizeof(uint32_t), cudaMemcpyHostToDevice, s.st));
    } else if (rc != 1) {
        return rc;
    }
    return df_record_segment_host(s, d, k, tp, !forward);
}

// Lanes per row of the adjoint's neighbour passes: enough rows x lanes to fill the GPU's
// thread slots (148 SMs x 2048), at most 8.
int df_lanes(uint32_t nf) {
    const uint64_t slots = 148ull * 2048ull;
    int l = 1;
    while (l < 8 && (uint64_t)nf * l < slots) l *= 2;
    return l;
}

template <int L>
int df_adjoint_segment_l(vtp_solver &s, DfDiffState &d, uint32_t k, int tp) {
    const uint32_t nf = d.nf;
    const DfTape &tape = d.tapes[tp];
    const unsigned G = vtp::nblk(nf, 256), GL = vtp::nblk(nf * (uint32_t)L, 256);
    vtp::DfdArgs a{};
    a.nf = nf; a.ell_stride = s.L.ell_stride; a.k = s.kc;
    a.dt = s.dt; a.mass_f = s.rho_f * s.vol0;
    a.vis10 = 10.f * ((s.viscosity + s.viscosity) / 2 * a.mass_f / s.rho_f);
    a.eps = 0.001f * (s.h * s.h);
    a.xbar = d.xbar; a.a1b = d.a1b; a.db = d.db; a.rbar = d.rbar; a.abar = d.abar;
    a.xbar_a = d.xbar_a; a.vbar_a = d.vbar_a; a.vpart = d.vpart;
    for (int t = (int)k - 1; t >= 0; --t) {
        const DfTapeSlot &T = tape.slots[t];
        a.nbr = T.nbr; a.ncnt = T.ncnt; a.orig = T.orig; a.x = T.x; a.vp = T.vp; a.alpha = T.alpha;
        int cur = 0;
        a.vb = d.vb[cur];
        vtp::k_dfd_gather<<<G, 256, 0, s.st>>>(a);
        for (int w = 1; w >= 0; --w) {
            for (int it = (int)T.iters[w] - 1; it >= 0; --it) {
                a.rec = tape.recs[T.first[w] + it];
                vtp::k_dfd_iter_a<L><<<GL, 256, 0, s.st>>>(a);
                vtp::k_dfd_iter_b<L><<<GL, 256, 0, s.st>>>(a);
            }
            if (w == 1) {
                a.vb_out = d.vb[cur ^ 1];
                vtp::k_dfd_visc<L><<<GL, 256, 0, s.st>>>(a);
                vtp::k_dfd_vreduce<<<1, 256, 0, s.st>>>(d.vpart, GL, (double)s.vol0, d.vacc);
                cur ^= 1;
                a.vb = d.vb[cur];
            }
        }
        vtp::k_dfd_a1<L><<<GL, 256, 0, s.st>>>(a);
        vtp::k_dfd_ratio_x<L><<<GL, 256, 0, s.st>>>(a);
    }
    CU(cudaGetLastError());
    return VTP_OK;
}

int df_adjoint_segment(vtp_solver &s, DfDiffState &d, uint32_t k, int tp) {
    if (!d.nf) return VTP_OK;
    switch (df_lanes(d.nf)) {
        case 1: return df_adjoint_segment_l<1>(s, d, k, tp);
        case 2: return df_adjoint_segment_l<2>(s, d, k, tp);
        case 4: return df_adjoint_segment_l<4>(s, d, k, tp);
        default: return df_adjoint_segment_l<8>(s, d, k, tp);
    }
}

// Forward of a recorded rollout: checkpoint, then the ordinary substeps up to the next
// checkpoint, or (the last segments) recording substeps into the tapes.
int df_record_rollout(vtp_solver &s, DfDiffState &d) {
    const uint32_t nchk = (d.steps + d.every - 1) / d.every;
    const uint32_t ntapes = (uint32_t)d.tapes.size();
    int rc;
    d.taped.assign(nchk, -1);
    for (uint32_t c = 0; c < nchk; ++c) {
        if ((rc = df_save(s, d.ck_pos[c], d.ck_vel[c], d.ck_orig[c]))) return rc;
        const uint32_t k = std::min(d.every, d.steps - c * d.every);
        if (c + ntapes >= nchk) {
            const int tp = (int)(c + ntapes - nchk);
            if ((rc = df_record_segment(s, d, k, tp, true, d.ck_pos[c], d.ck_vel[c], d.ck_orig[c]))) return rc;
            for (uint32_t t = 0; t < k; ++t) {   // as tick_n advances them for the segments before
                s.sim_time += s.dt;
                ++s.steps_done;
            }
            s.stats.steps_done = s.steps_done;
            s.stats.sim_time = s.sim_time;
            d.taped[c] = tp;
            continue;
        }
        if ((rc = s.tick_n(k))) return rc;
    }
    if ((rc = df_save(s, d.ck_pos[nchk], d.ck_vel[nchk], d.ck_orig[nchk]))) return rc;
    CU(cudaStreamSynchronize(s.st));
    return s.check_status();
}

}  // namespace

namespace vtp {

int dfsph_diff_ready(vtp_solver *s) {
    if (s->nscenes() != 1) return fail(VTP_ERR_CONFIG, "differentiable mode runs a single scene");
    if (s->cfl > 0.f) return fail(VTP_ERR_CONFIG, "differentiable DFSPH takes the fixed time step (no \"cfl\")");
    if (s->gamma != 0.f)
        return fail(VTP_ERR_CONFIG, "differentiable DFSPH has no surface-tension adjoint (surfaceTensionCoefficient must be 0)");
    return VTP_OK;
}

int dfsph_diff_forward(vtp_solver *s, uint32_t n_steps, uint32_t checkpoint_every, int keep_lists) {
    const NvtxRange nvtx_range("vtp DFSPH diff forward");
    int rc = dfsph_diff_ready(s);
    if (rc) return rc;
    if (!s->initialized && (rc = s->initialize())) return rc;
    if (s->crashed) return fail(VTP_ERR_STATE, "solver is crashed");
    if (n_steps == 0 || checkpoint_every == 0) return fail(VTP_ERR_ARG, "n_steps and checkpoint_every must be > 0");
    const uint32_t every = std::min(checkpoint_every, n_steps);
    const uint32_t nchk = (n_steps + every - 1) / every;
    const size_t nf = std::max<uint32_t>(s->L.nf, 1), n = std::max<uint32_t>(s->L.n, 1);
    const size_t lrows = ((size_t)s->L.nf + 31) / 32 * 32 * s->L.ell_stride;
    // Tapes kept resident: as many segments' as the budget and half the free memory allow
    // (all of them with keep_lists), estimated at 8 iteration records per substep.
    const size_t slot_bytes = 4 * nf * 2 + 4 * std::max<size_t>(lrows, 1) + 16 * n + 16 * nf + 4 * nf + 16 * n * 8;
    const size_t tape_bytes = std::max<size_t>(slot_bytes * every, 1);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    const size_t budget = std::min<size_t>((size_t)s->tape_budget_mb << 20, free_b / 2);
    const uint32_t ntapes =
        keep_lists ? nchk : (uint32_t)std::min<size_t>(std::max<size_t>(budget / tape_bytes, 1), nchk);
    // A rollout of the same shape as the previous one reuses its checkpoints, tapes and work
    // arrays (the free memory the estimate reads has shrunk by them since).
    if (s->dfdiff && s->dfdiff->steps == n_steps && s->dfdiff->every == every &&
        s->dfdiff->keep_lists == (keep_lists != 0) && s->dfdiff->nf == s->L.nf && s->dfdiff->n == s->L.n)
        return df_record_rollout(*s, *s->dfdiff);
    auto d = std::make_shared<DfDiffState>();
    d->steps = n_steps;
    d->every = every;
    d->keep_lists = keep_lists != 0;
    d->nf = s->L.nf;
    d->n = s->L.n;
    d->ck_pos.resize(nchk + 1);
    d->ck_vel.resize(nchk + 1);
    d->ck_orig.resize(nchk + 1);
    for (uint32_t c = 0; c <= nchk; ++c)
        if ((rc = d->alloc(&d->ck_pos[c], nf)) || (rc = d->alloc(&d->ck_vel[c], nf)) ||
            (rc = d->alloc(&d->ck_orig[c], nf)))
            return rc;
    if ((rc = d->alloc(&d->bstat, n))) return rc;
    if (s->L.n > s->L.nf)
        k_bstat<<<nblk(s->L.n - s->L.nf, 256), 256, 0, s->st>>>(s->L.nf, s->L.n, s->vadv.c(), d->bstat);
    d->tapes.resize(ntapes);
    if (cudaMallocHost((void **)&d->h_info, (4 * (size_t)every + 2) * sizeof(uint32_t)) != cudaSuccess) {
        d->h_info = nullptr;
        return fail(VTP_ERR_NOMEM, "differentiable DFSPH: page-locked readback buffer");
    }
    for (auto &tape : d->tapes) {
        if ((rc = d->alloc(&tape.d_recs, kRecTable)) || (rc = d->alloc(&tape.d_cap, 1)) ||
            (rc = d->alloc(&tape.d_ctl, 2)) || (rc = d->alloc(&tape.d_info, 4 * (size_t)every)))
            return rc;
        CU(cudaMemsetAsync(tape.d_cap, 0, sizeof(uint32_t), s->st));
        tape.slots.resize(every);
        for (auto &slot : tape.slots) {
            if ((rc = d->alloc(&slot.orig, nf)) || (rc = d->alloc(&slot.nbr, std::max<size_t>(lrows, 1))) ||
                (rc = d->alloc(&slot.ncnt, nf)) || (rc = d->alloc(&slot.x, n)) || (rc = d->alloc(&slot.vp, nf)) ||
                (rc = d->alloc(&slot.alpha, nf)))
                return rc;
            if (s->L.nb)   // boundary rows are static: copy them once
                CU(cudaMemcpyAsync(slot.x + s->L.nf, s->pos.c() + s->L.nf, (size_t)s->L.nb * sizeof(float4),
                                   cudaMemcpyDeviceToDevice, s->st));
        }
    }
    d->blocks = nblk((uint32_t)nf * 8u, 256);   // viscosity partials: one per block at up to 8 lanes per row
    if ((rc = d->alloc(&d->xbar_a, n)) || (rc = d->alloc(&d->vbar_a, n)) || (rc = d->alloc(&d->xbar, nf)) ||
        (rc = d->alloc(&d->vb[0], nf)) || (rc = d->alloc(&d->vb[1], nf)) || (rc = d->alloc(&d->a1b, nf)) ||
        (rc = d->alloc(&d->db, nf)) || (rc = d->alloc(&d->rbar, nf)) || (rc = d->alloc(&d->abar, nf)) ||
        (rc = d->alloc(&d->vpart, d->blocks)) || (rc = d->alloc(&d->vacc, 1)))
        return rc;
    s->dfdiff.reset();
    if ((rc = df_record_rollout(*s, *d))) return rc;
    s->dfdiff = d;
    return VTP_OK;
}

int dfsph_diff_backward(vtp_solver *s, const float *dl_dpos, const float *dl_dvel, float *dl_dpos0,
                        float *dl_dvel0, double *dl_dvis) {
    const NvtxRange nvtx_range("vtp DFSPH diff backward");
    int rc = dfsph_diff_ready(s);
    if (rc) return rc;
    if (!s->dfdiff) return fail(VTP_ERR_STATE, "diff_backward before diff_forward");
    DfDiffState &d = *s->dfdiff;
    const uint32_t n = d.n;
    const size_t n3 = (size_t)n * 3 * sizeof(float);
    if ((rc = s->ensure_stage(n3))) return rc;
    if (dl_dpos) CU(cudaMemcpyAsync(s->stage, dl_dpos, n3, cudaMemcpyHostToDevice, s->st));
    k_f3_to_f4<<<nblk(n, 256), 256, 0, s->st>>>(n, dl_dpos ? s->stage : nullptr, d.xbar_a);
    if (dl_dvel) CU(cudaMemcpyAsync(s->stage, dl_dvel, n3, cudaMemcpyHostToDevice, s->st));
    k_f3_to_f4<<<nblk(n, 256), 256, 0, s->st>>>(n, dl_dvel ? s->stage : nullptr, d.vbar_a);
    CU(cudaMemsetAsync(d.vacc, 0, sizeof(double), s->st));
    const uint32_t nchk = (d.steps + d.every - 1) / d.every;
    for (int c = (int)nchk - 1; c >= 0; --c) {
        const uint32_t t0 = (uint32_t)c * d.every, k = std::min(d.every, d.steps - t0);
        int tp = c < (int)d.taped.size() ? d.taped[c] : -1;
        if (tp < 0) {
            // Recompute the segment from its checkpoint into tape 0 (whose own segment, the
            // earliest one the forward recorded, has been consumed already).  Its iteration
            // counts come from the stop test, which sees the forward's bits again.
            tp = 0;
            if ((rc = df_restore(*s, d.ck_pos[c], d.ck_vel[c], d.ck_orig[c]))) return rc;
            if ((rc = df_record_segment(*s, d, k, 0, false, d.ck_pos[c], d.ck_vel[c], d.ck_orig[c]))) return rc;
        }
        if ((rc = df_adjoint_segment(*s, d, k, tp))) return rc;
    }
    if (!d.keep_lists) d.taped.assign(d.taped.size(), -1);   // tape 0 now holds the first segment's recompute
    if (dl_dpos0) {
        k_f4_to_f3<<<nblk(n, 256), 256, 0, s->st>>>(n, d.xbar_a, s->stage);
        CU(cudaMemcpyAsync(dl_dpos0, s->stage, n3, cudaMemcpyDeviceToHost, s->st));
        CU(cudaStreamSynchronize(s->st));
    }
    if (dl_dvel0) {
        k_f4_to_f3<<<nblk(n, 256), 256, 0, s->st>>>(n, d.vbar_a, s->stage);
        CU(cudaMemcpyAsync(dl_dvel0, s->stage, n3, cudaMemcpyDeviceToHost, s->st));
        CU(cudaStreamSynchronize(s->st));
    }
    double vb = 0.0;
    CU(cudaMemcpyAsync(&vb, d.vacc, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    // Put the forward's final state back so the solver can continue.
    if ((rc = df_restore(*s, d.ck_pos[nchk], d.ck_vel[nchk], d.ck_orig[nchk]))) return rc;
    CU(cudaStreamSynchronize(s->st));
    if (dl_dvis) *dl_dvis = vb;
    return s->check_status();
}

int dfsph_diff_slot(vtp_solver *s, uint32_t step, const uint32_t **orig, const uint32_t **nbr,
                    const uint32_t **ncnt, uint32_t *div_iters, uint32_t *inc_iters) {
    if (!s->dfdiff || !s->dfdiff->keep_lists)
        return fail(VTP_ERR_STATE, "the substep records need diff_forward with keep_lists");
    DfDiffState &d = *s->dfdiff;
    if (step >= d.steps) return fail(VTP_ERR_ARG, "step out of range");
    const uint32_t c = step / d.every, t = step % d.every;
    const int tp = c < d.taped.size() ? d.taped[c] : -1;
    if (tp < 0) return fail(VTP_ERR_STATE, "substep not recorded");
    const DfTapeSlot &slot = d.tapes[tp].slots[t];
    if (orig) *orig = slot.orig;
    if (nbr) *nbr = slot.nbr;
    if (ncnt) *ncnt = slot.ncnt;
    if (div_iters) *div_iters = slot.iters[0];
    if (inc_iters) *inc_iters = slot.iters[1];
    return VTP_OK;
}

}  // namespace vtp

extern "C" int vtp_solver_diff_iterations(vtp_solver *s, uint32_t step, uint32_t *div_iters, uint32_t *inc_iters) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    if (s->type != VTP_SOLVER_DFSPH) return fail(VTP_ERR_CONFIG, "pressure-solve iteration counts are DFSPH records");
    return vtp::dfsph_diff_slot(s, step, nullptr, nullptr, nullptr, div_iters, inc_iters);
}
