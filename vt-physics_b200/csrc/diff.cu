// Differentiable PBF: a recorded forward with checkpoints and the hand-written
// adjoint of the PBF substep (no counterpart in the reference).
//
// Forward (vtp_solver_diff_forward): the ordinary substep graphs, with the
// fluid state (positions, velocities, sorted order) saved every k substeps.
// Backward (vtp_solver_diff_backward): for each checkpoint segment, last to
// first, the segment is recomputed from its checkpoint with the substep
// kernels themselves (so the neighbour lists and every intermediate state are
// exactly the forward's) into a tape, then the adjoint substeps run in reverse.
//
// One substep (PBFSolver::tick, PBFSolver.cpp:326-376, as the library runs it):
//   v0 = v + g dt, x0 = x + v0 dt                         (apply_ext_force)
//   for it < I:  rho_i = m_i W0 + sum_j m_j W_ij,  C_i = max(rho_i, rho0)/rho0 - 1
//                e_ij = g_ij r_ij / rho0,  G_i = sum_j e_ij,  s2_i = sum_j |e_ij|^2 + |G_i|^2
//                lambda_i = -C_i / (s2_i + eps)
//                D_i = sum_j (lambda_i + lambda_j) e_ij   (lambda_j = 0 for boundary j)
//                x <- x + D,  v <- v + D / dt
//   a_i = c sum_j V_j (v_j - v_i) W_ij,  x <- x + a dt,  v <- v + a       (XSPH)
// with gradW_ij = g_ij r_ij and d(g r)/dr = g I + hh r r^T (hh = g'(|r|)/|r|).
// The adjoint of every neighbour sum is evaluated in gather form over the
// same lists (pair (i, j) is in i's list iff (j, i) is in j's list while no
// list overflows), so no pass needs atomics: each row reads its neighbours'
// adjoint values of the previous pass.  Boundary rows are static and get no
// adjoint.
#include "solver.h"
#include "diff_dfsph.h"

#include <algorithm>
#include <array>
#include <string>
#include <vector>

namespace vtp {

struct DiffState {
    uint32_t steps = 0, every = 0;     // recorded substeps, checkpoint interval
    bool keep_lists = false;
    uint32_t nf = 0, n = 0;
    std::vector<void *> mem;
    // checkpoints: fluid rows of (pos, vel, orig) at substeps 0, k, 2k, ... and at the end
    std::vector<float4 *> ck_pos, ck_vel;
    std::vector<uint32_t *> ck_orig;
    // Tapes of checkpoint segments (lists and intermediate states of `every` substeps each).
    // The forward records its last `tapes.size()` segments straight into them (segment c into
    // tape taped[c]); every other segment is recomputed from its checkpoint into tape 0 by
    // the backward, after the segments the tapes hold have been consumed.
    std::vector<std::vector<PbfTapeSlot>> tapes;
    std::vector<int> taped;
    // all substeps' lists (keep_lists)
    std::vector<uint32_t *> kl_orig, kl_nbr, kl_cnt;
    // adjoint work arrays
    float4 *xbar_a = nullptr, *vbar_a = nullptr;   // attach order [n]
    float4 *xbar = nullptr, *vbar = nullptr, *abar = nullptr, *D[2] = {nullptr, nullptr}, *A2 = nullptr;
    float *sbar = nullptr;
    double *kpart = nullptr, *kacc = nullptr;
    uint32_t kblocks = 0;
    // DFSPH pressure-solve operator: per-iteration delta (clamp pattern) and work arrays
    int df_which = -1;
    uint32_t df_iters = 0;
    uint64_t df_steps = 0;
    std::vector<float *> df_delta;
    float4 *df_vb = nullptr, *df_save = nullptr;
    float *df_kb = nullptr;

    // A full checkpoint segment's two halves, for each tape, captured once as graphs and
    // replayed for every segment of that length (their pointers are all fixed: the tape, the
    // adjoint arrays, the solver's buffers at the parity a segment starts from): `rec` runs
    // the segment's substeps recording into the tape, `adj` runs the adjoint substeps over it.
    std::vector<cudaGraphExec_t> rec_exec, adj_exec;
    std::vector<std::array<int, 3>> rec_parity;   // pos / vel / orig buffer parity `rec` starts from

    ~DiffState() {
        for (auto e : rec_exec)
            if (e) cudaGraphExecDestroy(e);
        for (auto e : adj_exec)
            if (e) cudaGraphExecDestroy(e);
        for (void *p : mem) cudaFree(p);
    }
    template <class T>
    int alloc(T **p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
        if (e != cudaSuccess) return fail(VTP_ERR_NOMEM, std::string("differentiable mode: ") + cudaGetErrorString(e));
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

// Gathered neighbour data of the adjoint passes.
struct XN {
    float4 q, v, a;
    float vol;
};
struct LN {
    float4 q, d;
};
struct DN {
    float4 q, d, A;
    float l, s;
    bool fj;
};

struct AdjArgs {
    uint32_t nf, ell_stride;
    Cubic k;
    float dt, inv_dt, rho0, eps, c;
    const uint32_t *nbr, *ncnt, *orig;
    const float4 *x;        // positions of the pass (n rows, w = mass)
    const float4 *v;        // velocities before XSPH (n rows)
    const float *vol;       // [n]
    const float *lam, *rho; // [nf] of the iteration
    float4 *xbar, *vbar, *abar, *Dcur, *Dnext, *A2;
    float *sbar;
    float4 *xbar_a, *vbar_a;
    double *kpart;
};

// Attach order -> this substep's rows; abar = xbar dt + vbar (XSPH output adjoint).
__global__ void k_adj_gather(AdjArgs a) {
    pdl_enter();
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const uint32_t id = a.orig[r];
    const float4 xo = a.xbar_a[id], vo = a.vbar_a[id];
    a.xbar[r] = xo;
    a.vbar[r] = vo;
    a.abar[r] = make_float4(xo.x * a.dt + vo.x, xo.y * a.dt + vo.y, xo.z * a.dt + vo.z, 0.f);
}

// The three neighbour passes take L lanes per row ("adjointLanes"; lane_group_mask /
// nbr_loop_lanes / lane_sum of common.cuh): with L = 1 one thread walks the row with four
// neighbours' gathers in flight; with L > 1 the row's lanes take entries lane, lane + L, ...
// (AU gathers in flight each, fewer registers) and a butterfly adds their partials.
template <int L>
constexpr int adj_unroll() { return L == 1 ? 4 : (L == 2 ? 2 : 1); }

// XSPH adjoint; epilogue: Delta-bar of the last constraint iteration.
template <int L>
__global__ void __launch_bounds__(256) k_adj_xsph(AdjArgs a) {
    pdl_enter();
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = gt / L;
    const int lane = (int)(gt % L);
    double kl = 0.0;
    if (r < a.nf) {
        const float4 p = a.x[r], vi = a.v[r], ai = a.abar[r];
        const float Vi = a.vol[r];
        const uint32_t n = a.ncnt[r];
        const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
        float vx = 0.f, vy = 0.f, vz = 0.f, xx = 0.f, xy = 0.f, xz = 0.f, ksum = 0.f;
        nbr_loop_lanes<adj_unroll<L>(), L>(lst, n > 0 ? n - 1 : 0, lane,
                             [&](uint32_t j) {
                                 XN e;
                                 e.q = __ldg(a.x + j);
                                 e.v = __ldg(a.v + j);
                                 e.vol = __ldg(a.vol + j);
                                 e.a = j < a.nf ? __ldg(a.abar + j) : make_float4(0.f, 0.f, 0.f, 0.f);
                                 return e;
                             },
                             [&](uint32_t, const XN &e) {
                                 const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                                 const float d2 = dist2(rx, ry, rz);
                                 const float w = cubic_w(d2, a.k), g = cubic_g(d2, a.k);
                                 const float Vj = e.vol;
                                 const float dx = e.v.x - vi.x, dy = e.v.y - vi.y, dz = e.v.z - vi.z;
                                 const float di = dx * ai.x + dy * ai.y + dz * ai.z;
                                 const float dj = dx * e.a.x + dy * e.a.y + dz * e.a.z;
                                 const float ci = -a.c * Vj * w, cj = a.c * Vi * w;
                                 vx += ci * ai.x + cj * e.a.x;
                                 vy += ci * ai.y + cj * e.a.y;
                                 vz += ci * ai.z + cj * e.a.z;
                                 const float s = a.c * g * (Vj * di - Vi * dj);
                                 xx += s * rx;
                                 xy += s * ry;
                                 xz += s * rz;
                                 ksum += Vj * w * di;
                             });
        const unsigned m = lane_group_mask<L>();
        vx = lane_sum<L>(vx, m); vy = lane_sum<L>(vy, m); vz = lane_sum<L>(vz, m);
        xx = lane_sum<L>(xx, m); xy = lane_sum<L>(xy, m); xz = lane_sum<L>(xz, m);
        ksum = lane_sum<L>(ksum, m);
        if (lane == 0) {
            float4 xb = a.xbar[r], vb = a.vbar[r];
            xb.x += xx; xb.y += xy; xb.z += xz;
            vb.x += vx; vb.y += vy; vb.z += vz;
            a.xbar[r] = xb;
            a.vbar[r] = vb;
            a.Dcur[r] = make_float4(xb.x + vb.x * a.inv_dt, xb.y + vb.y * a.inv_dt, xb.z + vb.z * a.inv_dt, 0.f);
            kl = (double)ksum;
        }
    }
    const double s = block_sum_d(kl);
    if (threadIdx.x == 0) a.kpart[blockIdx.x] = s;
}

// Constraint iteration adjoint, pass A: lambda-bar -> s2-bar, rho-bar; G recomputed.
template <int L>
__global__ void __launch_bounds__(256) k_adj_lambda(AdjArgs a) {
    pdl_enter();
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = gt / L;
    const int lane = (int)(gt % L);
    if (r >= a.nf) return;   // the same for every lane of the row
    const float4 p = a.x[r], di = a.Dcur[r];
    const uint32_t n = a.ncnt[r];
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    const float ir = 1.f / a.rho0;
    float lb = 0.f, gx = 0.f, gy = 0.f, gz = 0.f, s2 = 0.f;
    nbr_loop_lanes<adj_unroll<L>(), L>(lst, n > 0 ? n - 1 : 0, lane,
                         [&](uint32_t j) {
                             LN e;
                             e.q = __ldg(a.x + j);
                             e.d = j < a.nf ? __ldg(a.Dcur + j) : make_float4(0.f, 0.f, 0.f, 0.f);
                             return e;
                         },
                         [&](uint32_t, const LN &e) {
                             const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                             const float g = cubic_g(dist2(rx, ry, rz), a.k) * ir;
                             const float ex = g * rx, ey = g * ry, ez = g * rz;
                             gx += ex; gy += ey; gz += ez;
                             s2 += ex * ex + ey * ey + ez * ez;
                             lb += ex * (di.x - e.d.x) + ey * (di.y - e.d.y) + ez * (di.z - e.d.z);
                         });
    const unsigned m = lane_group_mask<L>();
    lb = lane_sum<L>(lb, m); s2 = lane_sum<L>(s2, m);
    gx = lane_sum<L>(gx, m); gy = lane_sum<L>(gy, m); gz = lane_sum<L>(gz, m);
    if (lane != 0) return;
    s2 += gx * gx + gy * gy + gz * gz;
    const float den = s2 + a.eps;
    const float lam = a.lam[r];
    a.sbar[r] = -lb * lam / den;
    const float rb = a.rho[r] <= a.rho0 ? 0.f : -lb / (den * a.rho0);   // clamped density: no gradient
    a.A2[r] = make_float4(gx, gy, gz, rb);
}

// Constraint iteration adjoint, pass B: xbar of the iteration's input positions;
// epilogue: Delta-bar of the previous iteration.
template <int L>
__global__ void __launch_bounds__(256) k_adj_dx(AdjArgs a) {
    pdl_enter();
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = gt / L;
    const int lane = (int)(gt % L);
    if (r >= a.nf) return;   // the same for every lane of the row
    const float4 p = a.x[r], di = a.Dcur[r], Ai = a.A2[r];
    const float li = a.lam[r], sbi = a.sbar[r];
    const uint32_t n = a.ncnt[r];
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    const float ir = 1.f / a.rho0;
    float ax = 0.f, ay = 0.f, az = 0.f;
    nbr_loop_lanes<adj_unroll<L>(), L>(lst, n > 0 ? n - 1 : 0, lane,
                         [&](uint32_t j) {
                             DN e;
                             e.q = __ldg(a.x + j);
                             e.fj = j < a.nf;
                             if (e.fj) {
                                 e.l = __ldg(a.lam + j);
                                 e.s = __ldg(a.sbar + j);
                                 e.d = __ldg(a.Dcur + j);
                                 e.A = __ldg(a.A2 + j);
                             } else {
                                 e.l = e.s = 0.f;
                                 e.d = e.A = make_float4(0.f, 0.f, 0.f, 0.f);
                             }
                             return e;
                         },
                         [&](uint32_t, const DN &e) {
                             const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                             const float d2 = dist2(rx, ry, rz);
                             const float g = cubic_g(d2, a.k), hh = cubic_hh(d2, a.k);
                             const float ex = g * rx * ir, ey = g * ry * ir, ez = g * rz * ir;
                             const float ll = li + e.l;
                             // e-bar of pair (i, j) minus e-bar of pair (j, i) (zero for a boundary j)
                             float bx = ll * di.x + 2.f * sbi * (ex + Ai.x);
                             float by = ll * di.y + 2.f * sbi * (ey + Ai.y);
                             float bz = ll * di.z + 2.f * sbi * (ez + Ai.z);
                             if (e.fj) {
                                 bx -= ll * e.d.x + 2.f * e.s * (e.A.x - ex);
                                 by -= ll * e.d.y + 2.f * e.s * (e.A.y - ey);
                                 bz -= ll * e.d.z + 2.f * e.s * (e.A.z - ez);
                             }
                             const float rdot = rx * bx + ry * by + rz * bz;
                             const float dens = e.q.w * Ai.w + (e.fj ? p.w * e.A.w : 0.f);   // m_j rho-bar_i + m_i rho-bar_j
                             const float cg = g * dens;
                             ax += cg * rx + (g * bx + hh * rx * rdot) * ir;
                             ay += cg * ry + (g * by + hh * ry * rdot) * ir;
                             az += cg * rz + (g * bz + hh * rz * rdot) * ir;
                         });
    const unsigned m = lane_group_mask<L>();
    ax = lane_sum<L>(ax, m); ay = lane_sum<L>(ay, m); az = lane_sum<L>(az, m);
    if (lane != 0) return;
    float4 xb = a.xbar[r];
    xb.x += ax; xb.y += ay; xb.z += az;
    a.xbar[r] = xb;
    const float4 vb = a.vbar[r];
    a.Dnext[r] = make_float4(xb.x + vb.x * a.inv_dt, xb.y + vb.y * a.inv_dt, xb.z + vb.z * a.inv_dt, 0.f);
}

// External force adjoint, then this substep's rows -> attach order.
__global__ void k_adj_force_scatter(AdjArgs a) {
    pdl_enter();
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const uint32_t id = a.orig[r];
    const float4 xb = a.xbar[r], vb = a.vbar[r];
    a.xbar_a[id] = xb;
    a.vbar_a[id] = make_float4(vb.x + a.dt * xb.x, vb.y + a.dt * xb.y, vb.z + a.dt * xb.z, 0.f);
}

__global__ void k_adj_kreduce(const double *part, uint32_t nb, double *acc) {
    pdl_enter();
    double s = 0.0;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) s += part[b];
    s = block_sum_d(s);
    if (threadIdx.x == 0) *acc += s;
}

// DFSPH pressure-solve adjoint.  One iteration maps v -> v - B kappa(v) with
// kappa_i = P_i max(0, c_i + (A v)_i), (A v)_i = dt sum_j V_j g_ij r_ij.(v_i - v_j),
// (B kappa)_i = c_i sum_j V_j (kappa_i + kappa_j) g_ij r_ij, c_i = dt V_i / m_i,
// P_i = 1 / (alpha_i dt^2 V_i) (vf_update_vel_adv_from_kappa_*, compute_kappa_*,
// DFSPHCudaImpl.cu:142-220); the clamp pattern of each iteration is recorded.
struct DfAdjArgs {
    uint32_t nf, ell_stride;
    Cubic k;
    float dt, inv_dt2, mass_f;
    const uint32_t *nbr, *ncnt;
    const float4 *pos;      // w = volume
    const float *alpha, *delta;
    float4 *vb;
    float *kb;
};

// kappa-bar = -B^T vbar, then delta-bar = P mask kappa-bar (stored in kb).
__global__ void __launch_bounds__(256) k_dadj_kappa(DfAdjArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const float4 p = a.pos[r], vi = a.vb[r];
    const float ci = a.dt * p.w / a.mass_f;
    const uint32_t n = a.ncnt[r];
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    float s = 0.f;
    for (uint32_t t = 0; t + 1 < n; ++t) {
        const uint32_t j = lst[(size_t)t * 32u];
        const float4 q = a.pos[j];
        const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
        const float g = cubic_g(dist2(rx, ry, rz), a.k);
        s -= g * q.w * ci * (rx * vi.x + ry * vi.y + rz * vi.z);
        if (j < a.nf) {
            const float4 vj = a.vb[j];
            s += g * (a.dt * q.w / a.mass_f) * p.w * (rx * vj.x + ry * vj.y + rz * vj.z);
        }
    }
    a.kb[r] = a.delta[r] > 0.f ? s / a.alpha[r] * a.inv_dt2 / p.w : 0.f;
}

// vbar += A^T delta-bar.
__global__ void __launch_bounds__(256) k_dadj_vel(DfAdjArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const float4 p = a.pos[r];
    const float ki = a.kb[r];
    const uint32_t n = a.ncnt[r];
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    float ax = 0.f, ay = 0.f, az = 0.f;
    for (uint32_t t = 0; t + 1 < n; ++t) {
        const uint32_t j = lst[(size_t)t * 32u];
        const float4 q = a.pos[j];
        const float rx = p.x - q.x, ry = p.y - q.y, rz = p.z - q.z;
        const float g = cubic_g(dist2(rx, ry, rz), a.k);
        const float c = a.dt * g * (q.w * ki + (j < a.nf ? p.w * a.kb[j] : 0.f));
        ax += c * rx;
        ay += c * ry;
        az += c * rz;
    }
    float4 v = a.vb[r];
    v.x += ax; v.y += ay; v.z += az;
    a.vb[r] = v;
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

int save_fluid(vtp_solver &s, float4 *p, float4 *v, uint32_t *o) {
    const size_t nf = s.L.nf;
    if (!nf) return VTP_OK;
    CU(cudaMemcpyAsync(p, s.pos.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(v, s.vel.c(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(o, s.orig.c(), nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s.st));
    return VTP_OK;
}

int restore_fluid(vtp_solver &s, const float4 *p, const float4 *v, const uint32_t *o) {
    const size_t nf = s.L.nf;
    if (!nf) return VTP_OK;
    CU(cudaMemcpyAsync(s.pos.c(), p, nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(s.vel.c(), v, nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
    CU(cudaMemcpyAsync(s.orig.c(), o, nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s.st));
    return VTP_OK;
}

int record_rollout(vtp_solver *s, vtp::DiffState &d);

// The k substeps of a checkpoint segment, recording into tape `tp`.
int record_segment(vtp_solver *s, vtp::DiffState &d, uint32_t k, int tp) {
    int rc;
    for (uint32_t t = 0; t < k; ++t)
        if ((rc = s->enqueue_pbf_substep(s->st, &d.tapes[tp][t]))) return rc;
    return VTP_OK;
}

// The adjoint substeps of a recorded segment of k substeps, last to first (programmatic
// launch between their kernels, as in the forward substep).
template <int L>
int adjoint_segment_l(vtp_solver *s, vtp::DiffState &d, uint32_t k, unsigned G, int tp) {
    const uint32_t nf = d.nf;
    const int I = s->iterations;
    const unsigned GL = vtp::nblk(nf * (uint32_t)L, 256);
    const vtp::PdlScope pdl_scope(s->pdl);
    for (int t = (int)k - 1; t >= 0 && nf; --t) {
        const PbfTapeSlot &T = d.tapes[tp][t];
        vtp::AdjArgs a{};
        a.nf = nf; a.ell_stride = s->L.ell_stride; a.k = s->kc;
        a.dt = s->dt; a.inv_dt = 1.f / s->dt; a.rho0 = s->rho_f; a.eps = 1e-6f; a.c = s->xsph_k;
        a.nbr = T.nbr; a.ncnt = T.ncnt; a.orig = T.orig;
        a.v = T.v; a.vol = s->vol;
        a.xbar = d.xbar; a.vbar = d.vbar; a.abar = d.abar; a.A2 = d.A2; a.sbar = d.sbar;
        a.xbar_a = d.xbar_a; a.vbar_a = d.vbar_a; a.kpart = d.kpart;
        int cur = 0;
        a.x = T.x[I];
        a.Dcur = d.D[cur];
        vtp::launch(vtp::k_adj_gather, G, 256, 0, s->st, a);
        vtp::launch(vtp::k_adj_xsph<L>, GL, 256, 0, s->st, a);
        vtp::launch(vtp::k_adj_kreduce, 1, 256, 0, s->st, d.kpart, GL, d.kacc);
        for (int it = I - 1; it >= 0; --it) {
            a.x = T.x[it];
            a.lam = T.lam[it];
            a.rho = T.rho[it];
            a.Dcur = d.D[cur];
            a.Dnext = d.D[cur ^ 1];
            vtp::launch(vtp::k_adj_lambda<L>, GL, 256, 0, s->st, a);
            vtp::launch(vtp::k_adj_dx<L>, GL, 256, 0, s->st, a);
            cur ^= 1;
        }
        vtp::launch(vtp::k_adj_force_scatter, G, 256, 0, s->st, a);
    }
    return VTP_OK;
}

int adjoint_segment(vtp_solver *s, vtp::DiffState &d, uint32_t k, unsigned G, int tp) {
    switch (s->adj_lanes) {
        case 2: return adjoint_segment_l<2>(s, d, k, G, tp);
        case 4: return adjoint_segment_l<4>(s, d, k, G, tp);
        case 8: return adjoint_segment_l<8>(s, d, k, G, tp);
        default: return adjoint_segment_l<1>(s, d, k, G, tp);
    }
}

// Runs `body` (enqueueing a full segment's work on s->st) through the graph `exec`, capturing
// it on first use.  The substep swaps the position buffers 6 times, the velocities twice and
// the sorted order once, so a segment of even length ends at the parity it started from;
// `parity` (when given) records the parity the graph was captured at, and a segment starting
// at another parity, of odd or partial length, or with graphs off, runs `body` directly.
template <class Body>
int run_segment_graph(vtp_solver *s, vtp::DiffState &d, uint32_t k, cudaGraphExec_t &exec, int *parity, Body body) {
    // (parity: 3 ints, or null for a graph that does not touch the solver's buffers)
    const int par[3] = {s->pos.cur, s->vel.cur, s->orig.cur};
    const bool graph_ok = s->use_graphs && k == d.every && k % 2 == 0 && d.nf;
    if (!graph_ok || (exec && parity && !std::equal(par, par + 3, parity))) return body();
    if (!exec) {
        CU(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeRelaxed));
        const int rc = body();
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(s->st, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        const bool same = s->pos.cur == par[0] && s->vel.cur == par[1] && s->orig.cur == par[2];
        cudaError_t e = ec == cudaSuccess && same ? cudaGraphInstantiate(&exec, g, 0) : cudaErrorInvalidValue;
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) {   // run the segment with direct launches instead
            cudaGetLastError();
            exec = nullptr;
            s->pos.cur = par[0]; s->vel.cur = par[1]; s->orig.cur = par[2];
            return body();
        }
        if (parity) std::copy(par, par + 3, parity);
    }
    CU(cudaGraphLaunch(exec, s->st));
    return VTP_OK;
}

int check_ready(vtp_solver *s) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    if (s->type != VTP_SOLVER_PBF) return fail(VTP_ERR_CONFIG, "differentiable mode supports the PBF solver");
    if (s->nscenes() != 1) return fail(VTP_ERR_CONFIG, "differentiable mode runs a single scene");
    if (s->pbf_form != 0) return fail(VTP_ERR_CONFIG, "differentiable mode follows the reference's PBF formulation");
    return VTP_OK;
}

}  // namespace

extern "C" {

int vtp_solver_diff_forward(vtp_solver *s, uint32_t n_steps, uint32_t checkpoint_every, int keep_lists) {
    if (s && s->type == VTP_SOLVER_DFSPH) return vtp::dfsph_diff_forward(s, n_steps, checkpoint_every, keep_lists);
    const vtp::NvtxRange nvtx_range("vtp diff forward");
    int rc = check_ready(s);
    if (rc) return rc;
    if (!s->initialized && (rc = s->initialize())) return rc;
    if (s->crashed) return fail(VTP_ERR_STATE, "solver is crashed");
    if (n_steps == 0 || checkpoint_every == 0) return fail(VTP_ERR_ARG, "n_steps and checkpoint_every must be > 0");
    // Tapes kept in device memory: as many segments' as the budget ("tapeBudgetMB") and half
    // the free device memory allow, at least one (the recompute tape).
    const uint32_t every = std::min(checkpoint_every, n_steps);
    const uint32_t nchk_all = (n_steps + every - 1) / every;
    const int I_it = s->iterations;
    const size_t lrows_all = ((size_t)s->L.nf + 31) / 32 * 32 * s->L.ell_stride;
    const size_t slot_bytes = 4 * (size_t)s->L.nf * 2 + 4 * lrows_all + 16 * (size_t)s->L.n * (I_it + 2) +
                              8 * (size_t)s->L.nf * I_it;
    const size_t tape_bytes = std::max<size_t>(slot_bytes * every, 1);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    const size_t budget = std::min<size_t>((size_t)s->tape_budget_mb << 20, free_b / 2);
    uint32_t ntapes = keep_lists ? 1u : (uint32_t)std::min<size_t>(std::max<size_t>(budget / tape_bytes, 1), nchk_all);
    // A rollout of the same shape as the previous one reuses its checkpoints, tapes and adjoint
    // arrays (a training loop records the same horizon again and again); device memory is
    // allocated only when the shape changes.
    if (s->diff && s->diff->steps == n_steps && s->diff->every == every && s->diff->keep_lists == (keep_lists != 0) &&
        s->diff->nf == s->L.nf && s->diff->n == s->L.n && !s->diff->tapes.empty() &&
        s->diff->tapes.size() <= ntapes) {
        std::shared_ptr<vtp::DiffState> d = s->diff;
        d->df_which = -1;
        return record_rollout(s, *d);
    }
    auto d = std::make_shared<vtp::DiffState>();
    d->steps = n_steps;
    d->every = every;
    d->keep_lists = keep_lists != 0;
    d->nf = s->L.nf;
    d->n = s->L.n;
    const uint32_t nchk = (n_steps + d->every - 1) / d->every;
    const size_t nf = std::max<uint32_t>(d->nf, 1), n = d->n;
    const size_t lrows = ((size_t)d->nf + 31) / 32 * 32 * s->L.ell_stride;
    d->ck_pos.resize(nchk + 1);
    d->ck_vel.resize(nchk + 1);
    d->ck_orig.resize(nchk + 1);
    for (uint32_t c = 0; c <= nchk; ++c) {
        if ((rc = d->alloc(&d->ck_pos[c], nf)) || (rc = d->alloc(&d->ck_vel[c], nf)) ||
            (rc = d->alloc(&d->ck_orig[c], nf)))
            return rc;
    }
    if (d->keep_lists) {
        d->kl_orig.resize(n_steps);
        d->kl_nbr.resize(n_steps);
        d->kl_cnt.resize(n_steps);
        for (uint32_t t = 0; t < n_steps; ++t)
            if ((rc = d->alloc(&d->kl_orig[t], nf)) || (rc = d->alloc(&d->kl_nbr[t], std::max<size_t>(lrows, 1))) ||
                (rc = d->alloc(&d->kl_cnt[t], nf)))
                return rc;
    }
    // The tapes: lists and intermediate states of `every` substeps each.
    const int I = s->iterations;
    d->tapes.resize(ntapes);
    for (auto &tape : d->tapes) {
    tape.resize(d->every);
    for (auto &slot : tape) {
        if ((rc = d->alloc(&slot.orig, nf)) || (rc = d->alloc(&slot.nbr, std::max<size_t>(lrows, 1))) ||
            (rc = d->alloc(&slot.ncnt, nf)) || (rc = d->alloc(&slot.v, n)))
            return rc;
        slot.x.resize(I + 1);
        slot.lam.resize(I);
        slot.rho.resize(I);
        for (auto &x : slot.x) {
            if ((rc = d->alloc(&x, n))) return rc;
            // boundary rows are static: copy them once
            if (s->L.nb)
                CU(cudaMemcpyAsync(x + s->L.nf, s->pos.c() + s->L.nf, (size_t)s->L.nb * sizeof(float4),
                                   cudaMemcpyDeviceToDevice, s->st));
        }
        if (s->L.nb)
            CU(cudaMemcpyAsync(slot.v + s->L.nf, s->vel.c() + s->L.nf, (size_t)s->L.nb * sizeof(float4),
                               cudaMemcpyDeviceToDevice, s->st));
        for (int it = 0; it < I; ++it)
            if ((rc = d->alloc(&slot.lam[it], nf)) || (rc = d->alloc(&slot.rho[it], nf))) return rc;
    }
    }
    d->rec_exec.assign(ntapes, nullptr);
    d->adj_exec.assign(ntapes, nullptr);
    d->rec_parity.assign(ntapes, {-1, -1, -1});
    d->kblocks = vtp::nblk(std::max<uint32_t>(d->nf, 1) * 8u, 256);   // XSPH partials at up to 8 lanes per row
    if ((rc = d->alloc(&d->xbar_a, n)) || (rc = d->alloc(&d->vbar_a, n)) || (rc = d->alloc(&d->xbar, nf)) ||
        (rc = d->alloc(&d->vbar, nf)) || (rc = d->alloc(&d->abar, nf)) || (rc = d->alloc(&d->D[0], nf)) ||
        (rc = d->alloc(&d->D[1], nf)) || (rc = d->alloc(&d->A2, nf)) || (rc = d->alloc(&d->sbar, nf)) ||
        (rc = d->alloc(&d->kpart, d->kblocks)) || (rc = d->alloc(&d->kacc, 1)))
        return rc;
    s->diff.reset();
    if ((rc = record_rollout(s, *d))) return rc;
    s->diff = d;
    return VTP_OK;
}

}  // extern "C"

namespace {
// Forward of a recorded rollout: checkpoint, then the ordinary substeps up to the next checkpoint.
int record_rollout(vtp_solver *s, vtp::DiffState &dd) {
    vtp::DiffState *d = &dd;
    const uint32_t n_steps = d->steps;
    const uint32_t nchk = (n_steps + d->every - 1) / d->every;
    int rc;
    const uint32_t ntapes = (uint32_t)d->tapes.size();
    d->taped.assign(nchk, -1);
    for (uint32_t c = 0; c < nchk; ++c) {
        if ((rc = save_fluid(*s, d->ck_pos[c], d->ck_vel[c], d->ck_orig[c]))) return rc;
        const uint32_t k = std::min(d->every, n_steps - c * d->every);
        if (!d->keep_lists && c + ntapes >= nchk) {
            // The last segments run their substeps recording into the tapes, so the backward
            // starts from them without recomputing them.
            const int tp = (int)(c + ntapes - nchk);
            if (!s->initialized && (rc = s->initialize())) return rc;
            if ((rc = run_segment_graph(s, *d, k, d->rec_exec[tp], d->rec_parity[tp].data(),
                                        [&] { return record_segment(s, *d, k, tp); })))
                return rc;
            for (uint32_t t = 0; t < k; ++t) {   // as tick_n advances them for the segments before
                s->sim_time += s->dt;
                ++s->steps_done;
            }
            s->stats.steps_done = s->steps_done;
            s->stats.sim_time = s->sim_time;
            d->taped[c] = tp;
            continue;
        }
        if (!d->keep_lists) {
            if ((rc = s->tick_n(k))) return rc;
            continue;
        }
        // keep_lists: direct launches, every substep's lists kept
        for (uint32_t t = 0; t < k; ++t) {
            const uint32_t step = c * d->every + t;
            PbfTapeSlot slot = d->tapes[0][0];
            slot.nbr = d->kl_nbr[step];
            slot.ncnt = d->kl_cnt[step];
            slot.orig = d->kl_orig[step];
            if ((rc = s->enqueue_pbf_substep(s->st, &slot))) return rc;
            s->sim_time += s->dt;
            ++s->steps_done;
        }
        CU(cudaStreamSynchronize(s->st));
        if ((rc = s->check_status())) return rc;
    }
    if ((rc = save_fluid(*s, d->ck_pos[nchk], d->ck_vel[nchk], d->ck_orig[nchk]))) return rc;
    CU(cudaStreamSynchronize(s->st));
    return s->check_status();
}
}  // namespace

extern "C" {

int vtp_solver_diff_backward(vtp_solver *s, const float *dl_dpos, const float *dl_dvel, float *dl_dpos0,
                             float *dl_dvel0, double *dl_dxsph_k) {
    if (s && s->type == VTP_SOLVER_DFSPH)
        return vtp::dfsph_diff_backward(s, dl_dpos, dl_dvel, dl_dpos0, dl_dvel0, dl_dxsph_k);
    const vtp::NvtxRange nvtx_range("vtp diff backward");
    int rc = check_ready(s);
    if (rc) return rc;
    if (!s->diff) return fail(VTP_ERR_STATE, "diff_backward before diff_forward");
    vtp::DiffState &d = *s->diff;
    const uint32_t n = d.n, nf = d.nf;
    const size_t n3 = (size_t)n * 3 * sizeof(float);
    const int I = s->iterations;
    int r2 = s->ensure_stage(n3);
    if (r2) return r2;
    // dL/d(final state), attach order
    if (dl_dpos) CU(cudaMemcpyAsync(s->stage, dl_dpos, n3, cudaMemcpyHostToDevice, s->st));
    vtp::k_f3_to_f4<<<vtp::nblk(n, 256), 256, 0, s->st>>>(n, dl_dpos ? s->stage : nullptr, d.xbar_a);
    if (dl_dvel) CU(cudaMemcpyAsync(s->stage, dl_dvel, n3, cudaMemcpyHostToDevice, s->st));
    vtp::k_f3_to_f4<<<vtp::nblk(n, 256), 256, 0, s->st>>>(n, dl_dvel ? s->stage : nullptr, d.vbar_a);
    CU(cudaMemsetAsync(d.kacc, 0, sizeof(double), s->st));
    const uint32_t nchk = (d.steps + d.every - 1) / d.every;
    const unsigned G = vtp::nblk(std::max<uint32_t>(nf, 1), 256);
    for (int c = (int)nchk - 1; c >= 0; --c) {
        const uint32_t t0 = (uint32_t)c * d.every, k = std::min(d.every, d.steps - t0);
        int tp = c < (int)d.taped.size() ? d.taped[c] : -1;
        if (tp < 0) {
            // Recompute the segment from its checkpoint into tape 0 (whose own segment, the
            // earliest one the forward recorded, has been consumed already).
            tp = 0;
            if ((rc = restore_fluid(*s, d.ck_pos[c], d.ck_vel[c], d.ck_orig[c]))) return rc;
            if ((rc = run_segment_graph(s, d, k, d.rec_exec[0], d.rec_parity[0].data(),
                                        [&] { return record_segment(s, d, k, 0); })))
                return rc;
        }
        if ((rc = run_segment_graph(s, d, k, d.adj_exec[tp], nullptr,
                                    [&] { return adjoint_segment(s, d, k, G, tp); })))
            return rc;
    }
    d.taped.assign(d.taped.size(), -1);   // tape 0 now holds the first segment's recompute
    CU(cudaGetLastError());
    // Outputs: dL/d(state at the start of the recorded forward), attach order.
    if (dl_dpos0) {
        vtp::k_f4_to_f3<<<vtp::nblk(n, 256), 256, 0, s->st>>>(n, d.xbar_a, s->stage);
        CU(cudaMemcpyAsync(dl_dpos0, s->stage, n3, cudaMemcpyDeviceToHost, s->st));
        CU(cudaStreamSynchronize(s->st));
    }
    if (dl_dvel0) {
        vtp::k_f4_to_f3<<<vtp::nblk(n, 256), 256, 0, s->st>>>(n, d.vbar_a, s->stage);
        CU(cudaMemcpyAsync(dl_dvel0, s->stage, n3, cudaMemcpyDeviceToHost, s->st));
        CU(cudaStreamSynchronize(s->st));
    }
    double kb = 0.0;
    CU(cudaMemcpyAsync(&kb, d.kacc, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    // Put the forward's final state back so the solver can continue.
    if ((rc = restore_fluid(*s, d.ck_pos[nchk], d.ck_vel[nchk], d.ck_orig[nchk]))) return rc;
    CU(cudaStreamSynchronize(s->st));
    if (dl_dxsph_k) *dl_dxsph_k = kb;
    return s->check_status();
}

int vtp_solver_diff_lists(vtp_solver *s, uint32_t step, uint32_t *counts, uint32_t *nbrs, uint32_t max_nbr) {
    const uint32_t *l_orig = nullptr, *l_nbr = nullptr, *l_cnt = nullptr;
    uint32_t n = 0, nf = 0;
    if (s && s->type == VTP_SOLVER_DFSPH) {
        int rc = vtp::dfsph_diff_slot(s, step, &l_orig, &l_nbr, &l_cnt, nullptr, nullptr);
        if (rc) return rc;
        n = s->L.n;
        nf = s->L.nf;
    } else {
        int rc = check_ready(s);
        if (rc) return rc;
        if (!s->diff || !s->diff->keep_lists) return fail(VTP_ERR_STATE, "diff_lists needs diff_forward with keep_lists");
        vtp::DiffState &d = *s->diff;
        if (step >= d.steps) return fail(VTP_ERR_ARG, "step out of range");
        n = d.n;
        nf = d.nf;
        l_orig = d.kl_orig[step];
        l_nbr = d.kl_nbr[step];
        l_cnt = d.kl_cnt[step];
    }
    if (!counts || !nbrs) return fail(VTP_ERR_ARG, "null argument");
    if (max_nbr != s->maxnbr) return fail(VTP_ERR_ARG, "max_nbr must equal maxNeighborNum");
    // Row -> attach id map of that substep: fluid rows from the record, boundary rows static.
    uint32_t *omap = nullptr, *dc = nullptr, *dn = nullptr;
    CU(cudaMalloc(&omap, (size_t)n * 4));
    cudaError_t e = cudaMalloc(&dc, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dn, (size_t)n * max_nbr * 4);
    if (e == cudaSuccess && nf) e = cudaMemcpyAsync(omap, l_orig, (size_t)nf * 4, cudaMemcpyDeviceToDevice, s->st);
    if (e == cudaSuccess && n > nf)
        e = cudaMemcpyAsync(omap + nf, s->orig.c() + nf, (size_t)(n - nf) * 4, cudaMemcpyDeviceToDevice, s->st);
    if (e == cudaSuccess) {
        vtp::export_neighbors(s->st, s->L, 0, nf, l_nbr, l_cnt, omap, max_nbr, dc, dn);
        vtp::export_neighbors(s->st, s->L, nf, n - nf, s->u.bnbr, s->u.bncnt, omap, max_nbr, dc, dn);
        e = cudaMemcpyAsync(counts, dc, (size_t)n * 4, cudaMemcpyDeviceToHost, s->st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(nbrs, dn, (size_t)n * max_nbr * 4, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    cudaFree(omap);
    cudaFree(dc);
    cudaFree(dn);
    if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    return VTP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- DFSPH pressure solve as an operator

namespace {

int dfsph_op_ready(vtp_solver *s) {
    if (!s) return fail(VTP_ERR_ARG, "null solver");
    if (s->type != VTP_SOLVER_DFSPH) return fail(VTP_ERR_CONFIG, "the pressure-solve operator is a DFSPH operator");
    if (s->nscenes() != 1) return fail(VTP_ERR_CONFIG, "the pressure-solve operator runs a single scene");
    if (s->cfl > 0.f) return fail(VTP_ERR_CONFIG, "the pressure-solve operator takes the fixed time step (no \"cfl\")");
    return VTP_OK;
}

}  // namespace

extern "C" {

int vtp_solver_dfsph_solve_forward(vtp_solver *s, int which, const float *v_in, float *v_out, uint32_t force_iters,
                                   uint32_t *iterations) {
    int rc = dfsph_op_ready(s);
    if (rc) return rc;
    if (!s->initialized && (rc = s->initialize())) return rc;
    if (which != 0 && which != 1) return fail(VTP_ERR_ARG, "which must be 0 (divergence) or 1 (density)");
    if (!v_in) return fail(VTP_ERR_ARG, "null v_in");
    if (!s->diff) s->diff = std::make_shared<vtp::DiffState>();
    vtp::DiffState &d = *s->diff;
    const uint32_t n = s->L.n, nf = s->L.nf;
    const size_t nfa = std::max<uint32_t>(nf, 1);
    if (!d.df_vb && ((rc = d.alloc(&d.df_vb, nfa)) || (rc = d.alloc(&d.df_save, nfa)) ||
                     (rc = d.alloc(&d.df_kb, nfa))))
        return rc;
    // Neighbour search of the current state (the next substep's lists), re-sorted rows copied
    // back so the substep graphs' buffer parity is kept, then compression ratio and alpha.
    vtp::Carry carry{};
    carry.nf4 = 1;
    carry.src4[0] = s->vadv.c();
    carry.dst4[0] = s->vadv.n();
    vtp::ugns_sort(s->st, s->scn(), s->nbuckets, 0, nf, s->pos.c(), s->pos.n(), s->vel.c(), s->vel.n(),
                   s->orig.c(), s->orig.n(), carry, 0.f, s->u, s->u.fstart);
    if (nf) {
        CU(cudaMemcpyAsync(s->pos.c(), s->pos.n(), (size_t)nf * sizeof(float4), cudaMemcpyDeviceToDevice, s->st));
        CU(cudaMemcpyAsync(s->vel.c(), s->vel.n(), (size_t)nf * sizeof(float4), cudaMemcpyDeviceToDevice, s->st));
        CU(cudaMemcpyAsync(s->orig.c(), s->orig.n(), (size_t)nf * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s->st));
        CU(cudaMemcpyAsync(s->vadv.c(), s->vadv.n(), (size_t)nf * sizeof(float4), cudaMemcpyDeviceToDevice, s->st));
        CU(cudaMemcpyAsync(d.df_save, s->vadv.c(), (size_t)nf * sizeof(float4), cudaMemcpyDeviceToDevice, s->st));
    }
    if (s->staged)   // the staged solve passes below read the slot lists too
        vtp::ugns_build_lists_staged(s->st, s->scn(), s->L, s->stg, s->pos.c(), s->u.nbr, s->u.ncnt, s->d_status,
                                     s->d_overflow);
    else
        vtp::ugns_build_lists(s->st, s->scn(), s->L, 0, nf, s->pos.c(), s->orig.c(), s->u, s->u.nbr, s->u.ncnt,
                              s->d_status, s->d_overflow, s->block);
    vtp::dfsph_ratio_alpha(s->st, s->dfsph_args(which), s->block);
    const size_t n3 = (size_t)n * 3 * sizeof(float);
    if ((rc = s->ensure_stage(n3))) return rc;
    CU(cudaMemcpyAsync(s->stage, v_in, n3, cudaMemcpyHostToDevice, s->st));
    vtp::gather_orig_to_f4(s->st, nf, s->stage, s->orig.c(), s->vadv.c(), 1);
    // The solve loop, host-driven, with each iteration's delta recorded.
    vtp::DfsphArgs a = s->dfsph_args(which);
    vtp::SolveCtl c = s->solve_ctl(which, cudaGraphConditionalHandle{}, 0);
    c.force_iters = force_iters;
    c.force_seq = nullptr;
    vtp::dfsph_solve_begin(s->st, s->solve + (size_t)which * s->scenes.size(), s->loop + which, s->nscenes());
    vtp::dfsph_solve_pack(s->st, a);
    uint32_t it = 0;
    for (; it < 101; ++it) {
        if (d.df_delta.size() <= it) {
            float *p = nullptr;
            if ((rc = d.alloc(&p, nfa))) return rc;
            d.df_delta.push_back(p);
        }
        vtp::dfsph_solve_a(s->st, a, s->block);
        if (nf) CU(cudaMemcpyAsync(d.df_delta[it], s->delta, (size_t)nf * sizeof(float), cudaMemcpyDeviceToDevice, s->st));
        vtp::dfsph_solve_b(s->st, a, s->block);
        vtp::dfsph_solve_end(s->st, c, s->partials, s->d_status);
        CU(cudaMemcpyAsync(s->h_pinned + 2, &s->loop[which].running, sizeof(uint32_t), cudaMemcpyDeviceToHost, s->st));
        CU(cudaStreamSynchronize(s->st));
        if (!s->h_pinned[2]) break;
    }
    const uint32_t iters = std::min<uint32_t>(it + 1, 101);
    if (v_out) {
        CU(cudaMemsetAsync(s->stage, 0, n3, s->st));
        vtp::scatter_f4_to_orig(s->st, nf, s->vadv.c(), s->orig.c(), s->stage);
        CU(cudaMemcpyAsync(v_out, s->stage, n3, cudaMemcpyDeviceToHost, s->st));
    }
    // Leave v* as the solver had it.
    if (nf) CU(cudaMemcpyAsync(s->vadv.c(), d.df_save, (size_t)nf * sizeof(float4), cudaMemcpyDeviceToDevice, s->st));
    CU(cudaStreamSynchronize(s->st));
    CU(cudaGetLastError());
    d.df_which = which;
    d.df_iters = iters;
    d.df_steps = s->steps_done;
    if (iterations) *iterations = iters;
    return s->check_status();
}

int vtp_solver_dfsph_solve_backward(vtp_solver *s, const float *vbar_out, float *vbar_in) {
    int rc = dfsph_op_ready(s);
    if (rc) return rc;
    if (!s->diff || s->diff->df_which < 0) return fail(VTP_ERR_STATE, "dfsph_solve_backward before dfsph_solve_forward");
    vtp::DiffState &d = *s->diff;
    if (d.df_steps != s->steps_done) return fail(VTP_ERR_STATE, "the solver advanced since dfsph_solve_forward");
    if (!vbar_out || !vbar_in) return fail(VTP_ERR_ARG, "null argument");
    const uint32_t n = s->L.n, nf = s->L.nf;
    const size_t n3 = (size_t)n * 3 * sizeof(float);
    if ((rc = s->ensure_stage(n3))) return rc;
    CU(cudaMemcpyAsync(s->stage, vbar_out, n3, cudaMemcpyHostToDevice, s->st));
    vtp::gather_orig_to_f4(s->st, nf, s->stage, s->orig.c(), d.df_vb, 0);
    vtp::DfAdjArgs a{};
    a.nf = nf; a.ell_stride = s->L.ell_stride; a.k = s->kc;
    a.dt = s->dt; a.inv_dt2 = s->inv_dt2; a.mass_f = s->rho_f * s->vol0;
    a.nbr = s->u.nbr; a.ncnt = s->u.ncnt; a.pos = s->pos.c(); a.alpha = s->alpha;
    a.vb = d.df_vb; a.kb = d.df_kb;
    const unsigned G = vtp::nblk(std::max<uint32_t>(nf, 1), 256);
    for (int it = (int)d.df_iters - 1; it >= 0 && nf; --it) {
        a.delta = d.df_delta[it];
        vtp::k_dadj_kappa<<<G, 256, 0, s->st>>>(a);
        vtp::k_dadj_vel<<<G, 256, 0, s->st>>>(a);
    }
    CU(cudaMemsetAsync(s->stage, 0, n3, s->st));
    vtp::scatter_f4_to_orig(s->st, nf, d.df_vb, s->orig.c(), s->stage);
    CU(cudaMemcpyAsync(vbar_in, s->stage, n3, cudaMemcpyDeviceToHost, s->st));
    CU(cudaStreamSynchronize(s->st));
    CU(cudaGetLastError());
    return VTP_OK;
}

}  // extern "C"
