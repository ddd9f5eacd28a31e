// IMM (N-phase mixture) and IMM-CT (mixture + conformation-tensor phase) solver
// passes for sm_100a, fluid rows only, rows cell-sorted.
//
// Restates IMMCTSolver::tick (Simulator/Runtime/Source/Solvers/IMM-CT/IMMCTSolver.cpp:408-492)
// and IMMSolver::tick (Solvers/IMM/IMMSolver.cpp:400-466) over the kernels of
// IMMCTCudaImpl.cu / IMMCudaImpl.cu, regrouped:
//   rest_density  : update_rest_density_and_mass_cuda, fluid part (IMMCTCudaImpl.cu:83-106)
//   precompute    : compute_compression_ratio + compute_df_beta + update_Cd (:129-184, :782-804)
//   div / incomp  : the DFSPH solve passes with per-particle mass (:186-264, :442-478)
//   apply_pressure: get_acc_pressure + clear_phase_acc + distribute_acc_pressure_2_phase +
//                   phase_acc_2_phase_vel + update_vel_from_phase_vel (:266-282, :392-440),
//                   optionally + update_pos (:480-491)
//   vis / tension : clear + gravity + add_phase_acc_vis + surface normal + tension +
//                   phase velocity + mixture velocity (:284-424)
//   ct / pct      : compute_vel_grad + compute_rheological_factors + update_ct and
//                   add_phase_pct_acc (:687-780, :806-821)          (IMM-CT only)
//   phase transfer: drift + diffusion volume-fraction exchange, the negativity retry
//                   loop as a CUDA-graph WHILE node, update / release / regularize /
//                   rest density / mixture velocity (:526-685, :1065-1152)
//
// Determinism: the reference resets its "all positive" flag from one thread and
// reads neighbours' rest densities written by other blocks in the same kernel
// (IMMCTCudaImpl.cu:89-103, :616-641); here the negativity test counts newly
// flagged particles with a device counter that is cleared before each test, and
// rest densities are written before any kernel reads them.
#include <cmath>
#include <cstring>

#include "immct.h"
#include "solver.h"

using json = nlohmann::json;

namespace vtp {

constexpr int kMaxPhases = 7;

// The conformation tensor Q and the stress tau are symmetric (the reference keeps full 3x3
// matrices, IMMCTrtData.hpp:79; its update keeps Q symmetric in exact arithmetic): six
// components are stored, in the order 00, 01, 02, 11, 12, 22, and the 3x3 row-major
// component c = 3 row + col is symmetric component sym_of(c).
constexpr int kSym = 6;
__host__ __device__ constexpr int sym_of(int c) {
    return c == 0 ? 0 : c == 1 || c == 3 ? 1 : c == 2 || c == 6 ? 2 : c == 4 ? 3 : c == 5 || c == 7 ? 4 : 5;
}
__host__ __device__ constexpr bool sym_diag(int k) { return k == 0 || k == 3 || k == 5; }

struct ImmParams {
    int P;
    int ct;                   // 1: IMM-CT, 0: IMM
    float rho[kMaxPhases];    // phase rest densities
    float mu[kMaxPhases];     // phase rest viscosities
    float color[kMaxPhases][3];
    float Cd0;                // IMM-CT: Cd0; IMM: the constant Cd
    float Cf;
    float vis_base, vis_max;  // IMM-CT: solution viscosities after the x1000 scaling of init_data_cuda
    float inv_relax;          // 1 / relaxationTime
    float thin0, theta;
};

struct ImmArgs {
    uint32_t nf;
    uint32_t ell_stride;
    Cubic k;
    ImmParams p;
    float dt, inv_dt, h, gamma, csigma, h6_64;
    float3 g;
    const uint32_t *nbr, *ncnt;
    float4 *pos;              // w = volume
    float4 *vel, *vel_alt, *vadv, *vadv_alt;
    float4 *vph[kMaxPhases];  // phase velocities (fluid rows)
    float *frac[kMaxPhases];  // volume fractions
    float *Q[kSym];           // conformation tensor, symmetric components (kSymOrder)
    float *tau[kSym];         // viscoelastic stress, symmetric components
    float4 *acc_tmp[kMaxPhases];
    float4 *normal;
    float *rd;                // rest density
    float *cd;                // momentum-exchange coefficient
    float *ratio, *alpha;
    float *fin[kMaxPhases], *fout[kMaxPhases];
    uint32_t *flag;
    uint32_t *counter;        // [0] newly flagged, [1] retry iteration, [2] stop, [3] retries, [4] work rows,
                              // [5] retry-loop bodies run since initialize (wraps)
    uint32_t *work;           // rows the running retry recomputes (k_drift_mark)
    int retry_all;            // phase-transfer retries recompute every row (1) or rows near new flags (0)
    uint32_t *status;
    uint64_t *tick;           // substep counter (per-substep forced iteration schedules)
    int unroll;
    // Packed gather rows of the viscosity / tension / conformation passes, 2 float4 per
    // fluid row ({x, V}, then {v, per-row factor} or {n, rest density}): the launch reads
    // `pk_in` and writes `pk_out` (see immct_enqueue_tick for which pass writes which).
    float4 *pk_in, *pk_out;
    // IMM-CT: packed rows of the stress-divergence gathers, 3 float4 per fluid row:
    // {x, V}, then tau_c / rho_rest^2 for the 6 symmetric components (the last 2 floats
    // unused); written by the conformation-tensor pass, read by the stress-divergence pass.
    float4 *tpk;
};

struct ImmState {
    ImmParams p{};
    bool have_tension = false;
    DB<float4> vph[kMaxPhases];
    DB<float> frac[kMaxPhases];
    DB<float> Q[kSym];
    float *tau[kSym] = {nullptr};
    float4 *acc_tmp[kMaxPhases] = {nullptr};
    float *rd = nullptr, *cd = nullptr;
    float *fin[kMaxPhases] = {nullptr}, *fout[kMaxPhases] = {nullptr};
    uint32_t *flag = nullptr, *counter = nullptr;
    uint32_t *work = nullptr;        // [nf] rows a phase-transfer retry recomputes
    uint32_t bodies_seen = 0;        // counter[5] at the last launch count
    float4 *tpk = nullptr;
    float4 *pk2 = nullptr;           // [2 nf] packed gather rows (viscosity -> tension / conformation)
    std::vector<float> bfrac;        // boundary rows' phase fractions in attach order (host)
    cudaGraphConditionalHandle cond{};
};

namespace {

inline unsigned nblk(uint32_t n, int b) { return (unsigned)((n + b - 1) / b); }

#define VTP_UNROLL_DISPATCH(U, ...)                            \
    switch (U) {                                                \
        case 1: { constexpr int UU = 1; __VA_ARGS__; } break;  \
        case 2: { constexpr int UU = 2; __VA_ARGS__; } break;  \
        case 8: { constexpr int UU = 8; __VA_ARGS__; } break;  \
        default: { constexpr int UU = 4; __VA_ARGS__; } break; \
    }

// Phase count as a compile-time constant for the common mixtures (2: IMM-CT and
// two-phase IMM, 3: three-phase IMM), so the per-phase arrays of the neighbour
// passes live in registers; other counts use the runtime loop (PP = 0).
#define VTP_PHASE_DISPATCH(P, ...)                              \
    switch (P) {                                                \
        case 2: { constexpr int PP = 2; __VA_ARGS__; } break;   \
        case 3: { constexpr int PP = 3; __VA_ARGS__; } break;   \
        default: { constexpr int PP = 0; __VA_ARGS__; } break;  \
    }

__device__ __forceinline__ float rest_of(const ImmArgs &a, uint32_t r) {
    float s = 0.f;
    for (int k = 0; k < a.p.P; ++k) s = __fmaf_rn(a.frac[k][r], a.p.rho[k], s);
    return s;
}

// rest_density = sum_k alpha_k rho_k (update_rest_density_and_mass_cuda, fluid rows).
__global__ void k_rest_density(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    a.rd[r] = rest_of(a, r);
}

struct GP {
    float4 q;
    float rd, f1;
};

// compression ratio, df_alpha and (IMM-CT) the momentum-exchange coefficient Cd.
template <int U>
__global__ void __launch_bounds__(256) k_precompute(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const float4 p = a.pos[r];
    const uint32_t n = a.ncnt[r];
    const float mi = a.rd[r] * p.w;
    float ratio = n > 0 ? p.w * a.k.w0 : 0.f;
    float a1x = 0.f, a1y = 0.f, a1z = 0.f, a2 = 1e-6f, blocking = 0.f;
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop<U>(lst, n > 0 ? n - 1 : 0,
                [&](uint32_t j) {
                    const bool f = j < a.nf;
                    return GP{ldg4(a.pos + j), f ? __ldg(a.rd + j) : 0.f, f && a.p.P > 1 ? __ldg(a.frac[1] + j) : 0.f};
                },
                [&](uint32_t j, const GP &e) {
                    const float dx = p.x - e.q.x, dy = p.y - e.q.y, dz = p.z - e.q.z;
                    const float d2 = dist2(dx, dy, dz);
                    const float w = cubic_w(d2, a.k);
                    const float g = cubic_g(d2, a.k);
                    ratio = __fmaf_rn(e.q.w, w, ratio);
                    const float gx = g * dx, gy = g * dy, gz = g * dz;
                    a1x = __fmaf_rn(e.q.w, gx, a1x);
                    a1y = __fmaf_rn(e.q.w, gy, a1y);
                    a1z = __fmaf_rn(e.q.w, gz, a1z);
                    if (j < a.nf) {
                        const float mj = e.rd * e.q.w;
                        a2 += (gx * gx + gy * gy + gz * gz) * e.q.w * e.q.w / mj;
                        blocking = __fmaf_rn(e.q.w * e.f1, w, blocking);
                    }
                });
    float alpha = (a1x * a1x + a1y * a1y + a1z * a1z) / mi + a2;
    if (alpha < 1e-6f) alpha = 1e-6f;
    a.ratio[r] = ratio;
    a.alpha[r] = alpha;
    a.cd[r] = a.p.ct ? a.p.Cd0 + (1.f - a.p.Cd0) * blocking : a.p.Cd0;
}

// Phase velocities from the mixture acceleration, then v = sum_k alpha_k v_k, v* = v.
__device__ __forceinline__ float4 mix_velocity(const ImmArgs &a, uint32_t r, float4 v) {
    float vx = 0.f, vy = 0.f, vz = 0.f;
    for (int k = 0; k < a.p.P; ++k) {
        const float4 vk = a.vph[k][r];
        const float fk = a.frac[k][r];
        vx = __fmaf_rn(vk.x, fk, vx);
        vy = __fmaf_rn(vk.y, fk, vy);
        vz = __fmaf_rn(vk.z, fk, vz);
    }
    v.x = vx; v.y = vy; v.z = vz;
    return v;
}

// apply_pressure_acc (IMMCTCudaImpl.cu:919-937), optionally followed by update_pos.
__global__ void k_apply_pressure(ImmArgs a, int update_pos) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const float4 v = a.vel[r], va = a.vadv[r];
    const float ax = (va.x - v.x) * a.inv_dt, ay = (va.y - v.y) * a.inv_dt, az = (va.z - v.z) * a.inv_dt;
    const float cd = a.cd[r], rd = a.rd[r];
    for (int k = 0; k < a.p.P; ++k) {
        const float c = cd + (1.f - cd) * (rd / a.p.rho[k]);
        float4 vk = a.vph[k][r];
        vk.x = __fmaf_rn(ax * c, a.dt, vk.x);
        vk.y = __fmaf_rn(ay * c, a.dt, vk.y);
        vk.z = __fmaf_rn(az * c, a.dt, vk.z);
        a.vph[k][r] = vk;
    }
    const float4 o = mix_velocity(a, r, v);
    a.vel[r] = o;
    a.vadv[r] = o;
    if (!update_pos && a.pk_out) {
        // rows for the viscosity pass: {x, V}, {v, h m / rho} (the normal's per-neighbour factor,
        // evaluated as add_phase_acc_vis / compute_surface_normal do per pair)
        const float4 p = a.pos[r];
        a.pk_out[2 * (size_t)r] = p;
        a.pk_out[2 * (size_t)r + 1] = make_float4(o.x, o.y, o.z, a.h * (rd * p.w) / rd);
    }
    if (update_pos) {
        float4 p = a.pos[r];
        p.x = __fmaf_rn(o.x, a.dt, p.x);
        p.y = __fmaf_rn(o.y, a.dt, p.y);
        p.z = __fmaf_rn(o.z, a.dt, p.z);
        a.pos[r] = p;
    }
}

struct VisG {
    float4 q, v;
    float rd;
};

// Gravity + phase viscosity (+ normals when tension is on); without tension the
// phase and mixture velocities are advanced here as well.
template <bool SPLIT, int U, int PP>
__global__ void __launch_bounds__(256) k_vis(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const float4 p = a.pos[r];
    const float4 vi = a.vel[r];
    const float cd = a.cd[r];
    const int P = PP > 0 ? PP : a.p.P;
    float3 acc[PP > 0 ? PP : kMaxPhases];
    float4 vk_i[PP > 0 ? PP : kMaxPhases];
#pragma unroll
    for (int k = 0; k < P; ++k) {
        acc[k] = a.g;
        vk_i[k] = a.vph[k][r];
    }
    float nx = 0.f, ny = 0.f, nz = 0.f;
    const uint32_t n = a.ncnt[r];
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop<U>(lst, n > 0 ? n - 1 : 0,
                [&](uint32_t j) {
                    if (j >= a.nf) return VisG{};
                    const F4x2 e = ldg8(a.pk_in + 2 * (size_t)j);   // {x, V}, {v, h m / rho}
                    return VisG{e.a, e.b, e.b.w};
                },
                [&](uint32_t j, const VisG &e) {
                    if (j >= a.nf) return;   // same material, j != i
                    const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                    const float d2 = dist2(rx, ry, rz);
                    const float g = cubic_g(d2, a.k);
                    const float gx = g * rx, gy = g * ry, gz = g * rz;
                    const float vx = vi.x - e.v.x, vy = vi.y - e.v.y, vz = vi.z - e.v.z;
#pragma unroll
                    for (int k = 0; k < P; ++k) {
                        const float m1 = a.p.mu[k] * (1.f - cd), m2 = a.p.mu[k] * cd;
                        const float ux = m1 * (vk_i[k].x - e.v.x) + m2 * vx;
                        const float uy = m1 * (vk_i[k].y - e.v.y) + m2 * vy;
                        const float uz = m1 * (vk_i[k].z - e.v.z) + m2 * vz;
                        const float s = 10.f * e.q.w * (ux * rx + uy * ry + uz * rz);
                        acc[k].x += s * gx / d2;
                        acc[k].y += s * gy / d2;
                        acc[k].z += s * gz / d2;
                    }
                    if (SPLIT) {
                        const float sn = e.rd;   // h m_j / rho_j, from the packed row
                        nx = __fmaf_rn(sn, gx, nx);
                        ny = __fmaf_rn(sn, gy, ny);
                        nz = __fmaf_rn(sn, gz, nz);
                    }
                });
    if constexpr (SPLIT) {
#pragma unroll
        for (int k = 0; k < P; ++k) a.acc_tmp[k][r] = make_float4(acc[k].x, acc[k].y, acc[k].z, 0.f);
        a.normal[r] = make_float4(nx, ny, nz, 0.f);
        // rows for the tension pass: {x, V}, {n, rest density}
        a.pk_out[2 * (size_t)r] = p;
        a.pk_out[2 * (size_t)r + 1] = make_float4(nx, ny, nz, a.rd[r]);
    } else {
#pragma unroll
        for (int k = 0; k < P; ++k) {
            float4 vk = vk_i[k];
            vk.x = __fmaf_rn(acc[k].x, a.dt, vk.x);
            vk.y = __fmaf_rn(acc[k].y, a.dt, vk.y);
            vk.z = __fmaf_rn(acc[k].z, a.dt, vk.z);
            a.vph[k][r] = vk;
        }
        const float4 o = mix_velocity(a, r, vi);
        a.vel_alt[r] = o;
        a.vadv_alt[r] = o;
        // rows for the conformation pass: {x, V}, {v, m / rho}
        const float rdr = a.rd[r];
        a.pk_out[2 * (size_t)r] = p;
        a.pk_out[2 * (size_t)r + 1] = make_float4(o.x, o.y, o.z, (rdr * p.w) / rdr);
    }
}

struct TG {
    float4 q, n;
    float rd;
};

// Surface tension (add_phase_acc_surface_tension_cuda), then phase / mixture velocities.
template <int U>
__global__ void __launch_bounds__(256) k_tension(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const float4 p = a.pos[r];
    const float4 vi = a.vel[r];
    const float4 ni = a.normal[r];
    const float rdi = a.rd[r];
    const float mi = rdi * p.w;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    const uint32_t n = a.ncnt[r];
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop<U>(lst, n > 0 ? n - 1 : 0,
                [&](uint32_t j) {
                    if (j >= a.nf) return TG{};
                    const F4x2 e = ldg8(a.pk_in + 2 * (size_t)j);   // {x, V}, {n, rest density}
                    return TG{e.a, e.b, e.b.w};
                },
                [&](uint32_t j, const TG &e) {
                    if (j >= a.nf) return;
                    const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                    const float rl = sqrtf(dist2(rx, ry, rz));
                    const float kk = 2.f * rdi / (rdi + e.rd);
                    const float mj = e.rd * e.q.w;
                    const float cs = -a.gamma * mi * mj * tension_c(rl, a.h, a.csigma, a.h6_64) / rl;
                    const float c2 = -a.gamma * mi;
                    tx += kk * (cs * rx + c2 * (ni.x - e.n.x));
                    ty += kk * (cs * ry + c2 * (ni.y - e.n.y));
                    tz += kk * (cs * rz + c2 * (ni.z - e.n.z));
                });
    for (int k = 0; k < a.p.P; ++k) {
        const float4 acc = a.acc_tmp[k][r];
        float4 vk = a.vph[k][r];
        vk.x = __fmaf_rn(acc.x + tx, a.dt, vk.x);
        vk.y = __fmaf_rn(acc.y + ty, a.dt, vk.y);
        vk.z = __fmaf_rn(acc.z + tz, a.dt, vk.z);
        a.vph[k][r] = vk;
    }
    const float4 o = mix_velocity(a, r, vi);
    a.vel_alt[r] = o;
    a.vadv_alt[r] = o;
    // rows for the conformation pass: {x, V}, {v, m / rho}
    a.pk_out[2 * (size_t)r] = p;
    a.pk_out[2 * (size_t)r + 1] = make_float4(o.x, o.y, o.z, (rdi * p.w) / rdi);
}

struct CG {
    float4 q, v;
    float rd;
};

// Velocity gradient, rheological factors and the conformation-tensor update
// (compute_vel_grad_cuda, compute_rheological_factors_cuda, update_ct_cuda).
template <int U>
__global__ void __launch_bounds__(256) k_ct(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const float4 p = a.pos[r];
    const float4 vi = a.vel[r];
    float G[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) G[c] = 0.f;
    const uint32_t n = a.ncnt[r];
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop<U>(lst, n > 0 ? n - 1 : 0,
                [&](uint32_t j) {
                    if (j >= a.nf) return CG{};
                    const F4x2 e = ldg8(a.pk_in + 2 * (size_t)j);   // {x, V}, {v, m / rho}
                    return CG{e.a, e.b, e.b.w};
                },
                [&](uint32_t j, const CG &e) {
                    if (j >= a.nf) return;
                    const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                    const float g = cubic_g(dist2(rx, ry, rz), a.k);
                    const float w[3] = {g * rx, g * ry, g * rz};
                    const float vj = e.rd;   // m_j / rho_j, from the packed row
                    const float d[3] = {e.v.x - vi.x, e.v.y - vi.y, e.v.z - vi.z};
#pragma unroll
                    for (int row = 0; row < 3; ++row)
#pragma unroll
                        for (int col = 0; col < 3; ++col) G[row * 3 + col] += vj * (d[row] * w[col]);
                });
    const float f1 = a.frac[1][r];
    // thinning coefficient beta and viscosity increase kappa (compute_rheological_factors_cuda)
    const float beta = (float)((double)(a.p.thin0 * fmaxf(0.f, a.p.theta - f1)) / ((double)a.p.theta + 1e-6));
    const float kap = powf(1.f - f1, -1.2f);
    float Q[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) Q[c] = a.Q[sym_of(c)][r];
    float QmI[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) QmI[c] = Q[c] - ((c % 4) == 0 ? 1.f : 0.f);
    float dQ[9];
#pragma unroll
    for (int row = 0; row < 3; ++row) {
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            float qg = 0.f, gq = 0.f, qq = 0.f;
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                qg += Q[row * 3 + m] * G[m * 3 + col];        // Q G
                gq += G[m * 3 + row] * Q[m * 3 + col];        // G^T Q
                qq += QmI[row * 3 + m] * Q[m * 3 + col];      // (Q - I) Q
            }
            const int c = row * 3 + col;
            dQ[c] = (qg + gq - a.p.inv_relax * QmI[c] - beta * qq) * a.dt;
        }
    }
    // update_ct_cuda (IMMCTCudaImpl.cu:716-744) element by element; the upper triangle is kept
    // (the lower one differs from it only by the rounding of the (Q - I) Q products)
    float Qn[kSym];
#pragma unroll
    for (int row = 0; row < 3; ++row)
#pragma unroll
        for (int col = row; col < 3; ++col) {
            const int c = row * 3 + col;
            Qn[sym_of(c)] = Q[c] + dQ[c];
        }
#pragma unroll
    for (int k = 0; k < kSym; ++k) a.Q[k][r] = Qn[k];
    const float trD = 0.5f * (G[0] + G[0]) + 0.5f * (G[4] + G[4]) + 0.5f * (G[8] + G[8]);
    const float shear = sqrtf(0.5f * trD * trD);
    float vis = a.p.vis_base * kap;
    vis = fminf(vis, a.p.vis_max);
    vis = a.p.vis_base + (vis - a.p.vis_base) / (1.f + powf(10.f * shear, 5.f)) *
                             fminf(1.f, f1 / (a.p.theta + 1e-6f));
    float t[kSym];
    const float d = powf(a.rd[r], 2.f);
#pragma unroll
    for (int k = 0; k < kSym; ++k) {
        const float tc = vis * (Qn[k] - (sym_diag(k) ? 1.f : 0.f));
        a.tau[k][r] = tc;
        t[k] = tc / d;   // the tau_j / rho_j^2 term of add_phase_pct_acc_cuda, once per row
    }
    float4 *row = a.tpk + 3 * (size_t)r;
    row[0] = p;
    row[1] = make_float4(t[0], t[1], t[2], t[3]);
    row[2] = make_float4(t[4], t[5], 0.f, 0.f);
}

struct PG {
    float4 q;
    float t[kSym];   // tau_j / rho_j^2, symmetric components
};

// Viscoelastic stress divergence (add_phase_pct_acc_cuda) + phase / mixture velocities.
template <int U>
__global__ void __launch_bounds__(256) k_pct(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const float4 p = a.pos[r];
    const float rdi = a.rd[r];
    const float inv_i = powf(rdi, 2.f);
    float ti[kSym];
#pragma unroll
    for (int k = 0; k < kSym; ++k) ti[k] = a.tau[k][r] / inv_i;
    float ax = 0.f, ay = 0.f, az = 0.f;
    const uint32_t n = a.ncnt[r];
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop<(U > 2 ? 2 : U)>(lst, n > 0 ? n - 1 : 0,
                [&](uint32_t j) {
                    PG e{};
                    if (j >= a.nf) return e;
                    // the neighbour's packed row: {x, V}, tau_j / rho_j^2 (48 bytes)
                    const float4 *row = a.tpk + 3 * (size_t)j;
                    const float4 h1 = ldg4(row + 1), h2 = ldg4(row + 2);
                    e.q = ldg4(row);
                    e.t[0] = h1.x; e.t[1] = h1.y; e.t[2] = h1.z; e.t[3] = h1.w;
                    e.t[4] = h2.x; e.t[5] = h2.y;
                    return e;
                },
                [&](uint32_t j, const PG &e) {
                    if (j >= a.nf) return;
                    const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                    const float g = cubic_g(dist2(rx, ry, rz), a.k);
                    const float w0 = g * rx, w1 = g * ry, w2 = g * rz;
                    float M[kSym];
#pragma unroll
                    for (int k = 0; k < kSym; ++k) M[k] = ti[k] + e.t[k];
                    ax += M[0] * w0 + M[1] * w1 + M[2] * w2;
                    ay += M[1] * w0 + M[3] * w1 + M[4] * w2;
                    az += M[2] * w0 + M[4] * w1 + M[5] * w2;
                });
    const float s = a.frac[1][r] * rdi;
    ax *= s; ay *= s; az *= s;
    const float cd = a.cd[r];
    for (int k = 0; k < a.p.P; ++k) {
        const float c = cd + (1.f - cd) * (rdi / a.p.rho[k]);
        float4 vk = a.vph[k][r];
        vk.x = __fmaf_rn(ax * c, a.dt, vk.x);
        vk.y = __fmaf_rn(ay * c, a.dt, vk.y);
        vk.z = __fmaf_rn(az * c, a.dt, vk.z);
        a.vph[k][r] = vk;
    }
    const float4 o = mix_velocity(a, r, a.vel[r]);
    a.vel[r] = o;
    a.vadv[r] = o;
}

struct DG {
    float4 q, v;
    uint32_t flag;
};

// Rows a phase-transfer retry has to recompute.  Between passes only the flags
// change (fractions, phase velocities and positions are fixed until
// k_phase_finish), and a pair is skipped when either side is flagged, so a
// pass changes a row's result only when the row or one of its fluid
// neighbours was flagged by the check just before it (flag == that check's
// number); every other row would recompute the values it holds, bit for bit.
// Those rows are appended to `work` (one atomic per warp; the order does not
// matter, each row's result depends on its own list only).
__global__ void __launch_bounds__(256) k_drift_mark(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (a.counter[2]) return;   // the retry loop has stopped
    const uint32_t gen = a.counter[1] - 1u;
    bool redo = false;
    if (r < a.nf) {
        const uint32_t fr = a.flag[r];
        redo = fr == gen;
        if (fr == 0) {
            const uint32_t n = a.ncnt[r];
            const uint32_t cnt = n > 0 ? n - 1 : 0;
            const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
            // four entries, then their four flags, per round trip (gen >= 1, so rows without a
            // flag word (boundary rows) read as 0)
            uint32_t t = 0;
            for (; t + 4 <= cnt && !redo; t += 4) {
                uint32_t j[4], f[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) j[u] = lst[(size_t)(t + u) * 32u];
#pragma unroll
                for (int u = 0; u < 4; ++u) f[u] = j[u] < a.nf ? __ldg(a.flag + j[u]) : 0u;
                redo = f[0] == gen || f[1] == gen || f[2] == gen || f[3] == gen;
            }
            for (; t < cnt && !redo; ++t) {
                const uint32_t j = lst[(size_t)t * 32u];
                redo = j < a.nf && __ldg(a.flag + j) == gen;
            }
        }
    }
    const unsigned m = __ballot_sync(0xffffffffu, redo);
    if (m == 0) return;
    const int lane = (int)(threadIdx.x & 31u);
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&a.counter[4], (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);   // every lane of the warp is here
    if (redo) a.work[base + (uint32_t)__popc(m & ((1u << lane) - 1u))] = r;
}

// Drift and diffusion volume-fraction exchange (update_phase_change_from_drift_cuda
// and update_phase_change_from_diffuse_cuda, IMMCTCudaImpl.cu:541-614): two walks
// over the list so that drift terms are accumulated before diffusion terms, as
// the reference does.  Every fluid row on the first pass of a substep; on a
// retry every row ("phaseRetry": "all") or the rows k_drift_mark listed.
template <int U, int PP>
__global__ void __launch_bounds__(256) k_drift_diffuse(ImmArgs a, int retry) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (retry) {
        if (a.counter[2]) return;   // the retry loop has stopped
        if (!a.retry_all) {
            if (r >= a.counter[4]) return;
            r = a.work[r];
        }
    }
    if (r >= a.nf) return;
    constexpr int NP = PP > 0 ? PP : kMaxPhases;
    const int P = PP > 0 ? PP : a.p.P;
    float in[NP], out[NP];
#pragma unroll
    for (int k = 0; k < P; ++k) in[k] = out[k] = 0.f;
    if (a.flag[r] == 0) {
        const float4 p = a.pos[r];
        const float4 vi = a.vel[r];
        float fi[NP];
        float4 ui[NP];
#pragma unroll
        for (int k = 0; k < P; ++k) {
            fi[k] = a.frac[k][r];
            const float4 vk = a.vph[k][r];
            ui[k] = make_float4(vk.x - vi.x, vk.y - vi.y, vk.z - vi.z, 0.f);
        }
        const uint32_t n = a.ncnt[r];
        const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
        const float ndt = -a.dt;
        // drift
        nbr_loop<U>(lst, n > 0 ? n - 1 : 0,
                    [&](uint32_t j) {
                        if (j >= a.nf) return DG{};
                        return DG{ldg4(a.pos + j), ldg4(a.vel + j), __ldg(a.flag + j)};
                    },
                    [&](uint32_t j, const DG &e) {
                        if (j >= a.nf || e.flag != 0) return;
                        const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                        const float g = cubic_g(dist2(rx, ry, rz), a.k);
                        const float gx = g * rx, gy = g * ry, gz = g * rz;
#pragma unroll
                        for (int k = 0; k < P; ++k) {
                            const float fj = __ldg(a.frac[k] + j);
                            const float4 vkj = ldg4(a.vph[k] + j);
                            const float ujx = vkj.x - e.v.x, ujy = vkj.y - e.v.y, ujz = vkj.z - e.v.z;
                            const float sx = fi[k] * ui[k].x + fj * ujx;
                            const float sy = fi[k] * ui[k].y + fj * ujy;
                            const float sz = fi[k] * ui[k].z + fj * ujz;
                            const float ch = ndt * e.q.w * (sx * gx + sy * gy + sz * gz);
                            if (ch < 0.f) out[k] += ch;
                            else in[k] += ch;
                        }
                    });
        // diffusion
        const float dtcf = a.dt * a.p.Cf;
        nbr_loop<U>(lst, n > 0 ? n - 1 : 0,
                    [&](uint32_t j) {
                        if (j >= a.nf) return DG{};
                        return DG{ldg4(a.pos + j), make_float4(0.f, 0.f, 0.f, 0.f), __ldg(a.flag + j)};
                    },
                    [&](uint32_t j, const DG &e) {
                        if (j >= a.nf || e.flag != 0) return;
                        const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                        const float d2 = dist2(rx, ry, rz);
                        const float g = cubic_g(d2, a.k);
                        const float factor = (g * rx * rx + g * ry * ry + g * rz * rz) / d2;
#pragma unroll
                        for (int k = 0; k < P; ++k) {
                            const float fij = fi[k] - __ldg(a.frac[k] + j);
                            const float ch = dtcf * fij * e.q.w * factor;
                            if (ch < 0.f) out[k] += ch;
                            else in[k] += ch;
                        }
                    });
    }
#pragma unroll
    for (int k = 0; k < P; ++k) {
        a.fin[k][r] = in[k];
        a.fout[k][r] = out[k];
    }
}

// check_negative_cuda: flag particles whose fractions would turn negative.
__global__ void k_check_negative(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    if (a.counter[2] || a.flag[r] != 0) return;
    bool neg = false;
    for (int k = 0; k < a.p.P; ++k)
        if (a.frac[k][r] + a.fout[k][r] + a.fin[k][r] < 0.f) neg = true;
    if (neg) {
        a.flag[r] = a.counter[1];   // the check's number (>= 1): the next pass recomputes around it
        atomicAdd(&a.counter[0], 1u);
    }
}

// Retry decision of phase_transfer (IMMCTCudaImpl.cu:1084-1110): stop when no
// particle was newly flagged or after iteration 100.
__global__ void k_retry_decide(ImmArgs a, cudaGraphConditionalHandle h, int use_cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t *c = a.counter;
    c[5] += 1;   // one per body of the retry loop (launch accounting)
    if (c[2] == 0) {
        const uint32_t iter = c[1];
        const bool stop = c[0] == 0 || iter > 100;
        if (stop) {
            c[2] = 1;
            if (iter > 100) atomicOr(a.status, ST_NOT_CONVERGED);
        } else {
            c[1] = iter + 1;
            c[3] += 1;   // retries this substep
        }
    }
    c[0] = 0;
    c[4] = 0;
    if (use_cond) cudaGraphSetConditional(h, c[2] ? 0u : 1u);
}

__global__ void k_retry_begin(uint32_t *c) {
    if (threadIdx.x == 0) {
        c[0] = 0;
        c[1] = 1;
        c[2] = 0;
        c[3] = 0;
    }
}

// update_phase_change, release_unused_drift_vel, release_negative, regularize,
// rest density, mixture velocity; then update_mass_and_vel (regularize, rest
// density, mixture velocity) once more.
__global__ void k_phase_finish(ImmArgs a) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    const int P = a.p.P;
    float f[kMaxPhases];
    for (int k = 0; k < P; ++k) f[k] = a.frac[k][r] + (a.fout[k][r] + a.fin[k][r]);
    float4 v = a.vel[r];
    if (a.flag[r] != 0) {
        for (int k = 0; k < P; ++k) {
            float4 vk = a.vph[k][r];
            vk.x = v.x; vk.y = v.y; vk.z = v.z;
            a.vph[k][r] = vk;
        }
    }
    a.flag[r] = 0;
    for (int pass = 0; pass < 2; ++pass) {
        float s = 0.f;
        for (int k = 0; k < P; ++k) s += f[k];
        for (int k = 0; k < P; ++k) f[k] /= s;
    }
    for (int k = 0; k < P; ++k) a.frac[k][r] = f[k];
    a.rd[r] = rest_of(a, r);
    v = mix_velocity(a, r, v);
    a.vel[r] = v;
    a.vadv[r] = v;
    if (r == 0 && a.tick) *a.tick += 1;
}

}  // namespace

}  // namespace vtp

using vtp::ImmArgs;
using vtp::ImmState;
using vtp::kMaxPhases;

void immct_set_parity(vtp_solver &s, int cur);

static const std::vector<std::string> kImmctRequired = {
    "animationTime", "timeStep", "particleRadius", "simSpaceLB", "simSpaceSize", "maxNeighborNum",
    "divFreeThreshold", "incompThreshold", "surfaceTensionCoefficient", "diffusionCoefficientCf",
    "momentumExchangeCoefficientCd0", "solventViscosity", "phaseRestDensity", "phaseRestColor",
    "solutionBasicViscosity", "solutionMaxViscosity", "relaxationTime", "shearThinningBasicFactor",
    "rheologicalThreshold"};
static const std::vector<std::string> kImmRequired = {
    "animationTime", "timeStep", "particleRadius", "simSpaceLB", "simSpaceSize", "maxNeighborNum",
    "divFreeThreshold", "incompThreshold", "surfaceTensionCoefficient", "diffusionCoefficientCf",
    "momentumExchangeCoefficientCd", "phaseRestDensity", "phaseRestViscosity", "phaseRestColor"};

nlohmann::json immct_default_required(bool ct) {
    if (ct)
        return {{"animationTime", 5}, {"timeStep", 0.0008}, {"particleRadius", 0.05},
                {"simSpaceLB", {-10, -10, -10}}, {"simSpaceSize", {20, 20, 20}}, {"maxNeighborNum", 60},
                {"divFreeThreshold", 1e-4}, {"incompThreshold", 1e-4}, {"surfaceTensionCoefficient", 0.001},
                {"diffusionCoefficientCf", 0.15}, {"momentumExchangeCoefficientCd0", 0.5},
                {"solventViscosity", 0.01}, {"phaseRestDensity", {900, 1000}},
                {"phaseRestColor", {{255, 0, 0}, {0, 0, 255}}}, {"solutionBasicViscosity", 12},
                {"solutionMaxViscosity", 12}, {"relaxationTime", 0.001}, {"shearThinningBasicFactor", 0.5},
                {"rheologicalThreshold", 0.4}};
    return {{"animationTime", 10}, {"timeStep", 0.01}, {"particleRadius", 0.075},
            {"simSpaceLB", {-10, -10, -10}}, {"simSpaceSize", {20, 20, 20}}, {"maxNeighborNum", 60},
            {"divFreeThreshold", 1e-4}, {"incompThreshold", 1e-4}, {"surfaceTensionCoefficient", 0.001},
            {"diffusionCoefficientCf", 0.1}, {"momentumExchangeCoefficientCd", 0.5},
            {"phaseRestDensity", {1000, 1000, 1000}}, {"phaseRestViscosity", {0.01, 0.01, 0.01}},
            {"phaseRestColor", {{255, 0, 0}, {0, 255, 0}, {0, 0, 255}}}};
}

std::vector<std::string> immct_required_keys(bool ct) { return ct ? kImmctRequired : kImmRequired; }

int immct_parse(bool ct, const nlohmann::json &r, std::shared_ptr<ImmState> &imm) {
    auto st = std::make_shared<ImmState>();
    auto &p = st->p;
    p.ct = ct ? 1 : 0;
    auto rho = r["phaseRestDensity"].get<std::vector<float>>();
    if (rho.empty() || rho.size() > (size_t)kMaxPhases)
        return vtp::fail(VTP_ERR_CONFIG, "phaseRestDensity must have 1..7 entries");
    if (ct && rho.size() < 2) return vtp::fail(VTP_ERR_CONFIG, "IMMCT needs at least 2 phases");
    p.P = (int)rho.size();
    auto colors = r["phaseRestColor"].get<std::vector<std::vector<float>>>();
    for (int k = 0; k < p.P; ++k) {
        p.rho[k] = rho[k];
        for (int c = 0; c < 3; ++c) p.color[k][c] = (k < (int)colors.size() && c < (int)colors[k].size()) ? colors[k][c] : 0.f;
    }
    p.Cf = r["diffusionCoefficientCf"].get<float>();
    if (ct) {
        // IMMCTSolver::setConfig copies solventViscosity to every phase (IMMCTSolver.cpp:72).
        const float mu = r["solventViscosity"].get<float>();
        for (int k = 0; k < p.P; ++k) p.mu[k] = mu;
        p.Cd0 = r["momentumExchangeCoefficientCd0"].get<float>();
        // init_data_cuda scales the solution viscosities by 1000 on the device before use.
        p.vis_base = r["solutionBasicViscosity"].get<float>() * 1000.f;
        p.vis_max = r["solutionMaxViscosity"].get<float>() * 1000.f;
        p.inv_relax = 1.f / r["relaxationTime"].get<float>();
        p.thin0 = r["shearThinningBasicFactor"].get<float>();
        p.theta = r["rheologicalThreshold"].get<float>();
    } else {
        auto mu = r["phaseRestViscosity"].get<std::vector<float>>();
        if ((int)mu.size() != p.P) return vtp::fail(VTP_ERR_CONFIG, "phaseRestViscosity size must match phaseRestDensity");
        for (int k = 0; k < p.P; ++k) p.mu[k] = mu[k];
        p.Cd0 = r["momentumExchangeCoefficientCd"].get<float>();
    }
    imm = st;
    return VTP_OK;
}

int immct_phase_count(const vtp_solver &s) { return s.imm ? s.imm->p.P : 0; }

void immct_conservation_inputs(vtp_solver &s, const float **rd, const float **frac, float *rho_k, int *P) {
    ImmState &m = *s.imm;
    *rd = m.rd;
    *P = std::min(m.p.P, vtp::kConsPhases);
    for (int k = 0; k < *P; ++k) {
        frac[k] = m.frac[k].c();
        rho_k[k] = m.p.rho[k];
    }
}

#define CUI(call)                                                                               \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return vtp::fail(VTP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int immct_alloc(vtp_solver &s) {
    ImmState &m = *s.imm;
    const int P = m.p.P;
    const uint32_t nf = std::max<uint32_t>(s.L.nf, 1);
    int rc;
    for (int k = 0; k < P; ++k) {
        for (int b = 0; b < 2; ++b) {
            if ((rc = s.alloc(&m.vph[k].b[b], nf))) return rc;
            if ((rc = s.alloc(&m.frac[k].b[b], nf))) return rc;
        }
        if ((rc = s.alloc(&m.acc_tmp[k], nf))) return rc;
        if ((rc = s.alloc(&m.fin[k], nf))) return rc;
        if ((rc = s.alloc(&m.fout[k], nf))) return rc;
    }
    for (int c = 0; c < vtp::kSym; ++c) {
        for (int b = 0; b < 2; ++b)
            if ((rc = s.alloc(&m.Q[c].b[b], nf))) return rc;
        if ((rc = s.alloc(&m.tau[c], nf))) return rc;
        CUI(cudaMemsetAsync(m.tau[c], 0, nf * sizeof(float), s.st));
    }
    if ((rc = s.alloc(&m.rd, nf))) return rc;
    if ((rc = s.alloc(&m.cd, nf))) return rc;
    if ((rc = s.alloc(&m.flag, nf))) return rc;
    if ((rc = s.alloc(&m.counter, 6))) return rc;
    if ((rc = s.alloc(&m.work, nf))) return rc;
    if (m.p.ct && (rc = s.alloc(&m.tpk, 3 * (size_t)nf))) return rc;
    if ((rc = s.alloc(&m.pk2, 2 * (size_t)nf))) return rc;
    CUI(cudaMemsetAsync(m.flag, 0, nf * sizeof(uint32_t), s.st));
    CUI(cudaMemsetAsync(m.counter, 0, 6 * sizeof(uint32_t), s.st));
    return VTP_OK;
}

static ImmArgs imm_args(vtp_solver &s) {
    ImmState &m = *s.imm;
    ImmArgs a{};
    a.nf = s.L.nf;
    a.ell_stride = s.L.ell_stride;
    a.k = s.kc;
    a.p = m.p;
    a.retry_all = s.phase_retry_all ? 1 : 0;
    a.dt = s.dt;
    a.inv_dt = s.inv_dt;
    a.h = s.h;
    a.gamma = s.gamma;
    a.csigma = 32.f / 3.14159265f / std::pow(s.h, 9.f);
    a.h6_64 = std::pow(s.h, 6.f) / 64;
    a.g = s.gravity;
    a.nbr = s.u.nbr;
    a.ncnt = s.u.ncnt;
    a.pos = s.pos.c();
    a.vel = s.vel.c();
    a.vel_alt = s.vel.n();
    a.vadv = s.vadv.c();
    a.vadv_alt = s.vadv.n();
    for (int k = 0; k < m.p.P; ++k) {
        a.vph[k] = m.vph[k].c();
        a.frac[k] = m.frac[k].c();
        a.acc_tmp[k] = m.acc_tmp[k];
        a.fin[k] = m.fin[k];
        a.fout[k] = m.fout[k];
    }
    for (int c = 0; c < vtp::kSym; ++c) {
        a.Q[c] = m.Q[c].c();
        a.tau[c] = m.tau[c];
    }
    a.normal = s.normal;
    a.rd = m.rd;
    a.cd = m.cd;
    a.ratio = s.ratio;
    a.alpha = s.alpha;
    a.flag = m.flag;
    a.counter = m.counter;
    a.work = m.work;
    a.status = s.d_status;
    a.tick = s.d_tick;
    a.unroll = s.unroll;
    a.tpk = m.tpk;
    return a;
}

int immct_init(vtp_solver &s) {
    // init_data_cuda (IMMCTCudaImpl.cu:52-81): phase velocities = v, Q = I, fractions from the objects.
    ImmState &m = *s.imm;
    const int P = m.p.P;
    const uint32_t n = s.L.n, nf = s.L.nf;
    std::vector<uint32_t> ids(n);
    CUI(cudaMemcpyAsync(ids.data(), s.orig.c(), n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s.st));
    std::vector<float4> v4(n);
    CUI(cudaMemcpyAsync(v4.data(), s.vel.c(), n * sizeof(float4), cudaMemcpyDeviceToHost, s.st));
    CUI(cudaStreamSynchronize(s.st));
    std::vector<float> fr(nf);
    for (int k = 0; k < P; ++k) {
        for (uint32_t r = 0; r < nf; ++r) fr[r] = s.hphase[(size_t)ids[r] * P + k];
        for (int b = 0; b < 2; ++b) {
            CUI(cudaMemcpyAsync(m.frac[k].b[b], fr.data(), nf * sizeof(float), cudaMemcpyHostToDevice, s.st));
            CUI(cudaMemcpyAsync(m.vph[k].b[b], v4.data(), nf * sizeof(float4), cudaMemcpyHostToDevice, s.st));
        }
        CUI(cudaStreamSynchronize(s.st));
    }
    std::vector<float> one(nf, 1.f), zero(nf, 0.f);
    for (int c = 0; c < vtp::kSym; ++c)
        for (int b = 0; b < 2; ++b)
            CUI(cudaMemcpyAsync(m.Q[c].b[b], vtp::sym_diag(c) ? one.data() : zero.data(), nf * sizeof(float),
                                cudaMemcpyHostToDevice, s.st));
    m.bfrac.assign(s.hphase.begin(), s.hphase.end());
    m.have_tension = s.gamma != 0.f;
    // Both buffers hold the initial state; from here on the phase arrays swap in
    // lockstep with the row order (one swap per substep sort).
    immct_set_parity(s, s.orig.cur);
    ImmArgs a = imm_args(s);
    if (nf) vtp::k_rest_density<<<vtp::nblk(nf, 256), 256, 0, s.st>>>(a);
    CUI(cudaStreamSynchronize(s.st));
    return VTP_OK;
}

void immct_fill_carry(vtp_solver &s, vtp::Carry &carry) {
    ImmState &m = *s.imm;
    const int P = m.p.P;
    for (int k = 0; k < P; ++k) {
        carry.src4[carry.nf4] = m.vph[k].c();
        carry.dst4[carry.nf4++] = m.vph[k].n();
        carry.src1[carry.nf1] = m.frac[k].c();
        carry.dst1[carry.nf1++] = m.frac[k].n();
    }
    for (int c = 0; c < vtp::kSym; ++c) {
        carry.src1[carry.nf1] = m.Q[c].c();
        carry.dst1[carry.nf1++] = m.Q[c].n();
    }
}

int immct_copy_back(vtp_solver &s) {
    // After a re-sort into the second buffers, copy the fluid rows back (buffer parity kept).
    ImmState &m = *s.imm;
    const size_t nf = s.L.nf;
    for (int k = 0; k < m.p.P; ++k) {
        CUI(cudaMemcpyAsync(m.vph[k].c(), m.vph[k].n(), nf * sizeof(float4), cudaMemcpyDeviceToDevice, s.st));
        CUI(cudaMemcpyAsync(m.frac[k].c(), m.frac[k].n(), nf * sizeof(float), cudaMemcpyDeviceToDevice, s.st));
    }
    for (int c = 0; c < vtp::kSym; ++c)
        CUI(cudaMemcpyAsync(m.Q[c].c(), m.Q[c].n(), nf * sizeof(float), cudaMemcpyDeviceToDevice, s.st));
    return VTP_OK;
}

void immct_set_parity(vtp_solver &s, int cur) {
    // Phase arrays swap together with the row order once per substep.
    ImmState &m = *s.imm;
    for (int k = 0; k < m.p.P; ++k) m.vph[k].cur = cur, m.frac[k].cur = cur;
    for (int c = 0; c < vtp::kSym; ++c) m.Q[c].cur = cur;
}

uint32_t immct_last_retries(vtp_solver &s, uint64_t *body_launches) {
    uint32_t c[6] = {0, 0, 0, 0, 0, 0};
    if (body_launches) *body_launches = 0;
    if (cudaMemcpy(c, s.imm->counter, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    // Kernels of the retry loop's bodies since the last call: check, decide, (mark,) drift/diffuse.
    const uint32_t bodies = c[5] - s.imm->bodies_seen;
    s.imm->bodies_seen = c[5];
    if (body_launches) *body_launches = (uint64_t)bodies * (s.phase_retry_all ? 3u : 4u);
    return c[3];
}

void immct_color(vtp_solver &s, const float *frac_attach_order, float *rgb) {
    ImmState &m = *s.imm;
    const int P = m.p.P;
    const size_t n = s.L.n;
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            float v = 0.f;
            for (int k = 0; k < P; ++k) v = std::fma(frac_attach_order[i * P + k], m.p.color[k][c], v);
            rgb[i * 3 + c] = v;
        }
}

vtp::DfsphArgs immct_solve_args(vtp_solver &s, int which) {
    vtp::DfsphArgs a = s.dfsph_args(which);
    a.rest_density = s.imm->rd;
    return a;
}

void immct_solve_ab(vtp_solver &s, cudaStream_t st, int which) {
    const vtp::DfsphArgs a = immct_solve_args(s, which);
    vtp::dfsph_solve_a(st, a, s.block);
    vtp::dfsph_solve_b(st, a, s.block);
}

int immct_enqueue_tick(vtp_solver &s, cudaStream_t st, bool capture) {
    const vtp::NvtxRange nvtx_range("vtp IMM substep");
    ImmState &m = *s.imm;
    const int P = m.p.P;
    const int B = s.block;
    const uint32_t nf = s.L.nf;
    int rc;
    // Neighbour search; the sort carries v*, phase velocities, fractions and Q.
    vtp::Carry carry{};
    carry.nf4 = 1;
    carry.src4[0] = s.vadv.c();
    carry.dst4[0] = s.vadv.n();
    immct_fill_carry(s, carry);
    vtp::ugns_sort(st, s.scn(), s.nbuckets, 0, nf, s.pos.c(), s.pos.n(), s.vel.c(), s.vel.n(), s.orig.c(),
                   s.orig.n(), carry, 0.f, s.u, s.u.fstart, s.prof);
    s.pos.swap(); s.vel.swap(); s.orig.swap(); s.vadv.swap();
    for (int k = 0; k < P; ++k) m.vph[k].swap(), m.frac[k].swap();
    for (int c = 0; c < vtp::kSym; ++c) m.Q[c].swap();
    auto P_ = [&](const char *nm, auto &&fn) {
        if (s.prof) s.prof->begin();
        fn();
        if (s.prof) s.prof->end_(nm);
        s.launches_per_tick += 1;
    };
    P_("ugns_lists", [&] {
        vtp::ugns_build_lists(st, s.scn(), s.L, 0, nf, s.pos.c(), s.orig.c(), s.u, s.u.nbr, s.u.ncnt, s.d_status,
                              s.d_overflow, B);
    });
    s.launches_per_tick += 6;   // hash, 3 scan kernels, scatter, rank/reorder
    if (nf == 0) return VTP_OK;
    const unsigned G = vtp::nblk(nf, B), G256 = vtp::nblk(nf, 256);
    ImmArgs a = imm_args(s);
    P_("imm_rest_density", [&] { vtp::k_rest_density<<<G256, 256, 0, st>>>(a); });
    P_("imm_precompute", [&] { VTP_UNROLL_DISPATCH(s.unroll, vtp::k_precompute<UU><<<G, B, 0, st>>>(a)) });
    if ((rc = s.enqueue_solve(st, 0, capture))) return rc;
    // Packed gather rows between the solves: the pressure apply writes {x, v} rows into the
    // solver's packed solve rows (free until the next solve re-packs them), the viscosity
    // pass reads them and writes rows for the tension pass (or, without tension, for the
    // conformation pass) into m.pk2; the tension pass writes the conformation pass's rows
    // back into the solve rows.
    a = imm_args(s);
    a.pk_out = s.pva;
    P_("imm_apply_pressure", [&] { vtp::k_apply_pressure<<<G256, 256, 0, st>>>(a, 0); });
    a.pk_in = s.pva;
    a.pk_out = m.pk2;
    float4 *ct_rows = m.pk2;
    if (m.have_tension) {
        P_("imm_vis_normal", [&] { VTP_PHASE_DISPATCH(P, VTP_UNROLL_DISPATCH(s.unroll, vtp::k_vis<true, UU, PP><<<G, B, 0, st>>>(a))) });
        a.pk_in = m.pk2;
        a.pk_out = s.pva;
        ct_rows = s.pva;
        P_("imm_tension", [&] { VTP_UNROLL_DISPATCH(s.unroll, vtp::k_tension<UU><<<G, B, 0, st>>>(a)) });
    } else {
        P_("imm_vis", [&] { VTP_PHASE_DISPATCH(P, VTP_UNROLL_DISPATCH(s.unroll, vtp::k_vis<false, UU, PP><<<G, B, 0, st>>>(a))) });
    }
    s.vel.swap(); s.vadv.swap();
    if (m.p.ct) {
        a = imm_args(s);
        a.pk_in = ct_rows;
        P_("immct_ct", [&] { VTP_UNROLL_DISPATCH(s.unroll, vtp::k_ct<UU><<<G, B, 0, st>>>(a)) });
        P_("immct_pct", [&] { VTP_UNROLL_DISPATCH(s.unroll, vtp::k_pct<UU><<<G, B, 0, st>>>(a)) });
    }
    if ((rc = s.enqueue_solve(st, 1, capture))) return rc;
    a = imm_args(s);
    P_("imm_apply_pressure", [&] { vtp::k_apply_pressure<<<G256, 256, 0, st>>>(a, 1); });
    // Phase transfer with the negativity retry loop.
    P_("imm_retry_begin", [&] { vtp::k_retry_begin<<<1, 32, 0, st>>>(m.counter); });
    P_("imm_drift_diffuse", [&] { VTP_PHASE_DISPATCH(P, VTP_UNROLL_DISPATCH(s.unroll, vtp::k_drift_diffuse<UU, PP><<<G, B, 0, st>>>(a, 0))) });
    if (capture && s.device_loop) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        CUI(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
        cudaGraphConditionalHandle hnd;
        CUI(cudaGraphConditionalHandleCreate(&hnd, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hnd;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        CUI(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CUI(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
        CUI(cudaStreamBeginCaptureToGraph(s.side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        vtp::k_check_negative<<<G256, 256, 0, s.side>>>(a);
        vtp::k_retry_decide<<<1, 32, 0, s.side>>>(a, hnd, 1);
        if (!s.phase_retry_all) vtp::k_drift_mark<<<G256, 256, 0, s.side>>>(a);
        VTP_PHASE_DISPATCH(P, VTP_UNROLL_DISPATCH(s.unroll, vtp::k_drift_diffuse<UU, PP><<<G, B, 0, s.side>>>(a, 1)))
        cudaGraph_t out;
        CUI(cudaStreamEndCapture(s.side, &out));
    } else {
        for (int it = 0; it < 102; ++it) {
            P_("imm_check_negative", [&] { vtp::k_check_negative<<<G256, 256, 0, st>>>(a); });
            P_("imm_retry_decide", [&] { vtp::k_retry_decide<<<1, 32, 0, st>>>(a, cudaGraphConditionalHandle{}, 0); });
            if (!s.phase_retry_all) P_("imm_drift_mark", [&] { vtp::k_drift_mark<<<G256, 256, 0, st>>>(a); });
            P_("imm_drift_diffuse", [&] { VTP_PHASE_DISPATCH(P, VTP_UNROLL_DISPATCH(s.unroll, vtp::k_drift_diffuse<UU, PP><<<G, B, 0, st>>>(a, 1))) });
            CUI(cudaMemcpyAsync(s.h_pinned + 5, m.counter + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            CUI(cudaStreamSynchronize(st));
            if (s.h_pinned[5]) break;
        }
    }
    P_("imm_phase_finish", [&] { vtp::k_phase_finish<<<G256, 256, 0, st>>>(a); });
    return VTP_OK;
}

int immct_get_field(vtp_solver &s, int field, float *dev_out, size_t elems) {
    ImmState &m = *s.imm;
    const int P = m.p.P;
    const uint32_t n = s.L.n, nf = s.L.nf;
    std::vector<uint32_t> ids(n);
    CUI(cudaMemcpy(ids.data(), s.orig.c(), n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    std::vector<float> out(n * elems, 0.f);
    auto fetch = [&](const float *src, std::vector<float> &dst) -> int {
        dst.resize(nf);
        if (nf) CUI(cudaMemcpy(dst.data(), src, nf * sizeof(float), cudaMemcpyDeviceToHost));
        return VTP_OK;
    };
    std::vector<float> tmp;
    int rc;
    if (field == VTP_FIELD_VOL_FRAC) {
        for (uint32_t i = 0; i < n; ++i)
            for (int k = 0; k < P; ++k) out[(size_t)i * P + k] = m.bfrac[(size_t)i * P + k];
        for (int k = 0; k < P; ++k) {
            if ((rc = fetch(m.frac[k].c(), tmp))) return rc;
            for (uint32_t r = 0; r < nf; ++r) out[(size_t)ids[r] * P + k] = tmp[r];
        }
    } else if (field == VTP_FIELD_PHASE_VEL) {
        std::vector<float4> v4(nf);
        std::vector<float4> bv(n - nf);
        if (n > nf) CUI(cudaMemcpy(bv.data(), s.vel.c() + nf, (n - nf) * sizeof(float4), cudaMemcpyDeviceToHost));
        for (uint32_t r = nf; r < n; ++r)
            for (int k = 0; k < P; ++k) {
                float *o = &out[((size_t)ids[r] * P + k) * 3];
                o[0] = bv[r - nf].x; o[1] = bv[r - nf].y; o[2] = bv[r - nf].z;
            }
        for (int k = 0; k < P; ++k) {
            if (nf) CUI(cudaMemcpy(v4.data(), m.vph[k].c(), nf * sizeof(float4), cudaMemcpyDeviceToHost));
            for (uint32_t r = 0; r < nf; ++r) {
                float *o = &out[((size_t)ids[r] * P + k) * 3];
                o[0] = v4[r].x; o[1] = v4[r].y; o[2] = v4[r].z;
            }
        }
    } else if (field == VTP_FIELD_CONFORMATION || field == VTP_FIELD_STRESS) {
        if (!m.p.ct) return vtp::fail(VTP_ERR_ARG, "conformation / stress are IMM-CT fields");
        for (uint32_t r = nf; r < n; ++r)
            if (field == VTP_FIELD_CONFORMATION)
                for (int c = 0; c < 9; ++c) out[(size_t)ids[r] * 9 + c] = (c % 4) == 0 ? 1.f : 0.f;
        // returned as full 3x3 row-major matrices, as the reference stores them
        for (int k = 0; k < vtp::kSym; ++k) {
            if ((rc = fetch(field == VTP_FIELD_CONFORMATION ? m.Q[k].c() : m.tau[k], tmp))) return rc;
            for (int c = 0; c < 9; ++c)
                if (vtp::sym_of(c) == k)
                    for (uint32_t r = 0; r < nf; ++r) out[(size_t)ids[r] * 9 + c] = tmp[r];
        }
    } else if (field == VTP_FIELD_CD || field == VTP_FIELD_REST_DENSITY || field == VTP_FIELD_MASS) {
        std::vector<float> rdv, cdv;
        if ((rc = fetch(m.rd, rdv))) return rc;
        if ((rc = fetch(m.cd, cdv))) return rc;
        std::vector<float4> p4(n);
        CUI(cudaMemcpy(p4.data(), s.pos.c(), n * sizeof(float4), cudaMemcpyDeviceToHost));
        for (uint32_t r = 0; r < n; ++r) {
            float v;
            if (r < nf) {
                v = field == VTP_FIELD_CD ? cdv[r] : field == VTP_FIELD_REST_DENSITY ? rdv[r] : rdv[r] * p4[r].w;
            } else {
                float rb = 0.f;
                for (int k = 0; k < P; ++k) rb = std::fma(m.bfrac[(size_t)ids[r] * P + k], m.p.rho[k], rb);
                v = field == VTP_FIELD_CD ? 0.f : field == VTP_FIELD_REST_DENSITY ? rb : rb * p4[r].w;
            }
            out[ids[r]] = v;
        }
    } else {
        return vtp::fail(VTP_ERR_ARG, "field not available for this solver");
    }
    CUI(cudaMemcpy(dev_out, out.data(), out.size() * sizeof(float), cudaMemcpyHostToDevice));
    return VTP_OK;
}
