// DFSPH solver passes for sm_100a (fluid rows only; rows are cell-sorted).
//
// Restates DFSPHSolver::tick (DFSPHSolver.cpp:339-406) with the kernels of
// DFSPHCudaImpl.cu regrouped into neighbour passes:
//   ratio_alpha : compute_compression_ratio_cuda + compute_df_beta_cuda (:85-140)
//   solve_a     : compute_delta_compression_ratio_cuda +
//                 update_delta_compression_ratio_from_vel_adv_cuda +
//                 compute_kappa_{div,incomp}_... (:142-196, :355-367) and the
//                 per-block FP64 partial sums of the residual
//   solve_b     : vf_update_vel_adv_from_kappa_{div,incomp}_cuda (:198-220, :369-391)
//   solve_end   : the residual (mean over fluid objects of the object's mean
//                 clamped compression error, as vfsph_div computes it with
//                 cal_mean, :449-503) in FP64 on the device, the stop test
//                 (residual < threshold or iteration > 100) and the loop
//                 condition of the CUDA-graph WHILE node
//   viscosity   : apply_pressure_acc (:505-521) evaluated on the fly for i
//                 and j, then clear_acc + add_acc_gravity +
//                 add_acc_explicit_lap_vis + acc_2_vel (:222-296, :523-554)
//   vis_normal / tension : the same with compute_surface_normal_cuda and
//                 add_acc_surface_tension_cuda (:298-353) when gamma != 0
//   finalize    : apply_pressure_acc + update_pos_cuda (:393-404)
#include "dfsph.h"

#include <algorithm>

namespace vtp {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sm[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sm[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    double s = 0.0;
    if (wid == 0) {
        s = lane < nw ? sm[lane] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

__device__ __forceinline__ float4 pressure_applied(float4 v, float4 va, float inv_dt, float dt) {
    // add_acc_pressure_cuda + acc_2_vel: acc = (v* - v) / dt; v += acc dt.
    float4 o = v;
    o.x = __fmaf_rn((va.x - v.x) * inv_dt, dt, v.x);
    o.y = __fmaf_rn((va.y - v.y) * inv_dt, dt, v.y);
    o.z = __fmaf_rn((va.z - v.z) * inv_dt, dt, v.z);
    return o;
}

// Time step of the running substep: the fixed dt, or the adaptive one on the device
// (1/dt and 1/dt^2 formed as the host forms them for the fixed step).
struct StepDt {
    float dt, inv_dt, inv_dt2;
};
__device__ __forceinline__ StepDt step_dt(const DfsphArgs &a) {
    if (!a.dtp) return StepDt{a.dt, a.inv_dt, a.inv_dt2};
    const float dt = *a.dtp;
    const float inv = 1.f / dt;
    return StepDt{dt, inv, inv * inv};
}

__global__ void __launch_bounds__(256) k_rigid_volume(DfsphArgs a, const uint32_t *__restrict__ bncnt,
                                                      const uint32_t *__restrict__ bnbr,
                                                      float *__restrict__ rest_density_b) {
    // compute_rigid_volume_cuda (DFSPHCudaImpl.cu:63-83): V_b = 1 / sum_{boundary j} W_ij,
    // boundary rest_density = V_b * rho_b.
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nb) return;
    uint32_t i = a.nf + r;
    float4 p = a.pos[i];
    uint32_t n = bncnt[r];
    float delta = n > 0 ? a.k.w0 : 0.f;
    const uint32_t *lst = bnbr + ell_index(r, 0, a.ell_stride);
    for (uint32_t t = 0; t + 1 < n; ++t) {
        uint32_t j = lst[(size_t)t * 32u];
        if (j < a.nf) continue;
        float4 q = a.pos[j];
        delta += cubic_w(dist2(p.x - q.x, p.y - q.y, p.z - q.z), a.k);
    }
    float vb = 1.f / delta;
    p.w = vb;
    a.pos[i] = p;
    rest_density_b[r] = vb * a.rho_b;
}

// DFSPH compression ratio and alpha of one row (compute_compression_ratio_cuda +
// compute_df_beta_cuda, DFSPHCudaImpl.cu:85-140), accumulated entry by entry in list
// order, every rounding explicit.
struct RatioAlpha {
    float ratio, a1x, a1y, a1z, a2;

    // self_w: the self term V_i W(0) (0 for a row outside the grid, which has no list)
    __device__ __forceinline__ void begin(float self_w) {
        ratio = self_w;
        a1x = a1y = a1z = 0.f;
        a2 = 1e-6f;
    }
    // One list entry j: d2 = |x_i - x_j|^2, (dx, dy, dz) = x_i - x_j, vj = V_j.
    __device__ __forceinline__ void add(float d2, float dx, float dy, float dz, float vj, bool fluid_j,
                                        const Cubic &k, float inv_mf) {
        float w, g;
        cubic_wg(d2, k, w, g);
        ratio = __fmaf_rn(vj, w, ratio);
        const float gx = __fmul_rn(g, dx), gy = __fmul_rn(g, dy), gz = __fmul_rn(g, dz);
        a1x = __fmaf_rn(vj, gx, a1x);
        a1y = __fmaf_rn(vj, gy, a1y);
        a1z = __fmaf_rn(vj, gz, a1z);
        if (fluid_j) a2 = __fmaf_rn(__fmul_rn(__fmul_rn(dist2(gx, gy, gz), vj), vj), inv_mf, a2);
    }
    __device__ __forceinline__ float alpha(float mass_f) const {
        const float al = __fadd_rn(__fdiv_rn(dist2(a1x, a1y, a1z), mass_f), a2);
        return al < 1e-6f ? 1e-6f : al;
    }
};

struct PV {
    float4 q, v;
};
struct PN {
    float4 q, n;
};

template <int U>
__global__ void __launch_bounds__(256) k_ratio_alpha(DfsphArgs a) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf || halo_ghost(a, r)) return;
    const float4 p = a.pos[r];
    const uint32_t n = a.ncnt[r];
    RatioAlpha ra;
    ra.begin(n > 0 ? __fmul_rn(p.w, a.k.w0) : 0.f);   // self term V_i W(0)
    const float inv_mf = __fdiv_rn(1.f, a.mass_f);
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop<U>(lst, n > 0 ? n - 1 : 0, [&](uint32_t j) { return ldg4(a.pos + j); },
                [&](uint32_t j, const float4 &q) {
                    const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
                    ra.add(dist2(dx, dy, dz), dx, dy, dz, q.w, j < a.nf, a.k, inv_mf);
                });
    a.ratio[r] = ra.ratio;
    a.alpha[r] = ra.alpha(a.mass_f);
}

// Tile kernels run a persistent grid over the scene-offset tiles; a tile of a
// scene whose solve has stopped is skipped (block-uniform test).
template <bool MULTI, int U>
__global__ void __launch_bounds__(256) k_solve_a(DfsphArgs a) {
    const StepDt T = step_dt(a);
    for (uint32_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const uint4 tile = a.tiles[t];
        const bool stopped = a.state[tile.z].stopped != 0;
        if (a.tile_ran && threadIdx.x == 0) a.tile_ran[t] = stopped ? 0u : 1u;
        if (stopped) continue;
        const uint32_t r = tile.x + threadIdx.x;
        double contrib = 0.0;
        int obj = 0;
        if (threadIdx.x < tile.y && !halo_ghost(a, r)) {
            const float4 p = a.pos[r];
            const float4 vi = a.vadv[r];
            const uint32_t n = a.ncnt[r];
            float d = a.ratio[r] - 1.f;
            const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
            nbr_loop<U>(lst, n > 0 ? n - 1 : 0, [&](uint32_t j) { return ldg8(a.pva + 2 * (size_t)j); },
                        [&](uint32_t, const F4x2 &e) {
                            const float rx = p.x - e.a.x, ry = p.y - e.a.y, rz = p.z - e.a.z;
                            const float g = cubic_g(dist2(rx, ry, rz), a.k);
                            const float dot =
                                g * (rx * (vi.x - e.b.x) + ry * (vi.y - e.b.y) + rz * (vi.z - e.b.z));
                            d = __fmaf_rn(dot * e.a.w, T.dt, d);
                        });
            if (d < 0.f) d = 0.f;
            a.delta[r] = d;
            const float kap = d / a.alpha[r] * T.inv_dt2 / p.w;
            a.kappa[r] = kap;
            const float4 pkr = make_float4(p.x, p.y, p.z, kap);
            a.pk[r] = pkr;
            halo_each(a, r, [&](const PeerRows &P, uint32_t q) {
                P.kappa[q] = kap;
                P.pk[q] = pkr;
            });
            contrib = (double)d;
            if (MULTI) obj = (int)a.obj_of[a.orig[r]] - (int)a.scene_tiles[tile.z].obj0;
        }
        if (!MULTI) {
            double s = block_sum(contrib);
            if (threadIdx.x == 0) a.partials[t] = s;
        } else {
            const int no = (int)a.scene_tiles[tile.z].nobj;
            for (int o = 0; o < no; ++o) {
                double s = block_sum(obj == o ? contrib : 0.0);
                if (threadIdx.x == 0) a.partials[(size_t)t * a.nobj_max + o] = s;
            }
        }
    }
}

// Staged solve_a: one block per brick (staged.h); the block copies the
// packed {x, v*} rows of the group's neighbourhood into shared memory and each
// row gathers through its slot list, in list order, so delta and kappa are
// the bits the unstaged pass computes.  A group whose neighbourhood exceeds
// the capacity, and the rows outside the grid (block ngroups), gather from
// global memory.  The FP64 residual partials are per group.
template <bool MULTI, int U>
__global__ void __launch_bounds__(kStageBlock) k_solve_a_staged(DfsphArgs a) {
    extern __shared__ float4 stage[];   // slot s = {stage[2s], stage[2s + 1]}
    __shared__ GroupPlan P;
    if (a.state[0].stopped) return;
    const StepDt T = step_dt(a);
    const uint32_t grp = blockIdx.x;
    const SceneGrid g = a.sc.sg[0];
    uint32_t r0, r1;
    bool staged = false;
    if (grp == a.stg.ngroups) {
        const uint32_t k = g.key_base + g.nkey;
        r0 = __ldg(a.stg.fstart + k);
        r1 = __ldg(a.stg.fstart + k + 1);
    } else {
        const uint2 rows = group_rows(grp, g, a.stg);
        r0 = rows.x;
        r1 = rows.y;
        if (r0 != r1) {
            plan_group(P, grp, g, a.stg);
            staged = P.total <= a.stg.scap;
        }
    }
    if (staged) {
        for (uint32_t s = threadIdx.x; s < P.total; s += blockDim.x) {
            bool b;
            const uint32_t j = a.stg.mode == 0 ? slot_row<0>(P, slot_cell(P, s), s, b)
                                               : slot_row<1>(P, slot_cell(P, s), s, b);
            const F4x2 e = ldg8(a.pva + 2 * (size_t)j);
            stage[2 * s] = e.a;
            stage[2 * s + 1] = e.b;
        }
        __syncthreads();
    }
    double contrib = 0.0;
    for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
        const float4 p = a.pos[r];
        const float4 vi = a.vadv[r];
        const uint32_t n = a.ncnt[r];
        float d = a.ratio[r] - 1.f;
        auto use = [&](auto, const F4x2 &e) {
            const float rx = p.x - e.a.x, ry = p.y - e.a.y, rz = p.z - e.a.z;
            const float gw = cubic_g(dist2(rx, ry, rz), a.k);
            const float dot = gw * (rx * (vi.x - e.b.x) + ry * (vi.y - e.b.y) + rz * (vi.z - e.b.z));
            d = __fmaf_rn(dot * e.a.w, T.dt, d);
        };
        const uint32_t cnt = n > 0 ? n - 1 : 0;
        if (staged) {
            slot_loop<U>(a.stg.snbr + ell_index(r, 0, a.ell_stride), cnt,
                         [&](uint16_t s) {
                             uint32_t q = (uint32_t)(s & 0x7fffu);
#ifdef VTP_CHECKED
                             if (q >= P.total) {   // a slot outside the staged rows: record it, read slot 0
                                 atomicOr(a.status, ST_BOUNDS);
                                 q = 0;
                             }
#endif
                             q *= 2u;
                             return F4x2{stage[q], stage[q + 1]};
                         },
                         use);
        } else {
            nbr_loop<U>(a.nbr + ell_index(r, 0, a.ell_stride), cnt,
                        [&](uint32_t j) { return ldg8(a.pva + 2 * (size_t)j); }, use);
        }
        if (d < 0.f) d = 0.f;
        a.delta[r] = d;
        const float kap = d / a.alpha[r] * T.inv_dt2 / p.w;
        a.kappa[r] = kap;
        a.pk[r] = make_float4(p.x, p.y, p.z, kap);
        contrib += (double)d;
    }
    if (!MULTI) {
        const double s = block_sum(contrib);
        if (threadIdx.x == 0) a.partials[grp] = s;
    } else {
        const int no = (int)a.scene_tiles[0].nobj;
        for (int o = 0; o < no; ++o) {
            double c = 0.0;
            for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
                if ((int)a.obj_of[a.orig[r]] - (int)a.scene_tiles[0].obj0 == o) c += (double)a.delta[r];
            const double s = block_sum(c);
            if (threadIdx.x == 0) a.partials[(size_t)grp * a.nobj_max + o] = s;
        }
    }
}

// Staged solve_b: gathers the packed {x, kappa_j} (fluid) / {x, V_j}
// (boundary) rows from the group's staged copy; bit 15 of a slot marks a
// boundary neighbour.
template <int U>
__global__ void __launch_bounds__(kStageBlock) k_solve_b_staged(DfsphArgs a) {
    extern __shared__ float4 stage[];
    __shared__ GroupPlan P;
    if (a.state && a.state[0].stopped) return;
    const StepDt T = step_dt(a);
    const uint32_t grp = blockIdx.x;
    const SceneGrid g = a.sc.sg[0];
    uint32_t r0, r1;
    bool staged = false;
    if (grp == a.stg.ngroups) {
        const uint32_t k = g.key_base + g.nkey;
        r0 = __ldg(a.stg.fstart + k);
        r1 = __ldg(a.stg.fstart + k + 1);
    } else {
        const uint2 rows = group_rows(grp, g, a.stg);
        r0 = rows.x;
        r1 = rows.y;
        if (r0 == r1) return;
        plan_group(P, grp, g, a.stg);
        staged = P.total <= a.stg.scap;
    }
    if (staged) {
        for (uint32_t s = threadIdx.x; s < P.total; s += blockDim.x) {
            bool b;
            const uint32_t j = a.stg.mode == 0 ? slot_row<0>(P, slot_cell(P, s), s, b)
                                               : slot_row<1>(P, slot_cell(P, s), s, b);
            stage[s] = __ldg(a.pk + j);
        }
        __syncthreads();
    }
    for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
        const float4 p = a.pos[r];
        float4 v = a.vadv[r];
        const float ki = a.kappa[r];
        const uint32_t n = a.ncnt[r];
        const float mi = a.rest_density ? a.rest_density[r] * p.w : a.mass_f;
        const float ci = T.dt * p.w / mi;
        auto step = [&](bool fj, const float4 &e) {
            const float Vj = fj ? a.vol_f : e.w, kj = fj ? e.w : 0.f;
            const float rx = p.x - e.x, ry = p.y - e.y, rz = p.z - e.z;
            const float gw = cubic_g(dist2(rx, ry, rz), a.k);
            const float s = ci * Vj * (ki + kj) * gw;
            v.x = __fmaf_rn(-s, rx, v.x);
            v.y = __fmaf_rn(-s, ry, v.y);
            v.z = __fmaf_rn(-s, rz, v.z);
        };
        const uint32_t cnt = n > 0 ? n - 1 : 0;
        if (staged) {
            slot_loop<U>(a.stg.snbr + ell_index(r, 0, a.ell_stride), cnt,
                         [&](uint16_t s) {
                             uint32_t q = (uint32_t)(s & 0x7fffu);
#ifdef VTP_CHECKED
                             if (q >= P.total) {   // a slot outside the staged rows: record it, read slot 0
                                 atomicOr(a.status, ST_BOUNDS);
                                 q = 0;
                             }
#endif
                             return stage[q];
                         },
                         [&](uint16_t s, const float4 &e) { step(!(s & kSlotBoundary), e); });
        } else {
            nbr_loop<U>(a.nbr + ell_index(r, 0, a.ell_stride), cnt, [&](uint32_t j) { return ldg4(a.pk + j); },
                        [&](uint32_t j, const float4 &e) { step(j < a.nf, e); });
        }
        a.vadv[r] = v;
        a.pva[2 * (size_t)r + 1] = v;
    }
}

template <int U>
__global__ void __launch_bounds__(256) k_solve_b(DfsphArgs a) {
    const StepDt T = step_dt(a);
    for (uint32_t t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const uint4 tile = a.tiles[t];
        const bool skip = a.tile_ran ? a.tile_ran[t] == 0u : (a.state && a.state[tile.z].stopped);
        if (skip || threadIdx.x >= tile.y) continue;
        const uint32_t r = tile.x + threadIdx.x;
        if (halo_ghost(a, r)) continue;
        const float4 p = a.pos[r];
        float4 v = a.vadv[r];
        const float ki = a.kappa[r];
        const uint32_t n = a.ncnt[r];
        const float mi = a.rest_density ? a.rest_density[r] * p.w : a.mass_f;
        const float ci = T.dt * p.w / mi;   // dt V_i / m_i
        const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
        // Boundary kappa is 0 (kappa_div zeroed; kappa_incomp never written for boundary); the
        // packed row carries kappa_j for fluid rows (volume vol_f) and V_j for boundary rows.
        nbr_loop<U>(lst, n > 0 ? n - 1 : 0, [&](uint32_t j) { return ldg4(a.pk + j); },
                    [&](uint32_t j, const float4 &e) {
                        const bool fj = j < a.nf;
                        const float Vj = fj ? a.vol_f : e.w, kj = fj ? e.w : 0.f;
                        const float rx = p.x - e.x, ry = p.y - e.y, rz = p.z - e.z;
                        const float g = cubic_g(dist2(rx, ry, rz), a.k);
                        const float s = ci * Vj * (ki + kj) * g;
                        v.x = __fmaf_rn(-s, rx, v.x);
                        v.y = __fmaf_rn(-s, ry, v.y);
                        v.z = __fmaf_rn(-s, rz, v.z);
                    });
        a.vadv[r] = v;
        a.pva[2 * (size_t)r + 1] = v;
        halo_each(a, r, [&](const PeerRows &P, uint32_t q) {
            P.vadv[a.halo_vadv][q] = v;
            P.pva[2 * (size_t)q + 1] = v;
        });
    }
}

// After the divergence solve: the packed rows' second half becomes the
// velocity after apply_pressure_acc (DFSPHCudaImpl.cu:505-521) for fluid
// rows, so the viscosity pass gathers {x_j, v_j} with one 256-bit load; the
// first half still holds x_j from dfsph_solve_pack (positions do not change
// during the solve).
__global__ void k_pressure_pack(DfsphArgs a) {
    const StepDt T = step_dt(a);
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf) return;
    a.pva[2 * (size_t)r + 1] = pressure_applied(a.vel[r], a.vadv[r], T.inv_dt, T.dt);
}

__global__ void k_solve_pack(DfsphArgs a, uint32_t n) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float4 p = a.pos[r];
    a.pva[2 * (size_t)r] = p;
    a.pva[2 * (size_t)r + 1] = a.vadv[r];
    // With peer-store halos a ghost's {x, kappa} row is written only by its owner's solve_a
    // (which may already be storing it: no fence separates this pack from the peers' solve_a).
    if (r < a.nf && halo_ghost(a, r)) return;
    a.pk[r] = r < a.nf ? make_float4(p.x, p.y, p.z, 0.f) : p;
}

__global__ void k_solve_begin(SolveState *s, LoopState *loop, int nscenes) {
    for (int i = threadIdx.x; i < nscenes; i += blockDim.x) {
        s[i].iter = 0;
        s[i].stopped = 0;
    }
    if (threadIdx.x == 0) {
        loop->done = 0;
        loop->active = 0;
        loop->running = 1;
        loop->iters = 0;
    }
}

// One block per scene: FP64 residual of the scene from its tiles' partials,
// the stop test, and (last block to finish) the loop condition.
__global__ void __launch_bounds__(1024) k_solve_end(SolveCtl c, const double *__restrict__ partials,
                                                   uint32_t *status) {
    SolveState *st = c.state + blockIdx.x;
    const SceneTiles sct = c.scene_tiles[blockIdx.x];
    __shared__ uint32_t was_stopped;
    if (threadIdx.x == 0) was_stopped = st->stopped;
    __syncthreads();
    bool active = false;
    if (!was_stopped) {
        double acc = 0.0;
        for (uint32_t o = 0; o < sct.nobj; ++o) {
            // Each thread adds the partials b = tid, tid + blockDim, ... in that order; the
            // loads are issued eight at a time so that their latencies overlap.
            double s = 0.0;
            for (uint32_t b = threadIdx.x; b < sct.ntiles; b += 8u * blockDim.x) {
                double v[8];
#pragma unroll
                for (uint32_t u = 0; u < 8; ++u) {
                    const uint32_t bb = b + u * blockDim.x;
                    v[u] = bb < sct.ntiles ? partials[(size_t)(sct.tile0 + bb) * c.nobj_max + o] : 0.0;
                }
#pragma unroll
                for (uint32_t u = 0; u < 8; ++u)
                    if (b + u * blockDim.x < sct.ntiles) s += v[u];
            }
            s = block_sum(s);
            if (threadIdx.x == 0) acc += s * c.inv_count[sct.obj0 + o];
        }
        if (threadIdx.x == 0) {
            const double residual = sct.nobj ? acc / (double)sct.nobj : 0.0;
            const uint32_t iter = st->iter + 1;
            st->iter = iter;
            st->residual = residual;
            uint32_t force = c.force_iters;
            if (c.force_seq && c.tick) {
                const uint64_t t = *c.tick;
                if (t < c.force_seq_len) force = c.force_seq[2 * t + c.which];
            }
            bool stop;
            if (force > 0) stop = iter >= force;
            else stop = (residual < (double)c.threshold) || iter > c.max_iters - 1;
            if (!(residual == residual)) {  // NaN residual: stop and flag
                stop = true;
                atomicOr(status, ST_NAN);
            }
            st->stopped = stop ? 1u : 0u;
            if (stop) {
                st->last_iters = iter;
                st->total_iters += iter;
                // vfsph_div / vfsph_incomp flag a crash whenever the loop ran past 100 iterations.
                if (force == 0 && iter > c.max_iters - 1) atomicOr(status, ST_NOT_CONVERGED);
            }
            active = !stop;
        }
    }
    if (threadIdx.x != 0) return;
    if (active) atomicAdd(&c.loop->active, 1u);
    __threadfence();
    const uint32_t prev = atomicAdd(&c.loop->done, 1u);
    if (prev + 1 == gridDim.x) {
        __threadfence();
        const uint32_t act = atomicAdd(&c.loop->active, 0u);
        c.loop->done = 0;
        c.loop->active = 0;
        c.loop->iters += 1;
        c.loop->total += 1;
        c.loop->running = act ? 1u : 0u;
        if (c.use_cond) cudaGraphSetConditional(c.cond, act ? 1u : 0u);
    }
}

template <bool TENSION_SPLIT, int U>
__global__ void __launch_bounds__(256) k_viscosity(DfsphArgs a) {
    const StepDt T = step_dt(a);
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf || halo_ghost(a, r)) return;
    const float4 p = a.pos[r];
    const float4 vi = pressure_applied(a.vel[r], a.vadv[r], T.inv_dt, T.dt);
    const uint32_t n = a.ncnt[r];
    float ax = 0.f, ay = 0.f, az = 0.f;
    float nx = 0.f, ny = 0.f, nz = 0.f;
    const float ncoef = a.k.h * a.mass_f / a.rho0;   // h m_j / rho_rest_j (fluid)
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop<U>(lst, n > 0 ? n - 1 : 0,
                [&](uint32_t j) {
                    if (j >= a.nf) return F4x2{};   // same-material neighbours only
                    return ldg8(a.pva + 2 * (size_t)j);   // {x_j, v_j after the pressure step}
                },
                [&](uint32_t j, const F4x2 &e) {
                    if (j >= a.nf) return;
                    const float rx = p.x - e.a.x, ry = p.y - e.a.y, rz = p.z - e.a.z;
                    const float d2 = dist2(rx, ry, rz);
                    const float g = cubic_g(d2, a.k);
                    const float4 vj = e.b;
                    const float vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
                    const float pi = a.vis_coef * (vx * rx + vy * ry + vz * rz) / (d2 + a.h2_001);
                    const float s = 10.f * pi * g;
                    ax = __fmaf_rn(s, rx, ax);
                    ay = __fmaf_rn(s, ry, ay);
                    az = __fmaf_rn(s, rz, az);
                    if (TENSION_SPLIT) {
                        const float sn = ncoef * g;
                        nx = __fmaf_rn(sn, rx, nx);
                        ny = __fmaf_rn(sn, ry, ny);
                        nz = __fmaf_rn(sn, rz, nz);
                    }
                });
    const SceneGrid &sg = a.sc.sg[a.sc.row_scene[r]];
    const float accx = sg.grav_x + ax, accy = sg.grav_y + ay, accz = sg.grav_z + az;
    if (TENSION_SPLIT) {
        a.acc_tmp[r] = make_float4(accx, accy, accz, 0.f);
        const float4 nrm = make_float4(nx, ny, nz, 0.f);
        a.normal[r] = nrm;
        halo_each(a, r, [&](const PeerRows &P, uint32_t q) { P.normal[q] = nrm; });
        return;
    }
    float4 o = vi;
    o.x = __fmaf_rn(accx, T.dt, vi.x);
    o.y = __fmaf_rn(accy, T.dt, vi.y);
    o.z = __fmaf_rn(accz, T.dt, vi.z);
    a.vel_alt[r] = o;
    a.vadv_alt[r] = o;
    halo_each(a, r, [&](const PeerRows &P, uint32_t q) {
        P.vel[a.halo_vel ^ 1][q] = o;
        P.vadv[a.halo_vadv ^ 1][q] = o;
    });
}

template <int U>
__global__ void __launch_bounds__(256) k_tension(DfsphArgs a) {
    const StepDt T = step_dt(a);
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nf || halo_ghost(a, r)) return;
    const float4 p = a.pos[r];
    const float4 vi = pressure_applied(a.vel[r], a.vadv[r], T.inv_dt, T.dt);
    const float4 ni = a.normal[r];
    const uint32_t n = a.ncnt[r];
    // Fluid rest densities are equal, so k = 2 rho_i / (rho_i + rho_j) is evaluated once.
    const float kk = 2.f * a.rho0 / (a.rho0 + a.rho0);
    const float c1 = -a.gamma * a.mass_f * a.mass_f;
    const float c2 = -a.gamma * a.mass_f;
    float tx = 0.f, ty = 0.f, tz = 0.f;
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop<U>(lst, n > 0 ? n - 1 : 0,
                [&](uint32_t j) {
                    if (j >= a.nf) return PN{};
                    return PN{ldg4(a.pos + j), ldg4(a.normal + j)};
                },
                [&](uint32_t j, const PN &e) {
                    if (j >= a.nf) return;
                    const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                    const float rl = sqrtf(dist2(rx, ry, rz));
                    const float cs = c1 * tension_c(rl, a.k.h, a.csigma, a.h6_64) / rl;
                    tx += kk * (cs * rx + c2 * (ni.x - e.n.x));
                    ty += kk * (cs * ry + c2 * (ni.y - e.n.y));
                    tz += kk * (cs * rz + c2 * (ni.z - e.n.z));
                });
    const float4 acc = a.acc_tmp[r];
    float4 o = vi;
    o.x = __fmaf_rn(acc.x + tx, T.dt, vi.x);
    o.y = __fmaf_rn(acc.y + ty, T.dt, vi.y);
    o.z = __fmaf_rn(acc.z + tz, T.dt, vi.z);
    a.vel_alt[r] = o;
    a.vadv_alt[r] = o;
    halo_each(a, r, [&](const PeerRows &P, uint32_t q) {
        P.vel[a.halo_vel ^ 1][q] = o;
        P.vadv[a.halo_vadv ^ 1][q] = o;
    });
}

__global__ void __launch_bounds__(256) k_finalize(DfsphArgs a) {
    const StepDt T = step_dt(a);
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    float v2 = 0.f;
    if (r < a.nf && !halo_ghost(a, r)) {
        const float4 v = pressure_applied(a.vel[r], a.vadv[r], T.inv_dt, T.dt);
        a.vel[r] = v;
        a.vadv[r] = v;
        if (r == 0 && a.tick) *a.tick += 1;
        float4 p = a.pos[r];
        p.x = __fmaf_rn(v.x, T.dt, p.x);
        p.y = __fmaf_rn(v.y, T.dt, p.y);
        p.z = __fmaf_rn(v.z, T.dt, p.z);
        a.pos[r] = p;
        v2 = dist2(v.x, v.y, v.z);
    }
    if (a.vmax_bits) {   // adaptive step: max |v|^2 of the new velocities for the next substep
        __shared__ uint32_t wmax[8];
        uint32_t b = __reduce_max_sync(0xffffffffu, __float_as_uint(v2));
        if ((threadIdx.x & 31u) == 0) wmax[threadIdx.x >> 5] = b;
        __syncthreads();
        if (threadIdx.x < 32) {
            b = threadIdx.x < (blockDim.x >> 5) ? wmax[threadIdx.x] : 0u;
            b = __reduce_max_sync(0xffffffffu, b);
            if (threadIdx.x == 0 && b) atomicMax(a.vmax_bits, b);   // one atomic per block
        }
    }
}

// Largest |v|^2 over the fluid rows, folded into *vmax_bits (non-negative floats order like
// their bit patterns, so an unsigned atomicMax is a float max).
__global__ void __launch_bounds__(256) k_cfl_max(DfsphArgs a, uint32_t *vmax_bits) {
    float m = 0.f;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < a.nf; r += gridDim.x * blockDim.x) {
        const float4 v = a.vel[r];
        m = fmaxf(m, dist2(v.x, v.y, v.z));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31u) == 0 && m > 0.f) atomicMax(vmax_bits, __float_as_uint(m));
}

// dt = min(dt_max, cfl * diameter / vmax); the scratch word is cleared for the next substep.
// A step below dt_max * 1e-4 (velocities that have blown up) is held at that floor.
__global__ void k_cfl_step(uint32_t *vmax_bits, float cfl, float diameter, float dt_max, float *dtp,
                           float *sim_time) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const float vmax = sqrtf(__uint_as_float(*vmax_bits));
    *vmax_bits = 0u;
    float dt = dt_max;
    if (vmax > 0.f) dt = fmaxf(fminf(dt_max, cfl * diameter / vmax), dt_max * 1e-4f);
    *dtp = dt;
    *sim_time += dt;
}

inline unsigned nblk(uint32_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

unsigned dfsph_tile_grid(uint32_t ntiles, int block, bool persistent) {
    if (ntiles == 0) return 1u;
    if (!persistent) return ntiles;
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    const uint32_t resident = (uint32_t)sms * (uint32_t)(2048 / block);
    return ntiles < resident ? ntiles : resident;
}

void dfsph_rigid_volume(cudaStream_t st, const DfsphArgs &a, const uint32_t *bncnt, const uint32_t *bnbr,
                        float *rest_density_b) {
    if (a.nb) k_rigid_volume<<<nblk(a.nb, 256), 256, 0, st>>>(a, bncnt, bnbr, rest_density_b);
}
#define VTP_UNROLL_DISPATCH(U, ...)          \
    switch (U) {                                 \
        case 1: { constexpr int UU = 1; __VA_ARGS__; } break; \
        case 2: { constexpr int UU = 2; __VA_ARGS__; } break; \
        case 8: { constexpr int UU = 8; __VA_ARGS__; } break; \
        default: { constexpr int UU = 4; __VA_ARGS__; } break; \
    }

void dfsph_ratio_alpha(cudaStream_t st, const DfsphArgs &a, int block) {
    if (a.nf) VTP_UNROLL_DISPATCH(a.unroll, k_ratio_alpha<UU><<<nblk(a.nf, block), block, 0, st>>>(a))
}
void dfsph_solve_begin(cudaStream_t st, SolveState *s, LoopState *loop, int nscenes) {
    k_solve_begin<<<1, 256, 0, st>>>(s, loop, nscenes);
}
void dfsph_solve_pack(cudaStream_t st, const DfsphArgs &a) {
    const uint32_t n = a.nf + a.nb;
    if (n) k_solve_pack<<<nblk(n, 256), 256, 0, st>>>(a, n);
}
template <class K>
static void launch_staged(K kern, cudaStream_t st, const DfsphArgs &a, size_t row_bytes) {
    const size_t smem = (size_t)a.stg.scap * row_bytes;
    // the staged rows may exceed the 48 KB of dynamic shared memory a kernel gets by default
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<a.stg.ngroups + 1, kStageBlock, smem, st>>>(a);
}

void dfsph_solve_a(cudaStream_t st, const DfsphArgs &a, int block) {
    if (a.staged) {
        if (a.nobj_max > 1) VTP_UNROLL_DISPATCH(a.unroll, launch_staged(k_solve_a_staged<true, UU>, st, a, 32))
        else VTP_UNROLL_DISPATCH(a.unroll, launch_staged(k_solve_a_staged<false, UU>, st, a, 32))
        return;
    }
    const unsigned nb = dfsph_tile_grid(a.ntiles, block, a.persistent);
    if (a.nobj_max > 1) VTP_UNROLL_DISPATCH(a.unroll, k_solve_a<true, UU><<<nb, block, 0, st>>>(a))
    else VTP_UNROLL_DISPATCH(a.unroll, k_solve_a<false, UU><<<nb, block, 0, st>>>(a))
}
void dfsph_solve_b(cudaStream_t st, const DfsphArgs &a, int block) {
    if (a.staged) {
        VTP_UNROLL_DISPATCH(a.unroll, launch_staged(k_solve_b_staged<UU>, st, a, 16))
        return;
    }
    const unsigned nb = dfsph_tile_grid(a.ntiles, block, a.persistent);
    VTP_UNROLL_DISPATCH(a.unroll, k_solve_b<UU><<<nb, block, 0, st>>>(a))
}
void dfsph_solve_end(cudaStream_t st, const SolveCtl &c, const double *partials, uint32_t *status) {
    k_solve_end<<<c.nscenes, 1024, 0, st>>>(c, partials, status);
}
void dfsph_cfl_step(cudaStream_t st, float cfl, float diameter, float dt_max, uint32_t *vmax_bits, float *dtp,
                    float *sim_time) {
    k_cfl_step<<<1, 32, 0, st>>>(vmax_bits, cfl, diameter, dt_max, dtp, sim_time);
}
void dfsph_cfl_refresh(cudaStream_t st, const DfsphArgs &a, uint32_t *vmax_bits) {
    cudaMemsetAsync(vmax_bits, 0, sizeof(uint32_t), st);
    if (a.nf) {
        const unsigned g = std::min<unsigned>(nblk(a.nf, 256), 148u * 8u);
        k_cfl_max<<<g, 256, 0, st>>>(a, vmax_bits);
    }
}
void dfsph_pressure_pack(cudaStream_t st, const DfsphArgs &a) {
    if (a.nf) k_pressure_pack<<<nblk(a.nf, 256), 256, 0, st>>>(a);
}
void dfsph_viscosity(cudaStream_t st, const DfsphArgs &a, int block) {
    if (a.nf) VTP_UNROLL_DISPATCH(a.unroll, k_viscosity<false, UU><<<nblk(a.nf, block), block, 0, st>>>(a))
}
void dfsph_vis_normal(cudaStream_t st, const DfsphArgs &a, int block) {
    if (a.nf) VTP_UNROLL_DISPATCH(a.unroll, k_viscosity<true, UU><<<nblk(a.nf, block), block, 0, st>>>(a))
}
void dfsph_tension(cudaStream_t st, const DfsphArgs &a, int block) {
    if (a.nf) VTP_UNROLL_DISPATCH(a.unroll, k_tension<UU><<<nblk(a.nf, block), block, 0, st>>>(a))
}
void dfsph_finalize(cudaStream_t st, const DfsphArgs &a) {
    if (a.nf) k_finalize<<<nblk(a.nf, 256), 256, 0, st>>>(a);
}

}  // namespace vtp
