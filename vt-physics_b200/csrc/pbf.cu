// PBF solver passes for sm_100a (fluid rows only; rows are cell-sorted).
//
// Restates the reference's PBF substep (PBFSolver::tick, PBFSolver.cpp:326-376)
// with the kernels of PBFCudaImpl.cu:34-194 regrouped:
//   lambda pass  = compute_sph_density_and_error_cuda + update_lamb_cuda (:70-122)
//   dx pass      = compute_dx_cuda + apply_dx_cuda (:124-170), positions
//                  written to the second buffer so the pass stays Jacobi
//   xsph pass    = XSPH_cuda + apply_dx_cuda (:172-194, :267-281)
// apply_ext_force_cuda (:146-157) is fused into the neighbour-search sort.
#include "pbf.h"

namespace vtp {

namespace {

// Standard-PBF kernels (form 1): poly6 density, spiky gradient (gradW = g r).
__device__ __forceinline__ float poly6_w(float d2, const PbfArgs &a) {
    if (d2 > a.h2) return 0.f;
    const float d = a.h2 - d2;
    return a.c6 * d * d * d;
}
__device__ __forceinline__ float spiky_g(float d2, const PbfArgs &a) {
    if (!(d2 > 0.f)) return 0.f;
    const float r = sqrtf(d2);
    if (r < 1e-6f * a.k.h || r > a.k.h) return 0.f;
    const float d = a.k.h - r;
    return a.cs * d * d / r;
}
__device__ __forceinline__ float pbf_w(float d2, const PbfArgs &a) {
    return a.form ? poly6_w(d2, a) : cubic_w(d2, a.k);
}
__device__ __forceinline__ float pbf_w0(const PbfArgs &a) { return a.form ? a.c6 * a.h2 * a.h2 * a.h2 : a.k.w0; }

__global__ void __launch_bounds__(256) k_pbf_init_boundary(PbfArgs a, const uint32_t *__restrict__ bncnt,
                                                           const uint32_t *__restrict__ bnbr,
                                                           uint32_t ell_stride) {
    // compute_rigid_particle_volume_cuda (PBFCudaImpl.cu:47-68): V_b = 1 / sum_{boundary j} W_ij
    // (self included), m_b = rho_b V_b.  Only boundary neighbours count.
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nb) return;
    uint32_t i = a.nf + r;
    float4 p = a.pos[i];
    uint32_t n = bncnt[r];
    float delta = n > 0 ? pbf_w0(a) : 0.f;
    const uint32_t *lst = bnbr + ell_index(r, 0, ell_stride);
    for (uint32_t t = 0; t + 1 < n; ++t) {
        uint32_t j = lst[(size_t)t * 32u];
        if (j < a.nf) continue;
        float4 q = a.pos[j];
        delta += pbf_w(dist2(p.x - q.x, p.y - q.y, p.z - q.z), a);
    }
    float vb = 1.f / delta;
    a.vol[i] = vb;
    float mb = a.rho_b * vb;
    p.w = mb;
    a.pos[i] = p;
    a.pos_alt[i] = p;
}

struct PL {
    float4 q;
    float l;
};
struct PV2 {
    float4 q, v;
    float vol;
};

// Neighbour passes, U list entries in flight per thread and L lanes per row
// (L = 1: one thread walks the row's list in order; L > 1: the row's lanes
// take entries lane, lane + L, ... and their partial sums are added by a
// butterfly over the group, so a small scene keeps more of the GPU busy; the
// FP32 sums then group differently from the list order).
template <int U, int L>
__global__ void __launch_bounds__(256) k_pbf_lambda(PbfArgs a) {
    pdl_enter();
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = gt / L;
    const int lane = (int)(gt % L);
    if (r >= a.nf || halo_ghost(a, r)) return;   // the same for every lane of the row
    const float4 p = a.pos[r];
    const uint32_t n = a.ncnt[r];
    // Self is the first entry of every list: density gets m_i W(0), gradients 0.
    float rho = (n > 0 && lane == 0) ? p.w * pbf_w0(a) : 0.f;
    float gx = 0.f, gy = 0.f, gz = 0.f, s2 = 0.f;
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop_lanes<U, L>(lst, n > 0 ? n - 1 : 0, lane, [&](uint32_t j) { return ldg4(a.pos + j); },
                         [&](uint32_t, const float4 &q) {
                             const float dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
                             float w, g;
                             if (a.form == 0) {
                                 cubic_wg(dist2(dx, dy, dz), a.k, w, g);
                             } else {
                                 const float d2 = dist2(dx, dy, dz);
                                 w = poly6_w(d2, a);
                                 g = spiky_g(d2, a) * q.w;   // mass-weighted constraint gradient
                             }
                             rho = __fmaf_rn(q.w, w, rho);
                             const float ex = g * dx, ey = g * dy, ez = g * dz;
                             gx += ex; gy += ey; gz += ez;
                             const float fx = ex * a.inv_rho0, fy = ey * a.inv_rho0, fz = ez * a.inv_rho0;
                             s2 += fx * fx + fy * fy + fz * fz;
                         });
    if constexpr (L > 1) {
        const unsigned m = lane_group_mask<L>();
        rho = lane_sum<L>(rho, m);
        gx = lane_sum<L>(gx, m);
        gy = lane_sum<L>(gy, m);
        gz = lane_sum<L>(gz, m);
        s2 = lane_sum<L>(s2, m);
        if (lane != 0) return;
    }
    if (rho < a.rho0) rho = a.rho0;
    const float err = rho / a.rho0 - 1.f;
    gx /= a.rho0; gy /= a.rho0; gz /= a.rho0;
    s2 += gx * gx + gy * gy + gz * gz;
    a.density[r] = rho;
    const float lam = -err / (s2 + a.eps);
    a.lambda[r] = lam;
    halo_each(a, r, [&](const PeerRows &P, uint32_t q) { P.lambda[q] = lam; });
}

template <int U, int L>
__global__ void __launch_bounds__(256) k_pbf_dx(PbfArgs a) {
    pdl_enter();
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = gt / L;
    const int lane = (int)(gt % L);
    if (r >= a.nf || halo_ghost(a, r)) return;
    const float4 p = a.pos[r];
    const float li = a.lambda[r];
    const uint32_t n = a.ncnt[r];
    float dx = 0.f, dy = 0.f, dz = 0.f;
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    // Boundary lambda is never written by the reference; it is taken as 0.
    nbr_loop_lanes<U, L>(lst, n > 0 ? n - 1 : 0, lane,
                         [&](uint32_t j) { return PL{ldg4(a.pos + j), j < a.nf ? __ldg(a.lambda + j) : 0.f}; },
                         [&](uint32_t, const PL &e) {
                             const float rx = p.x - e.q.x, ry = p.y - e.q.y, rz = p.z - e.q.z;
                             float s;
                             if (a.form == 0) {
                                 s = (li + e.l) * cubic_g(dist2(rx, ry, rz), a.k);
                             } else {   // (lambda_i m_j + lambda_j m_i) gradW
                                 s = (li * e.q.w + e.l * p.w) * spiky_g(dist2(rx, ry, rz), a);
                             }
                             dx = __fmaf_rn(s, rx, dx);
                             dy = __fmaf_rn(s, ry, dy);
                             dz = __fmaf_rn(s, rz, dz);
                         });
    if constexpr (L > 1) {
        const unsigned m = lane_group_mask<L>();
        dx = lane_sum<L>(dx, m);
        dy = lane_sum<L>(dy, m);
        dz = lane_sum<L>(dz, m);
        if (lane != 0) return;
    }
    dx /= a.rho0; dy /= a.rho0; dz /= a.rho0;
    float4 o = p;
    o.x += dx; o.y += dy; o.z += dz;
    a.pos_alt[r] = o;
    float4 v = a.vel[r];
    v.x += dx / a.dt; v.y += dy / a.dt; v.z += dz / a.dt;
    a.vel[r] = v;
    halo_each(a, r, [&](const PeerRows &P, uint32_t q) {
        P.pos[a.halo_pos ^ 1][q] = o;   // the peer's second buffer, current after its swap
        P.vel[a.halo_vel][q] = v;
    });
}

template <int U, int L>
__global__ void __launch_bounds__(256) k_pbf_xsph(PbfArgs a) {
    pdl_enter();
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = gt / L;
    const int lane = (int)(gt % L);
    if (r >= a.nf || halo_ghost(a, r)) return;
    const float4 p = a.pos[r];
    const float4 vi = a.vel[r];
    const uint32_t n = a.ncnt[r];
    float ax = 0.f, ay = 0.f, az = 0.f;
    const uint32_t *lst = a.nbr + ell_index(r, 0, a.ell_stride);
    nbr_loop_lanes<U, L>(lst, n > 0 ? n - 1 : 0, lane,
                         [&](uint32_t j) { return PV2{ldg4(a.pos + j), ldg4(a.vel + j), __ldg(a.vol + j)}; },
                         [&](uint32_t, const PV2 &e) {
                             const float w = pbf_w(dist2(p.x - e.q.x, p.y - e.q.y, p.z - e.q.z), a);
                             const float c = a.xsph_k * e.vol;
                             ax = __fmaf_rn(c * (e.v.x - vi.x), w, ax);
                             ay = __fmaf_rn(c * (e.v.y - vi.y), w, ay);
                             az = __fmaf_rn(c * (e.v.z - vi.z), w, az);
                         });
    if constexpr (L > 1) {
        const unsigned m = lane_group_mask<L>();
        ax = lane_sum<L>(ax, m);
        ay = lane_sum<L>(ay, m);
        az = lane_sum<L>(az, m);
        if (lane != 0) return;
    }
    const float dx = ax * a.dt, dy = ay * a.dt, dz = az * a.dt;
    float4 o = p;
    o.x += dx; o.y += dy; o.z += dz;
    a.pos_alt[r] = o;
    float4 v = vi;
    v.x += dx / a.dt; v.y += dy / a.dt; v.z += dz / a.dt;
    a.vel_alt[r] = v;
}

inline unsigned nblk(uint32_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

void pbf_init_boundary(cudaStream_t st, const PbfArgs &a, const uint32_t *bncnt, const uint32_t *bnbr,
                       uint32_t ell_stride) {
    if (a.nb) k_pbf_init_boundary<<<nblk(a.nb, 256), 256, 0, st>>>(a, bncnt, bnbr, ell_stride);
}
#define VTP_UNROLL_DISPATCH(U, ...)          \
    switch (U) {                                 \
        case 1: { constexpr int UU = 1; __VA_ARGS__; } break; \
        case 2: { constexpr int UU = 2; __VA_ARGS__; } break; \
        case 8: { constexpr int UU = 8; __VA_ARGS__; } break; \
        default: { constexpr int UU = 4; __VA_ARGS__; } break; \
    }
#define VTP_LANES_DISPATCH(L, ...)           \
    switch (L) {                                 \
        case 4: { constexpr int LL = 4; __VA_ARGS__; } break; \
        case 8: { constexpr int LL = 8; __VA_ARGS__; } break; \
        default: { constexpr int LL = 1; __VA_ARGS__; } break; \
    }

void pbf_lambda(cudaStream_t st, const PbfArgs &a, int block) {
    if (a.nf)
        VTP_LANES_DISPATCH(a.lanes, VTP_UNROLL_DISPATCH(a.unroll, launch(k_pbf_lambda<UU, LL>, nblk(a.nf * LL, block), block, 0, st, a)))
}
void pbf_dx(cudaStream_t st, const PbfArgs &a, int block) {
    if (a.nf)
        VTP_LANES_DISPATCH(a.lanes, VTP_UNROLL_DISPATCH(a.unroll, launch(k_pbf_dx<UU, LL>, nblk(a.nf * LL, block), block, 0, st, a)))
}
void pbf_xsph(cudaStream_t st, const PbfArgs &a, int block) {
    if (a.nf)
        VTP_LANES_DISPATCH(a.lanes, VTP_UNROLL_DISPATCH(a.unroll, launch(k_pbf_xsph<UU, LL>, nblk(a.nf * LL, block), block, 0, st, a)))
}

}  // namespace vtp
