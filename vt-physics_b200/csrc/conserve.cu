// Conservation and density-error sums of the fluid, in FP64 on the device:
// total mass, momentum, kinetic energy, per-phase mass (IMM / IMM-CT) and the
// mean density error of the last substep, for one scene or the whole solver.
// These are the trajectory statistics that long runs are compared by; the sums run
// over the sorted rows in a fixed order (per-block tree sums, then one block
// over the blocks' partials), so repeated calls on the same state agree bit
// for bit.
#include "immct.h"
#include "solver.h"

namespace vtp {

namespace {

constexpr int kConsThreads = 256;
constexpr int kConsMax = 6 + kConsPhases;   // mass, momentum x3, kinetic energy, density error, phases

struct ConsArgs {
    uint32_t r0, r1;            // fluid rows [r0, r1)
    const float4 *pos, *vel;    // w = mass (PBF) or volume (DFSPH, IMM)
    int mass_kind;              // 0: pos.w, 1: the constant mf, 2: rest density * volume
    float mf;
    const float *rd;            // IMM: rest density per fluid row
    int P;                      // IMM phases
    const float *frac[kConsPhases];
    float rho_k[kConsPhases];
    const float *dens;          // density (PBF, scaled by 1/rho0) or compression ratio
    float dens_scale;
    int K;                      // quantities summed
    double *partials;           // [blocks][kConsMax]
};

__device__ __forceinline__ double block_sum_cons(double v) {
    __shared__ double sm[kConsThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sm[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (wid == 0) {
        s = lane < kConsThreads / 32 ? sm[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    return s;   // valid in thread 0
}

__global__ void __launch_bounds__(kConsThreads) k_cons_partials(ConsArgs a) {
    const uint32_t r = a.r0 + blockIdx.x * kConsThreads + threadIdx.x;
    double q[kConsMax];
#pragma unroll
    for (int k = 0; k < kConsMax; ++k) q[k] = 0.0;
    if (r < a.r1) {
        const float4 p = a.pos[r], v = a.vel[r];
        double m;
        if (a.mass_kind == 0) m = (double)p.w;
        else if (a.mass_kind == 1) m = (double)a.mf;
        else m = (double)a.rd[r] * (double)p.w;
        q[0] = m;
        q[1] = m * (double)v.x;
        q[2] = m * (double)v.y;
        q[3] = m * (double)v.z;
        q[4] = 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
        q[5] = (double)a.dens[r] * (double)a.dens_scale - 1.0;
        for (int k = 0; k < a.P; ++k) q[6 + k] = (double)p.w * (double)a.frac[k][r] * (double)a.rho_k[k];
    }
    for (int k = 0; k < a.K; ++k) {
        const double s = block_sum_cons(q[k]);
        if (threadIdx.x == 0) a.partials[(size_t)blockIdx.x * kConsMax + k] = s;
    }
}

__global__ void __launch_bounds__(kConsThreads) k_cons_total(const double *partials, uint32_t blocks, int K,
                                                             double *out) {
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (uint32_t b = threadIdx.x; b < blocks; b += kConsThreads) s += partials[(size_t)b * kConsMax + k];
        s = block_sum_cons(s);
        if (threadIdx.x == 0) out[k] = s;
    }
}

}  // namespace

}  // namespace vtp

int vtp_solver::conservation(int scene, vtp_conservation *out) {
    using namespace vtp;
    if (!initialized) return fail(VTP_ERR_STATE, "conservation sums before initialize");
    if (scene < -1 || scene >= nscenes()) return fail(VTP_ERR_ARG, "scene index out of range");
    ConsArgs a{};
    if (scene < 0) {
        a.r0 = 0;
        a.r1 = L.nf;
    } else {
        a.r0 = scenes[(size_t)scene].fbase;
        a.r1 = a.r0 + scenes[(size_t)scene].nf;
    }
    *out = vtp_conservation{};
    const uint32_t rows = a.r1 - a.r0;
    if (rows == 0) return VTP_OK;
    a.pos = pos.c();
    a.vel = vel.c();
    if (type == VTP_SOLVER_PBF) {
        a.mass_kind = 0;
        a.dens = density;
        a.dens_scale = 1.f / rho_f;
    } else if (!imm) {
        a.mass_kind = 1;
        a.mf = rho_f * vol0;
        a.dens = ratio;
        a.dens_scale = 1.f;
    } else {
        a.mass_kind = 2;
        a.dens = ratio;
        a.dens_scale = 1.f;
        immct_conservation_inputs(*this, &a.rd, a.frac, a.rho_k, &a.P);
    }
    a.K = 6 + a.P;
    const uint32_t blocks = (rows + kConsThreads - 1) / kConsThreads;
    if (cons_blocks < blocks) {
        if (d_cons) cudaFree(d_cons);
        d_cons = nullptr;
        cons_blocks = 0;
        cudaError_t e = cudaMalloc(&d_cons, ((size_t)blocks + 1) * kConsMax * sizeof(double));
        if (e != cudaSuccess) return fail(VTP_ERR_NOMEM, "conservation partials");
        cons_blocks = blocks;
    }
    a.partials = d_cons + kConsMax;   // [0, kConsMax) holds the totals
    k_cons_partials<<<blocks, kConsThreads, 0, st>>>(a);
    k_cons_total<<<1, kConsThreads, 0, st>>>(a.partials, blocks, a.K, d_cons);
    double h[kConsMax] = {0};
    cudaError_t e = cudaMemcpyAsync(h, d_cons, (size_t)a.K * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    out->fluid_mass = h[0];
    out->momentum[0] = h[1];
    out->momentum[1] = h[2];
    out->momentum[2] = h[3];
    out->kinetic_energy = h[4];
    out->mean_density_error = h[5] / (double)rows;
    out->fluid_particles = rows;
    out->phases = (uint32_t)a.P;
    for (int k = 0; k < a.P; ++k) out->phase_mass[k] = h[6 + k];
    return VTP_OK;
}

extern "C" VTP_API int vtp_solver_get_conservation(vtp_solver *s, int scene, vtp_conservation *out) {
    if (!s || !out) return vtp::fail(VTP_ERR_ARG, "null argument");
    return s->conservation(scene, out);
}
