// Scene generation on the device: the lattice cube and the hollow box of the
// reference's particle generators (ModelHandler.cpp:43-67 cube, :124-154 box),
// written straight into caller-owned device memory with the coordinates the
// host generators produce, bit for bit.
//
// The reference fills these objects in serial host loops; a million-particle
// scene then spends its set-up time generating and copying positions.  Here
// every particle is one thread:
//   cube: the per-axis coordinates are the reference's FP32 running sums
//         (start = r + lb, v += 2r while v < lb + size), so a thread replays
//         the sum up to its index (at most a few hundred additions) and gets
//         the same rounding; the optional jitter is the project's SplitMix64
//         stream (component e of particle p uses draw 3p + e + 1), added in
//         double and rounded once to float, as the host generator does;
//   box:  lattice points i = 0..n per axis at lb + r + 2 r i (double, rounded
//         to float), kept when within `layers` of a face; a kept point's
//         output slot is its grid index minus the interior points before it,
//         which has a closed form, so no scan or scratch memory is needed.
#include <algorithm>
#include <cmath>
#include <string>

#include "../../include/vtp.h"

namespace vtp {
int fail(int code, const std::string &msg);
}

namespace {

inline unsigned nblk(uint64_t n, int b) { return (unsigned)((n + (uint64_t)b - 1) / (uint64_t)b); }

// Number of values of the FP32 run start, start + step, ... below limit.
uint32_t f32_run_count(float start, float limit, float step) {
    uint32_t k = 0;
    for (float v = start; v < limit; v = v + step) {
        if (++k > (1u << 24)) break;   // step too small for the extent: reported as too large
    }
    return k;
}

__device__ __forceinline__ float f32_run_value(float start, float step, uint32_t k) {
    float v = start;
    for (uint32_t i = 0; i < k; ++i) v = __fadd_rn(v, step);
    return v;
}

__device__ __forceinline__ double splitmix64_uniform(uint64_t seed, uint64_t index) {
    uint64_t z = seed + index * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return __dmul_rn((double)(z >> 11), 1.0 / 9007199254740992.0);
}

// pos + (2u - 1) * amplitude * spacing in double, each operation rounded once.
__device__ __forceinline__ float jittered(float x, uint64_t seed, uint64_t draw, double amplitude, double spacing) {
    const double u = splitmix64_uniform(seed, draw);
    const double t = __dmul_rn(__dmul_rn(__dadd_rn(__dmul_rn(2.0, u), -1.0), amplitude), spacing);
    return (float)__dadd_rn((double)x, t);
}

struct CubeArgs {
    float sx, sy, sz;     // first coordinate per axis (r + lb)
    float step;           // 2 r
    uint32_t nx, ny, nz;
    double amplitude, spacing;
    uint64_t seed;
    int jitter;
};

__global__ void k_generate_cube(CubeArgs a, float *__restrict__ out) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t n = (uint64_t)a.nx * a.ny * a.nz;
    if (p >= n) return;
    // x fastest, then y, then z (the reference's loop nest order)
    const uint32_t ix = (uint32_t)(p % a.nx);
    const uint32_t iy = (uint32_t)((p / a.nx) % a.ny);
    const uint32_t iz = (uint32_t)(p / ((uint64_t)a.nx * a.ny));
    float v[3] = {f32_run_value(a.sx, a.step, ix), f32_run_value(a.sy, a.step, iy),
                  f32_run_value(a.sz, a.step, iz)};
    if (a.jitter)
        for (int c = 0; c < 3; ++c) v[c] = jittered(v[c], a.seed, 3 * p + (uint64_t)c + 1, a.amplitude, a.spacing);
    out[3 * p] = v[0];
    out[3 * p + 1] = v[1];
    out[3 * p + 2] = v[2];
}

struct BoxArgs {
    double base[3];       // lb + r (FP32 sum, widened)
    double step;          // 2 r
    int32_t n[3];         // lattice indices 0..n[a] per axis
    int32_t layers;
};

// Points of [lo, hi) below i.
__device__ __forceinline__ int64_t count_below(int32_t i, int32_t lo, int32_t hi) {
    const int32_t c = min(i, hi) - lo;
    return c > 0 ? c : 0;
}

__global__ void k_generate_box(BoxArgs a, float *__restrict__ out) {
    const int64_t N0 = a.n[0] + 1, N1 = a.n[1] + 1, N2 = a.n[2] + 1;
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N0 * N1 * N2) return;
    // first index slowest, third fastest
    const int32_t I = (int32_t)(q / (N1 * N2)), J = (int32_t)((q / N2) % N1), K = (int32_t)(q % N2);
    const int32_t L = a.layers;
    const bool keep = I < L || I >= a.n[0] - L || J < L || J >= a.n[1] - L || K < L || K >= a.n[2] - L;
    if (!keep) return;
    // interior = [L, n - L) per axis; kept points before q = q - interior points before q
    const int32_t ilo = L, ihi = a.n[0] - L, jlo = L, jhi = a.n[1] - L, klo = L, khi = a.n[2] - L;
    const int64_t nJ = jhi > jlo ? jhi - jlo : 0, nK = khi > klo ? khi - klo : 0;
    int64_t inner = count_below(I, ilo, ihi) * nJ * nK;
    if (I >= ilo && I < ihi) {
        inner += count_below(J, jlo, jhi) * nK;
        if (J >= jlo && J < jhi) inner += count_below(K, klo, khi);
    }
    const int64_t slot = q - inner;
    out[3 * slot] = (float)__dadd_rn(a.base[0], __dmul_rn(a.step, (double)I));
    out[3 * slot + 1] = (float)__dadd_rn(a.base[1], __dmul_rn(a.step, (double)J));
    out[3 * slot + 2] = (float)__dadd_rn(a.base[2], __dmul_rn(a.step, (double)K));
}

}  // namespace

extern "C" VTP_API int vtp_generate_cube(float radius, const float lb[3], const float size[3], double jitter_amp,
                                         double jitter_spacing, uint64_t seed, float *d_out, uint32_t capacity,
                                         uint32_t *count, void *stream) {
    if (!lb || !size || !count) return vtp::fail(VTP_ERR_ARG, "null argument");
    if (!(radius > 0.f)) return vtp::fail(VTP_ERR_ARG, "radius must be > 0");
    const float step = 2.f * radius;
    CubeArgs a{};
    a.sx = radius + lb[0];
    a.sy = radius + lb[1];
    a.sz = radius + lb[2];
    a.step = step;
    a.nx = f32_run_count(a.sx, lb[0] + size[0], step);
    a.ny = f32_run_count(a.sy, lb[1] + size[1], step);
    a.nz = f32_run_count(a.sz, lb[2] + size[2], step);
    const uint64_t n = (uint64_t)a.nx * a.ny * a.nz;
    if (a.nx > (1u << 24) || a.ny > (1u << 24) || a.nz > (1u << 24) || n > 0xffffffffull)
        return vtp::fail(VTP_ERR_BOUNDS, "vtp_generate_cube: more than 2^32 particles");
    *count = (uint32_t)n;
    if (n > capacity)
        return vtp::fail(VTP_ERR_BOUNDS, "vtp_generate_cube: " + std::to_string(n) + " particles, capacity " +
                                             std::to_string(capacity));
    if (n == 0) return VTP_OK;
    if (!d_out) return vtp::fail(VTP_ERR_ARG, "null output buffer");
    a.jitter = jitter_amp != 0.0;
    a.amplitude = jitter_amp;
    a.spacing = jitter_spacing;
    a.seed = seed;
    cudaStream_t st = (cudaStream_t)stream;
    k_generate_cube<<<nblk(n, 256), 256, 0, st>>>(a, d_out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VTP_OK : vtp::fail(VTP_ERR_CUDA, cudaGetErrorString(e));
}

extern "C" VTP_API int vtp_generate_box(float radius, const float lb[3], const float size[3], int32_t layers,
                                        float *d_out, uint32_t capacity, uint32_t *count, void *stream) {
    if (!lb || !size || !count) return vtp::fail(VTP_ERR_ARG, "null argument");
    if (!(radius > 0.f) || layers < 1) return vtp::fail(VTP_ERR_ARG, "radius must be > 0 and layers >= 1");
    BoxArgs a{};
    a.step = 2.0 * (double)radius;
    for (int k = 0; k < 3; ++k) {
        const double m = (double)(size[k] + radius) / (2.0 * (double)radius);
        if (!(m >= 0.0) || m > 2.0e6) return vtp::fail(VTP_ERR_BOUNDS, "vtp_generate_box: extent out of range");
        a.n[k] = (int32_t)m;
        a.base[k] = (double)(lb[k] + radius);
    }
    a.layers = layers;
    const int64_t N0 = a.n[0] + 1, N1 = a.n[1] + 1, N2 = a.n[2] + 1;
    const int64_t iI = std::max(0, a.n[0] - 2 * layers), iJ = std::max(0, a.n[1] - 2 * layers),
                  iK = std::max(0, a.n[2] - 2 * layers);
    const int64_t total = N0 * N1 * N2, n = total - iI * iJ * iK;
    if (n > 0xffffffffll || total > (int64_t)1 << 40)
        return vtp::fail(VTP_ERR_BOUNDS, "vtp_generate_box: more than 2^32 particles");
    *count = (uint32_t)n;
    if ((uint64_t)n > capacity)
        return vtp::fail(VTP_ERR_BOUNDS, "vtp_generate_box: " + std::to_string(n) + " particles, capacity " +
                                             std::to_string(capacity));
    if (n == 0) return VTP_OK;
    if (!d_out) return vtp::fail(VTP_ERR_ARG, "null output buffer");
    cudaStream_t st = (cudaStream_t)stream;
    k_generate_box<<<nblk((uint64_t)total, 256), 256, 0, st>>>(a, d_out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VTP_OK : vtp::fail(VTP_ERR_CUDA, cudaGetErrorString(e));
}
