// Shared device-side definitions: grid geometry, SPH kernel functions, the
// warp-interleaved neighbour-list layout and the device status word.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

namespace vtp {

// Programmatic dependent launch (sm_90 and later).  A kernel launched with
// launch() while the calling thread's PDL switch is on (PdlScope) has its
// launch processed while the kernel before it in the stream still runs, so its blocks start as that grid exits
// instead of a launch latency later; pdl_enter() (griddepcontrol.wait) then
// returns once the previous grid has completed and its memory is visible.
// Every kernel launched this way calls pdl_enter() before it reads or writes
// global memory, so the stream order of all accesses is unchanged.  No kernel
// triggers its dependents early (griddepcontrol.launch_dependents): waiting
// blocks of the next grid then held SM slots during the tail and the PBF
// substep was 10 % slower.  Without the launch attribute the wait returns at
// once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Host side: whether launch() adds the attribute (set per thread around a
// solver's enqueue by PdlScope).
bool &pdl_flag();
struct PdlScope {
    bool prev;
    explicit PdlScope(bool on) : prev(pdl_flag()) { pdl_flag() = on; }
    ~PdlScope() { pdl_flag() = prev; }
};

template <class... KArgs, class... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_flag() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Status bits set on the device (bit = 1 << vtp_status value).
enum : uint32_t {
    ST_NOT_CONVERGED = 1u << 3,
    ST_NAN = 1u << 4,
    ST_TIMEOUT = 1u << 5,
    ST_BOUNDS = 1u << 6,
};

// Uniform grid exactly as UniformGirdNeighborSearcher::setConfig builds it
// (UniformGridNeighborSearch.cpp:190-228): gridSize = ceil(simSpaceSize / cell),
// linear cell id = z*gy*gx + y*gx + x (UGNSCudaImpl.cu:58-63).
struct Grid {
    float lbx, lby, lbz;
    float cell;        // gridCellSize (= h)
    int gx, gy, gz;    // gridSize
    uint32_t nkey;     // number of key buckets; key nkey is the "outside" bucket
    float d2max;       // largest float d2 with sqrtf(d2) <= cell (IEEE sqrt)
    uint32_t maxnbr;   // maxNeighborNum (self included)
};

// Cell coordinate of a position: floor((p - LB) / cell) per component with
// IEEE division (UGNSCudaImpl.cu:28-48).
__device__ __forceinline__ int3 cell_of(float x, float y, float z, const Grid &g) {
    return make_int3((int)floorf(__fdiv_rn(__fsub_rn(x, g.lbx), g.cell)),
                     (int)floorf(__fdiv_rn(__fsub_rn(y, g.lby), g.cell)),
                     (int)floorf(__fdiv_rn(__fsub_rn(z, g.lbz), g.cell)));
}

// cellIsAvailable (UGNSCudaImpl.cu:73-81): the upper bound is inclusive.
__device__ __forceinline__ bool cell_available(int3 c, const Grid &g) {
    return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x <= g.gx && c.y <= g.gy && c.z <= g.gz;
}

__device__ __forceinline__ uint32_t cell_key(int3 c, const Grid &g) {
    return (uint32_t)c.z * (uint32_t)(g.gy * g.gx) + (uint32_t)c.y * (uint32_t)g.gx + (uint32_t)c.x;
}

// One scene of a solver.  A solver advances S >= 1 independent scenes that
// share the particle radius, time step and material constants but have their
// own domain (simSpaceLB / simSpaceSize) and gravity.  Each scene owns the
// global key buckets [key_base, key_base + nkey]; the last one is its
// "outside" bucket, so a scene's rows stay in one fixed contiguous range of
// the sorted order.  With S = 1 this is exactly the reference's single grid.
struct SceneGrid {
    float lbx, lby, lbz;
    int gx, gy, gz;
    uint32_t key_base;
    uint32_t nkey;             // buckets of in-grid cells (outside bucket excluded)
    float grav_x, grav_y, grav_z;
    int brick;                 // 1: bricked bucket order (cell_key), 0: the reference's linear key
    uint32_t bx, by;           // bricks along x and y
};

// Shared neighbour-search constants plus the per-row scene map.
struct Scenes {
    const SceneGrid *sg;       // [S]
    const uint16_t *row_scene; // [n] scene of each row (rows never change scene)
    float cell;
    float d2max;
    uint32_t maxnbr;
};

__device__ __forceinline__ int3 cell_of(float x, float y, float z, const SceneGrid &g, float cell) {
    return make_int3((int)floorf(__fdiv_rn(__fsub_rn(x, g.lbx), cell)),
                     (int)floorf(__fdiv_rn(__fsub_rn(y, g.lby), cell)),
                     (int)floorf(__fdiv_rn(__fsub_rn(z, g.lbz), cell)));
}

__device__ __forceinline__ bool cell_available(int3 c, const SceneGrid &g) {
    return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x <= g.gx && c.y <= g.gy && c.z <= g.gz;
}

// Scene-local linear cell id: the reference's cell index inside that scene's
// grid (getCellId, UGNSCudaImpl.cu:58-63), used for the exported keys.
__device__ __forceinline__ uint32_t ref_cell_key(int3 c, const SceneGrid &g) {
    return (uint32_t)c.z * (uint32_t)(g.gy * g.gx) + (uint32_t)c.y * (uint32_t)g.gx + (uint32_t)c.x;
}

// Bit i of a 2-bit value moved to bit 3i (Morton interleave of 3 coordinates).
__device__ __forceinline__ uint32_t morton_spread2(uint32_t v) { return (v & 1u) | ((v & 2u) << 2); }

// Scene-local bucket of a cell, the order rows are kept in.  Bricked order:
// the grid is cut into 4 x 4 x 4-cell bricks taken in linear order (x
// fastest), and the 64 cells of a brick follow the Morton (Z) curve, so
// consecutive rows - a warp, a 128-row tile - cover a compact block of cells
// and their neighbourhoods overlap in cache.  Every in-grid cell has its own
// bucket; the reference's linear id (ref_cell_key) instead lets cells on the
// inclusive upper x (y) face share a bucket with the first cell of the next
// row (plane), which only matters for grids under 4 cells wide in x or y:
// those keep the linear order (brick == 0), so that the candidates a row
// visits are the reference's in every grid.  A cell's run is sorted by attach
// id in either order and lists are walked cell by cell in the reference's
// offset order, so the lists do not depend on the bucket order.
__device__ __forceinline__ uint32_t cell_key(int3 c, const SceneGrid &g) {
    if (!g.brick) return ref_cell_key(c, g);
    const uint32_t x = (uint32_t)c.x, y = (uint32_t)c.y, z = (uint32_t)c.z;
    const uint32_t b = ((z >> 2) * g.by + (y >> 2)) * g.bx + (x >> 2);
    return b * 64u + (morton_spread2(x & 3u) | (morton_spread2(y & 3u) << 1) | (morton_spread2(z & 3u) << 2));
}

__device__ __forceinline__ SceneGrid load_scene(const Scenes &sc, uint32_t row) {
    return sc.sg[sc.row_scene[row]];
}

// Squared distance with a fixed FMA pattern; the neighbour-membership test
// `0 < |x_i - x_j| <= cell` (UGNSCudaImpl.cu:194) is evaluated as
// d2 > 0 && d2 <= d2max, which is equivalent for a correctly rounded sqrt.
__device__ __forceinline__ float dist2(float dx, float dy, float dz) {
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

// The 27 neighbour-cell offsets in the reference's order
// (UniformGridNeighborSearch.cpp:33-60): x slowest, z fastest.
__device__ __forceinline__ int3 nbr_offset(int t) {
    return make_int3(t / 9 - 1, (t / 3) % 3 - 1, t % 3 - 1);
}

// Warp-interleaved ELL neighbour list: for row r, slot t lives at
// base + (r/32)*32*stride + t*32 + r%32, so a warp reading slot t of 32
// consecutive rows touches one 128-byte line.
__device__ __forceinline__ size_t ell_index(uint32_t row, uint32_t t, uint32_t stride) {
    return (size_t)(row >> 5) * 32u * stride + (size_t)t * 32u + (row & 31u);
}

// Cubic spline (sph::cubic_value / cubic_gradient, KernelFunctions.cuh:13-57).
struct Cubic {
    float h;       // support radius
    float invh;    // 1 / h
    float sigma;   // 8 / pi / h^3 (FP32 as the reference computes it)
    float w0;      // W(0) = sigma
    int cube_powf = 0;   // outer branch: 1 = powf(1 - q, 3) as the reference, 0 = cube_rn
};

// t^3 rounded to the nearest float, for t >= 0 (no overflow or underflow in
// the range used here).  Compensated product (Ogita, Rump & Oishi, "Accurate
// sum and dot product", SIAM J. Sci. Comput. 2005): t*t = s + es and
// s*t = p + ep exactly by FMA, so t^3 = p + ep + es*t, and the small terms are
// folded into p with one rounding.  powf(t, 3.f) is within one ulp of it on
// the outer-branch domain of cubic_w (t = 1 - q, q in (0.5, 1], i.e.
// t = k * 2^-24, k in [0, 2^23]) and differs from it on about 6 % of those
// inputs; vtp_selftest_cube compares the two over all 2^23 + 1 inputs.
__device__ __forceinline__ float cube_rn(float t) {
    const float s = t * t;
    const float es = __fmaf_rn(t, t, -s);
    const float p = s * t;
    const float ep = __fmaf_rn(s, t, -p);
    return p + __fmaf_rn(es, t, ep);
}

// W(r) from r^2, rounded the way sph::cubic_value rounds it
// (KernelFunctions.cuh:13-34): IEEE sqrt, q = r * (1/h), the inner branch
// evaluated in double and rounded once, the outer branch as
// (sigma * 2) * (1 - q)^3.  The cube is powf(1 - q, 3) as the reference writes
// it when `cube_powf` is set (bit-identical W), else the correctly rounded
// cube_rn, which costs a few FMAs instead of a powf and is at most one ulp
// from it.  Density-ratio sums feed `ratio - 1`, where FP32 rounding is
// amplified ~1e3 times in the pressure solve, so W follows the reference's
// arithmetic; gradients use the faster form below.
__device__ __forceinline__ float cubic_w(float d2, const Cubic &k) {
    const float r = sqrtf(d2);
    const float q = r * k.invh;
    if (q > 1.f) return 0.f;
    if (q <= 0.5f) {
        const float q2 = q * q;
        const float q3 = q2 * q;
        return static_cast<float>((double)k.sigma * (6.0 * (double)q3 - 6.0 * (double)q2 + 1.0));
    }
    const float t = 1.f - q;
    return k.sigma * 2.f * (k.cube_powf ? powf(t, 3.f) : cube_rn(t));
}

// Scalar g with gradW(r_vec) = g * r_vec; zero for q < 1e-6 or q > 1.
// Every rounding is explicit, so g is the same bits in every kernel that
// evaluates it, whatever the compiler contracts around the call.
__device__ __forceinline__ float cubic_g(float d2, const Cubic &k) {
    if (!(d2 > 0.f)) return 0.f;   // coincident particles: q < 1e-6 -> 0
    const float rinv = rsqrtf(d2);
    const float r = __fmul_rn(d2, rinv);
    const float q = __fmul_rn(r, k.invh);
    if (q < 1e-6f || q > 1.f) return 0.f;
    float f;
    if (q <= 0.5f) f = __fmul_rn(__fmul_rn(6.f, q), __fmaf_rn(3.f, q, -2.f));
    else {
        const float t = __fsub_rn(1.f, q);
        f = __fmul_rn(__fmul_rn(-6.f, t), t);
    }
    return __fmul_rn(__fmul_rn(f, k.sigma), __fmul_rn(rinv, k.invh));
}

// W and g together.
__device__ __forceinline__ void cubic_wg(float d2, const Cubic &k, float &w, float &g) {
    w = cubic_w(d2, k);
    g = cubic_g(d2, k);
}

// sigma = 8 / pi / powf(h, 3) evaluated on the device, as every reference
// kernel evaluates it (KernelFunctions.cuh:16-17).
__global__ void k_cubic_sigma(float h, float *out);

// Akinci cohesion spline sph::surface_tension_C (KernelFunctions.cuh:59-70).
__device__ __forceinline__ float tension_c(float r, float h, float csigma, float h6_64) {
    if (r * 2.f > h && r <= h) {
        float a = h - r;
        return csigma * (a * a * a) * (r * r * r);
    }
    if (r > 0.f && r * 2.f <= h) {
        float a = h - r;
        return csigma * (2.f * (a * a * a) * (r * r * r) - h6_64);
    }
    return 0.f;
}

__device__ __forceinline__ float4 ldg4(const float4 *p) { return __ldg(p); }

// Two adjacent float4 (one 32-byte aligned row of a packed array) in one
// 256-bit read-only load.
struct F4x2 {
    float4 a, b;
};
__device__ __forceinline__ F4x2 ldg8(const float4 *p) {
    F4x2 r;
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(r.a.x), "=f"(r.a.y), "=f"(r.a.z), "=f"(r.a.w), "=f"(r.b.x), "=f"(r.b.y), "=f"(r.b.z), "=f"(r.b.w)
        : "l"(p));
    return r;
}

// Walks `cnt` list entries (warp-interleaved ELL, slot t at lst[t * 32]) in
// order, U at a time: the list indices of the next batch are loaded before the
// current batch's gathers (`load(j)`) are issued, so each thread keeps U
// gathers and U index loads in flight.  `use(j, data)` runs in list order,
// which keeps FP32 accumulation order identical for every U.
template <int U, class Load, class Use>
__device__ __forceinline__ void nbr_loop(const uint32_t *__restrict__ lst, uint32_t cnt, Load load, Use use) {
    if constexpr (U <= 1) {
        for (uint32_t t = 0; t < cnt; ++t) {
            const uint32_t j = __ldcs(lst + (size_t)t * 32u);
            use(j, load(j));
        }
    } else {
        using T = decltype(load(0u));
        uint32_t nxt[U];
#pragma unroll
        for (int u = 0; u < U; ++u) nxt[u] = (uint32_t)u < cnt ? __ldcs(lst + (size_t)u * 32u) : 0u;
        uint32_t t = 0;
        for (; t + U <= cnt; t += U) {
            uint32_t j[U];
#pragma unroll
            for (int u = 0; u < U; ++u) j[u] = nxt[u];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint32_t tt = t + U + (uint32_t)u;
                nxt[u] = tt < cnt ? __ldcs(lst + (size_t)tt * 32u) : 0u;
            }
            T d[U];
#pragma unroll
            for (int u = 0; u < U; ++u) d[u] = load(j[u]);
#pragma unroll
            for (int u = 0; u < U; ++u) use(j[u], d[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (t + (uint32_t)u < cnt) use(nxt[u], load(nxt[u]));
        }
    }
}

// Lane groups for rows walked by L lanes each (L divides 32; the L lanes of a
// row are one aligned group of a warp).
template <int L>
__device__ __forceinline__ unsigned lane_group_mask() {
    if constexpr (L >= 32) return 0xffffffffu;
    else return ((1u << L) - 1u) << ((threadIdx.x & 31u) & ~(unsigned)(L - 1));
}

// Butterfly sum over a row's L lanes; every lane gets the same bits (each
// step adds the same two values on both partner lanes).
template <int L>
__device__ __forceinline__ float lane_sum(float v, unsigned mask) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, L);
    return v;
}

// nbr_loop over a row's entries lane, lane + L, lane + 2L, ...: L lanes share
// one row's list and each keeps U gathers in flight.  With L == 1 this is
// nbr_loop itself (same order, same results).
template <int U, int L, class Load, class Use>
__device__ __forceinline__ void nbr_loop_lanes(const uint32_t *__restrict__ lst, uint32_t cnt, int lane, Load load,
                                               Use use) {
    if constexpr (L == 1) {
        nbr_loop<U>(lst, cnt, load, use);
    } else {
        using T = decltype(load(0u));
        uint32_t t = (uint32_t)lane;
        for (; t + (uint32_t)((U - 1) * L) < cnt; t += (uint32_t)(U * L)) {
            uint32_t j[U];
#pragma unroll
            for (int u = 0; u < U; ++u) j[u] = __ldcs(lst + (size_t)(t + (uint32_t)(u * L)) * 32u);
            T d[U];
#pragma unroll
            for (int u = 0; u < U; ++u) d[u] = load(j[u]);
#pragma unroll
            for (int u = 0; u < U; ++u) use(j[u], d[u]);
        }
        for (; t < cnt; t += (uint32_t)L) {
            const uint32_t j = __ldcs(lst + (size_t)t * 32u);
            use(j, load(j));
        }
    }
}

}  // namespace vtp
