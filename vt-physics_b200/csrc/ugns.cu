// Uniform-grid neighbour search for sm_100a.
//
// Replaces UniformGirdNeighborSearcher::update / cu_update
// (Simulator/Runtime/Source/Modules/NeighborSearch/UGNS/UGNSCudaImpl.cu:96-227).
// Instead of two thrust::sort_by_key calls, a 27-cell neighbour walk over
// particles in attach order and a padded N x maxNbr list, each substep does:
//   hash    : cell key per row + arrival rank inside the cell (atomicAdd)
//   scan    : exclusive scan of the per-cell counts -> cell start table
//   scatter : rows placed into their cell's segment (arrival order)
//   rank    : inside each segment, rank by attach id -> stable (cell, id)
//             order, identical to the reference's stable radix sort, and
//             move the particle state to its new row (float4 SoA)
//   lists   : neighbour list per row in the reference's order (27 offsets
//             in fixed order, ascending attach id inside a cell), stored as
//             a warp-interleaved ELL array of sorted row indices.
#include "internal.h"
#include "staged.h"

#include <type_traits>

namespace vtp {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
// Up to this many rows the list builder runs eight lanes per row.
constexpr uint32_t kSplitRows = 131072;

__device__ __forceinline__ float4 apply_force(float4 p, float4 &v, float dt, float3 g) {
    // apply_ext_force_cuda (PBFCudaImpl.cu:146-157): v += g dt; x += v dt.
    v.x = __fmaf_rn(g.x, dt, v.x);
    v.y = __fmaf_rn(g.y, dt, v.y);
    v.z = __fmaf_rn(g.z, dt, v.z);
    p.x = __fmaf_rn(v.x, dt, p.x);
    p.y = __fmaf_rn(v.y, dt, p.y);
    p.z = __fmaf_rn(v.z, dt, p.z);
    return p;
}

__global__ void k_hash(Scenes sc, uint32_t row0, uint32_t cnt, const float4 *__restrict__ pos,
                       const float4 *__restrict__ vel, float force_dt, uint32_t *__restrict__ key,
                       uint32_t *__restrict__ rank, uint32_t *__restrict__ count) {
    pdl_enter();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const SceneGrid g = load_scene(sc, row0 + i);
    float4 p = pos[row0 + i];
    if (force_dt > 0.f) {
        float4 v = vel[row0 + i];
        p = apply_force(p, v, force_dt, make_float3(g.grav_x, g.grav_y, g.grav_z));
    }
    int3 c = cell_of(p.x, p.y, p.z, g, sc.cell);
    const bool outside = !cell_available(c, g);
    uint32_t k = g.key_base + (outside ? g.nkey : cell_key(c, g));
    key[i] = k;
    const unsigned om = __ballot_sync(__activemask(), outside);
    if (outside) {
        // Every row outside its scene's grid counts into the scene's one outside bucket (whole
        // scenes can leave the box); one atomic per group of lanes with the same bucket keeps
        // that counter from serialising the kernel.  The order inside the outside bucket is
        // arbitrary either way: its rows have no neighbours and are nobody's neighbour.
        const unsigned grp = __match_any_sync(om, k);
        const unsigned lane = threadIdx.x & 31u;
        const int leader = __ffs(grp) - 1;
        uint32_t base = 0;
        if ((int)lane == leader) base = atomicAdd(&count[k], (uint32_t)__popc(grp));
        base = __shfl_sync(grp, base, leader);
        rank[i] = base + (uint32_t)__popc(grp & ((1u << lane) - 1u));
    } else {
        rank[i] = atomicAdd(&count[k], 1u);
    }
}

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t &total) {
    __shared__ uint32_t warp_sums[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    if (wid == 0) {
        uint32_t s = lane < nw ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t warp_off = wid > 0 ? warp_sums[wid - 1] : 0u;
    total = warp_sums[nw - 1];
    __syncthreads();
    return warp_off + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tile_sums(const uint32_t *__restrict__ in, size_t n,
                                                                 uint32_t *__restrict__ sums) {
    pdl_enter();
    size_t base = (size_t)blockIdx.x * kScanTile + threadIdx.x;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        size_t idx = base + (size_t)k * kScanThreads;
        if (idx < n) s += in[idx];
    }
    uint32_t total;
    block_excl_scan(s, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t *sums, size_t tiles) {
    pdl_enter();
    // One block; each thread owns a contiguous run of tiles.
    const size_t per = (tiles + blockDim.x - 1) / blockDim.x;
    size_t b = threadIdx.x * per;
    uint32_t local = 0;
    for (size_t k = 0; k < per; ++k)
        if (b + k < tiles) local += sums[b + k];
    uint32_t total;
    uint32_t off = block_excl_scan(local, total);
    for (size_t k = 0; k < per; ++k) {
        if (b + k < tiles) {
            uint32_t v = sums[b + k];
            sums[b + k] = off;
            off += v;
        }
    }
}

// Exclusive scan of the counters into `out` (plus `base_add`), out[n] = grand
// total.  The counters are zeroed after they are read, so the next hash starts
// from zero without a separate clear.
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(uint32_t *__restrict__ in, size_t n,
                                                             const uint32_t *__restrict__ sums, uint32_t base_add,
                                                             uint32_t *__restrict__ out) {
    pdl_enter();
    // Each thread scans kScanItems consecutive counters.
    __shared__ uint32_t tile[kScanTile];
    size_t t0 = (size_t)blockIdx.x * kScanTile;
    for (int k = 0; k < kScanItems; ++k) {
        size_t idx = t0 + (size_t)k * kScanThreads + threadIdx.x;
        tile[k * kScanThreads + threadIdx.x] = idx < n ? in[idx] : 0u;
        if (idx < n) in[idx] = 0u;
    }
    __syncthreads();
    uint32_t vals[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        vals[k] = tile[threadIdx.x * kScanItems + k];
        s += vals[k];
    }
    uint32_t total;
    uint32_t off = block_excl_scan(s, total) + sums[blockIdx.x] + base_add;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const size_t idx = t0 + (size_t)threadIdx.x * kScanItems + k;
        if (idx + 1 == n) out[n] = off + vals[k];
        tile[threadIdx.x * kScanItems + k] = off;
        off += vals[k];
    }
    __syncthreads();
    for (int k = 0; k < kScanItems; ++k) {
        size_t idx = t0 + (size_t)k * kScanThreads + threadIdx.x;
        if (idx < n) out[idx] = tile[k * kScanThreads + threadIdx.x];
    }
}

__global__ void k_scatter(uint32_t row0, uint32_t cnt, const uint32_t *__restrict__ key,
                          const uint32_t *__restrict__ rank, const uint32_t *__restrict__ start,
                          const uint32_t *__restrict__ orig, uint32_t *__restrict__ tmp_src,
                          uint32_t *__restrict__ tmp_orig, uint32_t *__restrict__ tmp_key, uint32_t *status) {
    pdl_enter();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    uint32_t k = key[i];
    uint32_t d = start[k] - row0 + rank[i];
#ifdef VTP_CHECKED
    if (d >= cnt) {   // a cell segment slot outside the sorted range: record it and skip the write
        if (status) atomicOr(status, ST_BOUNDS);
        return;
    }
#endif
    tmp_src[d] = i;
    tmp_orig[d] = orig[row0 + i];
    tmp_key[d] = k;
}

__global__ void k_rank_reorder(Scenes sc, uint32_t row0, uint32_t cnt, const uint32_t *__restrict__ start,
                               const uint32_t *__restrict__ tmp_src, const uint32_t *__restrict__ tmp_orig,
                               const uint32_t *__restrict__ tmp_key, const float4 *__restrict__ pos_in,
                               float4 *__restrict__ pos_out, const float4 *__restrict__ vel_in,
                               float4 *__restrict__ vel_out, uint32_t *__restrict__ orig_out, Carry carry,
                               float force_dt) {
    pdl_enter();
    uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= cnt) return;
    // A row keeps its scene: slot d lies in the same scene range as its source row.
    const SceneGrid g = load_scene(sc, row0 + d);
    uint32_t k = tmp_key[d];
    uint32_t my = tmp_orig[d];
    uint32_t dst = d;
    if (k < g.key_base + g.nkey) {
        // Stable order inside the cell: rank by attach id.
        uint32_t s0 = start[k] - row0, s1 = start[k + 1] - row0;
        uint32_t r = 0;
        for (uint32_t x = s0; x < s1; ++x) r += (tmp_orig[x] < my) ? 1u : 0u;
        dst = s0 + r;
    }
    uint32_t s = tmp_src[d];
    float4 p = pos_in[row0 + s];
    float4 v = vel_in[row0 + s];
    if (force_dt > 0.f) p = apply_force(p, v, force_dt, make_float3(g.grav_x, g.grav_y, g.grav_z));
    pos_out[row0 + dst] = p;
    vel_out[row0 + dst] = v;
    orig_out[row0 + dst] = my;
    for (int f = 0; f < carry.nf4; ++f) carry.dst4[f][row0 + dst] = carry.src4[f][row0 + s];
    for (int f = 0; f < carry.nf1; ++f) carry.dst1[f][row0 + dst] = carry.src1[f][row0 + s];
}

// Cell culling: distances from a row's position to the six faces of its own
// cell, shrunk by a safety margin.  A neighbour cell whose nearest point lies
// farther than h (d2 > d2max) holds no particle the membership test can accept
// (UGNSCudaImpl.cu:189-199 tests every particle of all 27 cells), so skipping
// it leaves the list unchanged.  The margin (1e-3 cell plus 1e-6 of the
// coordinate's magnitude) covers the rounding of the face positions and of
// the cell assignment floor((x - lb) / cell), both a few ulps of the
// coordinate; a cell inside the margin is simply walked.
struct FaceGaps {
    float lx, hx, ly, hy, lz, hz;   // clearance below / above along each axis (>= 0)

    __device__ __forceinline__ void init(const float4 &p, int3 c, const SceneGrid &g, float cell) {
        gap(p.x, c.x, g.lbx, cell, lx, hx);
        gap(p.y, c.y, g.lby, cell, ly, hy);
        gap(p.z, c.z, g.lbz, cell, lz, hz);
    }
    __device__ __forceinline__ static void gap(float x, int c, float lb, float cell, float &lo, float &hi) {
        const float f0 = __fmaf_rn((float)c, cell, lb);           // lower face of the cell
        const float m = __fmaf_rn(1e-6f, fabsf(f0) + cell, 1e-3f * cell);
        lo = fmaxf(x - f0 - m, 0.f);
        hi = fmaxf(f0 + cell - x - m, 0.f);
    }
    // Whether the neighbour cell at offset o can hold a particle within h.
    __device__ __forceinline__ bool reachable(int3 o, float d2max) const {
        const float ex = o.x < 0 ? lx : (o.x > 0 ? hx : 0.f);
        const float ey = o.y < 0 ? ly : (o.y > 0 ? hy : 0.f);
        const float ez = o.z < 0 ? lz : (o.z > 0 ? hz : 0.f);
        return dist2(ex, ey, ez) <= d2max;
    }
};

// One candidate of the neighbour walk (UGNSCudaImpl.cu:189-199).
struct Walker {
    float px, py, pz;
    uint32_t self;
    uint32_t cnt;        // entries written incl. self
    uint32_t maxnbr;
    uint32_t *out;       // ELL base for this row (slot t at out[t*32])
    bool overflow;

    // The row itself (d2 == 0) fails `d2 > 0` like every coincident particle,
    // as the reference's `0 < |x_i - x_j|` test excludes it.
    __device__ __forceinline__ void accept(uint32_t j, const float4 &q, float d2max) {
        float d2 = dist2(px - q.x, py - q.y, pz - q.z);
        if (d2 > 0.f && d2 <= d2max) {
            if (cnt < maxnbr) {
                out[(size_t)(cnt - 1) * 32u] = j;
                ++cnt;
            } else {
                overflow = true;
            }
        }
    }

    // Same test without the capacity check, for a cell whose candidates all fit
    // in the list.
    __device__ __forceinline__ void accept_room(uint32_t j, const float4 &q, float d2max) {
        const float d2 = dist2(px - q.x, py - q.y, pz - q.z);
        const bool acc = d2 > 0.f && d2 <= d2max;
        if (acc) out[(size_t)(cnt - 1) * 32u] = j;
        cnt += acc ? 1u : 0u;
    }

    template <bool ROOM>
    __device__ __forceinline__ void test(uint32_t j, const float4 &q, float d2max) {
        if (ROOM) accept_room(j, q, d2max);
        else accept(j, q, d2max);
    }

    template <bool ROOM>
    __device__ __forceinline__ void visit(uint32_t j, const float4 *__restrict__ pos, float d2max) {
        test<ROOM>(j, __ldg(pos + j), d2max);
    }

    // Candidates [j0, j1) in order; positions loaded four at a time.
    template <bool ROOM>
    __device__ __forceinline__ void visit_run(uint32_t j0, uint32_t j1, const float4 *__restrict__ pos,
                                              float d2max) {
        uint32_t j = j0;
        for (; j + 4 <= j1; j += 4) {
            const float4 q0 = __ldg(pos + j), q1 = __ldg(pos + j + 1), q2 = __ldg(pos + j + 2),
                         q3 = __ldg(pos + j + 3);
            test<ROOM>(j, q0, d2max);
            test<ROOM>(j + 1, q1, d2max);
            test<ROOM>(j + 2, q2, d2max);
            test<ROOM>(j + 3, q3, d2max);
        }
        for (; j < j1; ++j) visit<ROOM>(j, pos, d2max);
    }

    // One cell: fluid run [f0, f1) and boundary run [b0, b1) in MODE's order.
    template <int MODE, bool ROOM>
    __device__ __forceinline__ void visit_cell(uint32_t f0, uint32_t f1, uint32_t b0, uint32_t b1,
                                               const float4 *__restrict__ pos, const uint32_t *__restrict__ orig,
                                               float d2max) {
        if (MODE == 0) {
            visit_run<ROOM>(f0, f1, pos, d2max);
            visit_run<ROOM>(b0, b1, pos, d2max);
        } else if (MODE == 1) {
            visit_run<ROOM>(b0, b1, pos, d2max);
            visit_run<ROOM>(f0, f1, pos, d2max);
        } else {
            // Merge the two id-sorted runs by attach id.
            while (f0 < f1 || b0 < b1) {
                uint32_t j;
                if (b0 >= b1) j = f0++;
                else if (f0 >= f1) j = b0++;
                else j = (__ldg(orig + f0) < __ldg(orig + b0)) ? f0++ : b0++;
                visit<ROOM>(j, pos, d2max);
            }
        }
    }
};

template <int MODE, bool CULL>
__global__ void k_build_lists(Scenes sc, uint32_t row0, uint32_t cnt, uint32_t ell_stride,
                              const float4 *__restrict__ pos, const uint32_t *__restrict__ orig,
                              const uint32_t *__restrict__ fstart, const uint32_t *__restrict__ bstart,
                              uint32_t *__restrict__ nbr, uint32_t *__restrict__ ncnt,
                              uint32_t *__restrict__ status, uint32_t *__restrict__ overflow_count) {
    pdl_enter();
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cnt) return;
    uint32_t i = row0 + r;
    const SceneGrid g = load_scene(sc, i);
    float4 p = pos[i];
    int3 c = cell_of(p.x, p.y, p.z, g, sc.cell);
    if (!cell_available(c, g)) {  // outside the grid: no neighbours, not even self
        ncnt[r] = 0;
        return;
    }
    Walker w;
    w.px = p.x; w.py = p.y; w.pz = p.z;
    w.self = i;
    w.cnt = 1;
    w.maxnbr = sc.maxnbr;
    w.out = nbr + ell_index(r, 0, ell_stride);
    w.overflow = false;
    const float d2max = sc.d2max;
    FaceGaps fg;
    if (CULL) fg.init(p, c, g, sc.cell);
    for (int t = 0; t < 27; ++t) {
        int3 cc = c;
        int3 o = nbr_offset(t);
        cc.x += o.x; cc.y += o.y; cc.z += o.z;
        if (!cell_available(cc, g)) continue;
        if (CULL && !fg.reachable(o, d2max)) continue;
        uint32_t k = g.key_base + cell_key(cc, g);
        uint32_t f0 = __ldg(fstart + k), f1 = __ldg(fstart + k + 1);
        uint32_t b0 = __ldg(bstart + k), b1 = __ldg(bstart + k + 1);
        // The capacity check is needed only when the cell's candidates could
        // overflow the list.
        if (w.cnt + (f1 - f0) + (b1 - b0) <= w.maxnbr) w.visit_cell<MODE, true>(f0, f1, b0, b1, pos, orig, d2max);
        else w.visit_cell<MODE, false>(f0, f1, b0, b1, pos, orig, d2max);
    }
    ncnt[r] = w.cnt;
    if (w.overflow) {
        atomicAdd(overflow_count, 1u);
        atomicOr(status, ST_BOUNDS);
    }
}

// Lane-split walk for small row counts, where one thread per row leaves most
// of the GPU idle and the kernel time is one thread's serial walk: L lanes per
// row, lane l walking the contiguous group [27 l / L, 27 (l+1) / L) of the 27
// offsets.  Pass 1 counts the lane's accepted candidates, a shuffle scan over
// the row's lanes gives each lane its first slot, pass 2 walks again and
// writes.  The concatenation is the one-thread walk's list, truncation at
// maxNbr included, so both builders write identical lists.
// Passes of the lane-split walk: kCount tests every candidate, counts the
// accepted ones and keeps the first kSplitKeep of them in the block's shared
// buffer; kWrite tests again and writes every accepted candidate into its
// slot (only for a lane that accepted more than kSplitKeep).
enum SplitPass { kCount = 0, kWrite = 1 };
constexpr int kSplitBlock = 256;   // threads per block of the lane-split builder
constexpr uint32_t kSplitKeep = 16; // accepted candidates a lane keeps for the copy-out

template <int PASS>
struct SplitSink {
    float px, py, pz;
    uint32_t n;       // candidates accepted by this lane so far
    uint32_t base;    // kWrite: this lane's first slot
    uint32_t cap;     // list slots per row (maxNbr - 1)
    uint32_t *out;    // kCount: this thread's column of the shared buffer (stride kSplitBlock); kWrite: ELL row

    __device__ __forceinline__ void take(uint32_t j, const float4 &q, float d2max) {
        const float d2 = dist2(px - q.x, py - q.y, pz - q.z);
        if (d2 > 0.f && d2 <= d2max) {
            if (PASS == kCount) {
                if (n < kSplitKeep) out[n * kSplitBlock] = j;
            } else {
                const uint32_t slot = base + n;
                if (slot < cap) out[(size_t)slot * 32u] = j;
            }
            ++n;
        }
    }

    __device__ __forceinline__ void visit(uint32_t j, const float4 *__restrict__ pos, float d2max) {
        take(j, __ldg(pos + j), d2max);
    }

    __device__ __forceinline__ void run(uint32_t j0, uint32_t j1, const float4 *__restrict__ pos, float d2max) {
        uint32_t j = j0;
        for (; j + 4 <= j1; j += 4) {
            const float4 q0 = __ldg(pos + j), q1 = __ldg(pos + j + 1), q2 = __ldg(pos + j + 2),
                         q3 = __ldg(pos + j + 3);
            take(j, q0, d2max);
            take(j + 1, q1, d2max);
            take(j + 2, q2, d2max);
            take(j + 3, q3, d2max);
        }
        for (; j < j1; ++j) take(j, __ldg(pos + j), d2max);
    }
};

template <int MODE, bool CULL, int PASS>
__device__ __forceinline__ void split_walk(SplitSink<PASS> &k, int3 c, const SceneGrid &g, int t0, int t1,
                                           const float4 *__restrict__ pos, const uint32_t *__restrict__ orig,
                                           const uint32_t *__restrict__ fstart, const uint32_t *__restrict__ bstart,
                                           float d2max, const FaceGaps &fg) {
    for (int t = t0; t < t1; ++t) {
        int3 cc = c;
        const int3 o = nbr_offset(t);
        cc.x += o.x; cc.y += o.y; cc.z += o.z;
        if (!cell_available(cc, g)) continue;
        if (CULL && !fg.reachable(o, d2max)) continue;
        const uint32_t key = g.key_base + cell_key(cc, g);
        uint32_t f0 = __ldg(fstart + key), f1 = __ldg(fstart + key + 1);
        uint32_t b0 = __ldg(bstart + key), b1 = __ldg(bstart + key + 1);
        if (MODE == 0) {
            k.run(f0, f1, pos, d2max);
            k.run(b0, b1, pos, d2max);
        } else if (MODE == 1) {
            k.run(b0, b1, pos, d2max);
            k.run(f0, f1, pos, d2max);
        } else {
            while (f0 < f1 || b0 < b1) {
                uint32_t j;
                if (b0 >= b1) j = f0++;
                else if (f0 >= f1) j = b0++;
                else j = (__ldg(orig + f0) < __ldg(orig + b0)) ? f0++ : b0++;
                k.visit(j, pos, d2max);
            }
        }
    }
}

template <int MODE, bool CULL, int L>
__global__ void __launch_bounds__(kSplitBlock) k_build_lists_split(
    Scenes sc, uint32_t row0, uint32_t cnt, uint32_t ell_stride, const float4 *__restrict__ pos,
    const uint32_t *__restrict__ orig, const uint32_t *__restrict__ fstart, const uint32_t *__restrict__ bstart,
    uint32_t *__restrict__ nbr, uint32_t *__restrict__ ncnt, uint32_t *__restrict__ status,
    uint32_t *__restrict__ overflow_count) {
    pdl_enter();
    static_assert(L >= 2 && L <= 16 && (L & (L - 1)) == 0, "L divides the warp");
    // Accepted candidates of each thread, [kSplitKeep][kSplitBlock] (a thread's column is strided, so
    // a warp's stores and loads of entry k fall in 32 consecutive words).
    __shared__ uint32_t keep[kSplitKeep * kSplitBlock];
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t r = gt / L;
    const int lane = (int)(gt % L);
    // The L lanes of a row are one aligned group of a warp and leave together.
    if (r >= cnt) return;
    const unsigned gmask = ((1u << L) - 1u) << ((threadIdx.x & 31u) & ~(unsigned)(L - 1));
    const uint32_t i = row0 + r;
    const SceneGrid g = load_scene(sc, i);
    const float4 p = pos[i];
    const int3 c = cell_of(p.x, p.y, p.z, g, sc.cell);
    if (!cell_available(c, g)) {  // outside the grid: no neighbours, not even self
        if (lane == 0) ncnt[r] = 0;
        return;
    }
    const int t0 = 27 * lane / L, t1 = 27 * (lane + 1) / L;
    const float d2max = sc.d2max;
    FaceGaps fg;
    if (CULL) fg.init(p, c, g, sc.cell);
    SplitSink<kCount> cnt1{p.x, p.y, p.z, 0u, 0u, 0u, keep + threadIdx.x};
    split_walk<MODE, CULL>(cnt1, c, g, t0, t1, pos, orig, fstart, bstart, d2max, fg);
    uint32_t x = cnt1.n;
#pragma unroll
    for (int o = 1; o < L; o <<= 1) {
        const uint32_t y = __shfl_up_sync(gmask, x, o, L);
        if (lane >= o) x += y;
    }
    const uint32_t total = __shfl_sync(gmask, x, L - 1, L);
    const uint32_t cap = sc.maxnbr - 1u;
    uint32_t *const out = nbr + ell_index(r, 0, ell_stride);
    const uint32_t base = x - cnt1.n;
    if (base < cap && cnt1.n > 0) {
        if (cnt1.n <= kSplitKeep) {   // the lane's accepted candidates are in shared memory
            const uint32_t m = min(cnt1.n, cap - base);
            for (uint32_t k = 0; k < m; ++k) out[(size_t)(base + k) * 32u] = keep[k * kSplitBlock + threadIdx.x];
        } else {
            SplitSink<kWrite> wr{p.x, p.y, p.z, 0u, base, cap, out};
            split_walk<MODE, CULL>(wr, c, g, t0, t1, pos, orig, fstart, bstart, d2max, fg);
        }
    }
    if (lane == 0) {
        ncnt[r] = total < cap ? total + 1u : sc.maxnbr;
        if (total > cap) {
            atomicAdd(overflow_count, 1u);
            atomicOr(status, ST_BOUNDS);
        }
    }
}

#ifdef VTP_CHECKED
// Checked build (-DVTP_CHECKED): every list entry of rows [row0, row0 + cnt)
// after each build - count <= maxNbr, entries inside the solver's rows, no
// row listed as its own neighbour - with the first offence recorded in
// `status` (ST_BOUNDS); the passes consume only validated lists.
__global__ void k_check_lists(uint32_t row0, uint32_t cnt, uint32_t nrows, uint32_t ell_stride, uint32_t maxnbr,
                              const uint32_t *__restrict__ nbr, const uint32_t *__restrict__ ncnt,
                              uint32_t *__restrict__ status) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cnt) return;
    const uint32_t n = ncnt[r];
    bool bad = n > maxnbr;
    for (uint32_t t = 0; !bad && t + 1 < n; ++t) {
        const uint32_t j = nbr[ell_index(r, t, ell_stride)];
        bad = j >= nrows || j == row0 + r;
    }
    if (bad) atomicOr(status, ST_BOUNDS);
}
#endif

// Staged list builder: one block per brick (staged.h).  The block stages
// the brick's 6 x 6 x 6-cell neighbourhood - positions, with each row's index
// in w - in shared memory once, and every row of the group walks its 27 cells
// (the reference's offset order, a cell's runs in list order, cells beyond h
// culled) over the staged copy, writing the global list entry and the slot
// list entry of each accepted candidate.  A group whose neighbourhood exceeds
// the staging capacity walks global memory with the one-thread walker and
// writes no slot list (the solve passes then gather it from global memory);
// block `ngroups` gives the rows outside the grid empty lists.
template <int MODE, bool CULL>
__global__ void __launch_bounds__(kStageBlock) k_build_lists_staged(
    Scenes sc, Staging stg, uint32_t ell_stride, const float4 *__restrict__ pos, uint32_t *__restrict__ nbr,
    uint32_t *__restrict__ ncnt, uint32_t *__restrict__ status, uint32_t *__restrict__ overflow_count) {
    pdl_enter();
    extern __shared__ float4 stage[];
    __shared__ GroupPlan P;
    const uint32_t grp = blockIdx.x;
    const SceneGrid g = sc.sg[0];
    if (grp == stg.ngroups) {   // rows outside the grid: no neighbours, not even self
        const uint32_t k = g.key_base + g.nkey;
        const uint32_t r1 = __ldg(stg.fstart + k + 1);
        for (uint32_t r = __ldg(stg.fstart + k) + threadIdx.x; r < r1; r += blockDim.x) ncnt[r] = 0;
        return;
    }
    const uint2 rows = group_rows(grp, g, stg);
    if (rows.x == rows.y) return;
    plan_group(P, grp, g, stg);
    const bool staged = P.total <= stg.scap;
    if (staged) {
        for (uint32_t s = threadIdx.x; s < P.total; s += blockDim.x) {
            bool b;
            const uint32_t j = slot_row<MODE>(P, slot_cell(P, s), s, b);
            float4 q = __ldg(pos + j);
            q.w = __uint_as_float(j);
            stage[s] = q;
        }
    }
    __syncthreads();
    const float d2max = sc.d2max;
    const uint32_t maxnbr = sc.maxnbr;
    for (uint32_t r = P.r0 + threadIdx.x; r < P.r1; r += blockDim.x) {
        const float4 p = pos[r];
        const int3 c = cell_of(p.x, p.y, p.z, g, sc.cell);
        FaceGaps fg;
        if (CULL) fg.init(p, c, g, sc.cell);
        if (!staged) {
            Walker w;
            w.px = p.x; w.py = p.y; w.pz = p.z;
            w.self = r;
            w.cnt = 1;
            w.maxnbr = maxnbr;
            w.out = nbr + ell_index(r, 0, ell_stride);
            w.overflow = false;
            for (int t = 0; t < 27; ++t) {
                const int3 o = nbr_offset(t);
                const int3 cc = make_int3(c.x + o.x, c.y + o.y, c.z + o.z);
                if (!cell_available(cc, g)) continue;
                if (CULL && !fg.reachable(o, d2max)) continue;
                const uint32_t k = g.key_base + cell_key(cc, g);
                const uint32_t f0 = __ldg(stg.fstart + k), f1 = __ldg(stg.fstart + k + 1);
                const uint32_t b0 = __ldg(stg.bstart + k), b1 = __ldg(stg.bstart + k + 1);
                if (w.cnt + (f1 - f0) + (b1 - b0) <= w.maxnbr)
                    w.visit_cell<MODE, true>(f0, f1, b0, b1, pos, nullptr, d2max);
                else
                    w.visit_cell<MODE, false>(f0, f1, b0, b1, pos, nullptr, d2max);
            }
            ncnt[r] = w.cnt;
            if (w.overflow) {
                atomicAdd(overflow_count, 1u);
                atomicOr(status, ST_BOUNDS);
            }
            continue;
        }
        uint32_t *const out = nbr + ell_index(r, 0, ell_stride);
        uint16_t *const sout = stg.snbr + ell_index(r, 0, ell_stride);
        uint32_t cnt = 1;
        bool over = false;
        for (int t = 0; t < 27; ++t) {
            const int3 o = nbr_offset(t);
            const int3 cc = make_int3(c.x + o.x, c.y + o.y, c.z + o.z);
            if (!cell_available(cc, g)) continue;
            if (CULL && !fg.reachable(o, d2max)) continue;
            const int lx = cc.x - P.ox, ly = cc.y - P.oy, lz = cc.z - P.oz;
            if ((unsigned)lx >= (unsigned)kStageUx || (unsigned)ly >= (unsigned)kStageUy ||
                (unsigned)lz >= (unsigned)kStageUz) {   // a row outside its group's block: never expected
                atomicOr(status, ST_BOUNDS);
                continue;
            }
            const int u = (lz * kStageUy + ly) * kStageUx + lx;
            const uint32_t s0 = P.off[u], s1 = P.off[u + 1];
            // first boundary slot (mode 0) / first fluid slot (mode 1) of the cell
            const uint32_t sb = s0 + (MODE == 0 ? P.nfl[u] : P.nbl[u]);
            const bool room = cnt + (s1 - s0) <= maxnbr;
            for (uint32_t sl = s0; sl < s1; ++sl) {
                const float4 q = stage[sl];
                const float d2 = dist2(p.x - q.x, p.y - q.y, p.z - q.z);
                if (d2 > 0.f && d2 <= d2max) {
                    if (room || cnt < maxnbr) {
                        const bool bnd = MODE == 0 ? sl >= sb : sl < sb;
                        out[(size_t)(cnt - 1) * 32u] = __float_as_uint(q.w);
                        sout[(size_t)(cnt - 1) * 32u] = (uint16_t)(sl | (bnd ? kSlotBoundary : 0u));
                        ++cnt;
                    } else {
                        over = true;
                    }
                }
            }
        }
        ncnt[r] = cnt;
        if (over) {
            atomicAdd(overflow_count, 1u);
            atomicOr(status, ST_BOUNDS);
        }
    }
}

__global__ void k_scatter_f4(uint32_t n, const float4 *__restrict__ src, const uint32_t *__restrict__ orig,
                             float *__restrict__ dst3) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = src[i];
    size_t o = (size_t)orig[i] * 3;
    dst3[o] = v.x;
    dst3[o + 1] = v.y;
    dst3[o + 2] = v.z;
}

__global__ void k_scatter_f1(uint32_t n, const float *__restrict__ src, const uint32_t *__restrict__ orig,
                             float *__restrict__ dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[orig[i]] = src[i];
}

__global__ void k_gather_f4(uint32_t n, const float *__restrict__ src3, const uint32_t *__restrict__ orig,
                            float4 *__restrict__ dst, int keep_w) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    size_t o = (size_t)orig[i] * 3;
    float4 v = dst[i];
    v.x = src3[o];
    v.y = src3[o + 1];
    v.z = src3[o + 2];
    if (!keep_w) v.w = 0.f;
    dst[i] = v;
}

__global__ void k_gather_f1(uint32_t n, const float *__restrict__ src, const uint32_t *__restrict__ orig,
                            float *__restrict__ dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = src[orig[i]];
}

// Rows whose attach id lies in [first, first + count): scatter to / gather from a
// compact buffer indexed by id - first.
__global__ void k_scatter_f4_range(uint32_t n, const float4 *__restrict__ src, const uint32_t *__restrict__ orig,
                                   uint32_t first, uint32_t count, float *__restrict__ dst3) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = orig[i] - first;
    if (id >= count) return;
    const float4 v = src[i];
    dst3[3 * (size_t)id] = v.x;
    dst3[3 * (size_t)id + 1] = v.y;
    dst3[3 * (size_t)id + 2] = v.z;
}

__global__ void k_gather_f4_range(uint32_t n, const float *__restrict__ src3, const uint32_t *__restrict__ orig,
                                  uint32_t first, uint32_t count, float4 *__restrict__ dst,
                                  float4 *__restrict__ dst2) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = orig[i] - first;
    if (id >= count) return;
    float4 v = dst[i];
    v.x = src3[3 * (size_t)id];
    v.y = src3[3 * (size_t)id + 1];
    v.z = src3[3 * (size_t)id + 2];
    dst[i] = v;
    if (dst2) {
        float4 w = dst2[i];
        w.x = v.x; w.y = v.y; w.z = v.z;
        dst2[i] = w;
    }
}

// Positions and velocities of one attach-id range together (one pass each way).
__global__ void k_scatter_state_range(uint32_t n, const float4 *__restrict__ pos, const float4 *__restrict__ vel,
                                      const uint32_t *__restrict__ orig, uint32_t first, uint32_t count,
                                      float *__restrict__ p3, float *__restrict__ v3) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = orig[i] - first;
    if (id >= count) return;
    const float4 p = pos[i], v = vel[i];
    p3[3 * (size_t)id] = p.x;
    p3[3 * (size_t)id + 1] = p.y;
    p3[3 * (size_t)id + 2] = p.z;
    v3[3 * (size_t)id] = v.x;
    v3[3 * (size_t)id + 1] = v.y;
    v3[3 * (size_t)id + 2] = v.z;
}

__global__ void k_gather_state_range(uint32_t n, const float *__restrict__ p3, const float *__restrict__ v3,
                                     const uint32_t *__restrict__ orig, uint32_t first, uint32_t count,
                                     float4 *__restrict__ pos, float4 *__restrict__ vel, float4 *__restrict__ vadv) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = orig[i] - first;
    if (id >= count) return;
    float4 p = pos[i], v = vel[i];
    p.x = p3[3 * (size_t)id]; p.y = p3[3 * (size_t)id + 1]; p.z = p3[3 * (size_t)id + 2];
    v.x = v3[3 * (size_t)id]; v.y = v3[3 * (size_t)id + 1]; v.z = v3[3 * (size_t)id + 2];
    pos[i] = p;
    vel[i] = v;
    if (vadv) {
        float4 w = vadv[i];
        w.x = v.x; w.y = v.y; w.z = v.z;
        vadv[i] = w;
    }
}

// Slot of attach id `id` in buffers that hold several particle ranges back to back:
// tab[3k], tab[3k + 1], tab[3k + 2] = first, count, first slot of range k, the ranges
// ascending and disjoint; ~0u outside every range.
__device__ __forceinline__ uint32_t range_slot(uint32_t id, const uint32_t *__restrict__ tab, uint32_t nr) {
    uint32_t lo = 0, hi = nr;   // the first range that starts after id
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (tab[3 * mid] <= id) lo = mid + 1;
        else hi = mid;
    }
    if (lo == 0) return ~0u;
    const uint32_t k = lo - 1, d = id - tab[3 * k];
    return d < tab[3 * k + 1] ? tab[3 * k + 2] + d : ~0u;
}

__global__ void k_scatter_state_ranges(uint32_t n, const float4 *__restrict__ pos, const float4 *__restrict__ vel,
                                       const uint32_t *__restrict__ orig, const uint32_t *__restrict__ tab,
                                       uint32_t nr, float *__restrict__ p3, float *__restrict__ v3) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = range_slot(orig[i], tab, nr);
    if (id == ~0u) return;
    const float4 p = pos[i], v = vel[i];
    p3[3 * (size_t)id] = p.x;
    p3[3 * (size_t)id + 1] = p.y;
    p3[3 * (size_t)id + 2] = p.z;
    v3[3 * (size_t)id] = v.x;
    v3[3 * (size_t)id + 1] = v.y;
    v3[3 * (size_t)id + 2] = v.z;
}

__global__ void k_gather_state_ranges(uint32_t n, const float *__restrict__ p3, const float *__restrict__ v3,
                                      const uint32_t *__restrict__ orig, const uint32_t *__restrict__ tab,
                                      uint32_t nr, float4 *__restrict__ pos, float4 *__restrict__ vel,
                                      float4 *__restrict__ vadv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = range_slot(orig[i], tab, nr);
    if (id == ~0u) return;
    float4 p = pos[i], v = vel[i];
    p.x = p3[3 * (size_t)id]; p.y = p3[3 * (size_t)id + 1]; p.z = p3[3 * (size_t)id + 2];
    v.x = v3[3 * (size_t)id]; v.y = v3[3 * (size_t)id + 1]; v.z = v3[3 * (size_t)id + 2];
    pos[i] = p;
    vel[i] = v;
    if (vadv) {
        float4 w = vadv[i];
        w.x = v.x; w.y = v.y; w.z = v.z;
        vadv[i] = w;
    }
}

__global__ void k_iota(uint32_t n, uint32_t *dst, uint32_t base) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = base + i;
}

__global__ void k_export_neighbors(uint32_t row0, uint32_t cnt, uint32_t ell_stride,
                                   const uint32_t *__restrict__ nbr, const uint32_t *__restrict__ ncnt,
                                   const uint32_t *__restrict__ orig, uint32_t maxnbr,
                                   uint32_t *__restrict__ out_cnt, uint32_t *__restrict__ out_nbr) {
    uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= cnt) return;
    uint32_t i = row0 + r;
    uint32_t o = orig[i];
    uint32_t c = ncnt[r];
    out_cnt[o] = c;
    uint32_t *dst = out_nbr + (size_t)o * maxnbr;
    for (uint32_t t = 0; t < maxnbr; ++t) dst[t] = 0xffffffffu;
    if (c == 0) return;
    dst[0] = o;
    for (uint32_t t = 1; t < c; ++t) dst[t] = orig[nbr[ell_index(r, t - 1, ell_stride)]];
}

__global__ void k_export_sorted(Scenes sc, uint32_t n, const float4 *__restrict__ pos,
                                const uint32_t *__restrict__ orig, uint32_t *__restrict__ ids,
                                uint32_t *__restrict__ keys) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const SceneGrid g = load_scene(sc, i);
    float4 p = pos[i];
    int3 c = cell_of(p.x, p.y, p.z, g, sc.cell);
    ids[i] = orig[i];
    keys[i] = cell_available(c, g) ? ref_cell_key(c, g) : 0xffffffffu;
}

inline unsigned nblk(uint32_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

__global__ void k_cubic_sigma(float h, float *out) {
    const float PI = 3.14159265f;
    if (threadIdx.x == 0) out[0] = 8.f / PI / powf(h, 3.f);
}

// cube_rn against powf(t, 3.f) for every t = k * 2^-24, k in [0, 2^23]:
// number of differing inputs and the largest distance in ulps (both are
// positive floats, so the distance is the difference of the bit patterns).
__global__ void k_selftest_cube(uint32_t *mismatches, uint32_t *max_ulp) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > (1u << 23)) return;
    const float t = (float)k * 0x1p-24f;
    const int a = (int)__float_as_uint(cube_rn(t)), b = (int)__float_as_uint(powf(t, 3.f));
    if (a != b) {
        atomicAdd(mismatches, 1u);
        atomicMax(max_ulp, (uint32_t)(a > b ? a - b : b - a));
    }
}

int selftest_cube(cudaStream_t st, uint32_t *mismatches, uint32_t *max_ulp) {
    uint32_t *d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(uint32_t)) != cudaSuccess) return 1;
    uint32_t out[2] = {0u, 0u};
    cudaError_t e = cudaMemsetAsync(d, 0, 2 * sizeof(uint32_t), st);
    if (e == cudaSuccess) {
        k_selftest_cube<<<nblk((1u << 23) + 1u, 256), 256, 0, st>>>(d, d + 1);
        e = cudaMemcpyAsync(out, d, sizeof(out), cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    *mismatches = out[0];
    *max_ulp = out[1];
    return e == cudaSuccess ? 0 : 1;
}

int cubic_sigma_device(cudaStream_t st, float h, float *out_host) {
    float *d = nullptr;
    if (cudaMalloc(&d, sizeof(float)) != cudaSuccess) return 1;
    k_cubic_sigma<<<1, 32, 0, st>>>(h, d);
    cudaError_t e = cudaMemcpyAsync(out_host, d, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    return e == cudaSuccess ? 0 : 1;
}

static void scan_counts(cudaStream_t st, uint32_t *count, size_t n, uint32_t base_add, uint32_t *out,
                        UgnsBuffers &u) {
    size_t tiles = (n + kScanTile - 1) / kScanTile;
    launch(k_scan_tile_sums, (unsigned)tiles, kScanThreads, 0, st, count, n, u.scan_sums);
    launch(k_scan_sums, 1, 1024, 0, st, u.scan_sums, tiles);
    launch(k_scan_tiles, (unsigned)tiles, kScanThreads, 0, st, count, n, u.scan_sums, base_add, out);
}

void ugns_sort(cudaStream_t st, const Scenes &sc, uint32_t nbuckets, uint32_t row0, uint32_t cnt,
               const float4 *pos_in, float4 *pos_out, const float4 *vel_in, float4 *vel_out,
               const uint32_t *orig_in, uint32_t *orig_out, const Carry &carry, float force_dt, UgnsBuffers &u,
               uint32_t *start, Profiler *prof) {
    const size_t nb = nbuckets;  // buckets incl. every scene's outside bucket
    auto B = [&] { if (prof) prof->begin(); };
    auto E = [&](const char *nm) { if (prof) prof->end_(nm); };
    B();
    // u.count is all zero here: zeroed once at allocation and by every scan after reading it.
    if (cnt > 0) {
        launch(k_hash, nblk(cnt, 256), 256, 0, st, sc, row0, cnt, pos_in, vel_in, force_dt, u.key, u.rank, u.count);
    }
    E("ugns_clear_hash");
    B();
    scan_counts(st, u.count, nb, row0, start, u);
    E("ugns_cell_scan");
    if (cnt == 0) return;
    B();
    launch(k_scatter, nblk(cnt, 256), 256, 0, st, row0, cnt, u.key, u.rank, start, orig_in, u.tmp_src, u.tmp_orig,
           u.tmp_key, u.status);
    E("ugns_scatter");
    B();
    launch(k_rank_reorder, nblk(cnt, 256), 256, 0, st, sc, row0, cnt, start, u.tmp_src, u.tmp_orig, u.tmp_key, pos_in,
                                                   pos_out, vel_in, vel_out, orig_out, carry, force_dt);
    E("ugns_rank_reorder");
}

template <int MODE, bool CULL>
static void build_lists_as(cudaStream_t st, bool split, const Scenes &sc, const Layout &L, uint32_t row0,
                           uint32_t cnt, const float4 *pos, const uint32_t *orig, const UgnsBuffers &u, uint32_t *nbr,
                           uint32_t *ncnt, uint32_t *status, uint32_t *overflow, int block) {
    if (split) {
        constexpr int S = 8;
        launch(k_build_lists_split<MODE, CULL, S>, nblk(cnt * S, kSplitBlock), kSplitBlock, 0, st, sc, row0, cnt,
               L.ell_stride, pos, orig, u.fstart, u.bstart, nbr, ncnt, status, overflow);
    } else {
        launch(k_build_lists<MODE, CULL>, nblk(cnt, block), block, 0, st, sc, row0, cnt, L.ell_stride, pos, orig,
               u.fstart, u.bstart, nbr, ncnt, status, overflow);
    }
}

void ugns_build_lists(cudaStream_t st, const Scenes &sc, const Layout &L, uint32_t row0, uint32_t cnt,
                      const float4 *pos, const uint32_t *orig, const UgnsBuffers &u, uint32_t *nbr, uint32_t *ncnt,
                      uint32_t *status, uint32_t *overflow, int block) {
    if (cnt == 0) return;
    // Few rows: eight lanes per row (same lists, a quarter to an eighth of the
    // serial walk per thread).
    const bool split = L.list_lanes == 8 || (L.list_lanes == 0 && cnt <= kSplitRows);
    auto go = [&](auto mode, auto cull) {
        build_lists_as<decltype(mode)::value, decltype(cull)::value>(st, split, sc, L, row0, cnt, pos, orig, u, nbr,
                                                                     ncnt, status, overflow, block);
    };
    using T = std::true_type;
    using F = std::false_type;
    using M0 = std::integral_constant<int, 0>;
    using M1 = std::integral_constant<int, 1>;
    using M2 = std::integral_constant<int, 2>;
    switch (L.merge_mode) {
        case 0: L.cell_cull ? go(M0{}, T{}) : go(M0{}, F{}); break;
        case 1: L.cell_cull ? go(M1{}, T{}) : go(M1{}, F{}); break;
        default: L.cell_cull ? go(M2{}, T{}) : go(M2{}, F{}); break;
    }
#ifdef VTP_CHECKED
    k_check_lists<<<nblk(cnt, 256), 256, 0, st>>>(row0, cnt, L.n, L.ell_stride, sc.maxnbr, nbr, ncnt, status);
#endif
}

void ugns_build_lists_staged(cudaStream_t st, const Scenes &sc, const Layout &L, const Staging &stg,
                             const float4 *pos, uint32_t *nbr, uint32_t *ncnt, uint32_t *status,
                             uint32_t *overflow) {
    const size_t smem = (size_t)stg.scap * sizeof(float4);
    const unsigned grid = stg.ngroups + 1;
    // the staged rows may exceed the 48 KB of dynamic shared memory a kernel gets by default
    auto room = [&](auto kern) { cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); };
    if (stg.mode == 0 && L.cell_cull) {
        room(k_build_lists_staged<0, true>);
        launch(k_build_lists_staged<0, true>, grid, kStageBlock, smem, st, sc, stg, L.ell_stride, pos, nbr, ncnt,
               status, overflow);
    } else if (stg.mode == 0) {
        room(k_build_lists_staged<0, false>);
        launch(k_build_lists_staged<0, false>, grid, kStageBlock, smem, st, sc, stg, L.ell_stride, pos, nbr, ncnt,
               status, overflow);
    } else if (L.cell_cull) {
        room(k_build_lists_staged<1, true>);
        launch(k_build_lists_staged<1, true>, grid, kStageBlock, smem, st, sc, stg, L.ell_stride, pos, nbr, ncnt,
               status, overflow);
    } else {
        room(k_build_lists_staged<1, false>);
        launch(k_build_lists_staged<1, false>, grid, kStageBlock, smem, st, sc, stg, L.ell_stride, pos, nbr, ncnt,
               status, overflow);
    }
#ifdef VTP_CHECKED
    k_check_lists<<<nblk(L.nf, 256), 256, 0, st>>>(0, L.nf, L.n, L.ell_stride, sc.maxnbr, nbr, ncnt, status);
#endif
}

void scatter_f4_to_orig(cudaStream_t st, uint32_t n, const float4 *src, const uint32_t *orig, float *dst3) {
    if (n) k_scatter_f4<<<nblk(n, 256), 256, 0, st>>>(n, src, orig, dst3);
}
void scatter_f1_to_orig(cudaStream_t st, uint32_t n, const float *src, const uint32_t *orig, float *dst) {
    if (n) k_scatter_f1<<<nblk(n, 256), 256, 0, st>>>(n, src, orig, dst);
}
void gather_orig_to_f4(cudaStream_t st, uint32_t n, const float *src3, const uint32_t *orig, float4 *dst,
                       int keep_w) {
    if (n) k_gather_f4<<<nblk(n, 256), 256, 0, st>>>(n, src3, orig, dst, keep_w);
}
void gather_orig_to_f1(cudaStream_t st, uint32_t n, const float *src, const uint32_t *orig, float *dst) {
    if (n) k_gather_f1<<<nblk(n, 256), 256, 0, st>>>(n, src, orig, dst);
}
void scatter_f4_range(cudaStream_t st, uint32_t n, const float4 *src, const uint32_t *orig, uint32_t first,
                      uint32_t count, float *dst3) {
    if (n) k_scatter_f4_range<<<nblk(n, 256), 256, 0, st>>>(n, src, orig, first, count, dst3);
}
void gather_f4_range(cudaStream_t st, uint32_t n, const float *src3, const uint32_t *orig, uint32_t first,
                     uint32_t count, float4 *dst, float4 *dst2) {
    if (n) k_gather_f4_range<<<nblk(n, 256), 256, 0, st>>>(n, src3, orig, first, count, dst, dst2);
}
void scatter_state_range(cudaStream_t st, uint32_t n, const float4 *pos, const float4 *vel, const uint32_t *orig,
                         uint32_t first, uint32_t count, float *p3, float *v3) {
    if (n) k_scatter_state_range<<<nblk(n, 256), 256, 0, st>>>(n, pos, vel, orig, first, count, p3, v3);
}
void gather_state_range(cudaStream_t st, uint32_t n, const float *p3, const float *v3, const uint32_t *orig,
                        uint32_t first, uint32_t count, float4 *pos, float4 *vel, float4 *vadv) {
    if (n) k_gather_state_range<<<nblk(n, 256), 256, 0, st>>>(n, p3, v3, orig, first, count, pos, vel, vadv);
}
void scatter_state_ranges(cudaStream_t st, uint32_t n, const float4 *pos, const float4 *vel, const uint32_t *orig,
                          const uint32_t *tab, uint32_t nr, float *p3, float *v3) {
    if (n) k_scatter_state_ranges<<<nblk(n, 256), 256, 0, st>>>(n, pos, vel, orig, tab, nr, p3, v3);
}
void gather_state_ranges(cudaStream_t st, uint32_t n, const float *p3, const float *v3, const uint32_t *orig,
                         const uint32_t *tab, uint32_t nr, float4 *pos, float4 *vel, float4 *vadv) {
    if (n) k_gather_state_ranges<<<nblk(n, 256), 256, 0, st>>>(n, p3, v3, orig, tab, nr, pos, vel, vadv);
}
void fill_iota(cudaStream_t st, uint32_t n, uint32_t *dst, uint32_t base) {
    if (n) k_iota<<<nblk(n, 256), 256, 0, st>>>(n, dst, base);
}
void export_neighbors(cudaStream_t st, const Layout &L, uint32_t row0, uint32_t cnt, const uint32_t *nbr,
                      const uint32_t *ncnt, const uint32_t *orig, uint32_t maxnbr, uint32_t *out_cnt,
                      uint32_t *out_nbr) {
    if (cnt)
        k_export_neighbors<<<nblk(cnt, 256), 256, 0, st>>>(row0, cnt, L.ell_stride, nbr, ncnt, orig, maxnbr, out_cnt,
                                                           out_nbr);
}
void export_sorted(cudaStream_t st, const Scenes &sc, uint32_t n, const float4 *pos, const uint32_t *orig,
                   uint32_t *out_ids, uint32_t *out_keys) {
    if (n) k_export_sorted<<<nblk(n, 256), 256, 0, st>>>(sc, n, pos, orig, out_ids, out_keys);
}

}  // namespace vtp
