// Cell-group staging of neighbour data in shared memory (staged.cu).
//
// In the bricked bucket order a brick - 64 consecutive buckets - is a
// 4 x 4 x 4 block of cells, and its fluid rows are one contiguous range of
// the sorted order.  Every neighbour of those rows lies in the brick's
// 6 x 6 x 6-cell neighbourhood (the block grown by one cell on each side), so
// a block of threads working on one brick can copy the neighbourhood's rows
// into shared memory once - coalesced runs, one per cell, about 3.4 staged
// rows per row of the brick - and gather every neighbour from there.  The list builder writes, beside each global list, a
// slot list: entry t of a row is the neighbour's position in its group's
// staged copy (bit 15 set for a boundary row).  Both lists hold the same
// neighbours in the same order, so a pass gathering through either gets the
// same values and sums them in the same order.
#pragma once

#include "internal.h"

namespace vtp {

// The staged neighbourhood: 6 x 6 x 6 cells, x fastest.
constexpr int kStageUx = 6, kStageUy = 6, kStageUz = 6;
constexpr int kStageCells = kStageUx * kStageUy * kStageUz;   // 216
constexpr int kStageBlock = 512;                              // threads per brick block
constexpr uint32_t kStageBuckets = 64;                        // buckets of one brick
constexpr uint16_t kSlotBoundary = 0x8000u;                   // slot-list flag: the neighbour is a boundary row
constexpr uint32_t kStageMaxRows = 0x7fffu;                   // slots must fit in 15 bits

struct Staging {
    uint32_t ngroups = 0;           // bricks of the scene's grid (in-grid bucket count / 64)
    uint32_t scap = 0;              // staged rows per brick at most; a larger neighbourhood gathers from global memory
    int mode = 0;                   // 0: a cell's fluid run before its boundary run, 1: boundary first
    const uint32_t *fstart = nullptr, *bstart = nullptr;   // cell tables (absolute rows)
    uint16_t *snbr = nullptr;       // slot lists, ELL layout of the global lists, 2 B per entry
};

// Staging plan of one brick, in shared memory: the neighbourhood's cells
// (index u = (z * 6 + y) * 6 + x relative to the origin cell), each cell's
// fluid and boundary runs, and the offset of each cell's rows in the staged
// copy (a cell's runs are staged in the list order: fluid run first in mode
// 0, boundary run first in mode 1).
struct GroupPlan {
    uint32_t off[kStageCells + 1];
    uint32_t fs[kStageCells], nfl[kStageCells];   // fluid run: first row, length
    uint32_t bs[kStageCells], nbl[kStageCells];   // boundary run
    int ox, oy, oz;                               // origin cell of the neighbourhood
    uint32_t r0, r1;                              // the brick's fluid rows
    uint32_t total;                               // rows staged
};

// Fluid rows of brick `grp` (all threads get them; no synchronisation).
__device__ __forceinline__ uint2 group_rows(uint32_t grp, const SceneGrid &g, const Staging &s) {
    const uint32_t k0 = g.key_base + grp * kStageBuckets;
    return make_uint2(__ldg(s.fstart + k0), __ldg(s.fstart + k0 + kStageBuckets));
}

// Fills P for brick `grp`; every thread of the block calls it (it synchronises).
__device__ __forceinline__ void plan_group(GroupPlan &P, uint32_t grp, const SceneGrid &g, const Staging &s) {
    __shared__ uint32_t wsum[kStageBlock / 32];
    const int tid = (int)threadIdx.x;
    const int bx = (int)(grp % g.bx), byz = (int)(grp / g.bx);
    const int ox = 4 * bx - 1, oy = 4 * (byz % (int)g.by) - 1, oz = 4 * (byz / (int)g.by) - 1;
    uint32_t len = 0;
    if (tid < kStageCells) {
        const int3 c = make_int3(ox + tid % kStageUx, oy + (tid / kStageUx) % kStageUy, oz + tid / (kStageUx * kStageUy));
        uint32_t f0 = 0, f1 = 0, b0 = 0, b1 = 0;
        if (cell_available(c, g)) {
            const uint32_t k = g.key_base + cell_key(c, g);
            f0 = __ldg(s.fstart + k); f1 = __ldg(s.fstart + k + 1);
            b0 = __ldg(s.bstart + k); b1 = __ldg(s.bstart + k + 1);
        }
        P.fs[tid] = f0; P.nfl[tid] = f1 - f0;
        P.bs[tid] = b0; P.nbl[tid] = b1 - b0;
        len = (f1 - f0) + (b1 - b0);
    }
    const int lane = tid & 31, wid = tid >> 5;
    uint32_t x = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    uint32_t base = 0;
    for (int w = 0; w < wid; ++w) base += wsum[w];
    if (tid < kStageCells) P.off[tid] = base + x - len;
    if (tid == kStageCells - 1) {
        P.off[kStageCells] = base + x;
        P.total = base + x;
        P.ox = ox; P.oy = oy; P.oz = oz;
        const uint2 rr = group_rows(grp, g, s);
        P.r0 = rr.x; P.r1 = rr.y;
    }
    __syncthreads();
}

// Neighbourhood cell holding staged slot `s` (the last cell whose offset is <= s).
__device__ __forceinline__ int slot_cell(const GroupPlan &P, uint32_t s) {
    int lo = 0, hi = kStageCells;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (P.off[mid] <= s) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Global row staged at slot `s` of cell `u`, and whether it is a boundary row.
template <int MODE>
__device__ __forceinline__ uint32_t slot_row(const GroupPlan &P, int u, uint32_t s, bool &boundary) {
    const uint32_t l = s - P.off[u];
    if (MODE == 0) {
        boundary = l >= P.nfl[u];
        return boundary ? P.bs[u] + (l - P.nfl[u]) : P.fs[u] + l;
    }
    boundary = l < P.nbl[u];
    return boundary ? P.bs[u] + l : P.fs[u] + (l - P.nbl[u]);
}

// nbr_loop over a slot list (2-byte entries, ELL layout): U entries' loads in flight.
template <int U, class Load, class Use>
__device__ __forceinline__ void slot_loop(const uint16_t *__restrict__ lst, uint32_t cnt, Load load, Use use) {
    using T = decltype(load((uint16_t)0));
    uint32_t t = 0;
    for (; t + U <= cnt; t += U) {
        uint16_t j[U];
#pragma unroll
        for (int u = 0; u < U; ++u) j[u] = __ldcs(lst + (size_t)(t + u) * 32u);
        T d[U];
#pragma unroll
        for (int u = 0; u < U; ++u) d[u] = load(j[u]);
#pragma unroll
        for (int u = 0; u < U; ++u) use(j[u], d[u]);
    }
    for (; t < cnt; ++t) {
        const uint16_t j = __ldcs(lst + (size_t)t * 32u);
        use(j, load(j));
    }
}

// Lists of every fluid row: the global lists (nbr, ncnt) as ugns_build_lists
// writes them, plus the slot lists of stg.snbr, one block per group (and one
// for the rows outside the grid).  Single scene, bricked order, merge mode 0 / 1.
void ugns_build_lists_staged(cudaStream_t st, const Scenes &sc, const Layout &L, const Staging &stg,
                             const float4 *pos, uint32_t *nbr, uint32_t *ncnt, uint32_t *status,
                             uint32_t *overflow);

}  // namespace vtp
