// Internal host-side interfaces between the solver driver (capi.cu) and the
// kernel translation units (ugns.cu, pbf.cu, dfsph.cu, immct.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

#include <nvtx3/nvToolsExt.h>

namespace vtp {

// NVTX range over a host scope (solver stages: initialize, tick, the substep's
// enqueue stages, differentiation, export).  NVTX is header-only and does
// nothing unless a profiler is attached.  With graphs the enqueue stages are
// recorded once, at capture; every tick shows as one range around its graph
// launches.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

constexpr int kConsPhases = 8;   // phases the conservation sums report (vtp_conservation.phase_mass)

// Particles are kept sorted: fluid rows [0, nf) re-sorted by (cell, attach id)
// every substep, boundary rows [nf, n) sorted once at initialize.
struct Layout {
    uint32_t n = 0, nf = 0, nb = 0;
    uint32_t ell_stride = 0;   // slots per row in the ELL neighbour list (maxnbr - 1 others)
    int merge_mode = 0;        // 0: fluid ids < boundary ids, 1: boundary ids < fluid ids, 2: general
    int list_lanes = 0;        // list builder lanes per row: 0 = by row count, 1 or 8 = forced
    bool cell_cull = false;    // list builder skips neighbour cells beyond h of the row (same lists)
};

// Neighbour-search working set (one per solver).
struct UgnsBuffers {
    uint32_t *key = nullptr;       // [nf] cell key per old slot
    uint32_t *rank = nullptr;      // [nf] arrival rank within the cell (atomic)
    uint32_t *count = nullptr;     // [nbuckets] (all scenes' buckets incl. their outside buckets)
    uint32_t *fstart = nullptr;    // [nbuckets + 1] fluid cell starts (absolute rows)
    uint32_t *bstart = nullptr;    // [nbuckets + 1] boundary cell starts (absolute rows)
    uint32_t *tmp_src = nullptr;   // [max(nf, nb)] scattered: old slot
    uint32_t *tmp_orig = nullptr;  // [max(nf, nb)] scattered: attach id
    uint32_t *tmp_key = nullptr;   // [max(nf, nb)] scattered: key
    uint32_t *scan_sums = nullptr; // [tiles]
    uint32_t *nbr = nullptr;       // ELL list for fluid rows
    uint32_t *ncnt = nullptr;      // [nf] neighbour count incl. self (0 = outside the grid)
    uint32_t *bnbr = nullptr;      // ELL list for boundary rows (init / diagnostics)
    uint32_t *bncnt = nullptr;     // [nb]
    uint32_t *status = nullptr;    // the solver's device status word (checked-build guards report here)
    size_t scan_tiles = 0;
};

// Fields a reorder carries from old slot to new slot (float4 / float / uint).
struct Carry {
    static constexpr int kMaxF4 = 8, kMaxF1 = 16;
    int nf4 = 0, nf1 = 0;
    const float4 *src4[kMaxF4];
    float4 *dst4[kMaxF4];
    const float *src1[kMaxF1];
    float *dst1[kMaxF1];
};

// Optional per-kernel timing: CUDA events recorded around each launch.
struct Profiler {
    static constexpr int kMax = 4096;
    cudaStream_t st = nullptr;
    int n = 0;
    const char *names[kMax];
    cudaEvent_t beg[kMax], end[kMax];
    bool ready = false;
    void begin() {
        if (!ready || n >= kMax) return;
        cudaEventRecord(beg[n], st);
    }
    void end_(const char *name) {
        if (!ready || n >= kMax) return;
        cudaEventRecord(end[n], st);
        names[n++] = name;
    }
};

// --- ugns.cu ---
// Sort rows [row0, row0 + cnt) by (scene, cell, attach id) into the output
// arrays; `start` receives the cell-start table (absolute rows) over all
// `nbuckets` buckets.  With `force_dt` > 0 the rows' positions get
// v += g dt; x += v dt applied first with their scene's gravity (PBF external
// force fused into the sort).
void ugns_sort(cudaStream_t st, const Scenes &sc, uint32_t nbuckets, uint32_t row0, uint32_t cnt,
               const float4 *pos_in, float4 *pos_out, const float4 *vel_in, float4 *vel_out,
               const uint32_t *orig_in, uint32_t *orig_out, const Carry &carry,
               float force_dt, UgnsBuffers &u, uint32_t *start, Profiler *prof = nullptr);

// Build the neighbour lists of rows [row0, row0 + cnt) (reference order:
// 27 offsets, then ascending attach id inside a cell).
void ugns_build_lists(cudaStream_t st, const Scenes &sc, const Layout &L, uint32_t row0, uint32_t cnt,
                      const float4 *pos, const uint32_t *orig, const UgnsBuffers &u,
                      uint32_t *nbr, uint32_t *ncnt, uint32_t *status, uint32_t *overflow, int block);

// sigma of the cubic spline computed on the device (0 on success).
int cubic_sigma_device(cudaStream_t st, float h, float *out_host);
// cube_rn(t) vs powf(t, 3.f) over the outer-branch domain of cubic_w (0 on success).
int selftest_cube(cudaStream_t st, uint32_t *mismatches, uint32_t *max_ulp);

// Gather/scatter between attach order and sorted rows.
void scatter_f4_to_orig(cudaStream_t st, uint32_t n, const float4 *src, const uint32_t *orig, float *dst3);
void scatter_f1_to_orig(cudaStream_t st, uint32_t n, const float *src, const uint32_t *orig, float *dst);
void gather_orig_to_f4(cudaStream_t st, uint32_t n, const float *src3, const uint32_t *orig, float4 *dst,
                       int keep_w);
void gather_orig_to_f1(cudaStream_t st, uint32_t n, const float *src, const uint32_t *orig, float *dst);
void fill_iota(cudaStream_t st, uint32_t n, uint32_t *dst, uint32_t base);
// Attach-id range [first, first + count) <-> sorted rows [0, n) (float3 compact buffer).
void scatter_f4_range(cudaStream_t st, uint32_t n, const float4 *src, const uint32_t *orig, uint32_t first,
                      uint32_t count, float *dst3);
void gather_f4_range(cudaStream_t st, uint32_t n, const float *src3, const uint32_t *orig, uint32_t first,
                     uint32_t count, float4 *dst, float4 *dst2);
void scatter_state_range(cudaStream_t st, uint32_t n, const float4 *pos, const float4 *vel, const uint32_t *orig,
                         uint32_t first, uint32_t count, float *p3, float *v3);
void gather_state_range(cudaStream_t st, uint32_t n, const float *p3, const float *v3, const uint32_t *orig,
                        uint32_t first, uint32_t count, float4 *pos, float4 *vel, float4 *vadv);
// The same for several attach-id ranges held back to back in p3 / v3: tab (device) holds
// {first, count, first slot} per range, ascending and disjoint.
void scatter_state_ranges(cudaStream_t st, uint32_t n, const float4 *pos, const float4 *vel, const uint32_t *orig,
                          const uint32_t *tab, uint32_t nr, float *p3, float *v3);
void gather_state_ranges(cudaStream_t st, uint32_t n, const float *p3, const float *v3, const uint32_t *orig,
                         const uint32_t *tab, uint32_t nr, float4 *pos, float4 *vel, float4 *vadv);
void export_neighbors(cudaStream_t st, const Layout &L, uint32_t row0, uint32_t cnt, const uint32_t *nbr,
                      const uint32_t *ncnt, const uint32_t *orig, uint32_t maxnbr, uint32_t *out_cnt,
                      uint32_t *out_nbr);
void export_sorted(cudaStream_t st, const Scenes &sc, uint32_t n, const float4 *pos, const uint32_t *orig,
                   uint32_t *out_ids, uint32_t *out_keys);

}  // namespace vtp
