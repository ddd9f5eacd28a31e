// Allocation-free neighbour search: the uniform-grid neighbour search of the
// library as one call that allocates nothing.
//
// Some callers cannot call cudaMalloc at the moment they need neighbour lists:
// hosts that hand the GPU to this library under a fixed memory budget with
// their own pool allocator, and real-time loops that forbid allocation after
// start-up (cudaMalloc may synchronise the device and can fail under
// fragmentation in the middle of a frame).  They pass device buffers for
// the input positions and the output lists; everything else the search needs
// lives in the fixed scratch arena below, which every GPU that loads this
// library holds until the process exits.
//
// The arena is shared by every call on a device: two calls whose work
// overlaps on the GPU (different streams, or different host threads without
// ordering) corrupt each other's scratch.  Calls are ordered on one stream.
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/vtp.h"
#include "common.cuh"

namespace vtp {
int fail(int code, const std::string &msg);
}

namespace {

constexpr uint32_t kMaxParticles = VTP_NOALLOC_MAX_PARTICLES;
constexpr uint32_t kMaxKeys = VTP_NOALLOC_MAX_CELLS;   // cell buckets incl. the outside bucket
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;
constexpr uint32_t kMaxTiles = (kMaxKeys + 1 + kScanTile - 1) / kScanTile;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Arena layout (byte offsets).
constexpr size_t kOffKey = 0;
constexpr size_t kOffRank = kOffKey + align256(4ull * kMaxParticles);
constexpr size_t kOffTmp = kOffRank + align256(4ull * kMaxParticles);
constexpr size_t kOffSorted = kOffTmp + align256(4ull * kMaxParticles);
constexpr size_t kOffPos = kOffSorted + align256(4ull * kMaxParticles);
constexpr size_t kOffCount = kOffPos + align256(16ull * kMaxParticles);
constexpr size_t kOffStart = kOffCount + align256(4ull * (kMaxKeys + 1));
constexpr size_t kOffTiles = kOffStart + align256(4ull * (kMaxKeys + 2));
constexpr size_t kArenaBytes = kOffTiles + align256(4ull * kMaxTiles);

static_assert(kArenaBytes == VTP_NOALLOC_SCRATCH_BYTES, "scratch size in vtp.h out of date");

__device__ __align__(256) unsigned char g_noalloc_scratch[kArenaBytes];

struct Arena {
    uint32_t *key, *rank, *tmp, *sorted, *count, *start, *tiles;
    float4 *pos;
};

Arena arena_at(unsigned char *base) {
    Arena a;
    a.key = (uint32_t *)(base + kOffKey);
    a.rank = (uint32_t *)(base + kOffRank);
    a.tmp = (uint32_t *)(base + kOffTmp);
    a.sorted = (uint32_t *)(base + kOffSorted);
    a.pos = (float4 *)(base + kOffPos);
    a.count = (uint32_t *)(base + kOffCount);
    a.start = (uint32_t *)(base + kOffStart);
    a.tiles = (uint32_t *)(base + kOffTiles);
    return a;
}

// Device address of the arena on the current device.  In host code the
// symbol is a host-side stand-in, not a device address, so the address comes
// from cudaGetSymbolAddress.  It is looked up on every call rather than
// cached: after cudaDeviceReset (or in a new context on the same device) the
// module is loaded again and the array can sit at another address, and a
// cached pointer would then send the kernels into freed memory.  The lookup
// allocates nothing; only the first one in a context loads the module.
int arena_base(unsigned char **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
        return vtp::fail(VTP_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    *out = (unsigned char *)p;
    return VTP_OK;
}

__global__ void k_na_hash(vtp::Grid g, uint32_t n, const float *__restrict__ pos, Arena a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = pos[3 * (size_t)i], y = pos[3 * (size_t)i + 1], z = pos[3 * (size_t)i + 2];
    const int3 c = vtp::cell_of(x, y, z, g);
    const uint32_t k = vtp::cell_available(c, g) ? vtp::cell_key(c, g) : g.nkey;
    a.key[i] = k;
    a.rank[i] = atomicAdd(&a.count[k], 1u);
}

__device__ __forceinline__ uint32_t na_block_scan(uint32_t v, uint32_t &total) {
    __shared__ uint32_t ws[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < nw ? ws[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) ws[lane] = s;
    }
    __syncthreads();
    const uint32_t off = wid > 0 ? ws[wid - 1] : 0u;
    total = ws[nw - 1];
    __syncthreads();
    return off + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_na_tile_sums(uint32_t nb, Arena a) {
    const size_t base = (size_t)blockIdx.x * kScanTile + threadIdx.x;
    uint32_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const size_t idx = base + (size_t)k * kScanThreads;
        if (idx < nb) s += a.count[idx];
    }
    uint32_t total;
    na_block_scan(s, total);
    if (threadIdx.x == 0) a.tiles[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_na_scan_tiles(uint32_t tiles, Arena a) {
    const uint32_t per = (tiles + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per;
    uint32_t local = 0;
    for (uint32_t k = 0; k < per; ++k)
        if (b + k < tiles) local += a.tiles[b + k];
    uint32_t total;
    uint32_t off = na_block_scan(local, total);
    for (uint32_t k = 0; k < per; ++k)
        if (b + k < tiles) {
            const uint32_t v = a.tiles[b + k];
            a.tiles[b + k] = off;
            off += v;
        }
}

__global__ void __launch_bounds__(kScanThreads) k_na_scan(uint32_t nb, Arena a) {
    __shared__ uint32_t tile[kScanTile];
    const size_t t0 = (size_t)blockIdx.x * kScanTile;
    for (int k = 0; k < kScanItems; ++k) {
        const size_t idx = t0 + (size_t)k * kScanThreads + threadIdx.x;
        tile[k * kScanThreads + threadIdx.x] = idx < nb ? a.count[idx] : 0u;
    }
    __syncthreads();
    uint32_t v[kScanItems], s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = tile[threadIdx.x * kScanItems + k];
        s += v[k];
    }
    uint32_t total;
    uint32_t off = na_block_scan(s, total) + a.tiles[blockIdx.x];
    for (int k = 0; k < kScanItems; ++k) {
        tile[threadIdx.x * kScanItems + k] = off;
        off += v[k];
    }
    __syncthreads();
    for (int k = 0; k < kScanItems; ++k) {
        const size_t idx = t0 + (size_t)k * kScanThreads + threadIdx.x;
        if (idx < nb) a.start[idx] = tile[k * kScanThreads + threadIdx.x];
    }
}

__global__ void k_na_total(uint32_t nb, Arena a) {
    if (threadIdx.x == 0) a.start[nb] = a.start[nb - 1] + a.count[nb - 1];
}

__global__ void k_na_scatter(uint32_t n, Arena a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a.tmp[a.start[a.key[i]] + a.rank[i]] = i;
}

// Stable (cell, id) order: rank inside the cell segment by particle id.
__global__ void k_na_rank(vtp::Grid g, uint32_t n, const float *__restrict__ pos, Arena a) {
    const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const uint32_t me = a.tmp[d];
    const uint32_t k = a.key[me];
    uint32_t dst = d;
    if (k < g.nkey) {
        const uint32_t s0 = a.start[k], s1 = a.start[k + 1];
        uint32_t r = 0;
        for (uint32_t x = s0; x < s1; ++x) r += a.tmp[x] < me ? 1u : 0u;
        dst = s0 + r;
    }
    a.sorted[dst] = me;
    a.pos[dst] = make_float4(pos[3 * (size_t)me], pos[3 * (size_t)me + 1], pos[3 * (size_t)me + 2], 0.f);
}

// Lists in the reference layout: self first, then the 27 cells in the
// reference's offset order, particles of a cell by ascending id.
__global__ void k_na_walk(vtp::Grid g, uint32_t n, Arena a, uint32_t *__restrict__ counts,
                          uint32_t *__restrict__ nbrs) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t i = a.sorted[s];
    const uint32_t M = g.maxnbr;
    uint32_t *out = nbrs + (size_t)i * M;
    const float4 p = a.pos[s];
    const int3 c = vtp::cell_of(p.x, p.y, p.z, g);
    uint32_t cnt = 0;
    if (a.key[i] < g.nkey) {
        out[cnt++] = i;
        for (int t = 0; t < 27; ++t) {
            const int3 o = vtp::nbr_offset(t);
            const int3 cc = make_int3(c.x + o.x, c.y + o.y, c.z + o.z);
            if (!vtp::cell_available(cc, g)) continue;
            const uint32_t k = vtp::cell_key(cc, g);
            const uint32_t j0 = a.start[k], j1 = a.start[k + 1];
            for (uint32_t jj = j0; jj < j1; ++jj) {
                const uint32_t j = a.sorted[jj];
                if (j == i) continue;
                const float4 q = a.pos[jj];
                const float d2 = vtp::dist2(p.x - q.x, p.y - q.y, p.z - q.z);
                if (d2 > 0.f && d2 <= g.d2max && cnt < M) out[cnt++] = j;
            }
        }
    }
    counts[i] = cnt;
    for (uint32_t t = cnt; t < M; ++t) out[t] = 0xffffffffu;
}

inline unsigned nblk(uint32_t n, int b) { return (unsigned)((n + b - 1) / b); }

float sqrt_limit(float h) {
    float t = h * h;
    while (std::sqrt(t) > h) t = std::nextafter(t, 0.f);
    for (;;) {
        const float u = std::nextafter(t, INFINITY);
        if (std::sqrt(u) <= h) t = u;
        else break;
    }
    return t;
}

}  // namespace

extern "C" VTP_API int vtp_ugns_neighbors_noalloc(const float *d_pos, uint32_t n, const float lb[3],
                                                  const float size[3], float cell, uint32_t max_nbr,
                                                  uint32_t *d_counts, uint32_t *d_nbrs, void *stream) {
    if (!lb || !size || (n > 0 && (!d_pos || !d_counts || !d_nbrs)))
        return vtp::fail(VTP_ERR_ARG, "null argument");
    if (n > kMaxParticles)
        return vtp::fail(VTP_ERR_BOUNDS, "vtp_ugns_neighbors_noalloc: " + std::to_string(n) +
                                             " particles exceed the scratch limit of " +
                                             std::to_string(kMaxParticles));
    if (!(cell > 0.f) || !std::isfinite(cell) || max_nbr < 1 || max_nbr > 1024)
        return vtp::fail(VTP_ERR_ARG, "cell must be finite and > 0, and max_nbr in [1, 1024]");
    for (int a = 0; a < 3; ++a)
        if (!std::isfinite(lb[a]) || !std::isfinite(size[a]) || !(size[a] > 0.f))
            return vtp::fail(VTP_ERR_ARG, "vtp_ugns_neighbors_noalloc: lb must be finite and size finite and > 0");
    // Cells per axis, checked before the integer conversion (a tiny cell would
    // otherwise overflow int).
    double cells[3];
    for (int a = 0; a < 3; ++a) {
        cells[a] = std::ceil((double)(size[a] / cell));
        if (!(cells[a] >= 1.0) || cells[a] > (double)kMaxKeys)
            return vtp::fail(VTP_ERR_BOUNDS, "vtp_ugns_neighbors_noalloc: grid of " +
                                                 std::to_string(cells[a]) + " cells along one axis exceeds the "
                                                 "scratch limit of " + std::to_string(kMaxKeys) + " cell buckets");
    }
    vtp::Grid g{};
    g.lbx = lb[0]; g.lby = lb[1]; g.lbz = lb[2];
    g.cell = cell;
    g.gx = (int)cells[0];
    g.gy = (int)cells[1];
    g.gz = (int)cells[2];
    const uint64_t maxkey = (uint64_t)g.gz * g.gy * g.gx + (uint64_t)g.gy * g.gx + g.gx;
    if (maxkey + 2 > kMaxKeys)
        return vtp::fail(VTP_ERR_BOUNDS, "vtp_ugns_neighbors_noalloc: grid of " + std::to_string(maxkey + 2) +
                                             " cell buckets exceeds the scratch limit of " +
                                             std::to_string(kMaxKeys));
    g.nkey = (uint32_t)(maxkey + 1);
    g.d2max = sqrt_limit(cell);
    g.maxnbr = max_nbr;
    if (n == 0) return VTP_OK;
    unsigned char *base = nullptr;
    const int rc = arena_base(&base);
    if (rc) return rc;
    cudaError_t e;
    const Arena a = arena_at(base);
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t nb = g.nkey + 1;
    const uint32_t tiles = (nb + kScanTile - 1) / kScanTile;
    // The arena keeps the previous call's contents: the cell counters must start at zero.
    e = cudaMemsetAsync(a.count, 0, (size_t)nb * sizeof(uint32_t), st);
    if (e != cudaSuccess) return vtp::fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    k_na_hash<<<nblk(n, 256), 256, 0, st>>>(g, n, d_pos, a);
    k_na_tile_sums<<<tiles, kScanThreads, 0, st>>>(nb, a);
    k_na_scan_tiles<<<1, 1024, 0, st>>>(tiles, a);
    k_na_scan<<<tiles, kScanThreads, 0, st>>>(nb, a);
    k_na_total<<<1, 32, 0, st>>>(nb, a);
    k_na_scatter<<<nblk(n, 256), 256, 0, st>>>(n, a);
    k_na_rank<<<nblk(n, 256), 256, 0, st>>>(g, n, d_pos, a);
    k_na_walk<<<nblk(n, 128), 128, 0, st>>>(g, n, a, d_counts, d_nbrs);
    e = cudaGetLastError();
    if (e != cudaSuccess) return vtp::fail(VTP_ERR_CUDA, cudaGetErrorString(e));
    return VTP_OK;
}
