// Peer-store halos of a slab worker (vtp_domain_*, domain.cu): the stage kernels of the
// DFSPH and PBF passes write each value a peer's ghost row needs straight into that peer's
// buffers (plain stores to another GPU's memory over NVLink, or to another worker on the same
// GPU), instead of a pack / exchange / unpack after the pass.  Rows flagged as ghosts write
// nothing: their values arrive from their owners.  The host orders a peer's next stage after
// the stores (a collective on the stream, or a barrier).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vtp {

constexpr int kMaxPeers = 8;
constexpr int kMaxHaloTargets = 4;   // peers a row can be a ghost on

// A peer worker's buffers as mapped here (the fields its solver type uses).
struct PeerRows {
    float *kappa;                    // DFSPH: kappa
    float4 *pk, *pva, *normal;       // DFSPH: packed {x, kappa} / {x, v*} rows, surface normals
    float4 *vadv[2];                 // DFSPH: both v* buffers
    float4 *vel[2];                  // both velocity buffers
    float *lambda;                   // PBF: lambda
    float4 *pos[2];                  // PBF: both position buffers
};
struct HaloPush {
    const uint8_t *ghost;            // [rows] 1: ghost row (no writes)
    const uint32_t *ntarget;         // [rows] targets of the row (0..kMaxHaloTargets)
    const uint2 *target;             // [rows][kMaxHaloTargets] {peer, peer row}
    PeerRows peer[kMaxPeers];
};

#ifdef __CUDACC__
// A: an argument struct with a `const HaloPush *halo` member.
template <class A>
__device__ __forceinline__ bool halo_ghost(const A &a, uint32_t r) {
    return a.halo && a.halo->ghost[r];
}

// Hands `f(peer rows, the peer's row)` every peer the owned row r is a ghost on; the stores
// to other GPUs are ordered before what follows by a system fence.
template <class A, class F>
__device__ __forceinline__ void halo_each(const A &a, uint32_t r, F f) {
    if (!a.halo) return;
    const uint32_t n = min(a.halo->ntarget[r], (uint32_t)kMaxHaloTargets);
    for (uint32_t e = 0; e < n; ++e) {
        const uint2 t = a.halo->target[(size_t)r * kMaxHaloTargets + e];
        f(a.halo->peer[t.x], t.y);
    }
    if (n) __threadfence_system();
}
#endif

}  // namespace vtp
