// PBF pass launchers (pbf.cu).
#pragma once

#include "internal.h"
#include "halo.h"

namespace vtp {

struct PbfArgs {
    uint32_t nf, nb;
    uint32_t ell_stride;
    Cubic k;
    float rho0, inv_rho0, rho_b, eps, dt, xsph_k;
    int form;              // 0: the reference's formulation; 1: standard PBF (poly6 / spiky, mass-weighted)
    float h2, c6, cs;      // standard PBF: h^2, poly6 315/(64 pi h^9), spiky -45/(pi h^6)
    const uint32_t *nbr;   // fluid-row ELL list
    const uint32_t *ncnt;  // fluid-row counts (self included)
    float4 *pos;           // current positions, w = mass
    float4 *pos_alt;       // output positions (second buffer)
    float4 *vel;           // current velocities
    float4 *vel_alt;       // output velocities (XSPH pass)
    float *vol;            // [n] volume (fluid V0, boundary 1/sum W)
    float *density;        // [nf]
    float *lambda;         // [nf]
    int unroll;            // neighbours in flight per thread (1, 2, 4, 8)
    int lanes = 1;         // threads per row of the neighbour passes (1, 4, 8)
    const HaloPush *halo = nullptr;   // peer-store halos of a slab worker (halo.h; null: none)
    int halo_pos = 0, halo_vel = 0;   // current position / velocity buffer (the peers' parity equals ours)
};

void pbf_init_boundary(cudaStream_t st, const PbfArgs &a, const uint32_t *bncnt, const uint32_t *bnbr,
                       uint32_t ell_stride);
void pbf_lambda(cudaStream_t st, const PbfArgs &a, int block);
void pbf_dx(cudaStream_t st, const PbfArgs &a, int block);
void pbf_xsph(cudaStream_t st, const PbfArgs &a, int block);

}  // namespace vtp
