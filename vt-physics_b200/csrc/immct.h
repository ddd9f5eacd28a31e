// IMM / IMM-CT (mixture model + conformation tensor) solver hooks used by the driver.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

#include "dfsph.h"
#include "internal.h"

struct vtp_solver;

namespace vtp {
struct ImmState;
}

nlohmann::json immct_default_required(bool ct);
std::vector<std::string> immct_required_keys(bool ct);
int immct_parse(bool ct, const nlohmann::json &required, std::shared_ptr<vtp::ImmState> &imm);
int immct_alloc(vtp_solver &s);
int immct_init(vtp_solver &s);
int immct_enqueue_tick(vtp_solver &s, cudaStream_t st, bool capture);
void immct_solve_ab(vtp_solver &s, cudaStream_t st, int which);
// The pressure-solve arguments of a mixture solver: the DFSPH passes' with the per-row rest
// density (mass = rest density x volume).
vtp::DfsphArgs immct_solve_args(vtp_solver &s, int which);
int immct_phase_count(const vtp_solver &s);
int immct_get_field(vtp_solver &s, int field, float *dev_out, size_t elems);
void immct_fill_carry(vtp_solver &s, vtp::Carry &carry);
int immct_copy_back(vtp_solver &s);
void immct_set_parity(vtp_solver &s, int cur);
// Retries of the last substep; *body_launches (optional) receives the kernels
// the retry loop's bodies launched since the previous call.
uint32_t immct_last_retries(vtp_solver &s, uint64_t *body_launches = nullptr);
// Inputs of the conservation sums: rest density and phase fractions of the fluid rows, the
// phase rest densities (up to vtp::kConsPhases phases).
void immct_conservation_inputs(vtp_solver &s, const float **rd, const float **frac, float *rho_k, int *P);
void immct_color(vtp_solver &s, const float *frac_attach_order, float *rgb);
