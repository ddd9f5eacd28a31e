// Differentiable DFSPH rollout (diff_dfsph.cu): the DFSPH side of
// vtp_solver_diff_forward / _backward / _lists / _iterations.
#pragma once

#include <cstdint>

struct vtp_solver;

namespace vtp {

struct DfDiffState;

// Single scene, fixed time step, surface tension off; VTP_OK or the failure code.
int dfsph_diff_ready(vtp_solver *s);
int dfsph_diff_forward(vtp_solver *s, uint32_t n_steps, uint32_t checkpoint_every, int keep_lists);
// dl_dvis receives dL/d(fPartRestViscosity).
int dfsph_diff_backward(vtp_solver *s, const float *dl_dpos, const float *dl_dvel, float *dl_dpos0,
                        float *dl_dvel0, double *dl_dvis);
// Device pointers to the record of substep `step` (rollouts recorded with keep_lists): its
// sorted fluid rows' attach ids, lists, and iteration counts.
int dfsph_diff_slot(vtp_solver *s, uint32_t step, const uint32_t **orig, const uint32_t **nbr,
                    const uint32_t **ncnt, uint32_t *div_iters, uint32_t *inc_iters);

}  // namespace vtp
