// IMM / IMM-CT solver passes (not yet implemented: every entry reports VTP_ERR_CONFIG).
#include "immct.h"
#include "solver.h"

namespace vtp {
struct ImmState {
    bool ct = false;
};
}  // namespace vtp

nlohmann::json immct_default_required(bool) { return nlohmann::json::object(); }
std::vector<std::string> immct_required_keys(bool) { return {}; }
int immct_parse(bool, const nlohmann::json &, std::shared_ptr<vtp::ImmState> &) {
    return vtp::fail(VTP_ERR_CONFIG, "IMM / IMM-CT solvers are not available in this build");
}
int immct_alloc(vtp_solver &) { return vtp::fail(VTP_ERR_CONFIG, "IMM-CT not available"); }
int immct_init(vtp_solver &) { return vtp::fail(VTP_ERR_CONFIG, "IMM-CT not available"); }
int immct_enqueue_tick(vtp_solver &, cudaStream_t, bool) { return vtp::fail(VTP_ERR_CONFIG, "IMM-CT not available"); }
void immct_solve_ab(vtp_solver &, cudaStream_t, int) {}
int immct_phase_count(const vtp_solver &) { return 0; }
float immct_scalar_host(vtp_solver &, int, uint32_t, float, float) { return 0.f; }
int immct_get_field(vtp_solver &, int, float *, size_t) { return vtp::fail(VTP_ERR_CONFIG, "IMM-CT not available"); }
