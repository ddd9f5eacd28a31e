// The solver plugin interface of the reference (Simulator/Runtime/Include/
// Framework/Solver.hpp:27-62) with the four solvers implemented over the
// sm_100a library's C ABI (include/vtp.h).  Method names, JSON keys,
// boolean returns and the attach-order particle indexing are the
// reference's; failures log the library's message to stderr.
#ifndef VTP_HOST_SOLVER_HPP
#define VTP_HOST_SOLVER_HPP

#include <cstdint>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

#include "Framework/Material.hpp"
#include "Framework/Object.hpp"

struct vtp_solver;

namespace VT_Physics {

using json = nlohmann::json;

typedef enum eSolverType : uint8_t { PBF = 0, DFSPH = 1, IMM = 2, IMMCT = 3 } SolverType;

class Solver {
public:
    Solver() = default;
    virtual ~Solver() = 0;
    virtual json getSolverConfigTemplate() const = 0;
    virtual bool setConfig(json config) = 0;
    virtual bool setConfigByFile(std::string config_file) = 0;
    virtual json getSolverObjectComponentConfigTemplate() = 0;
    virtual bool run() = 0;
    [[maybe_unused]] virtual bool tickNsteps(uint32_t n) = 0;
    virtual bool attachObject(Object *obj) = 0;
    virtual bool attachObjects(std::vector<Object *> objs) = 0;
    virtual bool initialize() = 0;
    virtual bool reset() = 0;
    virtual void destroy() = 0;

protected:
    virtual bool tick() = 0;
    virtual bool checkConfig() const = 0;
};

// One implementation for the four solver types (the library dispatches on the type).
class VtpSolver : public Solver {
public:
    explicit VtpSolver(SolverType type);
    ~VtpSolver() override;
    json getSolverConfigTemplate() const override;
    bool setConfig(json config) override;
    bool setConfigByFile(std::string config_file) override;
    json getSolverObjectComponentConfigTemplate() override;
    bool run() override;
    bool tickNsteps(uint32_t n) override;
    bool attachObject(Object *obj) override;
    bool attachObjects(std::vector<Object *> objs) override;
    bool initialize() override;
    bool reset() override;
    void destroy() override;

    // Extensions of this library.
    std::vector<float> getField(int field) const;   // attach order, see vtp_field
    vtp_solver *handle() const { return m_h; }
    SolverType type() const { return m_type; }

protected:
    bool tick() override;
    bool checkConfig() const override;

private:
    bool ok(int rc, const char *what) const;
    SolverType m_type;
    vtp_solver *m_h = nullptr;
    json m_config;
    bool m_configured = false;
};

class PBFSolver : public VtpSolver {
public:
    PBFSolver() : VtpSolver(PBF) {}
};
class DFSPHSolver : public VtpSolver {
public:
    DFSPHSolver() : VtpSolver(DFSPH) {}
};
class IMMSolver : public VtpSolver {
public:
    IMMSolver() : VtpSolver(IMM) {}
};
class IMMCTSolver : public VtpSolver {
public:
    IMMCTSolver() : VtpSolver(IMMCT) {}
};

}  // namespace VT_Physics

#endif
