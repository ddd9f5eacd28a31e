// SolverManager, ObjectManager and the Simulator singleton of the reference
// (Simulator/Runtime/Source/Manager/SolverManager.cpp:19-40, Simulator.hpp),
// over the sm_100a library.
#ifndef VTP_HOST_SIMULATOR_HPP
#define VTP_HOST_SIMULATOR_HPP

#include <memory>
#include <vector>

#include "Framework/Object.hpp"
#include "Framework/Solver.hpp"

namespace VT_Physics {

class SolverManager {
public:
    Solver *createSolver(SolverType type);
    void clear() { m_solvers.clear(); }

private:
    std::vector<std::shared_ptr<Solver>> m_solvers;
};

// Copyable like the reference's (its examples copy the instance); the
// managers share ownership of what they created.
class Simulator final {
public:
    static Simulator &getInstance();
    ObjectManager *getObjectManager() { return &m_objectManager; }
    SolverManager *getSolverManager() { return &m_solverManager; }
    void terminate() {
        m_solverManager.clear();
        m_objectManager.clear();
    }
    static void clean() {}

private:
    ObjectManager m_objectManager;
    SolverManager m_solverManager;
};

}  // namespace VT_Physics

#endif
