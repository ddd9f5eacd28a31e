// Host interface over the C ABI (see Framework/Solver.hpp, Framework/Object.hpp).
#include <cmath>
#include <cstdio>
#include <fstream>

#include "../../../include/vtp.h"
#include "Framework/Object.hpp"
#include "Framework/Solver.hpp"
#include "Manager/Simulator.hpp"

namespace VT_Physics {

// ---------------------------------------------------------------- generators

std::vector<float> generateCube(float r, const float lb[3], const float size[3]) {
    // x = lb + r, then x += 2r while x < lb + size, each sum rounded to float.
    std::vector<float> axis[3];
    const float d = 2.f * r;
    for (int a = 0; a < 3; ++a) {
        const float lim = lb[a] + size[a];
        for (float v = r + lb[a]; v < lim; v = v + d) axis[a].push_back(v);
    }
    std::vector<float> out;
    out.reserve(axis[0].size() * axis[1].size() * axis[2].size() * 3);
    for (float z : axis[2])
        for (float y : axis[1])
            for (float x : axis[0]) out.insert(out.end(), {x, y, z});
    return out;
}

std::vector<float> generateBox(float r, const float lb[3], const float size[3], int layerNum) {
    // n = int((size + r) / 2r) lattice steps per axis from lb + r; keep the
    // layerNum outermost layers on every side.
    int n[3];
    double base[3];
    for (int a = 0; a < 3; ++a) {
        n[a] = (int)((double)(float)(size[a] + r) / (2.0 * (double)r));
        base[a] = (double)(float)(lb[a] + r);
    }
    std::vector<float> out;
    for (int i = 0; i <= n[0]; ++i)
        for (int j = 0; j <= n[1]; ++j)
            for (int k = 0; k <= n[2]; ++k) {
                const bool shell = i < layerNum || i >= n[0] - layerNum || j < layerNum || j >= n[1] - layerNum ||
                                   k < layerNum || k >= n[2] - layerNum;
                if (!shell) continue;
                out.push_back((float)(base[0] + 2.0 * r * i));
                out.push_back((float)(base[1] + 2.0 * r * j));
                out.push_back((float)(base[2] + 2.0 * r * k));
            }
    return out;
}

// ---------------------------------------------------------------- objects

long long Object::s_next_id = 0;

Object::Object(ObjectType type) : m_component(type) {
    m_id = ++s_next_id;
    m_name = "obj_" + std::to_string(m_id);
    m_objectComponentConfig = {{"epmMaterial", 255}, {"particleRadius", 0.05}};
}

json &Object::getObjectComponentConfig() { return m_objectComponentConfig; }
void Object::attachSpecificSolverObjectComponentConfig(json c) { m_solverSpecificComponentConfig = std::move(c); }
json &Object::getSolverObjectComponentConfig() { return m_solverSpecificComponentConfig; }
ObjectTypeComponent *Object::getObjectComponent() { return &m_component; }
long long Object::getID() const { return m_id; }
void Object::rename(std::string newName) { m_name = std::move(newName); }
std::string Object::getName() const { return m_name; }
void Object::reset() {
    m_component.m_pos.clear();
    m_vel.clear();
}
void Object::setElements(std::vector<float> xyz) { m_component.m_pos = std::move(xyz); }
void Object::setVelocities(std::vector<float> xyz) { m_vel = std::move(xyz); }

bool Object::update() {
    const json &c = m_objectComponentConfig;
    auto vec3 = [&](const char *k, float *v) {
        auto a = c.at(k).get<std::vector<float>>();
        if (a.size() != 3) throw std::runtime_error(std::string(k) + " needs 3 values");
        for (int i = 0; i < 3; ++i) v[i] = a[i];
    };
    // Sphere, cylinder and plane objects, and particle objects with a PLY file, go through the
    // library's host geometry calls (ModelHandler::generateObjectElements / loadObjectElements).
    auto from_library = [&](bool ply) {
        uint64_t n = 0;
        const std::string arg = ply ? c.at("particleGeometryPath").get<std::string>() : [&] {
            json g = c;
            g["genType"] = (int)m_component.getType();
            return g.dump();
        }();
        int rc = ply ? vtp_read_ply(arg.c_str(), nullptr, 0, &n) : vtp_generate_particles(arg.c_str(), nullptr, 0, &n);
        std::vector<float> xyz(3 * n);
        if (rc == VTP_OK && n)
            rc = ply ? vtp_read_ply(arg.c_str(), xyz.data(), n, &n)
                     : vtp_generate_particles(arg.c_str(), xyz.data(), n, &n);
        if (rc != VTP_OK) {
            std::fprintf(stderr, "[vtp] object %s: %s\n", m_name.c_str(), vtp_last_error());
            return false;
        }
        m_component.m_pos = std::move(xyz);
        return true;
    };
    try {
        switch (m_component.getType()) {
            case Particle_Common:
                return c.contains("particleGeometryPath") ? from_library(true) : true;
            case Particle_Sphere:
            case Particle_Cylinder:
            case Particle_Plane:
                return from_library(false);
            case Particle_Cube: {
                float lb[3], size[3];
                vec3("lb", lb);
                vec3("size", size);
                m_component.m_pos = generateCube(c.at("particleRadius").get<float>(), lb, size);
                return true;
            }
            case Particle_Box: {
                float lb[3], size[3];
                vec3("lb", lb);
                vec3("size", size);
                m_component.m_pos = generateBox(c.at("particleRadius").get<float>(), lb, size,
                                                c.at("layerNum").get<int>());
                return true;
            }
            default:
                std::fprintf(stderr, "[vtp] object type %d has no particle generator here\n",
                             (int)m_component.getType());
                return false;
        }
    } catch (const std::exception &e) {
        std::fprintf(stderr, "[vtp] object %s: %s\n", m_name.c_str(), e.what());
        return false;
    }
}

Object *ObjectManager::createObject(ObjectType type) {
    m_objects.push_back(std::make_shared<Object>(type));
    return m_objects.back().get();
}

// ---------------------------------------------------------------- solvers

Solver::~Solver() = default;

VtpSolver::VtpSolver(SolverType type) : m_type(type) {
    if (vtp_solver_create((int)type, &m_h) != VTP_OK) {
        std::fprintf(stderr, "[vtp] %s\n", vtp_last_error());
        m_h = nullptr;
    }
}

VtpSolver::~VtpSolver() {
    if (m_h) vtp_solver_destroy(m_h);
}

bool VtpSolver::ok(int rc, const char *what) const {
    if (rc == VTP_OK) return true;
    std::fprintf(stderr, "[vtp] %s: %s (%s)\n", what, vtp_last_error(), vtp_status_string(rc));
    return false;
}

json VtpSolver::getSolverConfigTemplate() const {
    if (!m_h) return {};
    size_t n = 0;
    vtp_solver_get_config(m_h, nullptr, 0, &n);
    std::string s(n, '\0');
    if (vtp_solver_get_config(m_h, s.data(), n, nullptr) != VTP_OK) return {};
    return json::parse(s.c_str());
}

bool VtpSolver::setConfig(json config) {
    if (!m_h) return false;
    if (!ok(vtp_solver_set_config(m_h, config.dump().c_str()), "setConfig")) return false;
    m_config = std::move(config);
    m_configured = true;
    return true;
}

bool VtpSolver::setConfigByFile(std::string config_file) {
    std::ifstream f(config_file);
    if (!f) {
        std::fprintf(stderr, "[vtp] cannot open %s\n", config_file.c_str());
        return false;
    }
    json c;
    try {
        f >> c;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "[vtp] %s: %s\n", config_file.c_str(), e.what());
        return false;
    }
    return setConfig(std::move(c));
}

json VtpSolver::getSolverObjectComponentConfigTemplate() {
    json t = {{"solverType", (int)m_type}, {"exportFlag", false}, {"velocityStart", {0, 0, 0}}};
    if (m_type == IMM || m_type == IMMCT) t["phaseFraction"] = json::array();
    else t["colorStart"] = {0, 0, 0};
    return t;
}

bool VtpSolver::attachObject(Object *obj) {
    if (!m_h || !obj) return false;
    const std::vector<float> pos = obj->getObjectComponent()->getElements();
    const std::vector<float> &vel = obj->getVelocities();
    if (!vel.empty() && vel.size() != pos.size()) {
        std::fprintf(stderr, "[vtp] attachObject: velocity count does not match the particle count\n");
        return false;
    }
    json meta = {{"name", obj->getName()},
                 {"ObjectComponentConfig", obj->getObjectComponentConfig()},
                 {"SolverObjectComponentConfig", obj->getSolverObjectComponentConfig()}};
    return ok(vtp_solver_attach_object(m_h, pos.data(), (uint32_t)(pos.size() / 3), vel.empty() ? nullptr : vel.data(),
                                       meta.dump().c_str()),
              "attachObject");
}

bool VtpSolver::attachObjects(std::vector<Object *> objs) {
    for (Object *o : objs)
        if (!attachObject(o)) return false;
    return true;
}

bool VtpSolver::initialize() { return m_h && ok(vtp_solver_initialize(m_h), "initialize"); }
bool VtpSolver::run() { return m_h && ok(vtp_solver_run(m_h), "run"); }
bool VtpSolver::tickNsteps(uint32_t n) { return m_h && ok(vtp_solver_tick_n_steps(m_h, n), "tickNsteps"); }
bool VtpSolver::tick() { return tickNsteps(1); }
bool VtpSolver::reset() { return m_h && ok(vtp_solver_reset(m_h), "reset"); }
void VtpSolver::destroy() {
    if (m_h) vtp_solver_destroy(m_h);
    m_h = nullptr;
}
bool VtpSolver::checkConfig() const { return m_configured; }

std::vector<float> VtpSolver::getField(int field) const {
    uint32_t n = 0, nf = 0, nb = 0, np = 0;
    if (!m_h || vtp_solver_particle_counts(m_h, &n, &nf, &nb, &np) != VTP_OK) return {};
    int width = 1;
    switch (field) {
        case VTP_FIELD_POS: case VTP_FIELD_VEL: case VTP_FIELD_COLOR: width = 3; break;
        case VTP_FIELD_VOL_FRAC: width = (int)np; break;
        case VTP_FIELD_PHASE_VEL: width = 3 * (int)np; break;
        case VTP_FIELD_CONFORMATION: case VTP_FIELD_VEL_GRAD: case VTP_FIELD_STRESS: width = 9; break;
        default: width = 1;
    }
    std::vector<float> out((size_t)n * width);
    if (!ok(vtp_solver_get_field(m_h, field, out.data(), out.size() * 4), "getField")) return {};
    return out;
}

Solver *SolverManager::createSolver(SolverType type) {
    std::shared_ptr<Solver> s;
    switch (type) {
        case PBF: s = std::make_shared<PBFSolver>(); break;
        case DFSPH: s = std::make_shared<DFSPHSolver>(); break;
        case IMM: s = std::make_shared<IMMSolver>(); break;
        case IMMCT: s = std::make_shared<IMMCTSolver>(); break;
        default: return nullptr;
    }
    m_solvers.push_back(s);
    return s.get();
}

Simulator &Simulator::getInstance() {
    static Simulator instance;
    return instance;
}

}  // namespace VT_Physics
