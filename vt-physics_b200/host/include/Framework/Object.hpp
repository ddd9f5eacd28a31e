// Particle objects of the host interface: the same class and method names as
// the reference's VT_Physics::Object (Simulator/Runtime/Include/Framework/
// Object.hpp:15-48) and ObjectManager, so programs written against the
// reference compile against this library.  Sphere, cube, cylinder, plane and
// box objects generate their particles with the reference generators'
// arithmetic (ModelHandler.cpp:43-175); Particle_Common objects take
// positions through setElements() or, with "particleGeometryPath" in their
// component config, from a PLY file (ModelHandler.cpp:177-228).
#ifndef VTP_HOST_OBJECT_HPP
#define VTP_HOST_OBJECT_HPP

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

#include "Framework/Material.hpp"

namespace VT_Physics {

using json = nlohmann::json;

// Object types (the reference's eObjectType, ObjectComponents.hpp:17-31), all
// with their particle generators.
typedef enum eObjectType : uint8_t {
    Particle_Common = 0,
    Particle_Sphere = 1,
    Particle_Cube = 2,
    Particle_Cylinder = 3,
    Particle_Plane = 4,
    Particle_Box = 5,
} ObjectType;

class Object;

// Geometry of an object (the reference's ObjectTypeComponent).
class ObjectTypeComponent {
public:
    explicit ObjectTypeComponent(ObjectType t) : m_type(t) {}
    ObjectType getType() const { return m_type; }
    // x, y, z of every particle (3 floats per particle)
    std::vector<float> getElements() const { return m_pos; }

private:
    friend class Object;
    ObjectType m_type;
    std::vector<float> m_pos;
};

class Object {
public:
    explicit Object(ObjectType type);

    json &getObjectComponentConfig();
    void attachSpecificSolverObjectComponentConfig(json specificSolverObjectComponentConfig);
    json &getSolverObjectComponentConfig();
    ObjectTypeComponent *getObjectComponent();
    long long getID() const;
    void rename(std::string newName);
    std::string getName() const;
    // Regenerates the particles from the component config (generators, or a PLY file).
    bool update();
    void reset();

    // Extensions: explicit positions (Particle_Common) and per-particle start velocities.
    void setElements(std::vector<float> xyz);
    void setVelocities(std::vector<float> xyz);
    const std::vector<float> &getVelocities() const { return m_vel; }

private:
    static long long s_next_id;
    long long m_id;
    std::string m_name;
    json m_objectComponentConfig{};
    json m_solverSpecificComponentConfig{};
    ObjectTypeComponent m_component;
    std::vector<float> m_vel;
};

class ObjectManager {
public:
    Object *createObject(ObjectType type);
    void clear() { m_objects.clear(); }

private:
    std::vector<std::shared_ptr<Object>> m_objects;
};

// The generators, shared with tests: n x 3 floats.
std::vector<float> generateCube(float r, const float lb[3], const float size[3]);
std::vector<float> generateBox(float r, const float lb[3], const float size[3], int layerNum);

}  // namespace VT_Physics

#endif
