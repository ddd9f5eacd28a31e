// Particle materials (the reference's Framework/Material.hpp:20-28).
#ifndef VTP_HOST_MATERIAL_HPP
#define VTP_HOST_MATERIAL_HPP

#include <string>
#include <unordered_map>

namespace VT_Physics {

enum class ParticleMaterial : int { epm_Fluid = 0, epm_Boundary = 1 };

#define EPM_FLUID static_cast<int>(VT_Physics::ParticleMaterial::epm_Fluid)
#define EPM_BOUNDARY static_cast<int>(VT_Physics::ParticleMaterial::epm_Boundary)

inline const std::unordered_map<int, std::string> EPMString = {{EPM_FLUID, "Fluid"}, {EPM_BOUNDARY, "Boundary"}};

}  // namespace VT_Physics

#endif
