/* Stub of the mesh importer used only by PLY geometry loading, which the
 * reference build driven from oracle/ref never calls. */
#pragma once
#include <string>
#include "scene.h"
namespace Assimp {
class Importer {
public:
    const aiScene *ReadFile(const std::string &, unsigned) { return nullptr; }
    const char *GetErrorString() const { return "mesh import is not available in this build"; }
};
}  // namespace Assimp
