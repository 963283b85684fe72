// Minimal stand-in for Assimp::Importer (see scene.h in this folder): loading always fails.
#pragma once
#include <string>
#include "scene.h"
namespace Assimp {
class Importer {
   public:
    const aiScene* ReadFile(const std::string&, unsigned int) { return nullptr; }
    const char* GetErrorString() const { return "mesh loading is unavailable in the oracle harness (no Assimp)"; }
};
}  // namespace Assimp
