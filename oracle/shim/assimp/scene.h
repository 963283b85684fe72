// Minimal stand-in for the Assimp scene types (project-written test infrastructure).
// Assimp is not installed here; the oracle harness only needs the reference's
// core/scene.cpp to compile.  Mesh files are never loaded through this stub:
// Importer::ReadFile always fails, so Scene::loadMesh throws its runtime_error.
#pragma once
struct aiVector3D { float x, y, z; };
struct aiString { const char* C_Str() const { return ""; } };
struct aiMesh {
    aiString mName;
    unsigned int mNumVertices = 0;
    aiVector3D* mVertices = nullptr;
    aiVector3D* mNormals = nullptr;
};
struct aiScene {
    unsigned int mNumMeshes = 0;
    aiMesh** mMeshes = nullptr;
    bool HasMeshes() const { return mNumMeshes > 0; }
};
