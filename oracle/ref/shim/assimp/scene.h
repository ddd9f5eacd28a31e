#pragma once
#define AI_SCENE_FLAGS_INCOMPLETE 0x1
struct aiVector3D { float x, y, z; };
struct aiMesh { unsigned mNumVertices; aiVector3D *mVertices; };
struct aiNode {};
struct aiScene { unsigned mFlags; aiNode *mRootNode; unsigned mNumMeshes; aiMesh **mMeshes; };
