// Stand-in for the assimp scene types the reference reads (TEST INFRASTRUCTURE
// for oracle/_ref).  Vertices are single precision, as assimp's default
// ai_real is float.
#pragma once
#include <vector>

struct aiVector3D {
  float x, y, z;
};
struct aiFace {
  unsigned int mNumIndices = 0;
  unsigned int* mIndices = nullptr;
};
struct aiMesh {
  unsigned int mNumVertices = 0;
  aiVector3D* mVertices = nullptr;
  unsigned int mNumFaces = 0;
  aiFace* mFaces = nullptr;
};
struct aiScene {
  unsigned int mNumMeshes = 0;
  aiMesh** mMeshes = nullptr;
};
