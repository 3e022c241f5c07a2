// Stand-in for assimp's post-processing flags (TEST INFRASTRUCTURE for oracle/_ref).
#pragma once
enum aiPostProcessSteps {
  aiProcess_CalcTangentSpace = 0x1,
  aiProcess_Triangulate = 0x8,
  aiProcess_GenNormals = 0x20,
  aiProcess_RemoveRedundantMaterials = 0x1000
};
