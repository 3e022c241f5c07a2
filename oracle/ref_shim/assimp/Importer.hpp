// Stand-in for Assimp::Importer (TEST INFRASTRUCTURE for oracle/_ref).
// Reads a Wavefront OBJ: "v x y z" lines parsed as float, "f" lines with
// 1-based or negative indices (the part before the first '/'), polygons
// fanned into triangles (v0, vk, vk+1).  One mesh, faces in file order.
#pragma once
#include <assimp/scene.h>

#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace Assimp {
class Importer {
 public:
  const aiScene* ReadFile(const std::string& path, unsigned int /*flags*/) {
    std::ifstream in(path);
    if (!in.is_open()) {
      err_ = "Unable to open file \"" + path + "\".";
      return nullptr;
    }
    std::string line;
    while (std::getline(in, line)) {
      std::istringstream ss(line);
      std::string tag;
      ss >> tag;
      if (tag == "v") {
        std::string a, b, c;
        ss >> a >> b >> c;
        verts_.push_back({std::strtof(a.c_str(), nullptr), std::strtof(b.c_str(), nullptr),
                          std::strtof(c.c_str(), nullptr)});
      } else if (tag == "f") {
        std::vector<long> ids;
        std::string tok;
        while (ss >> tok) {
          long k = std::strtol(tok.substr(0, tok.find('/')).c_str(), nullptr, 10);
          ids.push_back(k < 0 ? (long)verts_.size() + k : k - 1);
        }
        for (size_t k = 1; k + 1 < ids.size(); ++k) {
          idx_.push_back((unsigned)ids[0]);
          idx_.push_back((unsigned)ids[k]);
          idx_.push_back((unsigned)ids[k + 1]);
        }
      }
    }
    faces_.resize(idx_.size() / 3);
    for (size_t f = 0; f < faces_.size(); ++f) {
      faces_[f].mNumIndices = 3;
      faces_[f].mIndices = &idx_[3 * f];
    }
    mesh_.mNumVertices = (unsigned)verts_.size();
    mesh_.mVertices = verts_.data();
    mesh_.mNumFaces = (unsigned)faces_.size();
    mesh_.mFaces = faces_.data();
    mesh_ptr_ = &mesh_;
    scene_.mNumMeshes = 1;
    scene_.mMeshes = &mesh_ptr_;
    return &scene_;
  }
  const char* GetErrorString() const { return err_.c_str(); }

 private:
  std::vector<aiVector3D> verts_;
  std::vector<unsigned> idx_;
  std::vector<aiFace> faces_;
  aiMesh mesh_;
  aiMesh* mesh_ptr_ = nullptr;
  aiScene scene_;
  std::string err_;
};
}  // namespace Assimp
