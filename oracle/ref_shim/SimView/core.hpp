// Stand-in for the SimView viewer headers (TEST INFRASTRUCTURE for
// oracle/_ref).  The viewer submodule is absent from the reference and no
// graphics stack exists here; only the type names the containers mention
// are provided, as inert objects.
#pragma once
#include <array>
#include <memory>
#include <vector>

namespace simview {
using vec3f_t = std::array<float, 3>;
namespace model {
struct Primitive {
  virtual ~Primitive() = default;
};
using Primitive_t = std::shared_ptr<Primitive>;
struct Box : Primitive {
  Box(float, float, float, float, float, float) {}
  void initVAO() {}
};
struct Object : Primitive {
  template <class... A>
  void initVAO(A&&...) {}
};
using Object_t = std::shared_ptr<Object>;
struct Sphere : Primitive {};
using Sphere_t = std::shared_ptr<Sphere>;
}  // namespace model
namespace app {
struct ViewerGUIApp;  // named by Visualization.hpp only; never defined or used
using ViewerGUIApp_t = std::shared_ptr<ViewerGUIApp>;
}  // namespace app
}  // namespace simview
