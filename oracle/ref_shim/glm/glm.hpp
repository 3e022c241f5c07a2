// Stand-in for the glm headers the reference includes (include/Util/Math.hpp).
// TEST INFRASTRUCTURE: used only to compile the reference's own sources into
// oracle/_ref.  glm is not vendored in the reference and its version is not
// pinned there, so this implements only what the reference calls, from the
// documented definitions: componentwise +,-,*,/ ; dot(a,b) = (a.x*b.x +
// a.y*b.y) + a.z*b.z ; length(v) = sqrt(dot(v,v)) ; distance(a,b) =
// length(b-a) ; normalize(v) = v * (1/sqrt(dot(v,v))) ; cross as the
// determinant expansion ; min/max componentwise as (b < a ? b : a).
#pragma once
#include <cmath>
#include <string>

namespace glm {

struct dvec3 {
  double x, y, z;
  dvec3() : x(0.0), y(0.0), z(0.0) {}
  dvec3(double a, double b, double c) : x(a), y(b), z(c) {}
  explicit dvec3(double s) : x(s), y(s), z(s) {}
  double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  const double& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  dvec3& operator+=(const dvec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  dvec3& operator-=(const dvec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  dvec3& operator*=(double s) { x *= s; y *= s; z *= s; return *this; }
  dvec3& operator/=(double s) { x /= s; y /= s; z /= s; return *this; }
};

inline dvec3 operator+(const dvec3& a, const dvec3& b) { return dvec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline dvec3 operator-(const dvec3& a, const dvec3& b) { return dvec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline dvec3 operator*(const dvec3& a, const dvec3& b) { return dvec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline dvec3 operator+(const dvec3& a, double s) { return dvec3(a.x + s, a.y + s, a.z + s); }
inline dvec3 operator-(const dvec3& a, double s) { return dvec3(a.x - s, a.y - s, a.z - s); }
inline dvec3 operator*(const dvec3& a, double s) { return dvec3(a.x * s, a.y * s, a.z * s); }
inline dvec3 operator*(double s, const dvec3& a) { return dvec3(s * a.x, s * a.y, s * a.z); }
inline dvec3 operator/(const dvec3& a, double s) { return dvec3(a.x / s, a.y / s, a.z / s); }
inline dvec3 operator-(const dvec3& a) { return dvec3(-a.x, -a.y, -a.z); }

inline double dot(const dvec3& a, const dvec3& b) {
  const dvec3 t = a * b;
  return t.x + t.y + t.z;
}
inline double length(const dvec3& v) { return std::sqrt(dot(v, v)); }
inline double distance(const dvec3& a, const dvec3& b) { return length(b - a); }
inline dvec3 normalize(const dvec3& v) { return v * (1.0 / std::sqrt(dot(v, v))); }
inline dvec3 cross(const dvec3& a, const dvec3& b) {
  return dvec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
inline double min_(double a, double b) { return (b < a) ? b : a; }
inline double max_(double a, double b) { return (a < b) ? b : a; }
inline dvec3 min(const dvec3& a, const dvec3& b) { return dvec3(min_(a.x, b.x), min_(a.y, b.y), min_(a.z, b.z)); }
inline dvec3 max(const dvec3& a, const dvec3& b) { return dvec3(max_(a.x, b.x), max_(a.y, b.y), max_(a.z, b.z)); }
inline std::string to_string(const dvec3& v) {
  return "dvec3(" + std::to_string(v.x) + ", " + std::to_string(v.y) + ", " + std::to_string(v.z) + ")";
}

}  // namespace glm
