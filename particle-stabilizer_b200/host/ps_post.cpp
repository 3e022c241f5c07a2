// ps_post.cpp — the steps after the path that the reference CLI runs on the
// result (src/App/ParticleStabilizerMain.cpp:274-296):
//
//   ps_resolve_overlaps    ParticleModel::resolveOverlaps
//                          (src/ParticleStabilizer/ParticleModel.cpp:154-259)
//   ps_overlap_stats       its closing overlap check (same file, 232-256)
//   ps_write_obj_spheres   ObjData::write (src/ParticleStabilizer/ObjData.cpp:8-140)
//
// resolveOverlaps walks the spheres in ascending order along one axis and
// lifts each onto the first lower-ranked sphere it overlaps; a lift that
// moves the sphere past higher-ranked ones re-sorts that rank range and the
// same rank is processed again.  The reference scans every lower rank from
// the first one whose top reaches the sphere's bottom (O(N^2)); here the
// same decisions are taken with two indexes over the finalised ranks:
//   - a max segment tree of their tops (position + radius, computed as the
//     reference does) gives that first rank exactly, even where a lifted
//     sphere left the finalised ranks out of position order;
//   - a 2-D grid over the other two axes (cells of 2 r_max) gives every
//     sphere that can overlap in 3-D; the rest cannot pass the overlap test.
// Candidates are visited in rank order with the sphere's current position,
// the arithmetic is the reference's operation for operation, and the
// re-sorts are the same std::sort calls on the same ranking array, so the
// result is identical to the reference's.
//
// ObjData::write emits one triangulated unit sphere per particle (vertex
// table of (ndivs-1)(2 ndivs-1) quads, ndivs from the particle count), its
// normals once, then the faces.  The text is formatted here with the same
// float arithmetic and the same "%g" conversion that std::ostream applies,
// in parallel batches of particles written in order, so the file is
// byte-identical.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <limits>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#define _USE_MATH_DEFINES
#include <math.h>

#include "particle_stabilizer_b200.h"

extern "C" int ps_internal_fail(int code, const char* msg);  // ps_last_error() channel (ps_engine.cu)

namespace {

int post_fail(int code, const std::string& m) { return ps_internal_fail(code, m.c_str()); }

inline double P(const double* aos, int64_t i, int a) { return aos[8 * i + a]; }
inline double R(const double* aos, int64_t i) { return aos[8 * i + 6]; }

// Max segment tree over rank positions [0, n): value of a finalised rank is
// its top (position[axis] + radius); others hold -inf.
class TopTree {
 public:
  explicit TopTree(int64_t n) {
    size_ = 1;
    while (size_ < std::max<int64_t>(n, 1)) size_ <<= 1;
    t_.assign(2 * (size_t)size_, -std::numeric_limits<double>::infinity());
  }
  void set(int64_t i, double v) {
    int64_t k = i + size_;
    t_[(size_t)k] = v;
    for (k >>= 1; k >= 1; k >>= 1) t_[(size_t)k] = std::max(t_[(size_t)(2 * k)], t_[(size_t)(2 * k + 1)]);
  }
  // first index j < limit with bottom <= value[j]; limit if none
  int64_t first_at_least(double bottom, int64_t limit) const {
    if (limit <= 0 || !(bottom <= t_[1])) return limit;
    int64_t k = 1;
    while (k < size_) {
      k = bottom <= t_[(size_t)(2 * k)] ? 2 * k : 2 * k + 1;
    }
    const int64_t j = k - size_;
    return j < limit ? j : limit;
  }

 private:
  int64_t size_ = 1;
  std::vector<double> t_;
};

struct Grid2 {
  double cell = 1.0;
  int a0 = 0, a1 = 1;
  std::unordered_map<uint64_t, std::vector<std::pair<int64_t, int64_t>>> cells;  // (rank, particle), rank ascending

  static uint64_t key(int64_t x, int64_t y) { return ((uint64_t)(uint32_t)(int32_t)x << 32) | (uint32_t)(int32_t)y; }
  int64_t coord(double v) const { return (int64_t)std::floor(v / cell); }
  void insert(const double* aos, int64_t p, int64_t rank) {
    cells[key(coord(P(aos, p, a0)), coord(P(aos, p, a1)))].emplace_back(rank, p);
  }
};

}  // namespace

extern "C" int ps_overlap_stats(const double* aos, int64_t n, int64_t* n_collided, double* max_overlap) {
  if ((aos == nullptr && n > 0) || n < 0 || n_collided == nullptr || max_overlap == nullptr)
    return post_fail(PS_ERR_INVALID, "ps_overlap_stats: bad argument");
  double r_max = 0.0;
  for (int64_t i = 0; i < n; ++i) r_max = std::max(r_max, R(aos, i));
  // 3-D grid with cells of at least 2 r_max: every overlapping pair is in
  // neighbouring cells
  const double cell = r_max > 0.0 ? 2.0 * r_max * (1.0 + 1e-9) : 1.0;
  std::unordered_map<uint64_t, std::vector<int64_t>> grid;
  auto cc = [&](double v) { return (int64_t)std::floor(v / cell); };
  auto key = [](int64_t x, int64_t y, int64_t z) {
    return ((uint64_t)(x & 0x1fffff) << 42) | ((uint64_t)(y & 0x1fffff) << 21) | (uint64_t)(z & 0x1fffff);
  };
  // a particle with a non-finite coordinate overlaps nothing (its distances
  // are NaN or infinite), so it is left out
  auto finite = [&](int64_t i) {
    return std::isfinite(P(aos, i, 0)) && std::isfinite(P(aos, i, 1)) && std::isfinite(P(aos, i, 2));
  };
  for (int64_t i = 0; i < n; ++i)
    if (finite(i)) grid[key(cc(P(aos, i, 0)), cc(P(aos, i, 1)), cc(P(aos, i, 2)))].push_back(i);
  int64_t collided = 0;
  double max_d = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    if (!finite(i)) continue;
    bool hit = false;
    const int64_t x = cc(P(aos, i, 0)), y = cc(P(aos, i, 1)), z = cc(P(aos, i, 2));
    for (int64_t dx = -1; dx <= 1; ++dx)
      for (int64_t dy = -1; dy <= 1; ++dy)
        for (int64_t dz = -1; dz <= 1; ++dz) {
          auto it = grid.find(key(x + dx, y + dy, z + dz));
          if (it == grid.end()) continue;
          for (int64_t j : it->second) {
            if (j <= i) continue;  // the reference pairs i with every higher index
            // ParticleModel.cpp:240-245, glm::dot = (x*x + y*y) + z*z
            const double ddx = P(aos, i, 0) - P(aos, j, 0), ddy = P(aos, i, 1) - P(aos, j, 1),
                         ddz = P(aos, i, 2) - P(aos, j, 2);
            const double distance = std::sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
            const double cd = R(aos, i) + R(aos, j) - distance;
            if (cd > 0.0) {
              hit = true;
              max_d = std::max(max_d, cd);
            }
          }
        }
    if (hit) ++collided;
  }
  *n_collided = collided;
  *max_overlap = max_d;
  return PS_OK;
}

extern "C" int ps_resolve_overlaps(double* aos, int64_t n, int32_t axis, int64_t* n_collided, double* max_overlap) {
  if ((aos == nullptr && n > 0) || n < 0 || axis < 0 || axis > 2)
    return post_fail(PS_ERR_INVALID, "ps_resolve_overlaps: bad argument (axis must be 0, 1 or 2)");
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(P(aos, i, a))) return post_fail(PS_ERR_INVALID, "ps_resolve_overlaps: non-finite position");
  int oth[2], k2 = 0;
  for (int a = 0; a < 3; ++a)
    if (a != axis) oth[k2++] = a;
  auto pos = [&](int64_t p) -> double& { return aos[8 * p + axis]; };
  auto less = [&](int64_t i1, int64_t i2) { return pos(i1) < pos(i2); };

  std::vector<int64_t> rank((size_t)n);
  std::iota(rank.begin(), rank.end(), (int64_t)0);
  std::sort(rank.begin(), rank.end(), less);

  double r_max = 0.0;
  for (int64_t i = 0; i < n; ++i) r_max = std::max(r_max, R(aos, i));
  Grid2 grid;
  grid.cell = r_max > 0.0 ? 2.0 * r_max * (1.0 + 1e-9) : 1.0;
  grid.a0 = oth[0];
  grid.a1 = oth[1];
  TopTree tops(n);
  std::vector<std::pair<int64_t, int64_t>> cand;

  for (int64_t i = 0; i < n; ++i) {
    const int64_t ip = rank[(size_t)i];
    // minRank (ParticleModel.cpp:177-184): first lower rank whose top reaches
    // ip's bottom; 0 when there is none, and the reference then scans them all
    int64_t min_rank = tops.first_at_least(pos(ip) - R(aos, ip), i);
    if (min_rank == i) min_rank = 0;
    cand.clear();
    const int64_t gx = grid.coord(P(aos, ip, oth[0])), gy = grid.coord(P(aos, ip, oth[1]));
    for (int64_t dx = -1; dx <= 1; ++dx)
      for (int64_t dy = -1; dy <= 1; ++dy) {
        auto it = grid.cells.find(Grid2::key(gx + dx, gy + dy));
        if (it == grid.cells.end()) continue;
        const auto& v = it->second;
        auto first = std::lower_bound(v.begin(), v.end(), std::make_pair(min_rank, (int64_t)-1));
        cand.insert(cand.end(), first, v.end());
      }
    std::sort(cand.begin(), cand.end());
    bool again = false;
    for (const auto& rc : cand) {  // ParticleModel.cpp:186-229, in rank order
      const int64_t jp = rc.second;
      const double sumRadius = R(aos, ip) + R(aos, jp);
      const double sumRadiusSquared = sumRadius * sumRadius;
      const double deltaX = P(aos, ip, 0) - P(aos, jp, 0);
      const double deltaY = P(aos, ip, 1) - P(aos, jp, 1);
      const double deltaZ = P(aos, ip, 2) - P(aos, jp, 2);
      const double distanceSquared = deltaX * deltaX + deltaY * deltaY + deltaZ * deltaZ;
      if (!(sumRadiusSquared - distanceSquared > 0.0)) continue;
      const double delta0 = P(aos, ip, oth[0]) - P(aos, jp, oth[0]);
      const double delta1 = P(aos, ip, oth[1]) - P(aos, jp, oth[1]);
      pos(ip) = pos(jp) + std::sqrt(sumRadius * sumRadius - delta0 * delta0 - delta1 * delta1);
      // maxRankChanged (ParticleModel.cpp:209-217): first k > i with
      // pos[rank[k-1]] < pos(ip) < pos[rank[k]]; ranks above i are sorted
      const double p = pos(ip);
      auto kit = std::upper_bound(rank.begin() + i + 1, rank.end(), p,
                                  [&](double v, int64_t q) { return v < pos(q); });
      int64_t max_changed = i;
      const int64_t kk = (int64_t)(kit - rank.begin());
      if (kk < n && kk >= i + 2 && pos(rank[(size_t)(kk - 1)]) < p) max_changed = kk;
      if (max_changed != i) {
        std::sort(rank.begin() + i, rank.begin() + max_changed + 1, less);
        again = true;  // the reference's --i: process rank i again
        break;
      }
    }
    if (again) {
      --i;
      continue;
    }
    tops.set(i, pos(ip) + R(aos, ip));
    grid.insert(aos, ip, i);
  }
  if (n_collided != nullptr && max_overlap != nullptr) return ps_overlap_stats(aos, n, n_collided, max_overlap);
  return PS_OK;
}

extern "C" int ps_write_obj_spheres(const char* path, const double* aos, int64_t n) {
  if (path == nullptr || (aos == nullptr && n > 0) || n < 0) return post_fail(PS_ERR_INVALID, "ps_write_obj_spheres: bad argument");
  namespace fs = std::filesystem;
  std::error_code ec;
  const fs::path dir = fs::absolute(fs::path(path)).parent_path();
  if (!fs::exists(dir)) fs::create_directories(dir, ec);

  // unit sphere (ObjData.cpp:20-76), float arithmetic as the reference's
  const size_t nParticles = (size_t)n;
  const size_t MAX_NUM_VERTICES = 1000000;
  int ndivs = (int)sqrt((double)MAX_NUM_VERTICES / (6.0 + (double)nParticles)) + 1;
  ndivs = std::max(ndivs, 6);
  std::vector<std::array<float, 3>> vertices;
  size_t nFaces = 0;
  {
    const int nDivsTheta = ndivs;
    const int nDivsPhi = 2 * ndivs;
    const float deltaTheta = M_PI / (float)(nDivsTheta - 1);
    const float deltaPhi = 2 * M_PI / (float)(nDivsPhi - 1);
    for (int iTheta = 0; iTheta < nDivsTheta - 1; ++iTheta)
      for (int iPhi = 0; iPhi < nDivsPhi - 1; ++iPhi) {
        const float theta = (float)iTheta * deltaTheta;
        const float thetaNext = theta + deltaTheta;
        const float phi = (float)iPhi * deltaPhi;
        const float phiNext = phi + deltaPhi;
        const std::array<float, 3> p0 = {std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi),
                                         std::cos(theta)};
        const std::array<float, 3> p1 = {std::sin(thetaNext) * std::cos(phi), std::sin(thetaNext) * std::sin(phi),
                                         std::cos(thetaNext)};
        const std::array<float, 3> p2 = {std::sin(thetaNext) * std::cos(phiNext),
                                         std::sin(thetaNext) * std::sin(phiNext), std::cos(thetaNext)};
        const std::array<float, 3> p3 = {std::sin(theta) * std::cos(phiNext), std::sin(theta) * std::sin(phiNext),
                                         std::cos(theta)};
        vertices.push_back(p0);
        vertices.push_back(p1);
        vertices.push_back(p2);
        ++nFaces;
        vertices.push_back(p2);
        vertices.push_back(p3);
        vertices.push_back(p0);
        ++nFaces;
      }
  }
  std::FILE* f = std::fopen(path, "wb");
  if (f == nullptr) return post_fail(PS_ERR_IO, std::string("ps_write_obj_spheres: cannot open ") + path);
  std::fputs("o Generated particles\n", f);

  const unsigned n_threads = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const size_t batch = std::max<size_t>(1, (size_t)4 * 1024 * 1024 / std::max<size_t>(1, 3 * nFaces));  // ~ 4M lines
  std::vector<std::string> out(n_threads);
  auto emit = [&](auto&& format_one) {  // particles in batches, formatted in parallel, written in order
    for (size_t b0 = 0; b0 < nParticles; b0 += batch) {
      const size_t b1 = std::min(nParticles, b0 + batch);
      std::vector<std::thread> th;
      for (unsigned t = 0; t < n_threads; ++t)
        th.emplace_back([&, t] {
          std::string& s = out[t];
          s.clear();
          const size_t per = (b1 - b0 + n_threads - 1) / n_threads;
          const size_t lo = b0 + t * per, hi = std::min(b1, lo + per);
          for (size_t i = lo; i < hi; ++i) format_one(s, i);
        });
      for (auto& x : th) x.join();
      for (unsigned t = 0; t < n_threads; ++t) std::fwrite(out[t].data(), 1, out[t].size(), f);
    }
  };
  // 'v' (ObjData.cpp:84-101): float centre and radius, ostream's default
  // conversion of a float is %g of its value
  emit([&](std::string& s, size_t i) {
    char buf[160];
    const float cx = (float)aos[8 * i + 0], cy = (float)aos[8 * i + 1], cz = (float)aos[8 * i + 2];
    const float r = (float)aos[8 * i + 6];
    for (size_t v = 0; v < 3 * nFaces; ++v) {
      const float x = r * vertices[v][0] + cx, y = r * vertices[v][1] + cy, z = r * vertices[v][2] + cz;
      const int m = std::snprintf(buf, sizeof(buf), "v %g %g %g\n", (double)x, (double)y, (double)z);
      s.append(buf, (size_t)m);
    }
  });
  // 'vn' (ObjData.cpp:103-113): normals equal the unit-sphere vertices
  {
    char buf[160];
    std::string s;
    for (size_t v = 0; v < 3 * nFaces; ++v) {
      const int m = std::snprintf(buf, sizeof(buf), "vn %g %g %g\n", (double)vertices[v][0], (double)vertices[v][1],
                                  (double)vertices[v][2]);
      s.append(buf, (size_t)m);
    }
    std::fwrite(s.data(), 1, s.size(), f);
  }
  // 'f' (ObjData.cpp:115-131)
  emit([&](std::string& s, size_t i) {
    char buf[160];
    const size_t particleOffset = i * nFaces * 3;
    for (size_t iFace = 0; iFace < nFaces; ++iFace) {
      const size_t faceOffset = 3 * iFace, offset = particleOffset + faceOffset;
      const int m = std::snprintf(buf, sizeof(buf), "f %zu//%zu %zu//%zu %zu//%zu\n", offset + 1, faceOffset + 1,
                                  offset + 2, faceOffset + 2, offset + 3, faceOffset + 3);
      s.append(buf, (size_t)m);
    }
  });
  const bool ok = std::fflush(f) == 0;
  std::fclose(f);
  if (!ok) return post_fail(PS_ERR_IO, std::string("ps_write_obj_spheres: write failed for ") + path);
  return PS_OK;
}
