// ps_io.cpp — the file formats on either side of the DEM path.
//
//   CSV particles  ParticleData::readFromCSV / writeAsCSV
//                  (src/ParticleStabilizer/ParticleIO.cpp:39-144)
//   OBJ container  PolygonContainerCUDA::readFromFile + de-indexing
//                  (src/ParticleStabilizerCUDA/PolygonContainerCUDA.cpp:26-53, 314-350)
//   state file     binary checkpoint / resume (every record and the step
//                  count; no counterpart in the reference)
//
// Differences from the reference, by design: a malformed number makes the
// reader return PS_ERR_IO (std::stod would throw and abort the reference),
// and the OBJ reader is a self-contained triangle/polygon reader instead of
// assimp (n-gons are fanned from their first vertex).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "particle_stabilizer_b200.h"

// defined in ps_engine.cu: records the message returned by ps_last_error()
extern "C" int ps_internal_fail(int code, const char* msg);

namespace {
int io_fail(const std::string& m) { return ps_internal_fail(PS_ERR_IO, m.c_str()); }

// splitText (ParticleIO.cpp:8-19): tokens between delimiters, empty tokens
// and the literal "null" dropped.
std::vector<std::string> split_tokens(const std::string& s, char delim) {
  std::vector<std::string> out;
  std::stringstream ss(s);
  std::string item;
  while (std::getline(ss, item, delim))
    if (!item.empty() && item != "null") out.push_back(item);
  return out;
}

// std::stod semantics: leading whitespace, then a number; trailing text ignored.
bool parse_double(const std::string& s, double* v) {
  const char* b = s.c_str();
  char* e = nullptr;
  errno = 0;
  *v = std::strtod(b, &e);
  return e != b && errno != ERANGE;
}

// ParticleData::format(double, nChars) (ParticleIO.cpp:39-56): fixed
// notation with nChars - len(int part) - 1 decimals.
std::string fixed_field(double value, int n_chars) {
  int int_len = (int)std::to_string((int)std::fabs(value)).size();
  if (value < 0) int_len += 1;
  int decimals = n_chars - int_len - 1;
  if (decimals < 0) decimals = 0;
  char buf[128];
  std::snprintf(buf, sizeof(buf), "%.*f", decimals, value);
  return buf;
}
}  // namespace

extern "C" int ps_read_csv(const char* path, const double velocity[3], double density, double* aos_out, int64_t cap,
                           int64_t* n_out) {
  if (path == nullptr || velocity == nullptr || n_out == nullptr) return io_fail("ps_read_csv: null argument");
  std::ifstream file(path);
  if (!file.is_open()) return io_fail(std::string("Could not open file: ") + path);
  std::string line;
  std::getline(file, line);  // header
  int64_t n = 0;
  while (std::getline(file, line)) {
    const std::vector<std::string> tok = split_tokens(line, ',');
    if (tok.size() != 4) continue;  // "Invalid line" (ParticleIO.cpp:121-124)
    double v[4];
    for (int k = 0; k < 4; ++k)
      if (!parse_double(tok[k], &v[k])) return io_fail("ps_read_csv: bad number in line: " + line);
    if (aos_out != nullptr && n < cap) {
      double* q = aos_out + 8 * n;
      q[0] = v[0];
      q[1] = v[1];
      q[2] = v[2];
      q[3] = velocity[0];
      q[4] = velocity[1];
      q[5] = velocity[2];
      q[6] = v[3];
      q[7] = density * 4.0 / 3.0 * M_PI * std::pow(v[3], 3);  // ParticleIO.cpp:131
    }
    ++n;
  }
  *n_out = n;
  return PS_OK;
}

extern "C" int ps_write_csv(const char* path, const double* aos, int64_t n) {
  if (path == nullptr || (aos == nullptr && n > 0)) return io_fail("ps_write_csv: null argument");
  std::error_code ec;
  const std::filesystem::path dir = std::filesystem::absolute(path).parent_path();
  if (!std::filesystem::exists(dir)) std::filesystem::create_directories(dir, ec);
  std::ofstream file(path);
  if (!file) return io_fail(std::string("Could not open file ") + path);
  file << "x,y,z,radius\n";
  for (int64_t i = 0; i < n; ++i) {
    const double* q = aos + 8 * i;
    file << fixed_field(q[0], 10) << "," << fixed_field(q[1], 10) << "," << fixed_field(q[2], 10) << ","
         << fixed_field(q[6], 10) << "\n";
  }
  file.close();
  return file ? PS_OK : io_fail(std::string("write failed: ") + path);
}

namespace {
constexpr char kStateMagic[8] = {'P', 'S', 'B', '2', 'S', 'T', 'A', 'T'};
constexpr uint32_t kStateVersion = 1;
}  // namespace

extern "C" int ps_write_state_bin(const char* path, const double* aos, int64_t n, int64_t steps) {
  if (path == nullptr || (aos == nullptr && n > 0) || n < 0 || steps < 0)
    return io_fail("ps_write_state_bin: bad argument");
  std::error_code ec;
  const std::filesystem::path dir = std::filesystem::absolute(path).parent_path();
  if (!std::filesystem::exists(dir)) std::filesystem::create_directories(dir, ec);
  std::ofstream file(path, std::ios::binary);
  if (!file) return io_fail(std::string("Could not open file ") + path);
  const uint32_t version = kStateVersion, zero = 0;
  file.write(kStateMagic, sizeof kStateMagic);
  file.write(reinterpret_cast<const char*>(&version), sizeof version);
  file.write(reinterpret_cast<const char*>(&zero), sizeof zero);
  file.write(reinterpret_cast<const char*>(&n), sizeof n);
  file.write(reinterpret_cast<const char*>(&steps), sizeof steps);
  if (n > 0) file.write(reinterpret_cast<const char*>(aos), (std::streamsize)(8 * sizeof(double) * (size_t)n));
  file.close();
  return file ? PS_OK : io_fail(std::string("write failed: ") + path);
}

extern "C" int ps_read_state_bin(const char* path, double* aos_out, int64_t cap, int64_t* n_out, int64_t* steps_out) {
  if (path == nullptr || n_out == nullptr || cap < 0) return io_fail("ps_read_state_bin: bad argument");
  std::ifstream file(path, std::ios::binary);
  if (!file.is_open()) return io_fail(std::string("Could not open file: ") + path);
  char magic[8];
  uint32_t version = 0, zero = 0;
  int64_t n = -1, steps = -1;
  file.read(magic, sizeof magic);
  file.read(reinterpret_cast<char*>(&version), sizeof version);
  file.read(reinterpret_cast<char*>(&zero), sizeof zero);
  file.read(reinterpret_cast<char*>(&n), sizeof n);
  file.read(reinterpret_cast<char*>(&steps), sizeof steps);
  if (!file || std::memcmp(magic, kStateMagic, sizeof magic) != 0 || version != kStateVersion || n < 0 || steps < 0)
    return io_fail(std::string("ps_read_state_bin: not a state file (version 1): ") + path);
  file.seekg(0, std::ios::end);
  const std::streamoff payload = file.tellg() - (std::streamoff)(sizeof magic + 2 * sizeof(uint32_t) + 2 * sizeof(int64_t));
  if (payload != (std::streamoff)(8 * sizeof(double)) * n)
    return io_fail(std::string("ps_read_state_bin: truncated or oversized file: ") + path);
  if (aos_out != nullptr && cap > 0 && n > 0) {
    file.seekg((std::streamoff)(sizeof magic + 2 * sizeof(uint32_t) + 2 * sizeof(int64_t)), std::ios::beg);
    const int64_t m = std::min(n, cap);
    file.read(reinterpret_cast<char*>(aos_out), (std::streamsize)(8 * sizeof(double) * (size_t)m));
    if (!file) return io_fail(std::string("ps_read_state_bin: read failed: ") + path);
  }
  *n_out = n;
  if (steps_out != nullptr) *steps_out = steps;
  return PS_OK;
}

extern "C" int ps_read_obj(const char* path, double* tri_out, int64_t cap, int64_t* n_tri_out) {
  if (path == nullptr || n_tri_out == nullptr) return io_fail("ps_read_obj: null argument");
  std::ifstream in(path);
  if (!in.is_open()) return io_fail(std::string("Unable to open file \"") + path + "\".");
  std::vector<float> verts;
  int64_t nt = 0;
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string tag;
    ss >> tag;
    if (tag == "v") {
      std::string a, b, c;
      ss >> a >> b >> c;
      // single precision, as assimp's default ai_real
      verts.push_back(std::strtof(a.c_str(), nullptr));
      verts.push_back(std::strtof(b.c_str(), nullptr));
      verts.push_back(std::strtof(c.c_str(), nullptr));
    } else if (tag == "f") {
      std::vector<long> ids;
      std::string t;
      const long nv = (long)(verts.size() / 3);
      while (ss >> t) {
        const long k = std::strtol(t.substr(0, t.find('/')).c_str(), nullptr, 10);
        const long id = k < 0 ? nv + k : k - 1;
        if (id < 0 || id >= nv) return io_fail("ps_read_obj: face index out of range in line: " + line);
        ids.push_back(id);
      }
      for (size_t k = 1; k + 1 < ids.size(); ++k) {
        if (tri_out != nullptr && nt < cap) {
          const long c3[3] = {ids[0], ids[k], ids[k + 1]};
          for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a) tri_out[9 * nt + 3 * c + a] = (double)verts[3 * c3[c] + a];
        }
        ++nt;
      }
    }
  }
  *n_tri_out = nt;
  return PS_OK;
}
