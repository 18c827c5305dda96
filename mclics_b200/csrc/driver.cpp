// Whole-program driver behind mcl_run_input_file: reads a McLics input file, sets up the lattice and runs one of
// the *GPU evolution modes on this library's engine, writing the reference program's outputs.
//
// Behaviour kept from the reference, because it is the interface a user's files and scripts depend on:
//   input keys, aliases and defaults    src/io.cpp:135-310, include/parameters.h:18-98
//   derived flags                       src/main.cpp:86-107
//   validation and its messages         src/io.cpp:381-475 (all errors collected; nothing written on error)
//   geometries, anchoring, ICs          src/geometry_{bulk,slab,sphere,custom}.cpp, src/geometry.cpp:78-107,
//                                       src/ic.cpp
//   GHRL coefficients                   src/io.cpp:346-371
//   po.dat columns, snapshot names      src/evolve_{thermal,step,quench,electric}.cu, include/sweep.h
//   snapshot / ic.csv format            src/io.cpp:59-89, src/parameter_order.cpp:75-127
//   extra po.dat columns                src/parameter_order.cpp:129-295
// The structure is this driver's own: keys are a table (name, aliases, value kind, destination), validation is a
// list of rules, each geometry is a per-site classifier, and the four modes are one loop over a list of scan
// points. `ic random` runs on the device (mcl_random_directors). Errors come back as MCL_ERR_INPUT / MCL_ERR_IO
// with the message on stderr; the process is never terminated here.
#include <dirent.h>
#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include <algorithm>
#include <fstream>
#include <functional>
#include <map>
#include <sstream>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>

#include "eigen3.cuh"
#include "engine.h"

namespace {

using mcl::fail;

struct InputError {
  int code;
};

std::string fmt(const char *f, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, f);
  vsnprintf(buf, sizeof buf, f, ap);
  va_end(ap);
  return buf;
}

// Reports one input error ("  [ERROR] ..." on stderr, the library's last-error message) and abandons the run.
[[noreturn]] void reject(int code, const std::string &msg) {
  fprintf(stderr, "  [ERROR] %s\n", msg.c_str());
  fail(code, "%s", msg.c_str());
  throw InputError{code};
}

bool same(const std::string &a, const char *b) { return strcasecmp(a.c_str(), b) == 0; }

// ---- run parameters (the reference's keys and their defaults) ----------------------------------------------------
struct Params {
  std::string geometry = "bulk", xbound = "free", ybound = "free", zbound = "free", boundary_file;
  std::map<int, float> theta_s, phi_s, W;
  std::map<int, std::string> anchoring;
  std::string potential = "ll", evol = "thermal", ic = "random", ic_file, radial;
  int Nx = 16, Ny = 16, Nz = 16;
  float A = 1.0f, B1 = 0.04f, C = 0.3f;
  float Ti = 1.2f, Tf = 0.0f, dT = -0.02f;
  int MCS = 100, MCT = 100, MCQ = -1, fn = 1, first_file = 0, seed = 1;
  float phi_0 = 0, theta_0 = 0, p0_i = 0;
  float k11 = 1, k22 = 1, k33 = 1, p0 = 0;
  float elecX = 0, elecY = 0, elecZ = 0, elecA = 0, elecP = 0;
  float Ei = 0, Ef = 0, dE = 0;
  // derived
  int flip = 0;
  std::string mode;  // evol without its GPU suffix
};

// ---- input-file keys ----------------------------------------------------------------------------------------
// One entry per key: its names (the first is the canonical one), where the value goes, and for words the longest
// value the reference's fixed-size fields accept.
using Slot = std::variant<int *, float *, std::string *, std::map<int, std::string> *, std::map<int, float> *>;
struct Key {
  std::vector<const char *> names;
  Slot slot;
  size_t max_len = 0;  // words only
};

std::vector<Key> key_table(Params &p) {
  return {
      {{"nx"}, &p.Nx},
      {{"ny"}, &p.Ny},
      {{"nz"}, &p.Nz},
      {{"A"}, &p.A},
      {{"B1"}, &p.B1},
      {{"C"}, &p.C},
      {{"Ti"}, &p.Ti},
      {{"Tf"}, &p.Tf},
      {{"dT"}, &p.dT},
      {{"MCS"}, &p.MCS},
      {{"MCT"}, &p.MCT},
      {{"MCQ", "quench_steps"}, &p.MCQ},
      {{"seed"}, &p.seed},
      {{"fn"}, &p.fn},
      {{"first_file_number", "initial_output"}, &p.first_file},
      {{"k11"}, &p.k11},
      {{"k22"}, &p.k22},
      {{"k33"}, &p.k33},
      {{"p0"}, &p.p0},
      {{"phi_0"}, &p.phi_0},
      {{"theta_0"}, &p.theta_0},
      {{"p0_i"}, &p.p0_i},
      {{"elecX", "Electric_field_x", "EF_x"}, &p.elecX},
      {{"elecY", "Electric_field_y", "EF_y"}, &p.elecY},
      {{"elecZ", "Electric_field_z", "EF_z"}, &p.elecZ},
      {{"Ei", "initial_E"}, &p.Ei},
      {{"Ef", "final_E"}, &p.Ef},
      {{"dE", "E_variation"}, &p.dE},
      {{"elecA", "dielectric_anisotropy", "Aniso_E"}, &p.elecA},
      {{"elecP", "dipolar_coupling", "Polar_E"}, &p.elecP},
      {{"ic"}, &p.ic, 49},
      {{"ic_file"}, &p.ic_file, 1023},
      {{"xbound"}, &p.xbound, 19},
      {{"ybound"}, &p.ybound, 19},
      {{"zbound"}, &p.zbound, 19},
      {{"potential"}, &p.potential, 19},
      {{"evol", "mode"}, &p.evol, 19},
      {{"geometry"}, &p.geometry, 19},
      {{"boundary_file"}, &p.boundary_file, 1023},
      {{"radial"}, &p.radial, 19},
      {{"anchoring_type"}, &p.anchoring},
      {{"W"}, &p.W},
      {{"phi_s"}, &p.phi_s},
      {{"theta_s"}, &p.theta_s},
  };
}

// Numeric prefix of a token (stream-extraction semantics: "16.5" as an int is 16 with ".5" left over); false when
// the token does not start with a number. `rest` receives what follows the number.
bool parse_number(const std::string &tok, int &v, std::string &rest) {
  char *end = nullptr;
  errno = 0;
  const long x = strtol(tok.c_str(), &end, 10);
  if (end == tok.c_str() || errno || x < INT32_MIN || x > INT32_MAX) return false;
  v = (int)x;
  rest = end;
  return true;
}
bool parse_number(const std::string &tok, float &v, std::string &rest) {
  char *end = nullptr;
  const float x = strtof(tok.c_str(), &end);
  if (end == tok.c_str() || !isfinite(x)) return false;
  v = x;
  rest = end;
  return true;
}

// Reads one key's values from the tokens after it on its line; returns the unread text.
std::string read_values(const Key &k, const std::string &name, std::vector<std::string> &toks, size_t &at) {
  auto next = [&]() -> const std::string & {
    if (at >= toks.size()) reject(MCL_ERR_INPUT, fmt("Invalid value for parameter: %s", name.c_str()));
    return toks[at++];
  };
  auto number = [&](auto &dst) {
    std::string rest;
    if (!parse_number(next(), dst, rest)) reject(MCL_ERR_INPUT, fmt("Invalid value for parameter: %s", name.c_str()));
    return rest;
  };
  std::string rest;
  std::visit(
      [&](auto *dst) {
        using T = std::remove_pointer_t<decltype(dst)>;
        if constexpr (std::is_same_v<T, int> || std::is_same_v<T, float>) {
          rest = number(*dst);
        } else if constexpr (std::is_same_v<T, std::string>) {
          const std::string &w = next();
          if (w.size() > k.max_len)
            reject(MCL_ERR_INPUT, fmt("Value of '%s' is too long (%zu characters, maximum %zu): %.60s...", name.c_str(),
                                      w.size(), k.max_len, w.c_str()));
          *dst = w;
        } else {  // surface-indexed value: "<key> <surface> <value>"
          int sid = 0;
          std::string r1 = number(sid);
          if (!r1.empty()) reject(MCL_ERR_INPUT, fmt("Invalid value for parameter: %s", name.c_str()));
          if constexpr (std::is_same_v<T, std::map<int, float>>) {
            float v = 0;
            rest = number(v);
            (*dst)[sid] = v;
          } else {
            (*dst)[sid] = next();
          }
        }
      },
      k.slot);
  return rest;
}

Params read_input(const char *path) {
  Params p;
  std::ifstream in(path);
  if (!in) {
    perror(path);
    fail(MCL_ERR_IO, "cannot open input file %s", path);
    throw InputError{MCL_ERR_IO};
  }
  const std::vector<Key> keys = key_table(p);
  std::map<std::string, const Key *> by_name;  // lower-case name -> key
  for (const Key &k : keys)
    for (const char *n : k.names) {
      std::string l(n);
      for (char &c : l) c = (char)tolower((unsigned char)c);
      by_name[l] = &k;
    }
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::vector<std::string> toks;
    for (std::string t; ls >> t;) toks.push_back(t);
    if (toks.empty() || toks[0][0] == '#') continue;
    const std::string &name = toks[0];
    if (name.size() >= 200) reject(MCL_ERR_INPUT, fmt("Parameter name too long: %.60s...", name.c_str()));
    std::string lname(name);
    for (char &c : lname) c = (char)tolower((unsigned char)c);
    auto hit = by_name.find(lname);
    if (hit == by_name.end()) reject(MCL_ERR_INPUT, fmt("Unknown parameter: '%s'", name.c_str()));
    size_t at = 1;
    std::string extra = read_values(*hit->second, name, toks, at);
    for (; at < toks.size(); at++) extra += (extra.empty() ? "" : " ") + toks[at];
    if (!extra.empty() && extra[0] != '#')
      fprintf(stderr, "  [WARNING] Ignoring extra text after parameter '%s': %s\n", name.c_str(), extra.c_str());
    if (hit->second->slot == Slot(&p.MCQ) && p.MCQ < 0)
      reject(MCL_ERR_INPUT, fmt("MCQ (quench_steps) must be >= 0 (got %d)", p.MCQ));
  }
  return p;
}

// ---- derived values and validation ------------------------------------------------------------------------------
bool is_ghrl(const Params &p) { return same(p.potential, "ghrl") || same(p.potential, "gruhn-hess"); }

void derive(Params &p) {
  p.mode = p.evol;
  if (p.mode.size() > 3 && same(p.mode.substr(p.mode.size() - 3), "GPU")) p.mode.resize(p.mode.size() - 3);
  p.flip = (same(p.potential, "pear") || p.elecP != 0) ? 1 : 0;
  if (p.MCQ < 0) p.MCQ = p.MCT;
  if (p.radial.empty()) p.radial = same(p.geometry, "sphere") ? "sphere" : "none";
  static const char *kRadial[] = {"sphere", "cylinder", "both", "none"};
  bool ok = false;
  for (const char *r : kRadial) ok = ok || same(p.radial, r);
  if (!ok) reject(MCL_ERR_INPUT, fmt("radial must be sphere, cylinder, both or none (got '%s')", p.radial.c_str()));
  if (p.elecA != 0 || p.elecP != 0) {
    const float len = sqrtf(p.elecX * p.elecX + p.elecY * p.elecY + p.elecZ * p.elecZ);
    if (len == 0) reject(MCL_ERR_INPUT, "elecA or elecP is set but the field direction (elecX, elecY, elecZ) is zero");
    p.elecX /= len;
    p.elecY /= len;
    p.elecZ /= len;
  }
}

// A rule: when it applies, what makes the input invalid, and the message that says so.
struct Rule {
  bool (*applies)(const Params &);
  bool (*violated)(const Params &);
  std::string (*message)(const Params &);
};

bool always(const Params &) { return true; }
bool thermal_or_quench(const Params &p) { return same(p.mode, "thermal") || same(p.mode, "quench"); }

const Rule kRules[] = {
    {always, [](const Params &p) { return p.Nx < 1 || p.Ny < 1 || p.Nz < 1; },
     [](const Params &p) { return fmt("Grid sizes must be >= 1 (got %d x %d x %d).", p.Nx, p.Ny, p.Nz); }},
    {always, [](const Params &p) { return p.MCS < 1; },
     [](const Params &p) { return fmt("MCS must be >= 1 (got %d): averages are taken over the MCS steps.", p.MCS); }},
    {always, [](const Params &p) { return p.MCT < 0; },
     [](const Params &p) { return fmt("MCT must be >= 0 (got %d).", p.MCT); }},
    {[](const Params &p) { return same(p.mode, "step") || same(p.mode, "quench"); },
     [](const Params &p) { return p.fn < 1; },
     [](const Params &p) { return fmt("fn must be >= 1 in %s mode (got %d).", p.mode.c_str(), p.fn); }},
    {always, [](const Params &p) { return p.Ti < 0; },
     [](const Params &p) { return fmt("Ti must be >= 0 (got %g).", p.Ti); }},
    {thermal_or_quench, [](const Params &p) { return p.Tf < 0; },
     [](const Params &p) { return fmt("Tf must be >= 0 (got %g).", p.Tf); }},
    {[](const Params &p) { return same(p.mode, "thermal"); }, [](const Params &p) { return p.dT == 0; },
     [](const Params &) { return std::string("dT must be nonzero in thermal mode."); }},
    {[](const Params &p) { return same(p.mode, "thermal") && p.dT != 0; },
     [](const Params &p) { return (p.Tf - p.Ti) * p.dT < 0; },
     [](const Params &p) {
       return fmt("dT = %g does not lead from Ti = %g to Tf = %g (use dT < 0 to cool, dT > 0 to heat).", p.dT, p.Ti,
                  p.Tf);
     }},
    {[](const Params &p) { return same(p.mode, "electric"); }, [](const Params &p) { return p.dE == 0; },
     [](const Params &) { return std::string("dE must be nonzero in electric mode."); }},
    {[](const Params &p) { return same(p.mode, "electric") && p.dE != 0; },
     [](const Params &p) { return (p.Ef - p.Ei) * p.dE < 0; },
     [](const Params &p) { return fmt("dE = %g does not lead from Ei = %g to Ef = %g.", p.dE, p.Ei, p.Ef); }},
    {is_ghrl, [](const Params &p) { return p.k11 <= 0 || p.k22 <= 0 || p.k33 <= 0; },
     [](const Params &p) { return fmt("k11, k22 and k33 must be > 0 (got %g, %g, %g).", p.k11, p.k22, p.k33); }},
    {[](const Params &p) { return is_ghrl(p) && p.k11 > 0 && p.k22 > 0 && p.k33 > 0; },
     // nu = (S / 9)(k11 - 3 k22 - k33) must be negative
     [](const Params &p) { return p.k11 - 3 * p.k22 - p.k33 >= -1e-6 * p.k22; },
     [](const Params &p) {
       return fmt("The GHRL potential needs k11 < 3 k22 + k33 (got k11 = %g, k22 = %g, k33 = %g): otherwise its energy "
                  "scale nu is not negative and the pair potential is not nematic.",
                  p.k11, p.k22, p.k33);
     }},
    {[](const Params &p) { return same(p.ic, "cholesteric"); }, [](const Params &p) { return p.p0_i == 0 && p.p0 == 0; },
     [](const Params &) { return std::string("ic cholesteric needs a nonzero pitch: set p0_i (or p0)."); }},
};

void validate(const Params &p) {
  std::vector<std::string> errs;
  for (const Rule &r : kRules)
    if (r.applies(p) && r.violated(p)) errs.push_back(r.message(p));
  if (is_ghrl(p) && p.p0 != 0 && fabs(p.p0) < 2 * M_PI)
    fprintf(stderr,
            "  [WARNING] |p0| = %g < 2 pi: the twist per lattice bond exceeds 90 degrees and the lattice has no\n"
            "            equilibrium helix (sin(phi) = 2 pi / p0 > 1).\n",
            fabs(p.p0));
  if (errs.empty()) return;
  for (auto &s : errs) fprintf(stderr, "  [ERROR] %s\n", s.c_str());
  fprintf(stderr, "  %zu error(s) in the input file. Nothing was run and no file was changed.\n", errs.size());
  fail(MCL_ERR_INPUT, "%s", errs[0].c_str());
  throw InputError{MCL_ERR_INPUT};
}

// ---- lattice set-up -------------------------------------------------------------------------------------------
struct Lattice {
  int nx = 0, ny = 0, nz = 0;
  int geometry = MCL_GEOM_BULK;
  int periodic[3] = {0, 0, 0};
  int n_surfaces = 0;
  std::vector<int> pt;     // 0 empty, 1 bulk, s + 2 surface s
  std::vector<float> nrm;  // outward normals of surface sites
  std::vector<float> ni;   // directors (reference layout)
  mcl_model model;
  bool pear = false, sph = false, cyl = false;
  long long sites() const { return (long long)nx * ny * nz; }
  long long index(int i, int j, int k) const { return i + (long long)nx * (j + (long long)ny * k); }
};

// Point type and outward normal of one site.
struct SiteKind {
  int pt;
  float n[3];
};

// Geometries defined by a formula (src/geometry_{bulk,slab,sphere}.cpp): name, code, surfaces, axes forced free,
// and the per-site classifier.
struct Shape {
  const char *name;
  int code;
  int surfaces;
  bool force_free[3];
  std::function<SiteKind(const Lattice &, int, int, int)> classify;
};

const std::vector<Shape> &shapes() {
  static const std::vector<Shape> s = {
      {"bulk", MCL_GEOM_BULK, 0, {false, false, false},
       [](const Lattice &, int, int, int) { return SiteKind{1, {0, 0, 0}}; }},
      // plates at z = 0 (surface 0, normal -z) and z = nz - 1 (surface 1, normal +z; it wins when nz = 1)
      {"slab", MCL_GEOM_SLAB, 2, {false, false, true},
       [](const Lattice &L, int, int, int k) {
         if (k == L.nz - 1) return SiteKind{3, {0, 0, 1}};
         if (k == 0) return SiteKind{2, {0, 0, -1}};
         return SiteKind{1, {0, 0, 0}};
       }},
      // droplet of radius nz / 2 (integer halves as in the reference), a two-site shell as its surface
      {"sphere", MCL_GEOM_SPHERE, 1, {true, true, true},
       [](const Lattice &L, int i, int j, int k) {
         const float cx = (float)(L.nx / 2), cy = (float)(L.ny / 2), cz = (float)(L.nz / 2);
         const float dx = i - cx, dy = j - cy, dz = k - cz;
         const float r = sqrtf(dx * dx + dy * dy + dz * dz);
         if (r < cz - 1) return SiteKind{1, {0, 0, 0}};
         if (r < cz + 1) return SiteKind{2, {dx / r, dy / r, dz / r}};
         return SiteKind{0, {0, 0, 0}};
       }},
  };
  return s;
}

std::vector<std::string> csv_fields(const std::string &line) {
  std::vector<std::string> out(1);
  for (char c : line) {
    if (c == ',')
      out.emplace_back();
    else
      out.back() += c;
  }
  for (auto &f : out) {
    const size_t a = f.find_first_not_of(" \t\r"), b = f.find_last_not_of(" \t\r");
    f = a == std::string::npos ? "" : f.substr(a, b - a + 1);
  }
  return out;
}

// A CSV file of lattice points (boundary file, initial-condition file): a header naming its columns, then one
// row per point. `each` receives the 1-based line number and the row's values of the required columns; every
// complaint names the file and line.
void read_point_csv(const std::string &file, const std::vector<const char *> &cols,
                    const std::function<void(int, const std::vector<double> &)> &each) {
  std::ifstream in(file);
  if (!in) {
    perror(file.c_str());
    fail(MCL_ERR_IO, "cannot open %s", file.c_str());
    throw InputError{MCL_ERR_IO};
  }
  auto at = [&](int line, const std::string &msg) { reject(MCL_ERR_INPUT, fmt("%s, line %d: %s", file.c_str(), line, msg.c_str())); };
  std::string line;
  if (!std::getline(in, line)) at(1, "empty file (a header line is expected).");
  const std::vector<std::string> head = csv_fields(line);
  std::vector<int> where(cols.size(), -1);
  std::string missing, required;
  for (size_t c = 0; c < cols.size(); c++) {
    for (size_t h = 0; h < head.size(); h++)
      if (same(head[h], cols[c])) where[c] = (int)h;
    if (where[c] < 0) missing += std::string(missing.empty() ? "" : ", ") + cols[c];
    required += std::string(c ? "," : "") + cols[c];
  }
  if (!missing.empty()) at(1, fmt("missing column(s) in the header: %s (required: %s).", missing.c_str(), required.c_str()));
  std::vector<double> v(cols.size());
  for (int ln = 2; std::getline(in, line); ln++) {
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    const std::vector<std::string> f = csv_fields(line);
    if (f.size() != head.size()) at(ln, fmt("%zu fields, but the header has %zu.", f.size(), head.size()));
    for (size_t c = 0; c < cols.size(); c++) {
      const std::string &s = f[where[c]];
      char *end = nullptr;
      v[c] = strtod(s.c_str(), &end);
      if (s.empty() || *end) at(ln, fmt("column %s is not a number: '%s'.", cols[c], s.c_str()));
    }
    each(ln, v);
  }
}

// Lattice point (x, y, z) of a CSV row: integral and inside the grid, listed once.
long long csv_point(const Lattice &L, const std::string &file, int ln, const std::vector<double> &v,
                    std::vector<char> &seen) {
  auto at = [&](const std::string &msg) { reject(MCL_ERR_INPUT, fmt("%s, line %d: %s", file.c_str(), ln, msg.c_str())); };
  const int i = (int)v[0], j = (int)v[1], k = (int)v[2];
  if (v[0] != i || v[1] != j || v[2] != k) at("x, y and z must be integers.");
  if (i < 0 || i >= L.nx || j < 0 || j >= L.ny || k < 0 || k >= L.nz)
    at(fmt("point (%d, %d, %d) outside the %d x %d x %d grid.", i, j, k, L.nx, L.ny, L.nz));
  const long long q = L.index(i, j, k);
  if (seen[q]) at(fmt("point (%d, %d, %d) is listed twice.", i, j, k));
  seen[q] = 1;
  return q;
}

// src/geometry_custom.cpp:70-163: point types and normals from the boundary file; unlisted points are bulk.
void custom_shape(const Params &p, Lattice &L) {
  const std::string &file = p.boundary_file;
  std::vector<char> seen(L.sites(), 0);
  std::fill(L.pt.begin(), L.pt.end(), 1);
  int top = 0, renormalised = 0;
  long long listed = 0;
  read_point_csv(file, {"x", "y", "z", "nx", "ny", "nz", "pt"}, [&](int ln, const std::vector<double> &v) {
    const int type = (int)v[6];
    if (v[6] != type) reject(MCL_ERR_INPUT, fmt("%s, line %d: x, y, z and pt must be integers.", file.c_str(), ln));
    if (type < 0)
      reject(MCL_ERR_INPUT,
             fmt("%s, line %d: negative point type (use 0 empty, 1 bulk, 2+ surface).", file.c_str(), ln));
    const long long q = csv_point(L, file, ln, v, seen);
    listed++;
    double n[3] = {v[3], v[4], v[5]};
    const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (type >= 2) {
      if (len < 1e-6) reject(MCL_ERR_INPUT, fmt("%s, line %d: surface point with a zero normal vector.", file.c_str(), ln));
      if (fabs(len - 1) > 1e-3) {
        renormalised++;
        for (double &c : n) c /= len;
      }
    }
    for (int c = 0; c < 3; c++) L.nrm[3 * q + c] = (float)n[c];
    L.pt[q] = type;
    top = std::max(top, type);
  });
  if (listed < L.sites())
    fprintf(stderr, "  [WARNING] %lld of the %lld grid points are not listed in %s; they were set to bulk (pt = 1).\n",
            L.sites() - listed, L.sites(), file.c_str());
  if (renormalised)
    fprintf(stderr, "  [WARNING] %d surface normal(s) in %s did not have unit length and were normalized.\n",
            renormalised, file.c_str());
  L.n_surfaces = top > 1 ? top - 1 : 0;
}

// src/ic.cpp:103-200: directors from a CSV; every non-empty point must be listed.
void ic_from_file(const Params &p, Lattice &L) {
  const std::string &file = p.ic_file;
  std::vector<char> seen(L.sites(), 0);
  int renormalised = 0;
  read_point_csv(file, {"x", "y", "z", "nx", "ny", "nz"}, [&](int ln, const std::vector<double> &v) {
    const long long q = csv_point(L, file, ln, v, seen);
    double n[3] = {v[3], v[4], v[5]};
    if (!L.pt[q]) {
      n[0] = 0;
      n[1] = 0;
      n[2] = 1;
    } else {
      const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      if (len < 1e-6) reject(MCL_ERR_INPUT, fmt("%s, line %d: zero director on a non-empty site.", file.c_str(), ln));
      if (fabs(len - 1) > 1e-3) {
        renormalised++;
        for (double &c : n) c /= len;
      }
    }
    for (int c = 0; c < 3; c++) L.ni[3 * q + c] = (float)n[c];
  });
  long long unlisted = 0;
  for (long long q = 0; q < L.sites(); q++) {
    if (seen[q]) continue;
    unlisted += L.pt[q] != 0;
    L.ni[3 * q] = 0;
    L.ni[3 * q + 1] = 0;
    L.ni[3 * q + 2] = 1;
  }
  if (unlisted)
    reject(MCL_ERR_INPUT, fmt("%s: %lld non-empty grid point(s) are not listed (the grid is %d x %d x %d).",
                              file.c_str(), unlisted, L.nx, L.ny, L.nz));
  if (renormalised)
    fprintf(stderr, "  [WARNING] %d director(s) in %s did not have unit length and were normalized.\n", renormalised,
            file.c_str());
}

// Directors of the deterministic initial conditions (src/ic.cpp:67-92 homogeneous, :202-232 cholesteric);
// `ic random` is drawn on the device after the engine exists, `ic ic_file` read from its file.
void formula_ic(const Params &p, Lattice &L) {
  const double deg = M_PI / 180;
  const float pitch = p.p0_i ? p.p0_i : p.p0;
  const bool chol = same(p.ic, "cholesteric");
  for (int k = 0; k < L.nz; k++) {
    // the cholesteric twists the azimuth about z by 2 pi per pitch
    const double phi = chol ? (double)(float)(p.phi_0 * deg - 2 * M_PI * k / pitch) : p.phi_0 * deg;
    const float d[3] = {(float)(sin(p.theta_0 * deg) * cos(phi)), (float)(sin(p.theta_0 * deg) * sin(phi)),
                        (float)cos(p.theta_0 * deg)};
    for (int j = 0; j < L.ny; j++)
      for (int i = 0; i < L.nx; i++) {
        const long long q = L.index(i, j, k);
        for (int c = 0; c < 3; c++) L.ni[3 * q + c] = L.pt[q] ? d[c] : (c == 2 ? 1.f : 0.f);
      }
  }
}

// src/io.cpp:346-371: the GHRL coefficients from the elastic constants (float inputs, the scale in double).
void ghrl_coefficients(const Params &p, mcl_model &m) {
  const float k11 = p.k11, k22 = p.k22, k33 = p.k33;
  const float scale = fabs(9.0 / (k11 - 3 * k22 - k33));
  m.ghrl_lambda = (scale / 9) * (2 * k11 - 3 * k22 + k33);
  m.ghrl_mu = scale * (k22 - k11);
  m.ghrl_rho = (scale / 9) * (k11 - k33);
  m.ghrl_nu = (scale / 9) * (k11 - 3 * k22 - k33);
  m.ghrl_sigma = p.p0 ? -scale * k22 * (2 * M_PI / p.p0) : 0;
}

struct NamedCode {
  const char *name;
  int code;
};
const NamedCode kAnchorings[] = {{"homeotropic", MCL_ANCH_HOMEOTROPIC},
                                 {"rp", MCL_ANCH_RP},
                                 {"rp_tangent", MCL_ANCH_RP_TANGENT},
                                 {"fg", MCL_ANCH_FG},
                                 {"homeotropic_ghrl", MCL_ANCH_HOMEOTROPIC_GHRL},
                                 {"rp_ghrl", MCL_ANCH_RP_GHRL},
                                 {"fg_ghrl", MCL_ANCH_FG_GHRL}};
const NamedCode kPotentials[] = {
    {"ll", MCL_POT_LL}, {"lebwohl-lasher", MCL_POT_LL}, {"ghrl", MCL_POT_GHRL}, {"gruhn-hess", MCL_POT_GHRL}, {"pear", MCL_POT_PEAR}};
const char *kModes[] = {"thermal", "step", "quench", "electric"};

template <size_t N>
int code_of(const NamedCode (&table)[N], const std::string &name) {
  for (const NamedCode &e : table)
    if (same(name, e.name)) return e.code;
  return -1;
}

Lattice build_lattice(const Params &p) {
  bool mode_ok = false;
  for (const char *m : kModes) mode_ok = mode_ok || same(p.mode, m);
  if (!mode_ok)
    reject(MCL_ERR_INPUT, fmt("Evol mode '%s' not implemented. Options: thermal | step | quench | electric, or the same "
                              "with the GPU suffix (thermalGPU, ...)", p.evol.c_str()));
  Lattice L;
  L.nx = p.Nx;
  L.ny = p.Ny;
  L.nz = p.Nz;
  L.pt.assign(L.sites(), 1);
  L.nrm.assign(3 * L.sites(), 0.f);
  L.ni.assign(3 * L.sites(), 0.f);
  const std::string bounds[3] = {p.xbound, p.ybound, p.zbound};
  bool forced[3] = {false, false, false};
  if (same(p.geometry, "custom")) {
    L.geometry = MCL_GEOM_CUSTOM;
    custom_shape(p, L);
  } else {
    const Shape *shape = nullptr;
    for (const Shape &s : shapes())
      if (same(p.geometry, s.name)) shape = &s;
    if (!shape)
      reject(MCL_ERR_INPUT, fmt("Geometry '%s' not implemented. Options: bulk | slab | sphere | custom", p.geometry.c_str()));
    L.geometry = shape->code;
    L.n_surfaces = shape->surfaces;
    for (int a = 0; a < 3; a++) forced[a] = shape->force_free[a];
    for (int k = 0; k < L.nz; k++)
      for (int j = 0; j < L.ny; j++)
        for (int i = 0; i < L.nx; i++) {
          const SiteKind s = shape->classify(L, i, j, k);
          const long long q = L.index(i, j, k);
          L.pt[q] = s.pt;
          for (int c = 0; c < 3; c++) L.nrm[3 * q + c] = s.n[c];
        }
  }
  for (int a = 0; a < 3; a++) {
    if (forced[a]) continue;
    if (same(bounds[a], "periodic"))
      L.periodic[a] = 1;
    else if (!same(bounds[a], "free"))
      reject(MCL_ERR_INPUT, fmt("%c boundary '%s' not implemented. Options: free | periodic", "XYZ"[a], bounds[a].c_str()));
  }
  // src/io.cpp:462-475: the checkerboard needs an even number of sites along a periodic axis
  const int n[3] = {L.nx, L.ny, L.nz};
  for (int a = 0; a < 3; a++)
    if (L.periodic[a] && n[a] % 2) {
      fprintf(stderr,
              "  [ERROR] Periodic boundary along %c requires an even number of sites (N%c = %d).\n"
              "          The checkerboard update needs it; use an even size or a free boundary.\n",
              "xyz"[a], "xyz"[a], n[a]);
      fail(MCL_ERR_INPUT, "periodic boundary along %c requires an even number of sites", "xyz"[a]);
      throw InputError{MCL_ERR_INPUT};
    }
  // model: potential, field, anchorings of the geometry's surfaces
  mcl_model &m = L.model;
  memset(&m, 0, sizeof m);
  const int pot = code_of(kPotentials, p.potential);
  if (pot < 0) reject(MCL_ERR_INPUT, fmt("Potential '%s' not implemented. Options: ll | ghrl | pear", p.potential.c_str()));
  m.potential = pot;
  m.A = p.A;
  m.B1 = p.B1;
  m.C = p.C;
  if (pot == MCL_POT_GHRL) ghrl_coefficients(p, m);
  m.field_dir[0] = p.elecX;
  m.field_dir[1] = p.elecY;
  m.field_dir[2] = p.elecZ;
  m.elecA = p.elecA;
  m.elecP = p.elecP;
  m.flip_move = p.flip;
  if (L.n_surfaces > MCL_MAX_SURFACES)
    reject(MCL_ERR_INPUT, fmt("at most %d surfaces are supported (got %d)", MCL_MAX_SURFACES, L.n_surfaces));
  m.n_surfaces = L.n_surfaces;
  for (int s = 0; s < L.n_surfaces; s++) {
    auto a = p.anchoring.find(s);
    if (a == p.anchoring.end())
      reject(MCL_ERR_INPUT, fmt("The geometry has %d surface(s), but anchoring_type %d is not defined in the input file.",
                                L.n_surfaces, s));
    const int code = code_of(kAnchorings, a->second);
    if (code < 0)
      reject(MCL_ERR_INPUT, fmt("Anchoring type '%s' not implemented. Options: homeotropic | rp | rp_tangent | fg | "
                                "homeotropic_ghrl | rp_ghrl | fg_ghrl", a->second.c_str()));
    m.anch_type[s] = code;
    auto w = p.W.find(s);
    if (w == p.W.end()) reject(MCL_ERR_INPUT, fmt("Parameter W not defined for the boundary condition #%d.", s));
    m.anch_W[s] = w->second;
    if (code == MCL_ANCH_RP || code == MCL_ANCH_RP_TANGENT || code == MCL_ANCH_RP_GHRL) {
      auto ph = p.phi_s.find(s), th = p.theta_s.find(s);
      if (ph == p.phi_s.end()) reject(MCL_ERR_INPUT, fmt("Parameter phi_s not defined for the boundary condition #%d.", s));
      if (th == p.theta_s.end())
        reject(MCL_ERR_INPUT, fmt("Parameter theta_s not defined for the boundary condition #%d.", s));
      m.anch_theta[s] = th->second;
      m.anch_phi[s] = ph->second;
    }
  }
  // initial condition
  if (same(p.ic, "ic_file"))
    ic_from_file(p, L);
  else if (same(p.ic, "homogeneous") || same(p.ic, "cholesteric"))
    formula_ic(p, L);
  else if (!same(p.ic, "random"))
    reject(MCL_ERR_INPUT, fmt("Initial condition '%s' not implemented. Options: random | homogeneous | ic_file | "
                              "cholesteric", p.ic.c_str()));
  L.pear = same(p.potential, "pear");
  L.sph = same(p.radial, "sphere") || same(p.radial, "both");
  L.cyl = same(p.radial, "cylinder") || same(p.radial, "both");
  return L;
}

// ---- scan points and file names (include/sweep.h) -----------------------------------------------------------
// A scan from `first` to `last` in steps of `step`: the number of points tolerates a step that does not divide
// the range exactly (1e-3 of a step), and the last point is `last` itself when the range is a whole number of
// steps.
struct Scan {
  double first, last, step;
  int points() const { return 1 + (int)floor((last - first) / step + 1e-3); }
  double at(int i) const {
    const int n = points();
    const double steps = (last - first) / step;
    return (i == n - 1 && fabs(steps - (n - 1)) < 1e-3) ? last : first + i * step;
  }
};

// Snapshot file index of a scanned value: the value times a power of ten (at least 100) large enough that one
// step moves the index by at least one, truncated after a nudge of 1e-3 of a unit of the index.
struct SnapshotNames {
  int scale = 100;
  explicit SnapshotNames(double step) {
    while (scale < 100000000 && scale * fabs(step) < 1 - 1e-3) scale *= 10;
  }
  long index(double v) const { return (long)(scale * (v + 1e-3 / scale)); }
};

// ---- outputs --------------------------------------------------------------------------------------------------
// Local S of a site from its own director and its present, non-empty neighbours (src/parameter_order.cpp:75-127,
// accumulated in float as there); only ic.csv uses it: snapshots take the device's values (mcl_local_order).
float host_local_S(const Lattice &L, const float *ni, int i, int j, int k) {
  float q[6] = {0, 0, 0, 0, 0, 0};  // xx, xy, xz, yy, yz, zz of sum (3 n n - 1)
  int count = 0;
  static const int offs[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  const int n[3] = {L.nx, L.ny, L.nz};
  for (const auto &o : offs) {
    int c[3] = {i + o[0], j + o[1], k + o[2]};
    bool present = true;
    for (int a = 0; a < 3; a++) {
      if (c[a] >= 0 && c[a] < n[a]) continue;
      if (L.periodic[a])
        c[a] = (c[a] + n[a]) % n[a];
      else
        present = false;
    }
    if (!present) continue;
    const long long s = L.index(c[0], c[1], c[2]);
    if (!L.pt[s]) continue;
    const float *d = ni + 3 * s;
    const int ab[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int e = 0; e < 6; e++) q[e] = (float)(q[e] + 3.0 * (d[ab[e][0]] * d[ab[e][1]]));
    q[0] -= 1;
    q[3] -= 1;
    q[5] -= 1;
    count++;
  }
  double qd[6], v[3];
  for (int e = 0; e < 6; e++) qd[e] = (float)(q[e] / (2.0 * count));
  return (float)mcl::largest_eigen3(qd, v);
}

// Snapshot / ic.csv (src/io.cpp:59-89). S: per-site local order from the device, or null to compute it here.
int write_snapshot(const std::string &name, const Lattice &L, const float *ni, const float *S) {
  FILE *f = fopen(name.c_str(), "w");
  if (!f) {
    perror(name.c_str());
    return fail(MCL_ERR_IO, "cannot write %s", name.c_str());
  }
  fprintf(f, "x,y,z,nx,ny,nz,S,pt\n");
  for (int k = 0; k < L.nz; k++)
    for (int j = 0; j < L.ny; j++)
      for (int i = 0; i < L.nx; i++) {
        const long long q = L.index(i, j, k);
        const float s = L.pt[q] ? (S ? S[q] : host_local_S(L, ni, i, j, k)) : NAN;
        fprintf(f, "%d,%d,%d,%g,%g,%g,%g,%d\n", i, j, k, ni[3 * q], ni[3 * q + 1], ni[3 * q + 2], s, L.pt[q]);
      }
  fclose(f);
  printf("  Snapshot -> %s\n", name.c_str());
  fflush(stdout);
  return MCL_OK;
}

// Extra po.dat columns (src/parameter_order.cpp:129-295): one mcl_measure_extras per measurement sweep, summed
// as the reference sums them (P, dtheta, divn as float, the radial orders in double).
struct ExtraColumns {
  bool pear = false, sph = false, cyl = false;
  double sum[7] = {0, 0, 0, 0, 0, 0, 0};  // P, dtheta, divn, Sr_sph, Pr_sph, Sr_cyl, Pr_cyl
  bool any() const { return pear || sph || cyl; }
  void clear() { std::fill(sum, sum + 7, 0.0); }
  void add(const mcl_extras &x) {
    const double v[7] = {(float)x.P, (float)x.dtheta, (float)x.divn, x.Sr_sph, x.Pr_sph, x.Sr_cyl, x.Pr_cyl};
    for (int c = 0; c < 7; c++) sum[c] += v[c];
  }
  // columns in output order: the polar ones with pear, then each radial order (its polar twin with pear)
  std::vector<std::pair<const char *, int>> columns() const {
    std::vector<std::pair<const char *, int>> c;
    if (pear) c.insert(c.end(), {{"P", 0}, {"dtheta", 1}, {"divn", 2}});
    if (sph) {
      c.push_back({"Sr_sph", 3});
      if (pear) c.push_back({"Pr_sph", 4});
    }
    if (cyl) {
      c.push_back({"Sr_cyl", 5});
      if (pear) c.push_back({"Pr_cyl", 6});
    }
    return c;
  }
};

void remove_old_outputs() {
  printf("  Removing output files from previous run... ");
  int removed = 0;
  if (DIR *dir = opendir(".")) {
    while (struct dirent *ent = readdir(dir)) {
      const std::string n = ent->d_name;
      const bool snap = n.size() > 19 && n.compare(0, 15, "director_field_") == 0 && n.compare(n.size() - 4, 4, ".csv") == 0;
      if (n == "ic.csv" || n == "po.dat" || snap) removed += remove(n.c_str()) == 0;
    }
    closedir(dir);
  }
  printf("%d file(s) removed.\n\n", removed);
}

#define RUN_CK(call)               \
  do {                             \
    const int rc_ = (call);        \
    if (rc_ != MCL_OK) return rc_; \
  } while (0)

// Means over one measurement block of MCS sweeps (the inner loops of src/evolve_*.cu): S and E as the floats the
// reference's loops add up, their squares, the extra columns after every sweep.
struct BlockMeans {
  double S = 0, S2 = 0, E = 0, E2 = 0;
};

int measure_block(mcl_engine *e, int mcs, ExtraColumns &ex, BlockMeans &r) {
  RUN_CK(mcl_clear_series(e));
  std::vector<mcl_observables> obs(mcs);
  if (ex.any()) {
    for (int s = 0; s < mcs; s++) {  // the extra observables need the state after each sweep
      RUN_CK(mcl_sweeps(e, 1, 1));
      RUN_CK(mcl_read_series(e, 0, s, 1, &obs[s]));
      mcl_extras x;
      RUN_CK(mcl_measure_extras(e, 0, obs[s].director, &x));
      ex.add(x);
    }
  } else {
    RUN_CK(mcl_sweeps(e, mcs, 1));
    RUN_CK(mcl_read_series(e, 0, 0, mcs, obs.data()));
  }
  for (const auto &o : obs) {
    const float E = (float)o.energy, S = (float)o.S;
    r.E += E;
    r.E2 += E * E;
    r.S += S;
    r.S2 += S * S;
  }
  r.E /= mcs;
  r.E2 /= mcs;
  r.S /= mcs;
  r.S2 /= mcs;
  return MCL_OK;
}

// One point of a mode's scan: the po.dat label, the snapshot name, and what to do before measuring.
struct ScanPoint {
  std::string label, snapshot;
  std::function<int(mcl_engine *)> prepare;
};

// The four modes as scans (src/evolve_thermal.cu:37-112, src/evolve_step.cu:34-109, src/evolve_quench.cu:36-115,
// src/evolve_electric.cu:37-115): the first po.dat column and the points.
std::vector<ScanPoint> mode_points(const Params &p, const char *&column) {
  std::vector<ScanPoint> pts;
  const int MCT = p.MCT, MCQ = p.MCQ;
  if (same(p.mode, "thermal")) {
    column = "T";
    const Scan scan{p.Ti, p.Tf, p.dT};
    const SnapshotNames names(p.dT);
    if (names.scale != 100) printf("  Snapshot names: director_field_<int(%d T)>.csv (|dT| < 0.01)\n", names.scale);
    for (int i = 0; i < scan.points(); i++) {
      const float T = (float)scan.at(i);
      pts.push_back({fmt("%g", T), fmt("director_field_%ld.csv", names.index(T)), [=](mcl_engine *e) -> int {
                       RUN_CK(mcl_set_temperature(e, 0, T));
                       return mcl_sweeps(e, MCT, 0);
                     }});
    }
  } else if (same(p.mode, "electric")) {
    column = "field";
    const Scan scan{p.Ei, p.Ef, p.dE};
    const SnapshotNames names(p.dE);
    printf("  Snapshot names: director_field_<int(%d E)>.csv\n", names.scale);
    for (int i = 0; i < scan.points(); i++) {
      const float E = (float)scan.at(i);
      pts.push_back({fmt("%g", E), fmt("director_field_%ld.csv", names.index(E)), [=](mcl_engine *e) -> int {
                       RUN_CK(mcl_set_field(e, 0, E));
                       return mcl_sweeps(e, MCT, 0);
                     }});
    }
  } else {  // step: MCT at Ti per block; quench: MCT at Ti, MCQ at Tf per block
    column = "ii";
    const bool quench = same(p.mode, "quench");
    const float Ti = p.Ti, Tf = p.Tf;
    for (int ii = p.first_file; ii < p.first_file + p.fn; ii++)
      pts.push_back({fmt("%d", ii), fmt("director_field_%d.csv", ii), [=](mcl_engine *e) -> int {
                       RUN_CK(mcl_set_temperature(e, 0, Ti));
                       RUN_CK(mcl_sweeps(e, MCT, 0));
                       if (!quench) return MCL_OK;
                       RUN_CK(mcl_set_temperature(e, 0, Tf));
                       return mcl_sweeps(e, MCQ, 0);
                     }});
  }
  return pts;
}

int run(const Params &p, Lattice &L) {
  mcl_replica rep;
  memset(&rep, 0, sizeof rep);
  rep.nx = L.nx;
  rep.ny = L.ny;
  rep.nz = L.nz;
  rep.geometry = L.geometry;
  for (int a = 0; a < 3; a++) rep.periodic[a] = L.periodic[a];
  rep.T = p.Ti;
  rep.elecE = 1.f;
  rep.ang_var = 0.5f;  // once per run, not per scan point (src/evolve_thermal.cu:43)
  rep.seed = (unsigned long long)(long long)p.seed;
  mcl_engine *e = nullptr;
  RUN_CK(mcl_create(&L.model, &rep, 1, MCL_SCHED_CHECKER2, &e));
  struct Owner {
    mcl_engine *e;
    ~Owner() { mcl_destroy(e); }
  } owner{e};
  if (L.geometry == MCL_GEOM_CUSTOM || L.geometry == MCL_GEOM_SPHERE) RUN_CK(mcl_set_geometry(e, 0, L.pt.data(), L.nrm.data()));
  if (same(p.ic, "random")) {
    RUN_CK(mcl_random_directors(e, 0, rep.seed));
    RUN_CK(mcl_download_directors(e, 0, L.ni.data()));
  } else {
    RUN_CK(mcl_upload_directors(e, 0, L.ni.data()));
  }
  RUN_CK(write_snapshot("ic.csv", L, L.ni.data(), nullptr));

  ExtraColumns ex;
  ex.pear = L.pear;
  ex.sph = L.sph;
  ex.cyl = L.cyl;
  const char *column = "";
  const std::vector<ScanPoint> pts = mode_points(p, column);
  FILE *po = fopen("po.dat", "a");
  if (!po) return fail(MCL_ERR_IO, "cannot write po.dat");
  struct Closer {
    FILE *f;
    ~Closer() { fclose(f); }
  } closer{po};
  fprintf(po, "%s S varS E varE", column);
  for (auto &c : ex.columns()) fprintf(po, " %s", c.first);
  fprintf(po, "\n");
  fflush(po);
  std::vector<float> host(L.ni.size()), localS(L.sites());
  for (const ScanPoint &pt : pts) {
    RUN_CK(pt.prepare(e));
    ex.clear();
    BlockMeans r;
    RUN_CK(measure_block(e, p.MCS, ex, r));
    RUN_CK(mcl_download_directors(e, 0, host.data()));
    RUN_CK(mcl_local_order(e, 0, localS.data()));
    RUN_CK(write_snapshot(pt.snapshot, L, host.data(), localS.data()));
    fprintf(po, "%s %g %g %g %g", pt.label.c_str(), r.S, r.S2 - r.S * r.S, r.E, r.E2 - r.E * r.E);
    for (auto &c : ex.columns()) fprintf(po, " %g", ex.sum[c.second] / p.MCS);
    fprintf(po, "\n");
    fflush(po);
  }
  return MCL_OK;
}

}  // namespace

extern "C" int mcl_run_input_file(const char *path) {
  try {
    if (!path) return fail(MCL_ERR_ARG, "no input file");
    printf("  Parameter file : %s\n\n", path);
    Params p = read_input(path);
    derive(p);
    validate(p);
    Lattice L = build_lattice(p);
    printf("  Grid %dx%dx%d, geometry %s, potential %s, mode %s, MCT %d, MCS %d, seed %d\n\n", p.Nx, p.Ny, p.Nz,
           p.geometry.c_str(), p.potential.c_str(), p.evol.c_str(), p.MCT, p.MCS, p.seed);
    remove_old_outputs();
    return run(p, L);
  } catch (const InputError &err) {
    return err.code;
  } catch (const std::exception &ex) {
    return fail(MCL_ERR_NOMEM, "host exception: %s", ex.what());
  }
}
