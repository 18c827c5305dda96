// Whole-program driver behind mcl_run_input_file: the reference program's behaviour for the *GPU evolution
// modes, on this library's engine.
//
//   input grammar and defaults   src/io.cpp:135-310, include/parameters.h:18-98
//   derived flags                src/main.cpp:86-107
//   validation                   src/io.cpp:381-475 (errors are collected; nothing is written on error)
//   geometry, anchoring, IC      src/simulator.cpp:32-126, src/geometry_*.cpp, src/geometry.cpp:78-107, src/ic.cpp
//   GHRL coefficients            src/io.cpp:346-371
//   mode loops and po.dat        src/evolve_{thermal,step,quench,electric}.cu, include/sweep.h
//   snapshots / ic.csv           src/io.cpp:59-89, src/parameter_order.cpp:75-127
//   extra po.dat columns         src/parameter_order.cpp:129-295
// Errors are returned as MCL_ERR_INPUT / MCL_ERR_IO with the reference's message text on stderr; the process is
// never terminated here.
#include <dirent.h>
#include <stdarg.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <strings.h>

#include <fstream>
#include <map>
#include <string>
#include <vector>

#include "eigen3.cuh"
#include "engine.h"

namespace {

using mcl::fail;

// Run parameters with the reference defaults (include/parameters.h:18-98).
struct Params {
  char geometry[20] = "bulk";
  int Nx = 16, Ny = 16, Nz = 16;
  char XB[20] = "free", YB[20] = "free", ZB[20] = "free";
  char bound_file[1024] = "";
  std::map<int, float> theta_s, phi_s, W;
  std::map<int, std::string> anchoring_type;
  char potential[20] = "ll";
  float A = 1.0f, B1 = 0.04f, C = 0.3f;
  float Ti = 1.2f, Tf = 0.0f, dT = -0.02f, T = 0.f;
  float ghrl_rho = 0, ghrl_lambda = 0, ghrl_mu = 0, ghrl_nu = 1, ghrl_sigma = 0;
  char evol[20] = "thermal";
  int MCS = 100, MCT = 100, MCQ = -1, fn = 1, first_file = 0, seed = 1;
  char ic[50] = "random";
  char ic_file[1024] = "";
  float phi_0 = 0, theta_0 = 0, p0_i = 0;
  float k11 = 1, k22 = 1, k33 = 1, p0 = 0;
  float elecX = 0, elecY = 0, elecZ = 0, elecA = 0, elecP = 0;
  int flipMove = 0;
  char radial[20] = "";
  float elecEi = 0, elecEf = 0, elecdE = 0, elecE = 1;
};

struct InputError {
  int code;
};

[[noreturn]] void input_fail(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  fprintf(stderr, "  [ERROR] %s\n", buf);
  fail(MCL_ERR_INPUT, "%s", buf);
  throw InputError{MCL_ERR_INPUT};
}

// ---- input file (src/io.cpp:107-310) ------------------------------------------------------------------------
void read_word(std::ifstream &in, char *dest, size_t size, const char *name) {
  std::string v;
  if (!(in >> v)) return;
  if (v.size() >= size)
    input_fail("Value of '%s' is too long (%zu characters, maximum %zu): %.60s...", name, v.size(), size - 1, v.c_str());
  strcpy(dest, v.c_str());
}

void finish_line(std::ifstream &in, const char *name) {
  if (in.fail()) return;
  std::string rest;
  std::getline(in, rest);
  size_t s = rest.find_first_not_of(" \t\r");
  if (s != std::string::npos && rest[s] != '#')
    fprintf(stderr, "  [WARNING] Ignoring extra text after parameter '%s': %s\n", name, rest.c_str() + s);
}

void check_stream(std::ifstream &in, const char *name) {
  if (in.eof()) return;
  if (in.fail() || in.bad()) input_fail("Invalid value for parameter: %s", name);
}

bool is(const char *a, const char *b) { return strcasecmp(a, b) == 0; }

template <typename T>
void num(std::ifstream &in, T &v, const char *name) {
  in >> v;
  finish_line(in, name);
}

Params read_input(const char *path) {
  Params p;
  std::ifstream in(path);
  if (!in) {
    perror(path);
    fail(MCL_ERR_IO, "cannot open input file %s", path);
    throw InputError{MCL_ERR_IO};
  }
  std::string tok;
  while (in >> tok) {
    if (tok.size() >= 200) input_fail("Parameter name too long: %.60s...", tok.c_str());
    const char *k = tok.c_str();
    int nn;
    if (is(k, "nx")) num(in, p.Nx, k);
    else if (is(k, "ny")) num(in, p.Ny, k);
    else if (is(k, "nz")) num(in, p.Nz, k);
    else if (is(k, "A")) num(in, p.A, k);
    else if (is(k, "B1")) num(in, p.B1, k);
    else if (is(k, "C")) num(in, p.C, k);
    else if (is(k, "Ti")) num(in, p.Ti, k);
    else if (is(k, "Tf")) num(in, p.Tf, k);
    else if (is(k, "dT")) num(in, p.dT, k);
    else if (is(k, "MCS")) num(in, p.MCS, k);
    else if (is(k, "MCT")) num(in, p.MCT, k);
    else if (is(k, "MCQ") || is(k, "quench_steps")) {
      num(in, p.MCQ, k);
      if (!in.fail() && p.MCQ < 0) input_fail("MCQ (quench_steps) must be >= 0 (got %d)", p.MCQ);
    } else if (is(k, "seed")) num(in, p.seed, k);
    else if (is(k, "ic")) { read_word(in, p.ic, sizeof p.ic, k); finish_line(in, k); }
    else if (is(k, "ic_file")) { read_word(in, p.ic_file, sizeof p.ic_file, k); finish_line(in, k); }
    else if (is(k, "xbound")) { read_word(in, p.XB, sizeof p.XB, k); finish_line(in, k); }
    else if (is(k, "ybound")) { read_word(in, p.YB, sizeof p.YB, k); finish_line(in, k); }
    else if (is(k, "zbound")) { read_word(in, p.ZB, sizeof p.ZB, k); finish_line(in, k); }
    else if (is(k, "potential")) { read_word(in, p.potential, sizeof p.potential, k); finish_line(in, k); }
    else if (is(k, "evol") || is(k, "mode")) { read_word(in, p.evol, sizeof p.evol, k); finish_line(in, k); }
    else if (is(k, "k11")) num(in, p.k11, k);
    else if (is(k, "k22")) num(in, p.k22, k);
    else if (is(k, "k33")) num(in, p.k33, k);
    else if (is(k, "p0")) num(in, p.p0, k);
    else if (is(k, "phi_0")) num(in, p.phi_0, k);
    else if (is(k, "theta_0")) num(in, p.theta_0, k);
    else if (is(k, "p0_i")) num(in, p.p0_i, k);
    else if (is(k, "fn")) num(in, p.fn, k);
    else if (is(k, "first_file_number") || is(k, "initial_output")) num(in, p.first_file, k);
    else if (k[0] == '#') { std::string c; std::getline(in, c); }
    else if (is(k, "geometry")) { read_word(in, p.geometry, sizeof p.geometry, k); finish_line(in, k); }
    else if (is(k, "boundary_file")) { read_word(in, p.bound_file, sizeof p.bound_file, k); finish_line(in, k); }
    else if (is(k, "anchoring_type")) {
      in >> nn;
      std::string v;
      in >> v;
      if (!in.fail()) p.anchoring_type[nn] = v;
      finish_line(in, k);
    } else if (is(k, "W")) { in >> nn; float v; in >> v; if (!in.fail()) p.W[nn] = v; finish_line(in, k); }
    else if (is(k, "phi_s")) { in >> nn; float v; in >> v; if (!in.fail()) p.phi_s[nn] = v; finish_line(in, k); }
    else if (is(k, "theta_s")) { in >> nn; float v; in >> v; if (!in.fail()) p.theta_s[nn] = v; finish_line(in, k); }
    else if (is(k, "elecX") || is(k, "Electric_field_x") || is(k, "EF_x")) num(in, p.elecX, k);
    else if (is(k, "elecY") || is(k, "Electric_field_y") || is(k, "EF_y")) num(in, p.elecY, k);
    else if (is(k, "elecZ") || is(k, "Electric_field_z") || is(k, "EF_z")) num(in, p.elecZ, k);
    else if (is(k, "Ei") || is(k, "initial_E")) num(in, p.elecEi, k);
    else if (is(k, "Ef") || is(k, "final_E")) num(in, p.elecEf, k);
    else if (is(k, "dE") || is(k, "E_variation")) num(in, p.elecdE, k);
    else if (is(k, "elecA") || is(k, "dielectric_anisotropy") || is(k, "Aniso_E")) num(in, p.elecA, k);
    else if (is(k, "elecP") || is(k, "dipolar_coupling") || is(k, "Polar_E")) num(in, p.elecP, k);
    else if (is(k, "radial")) { read_word(in, p.radial, sizeof p.radial, k); finish_line(in, k); }
    else input_fail("Unknown parameter: '%s'", k);
    check_stream(in, k);
  }
  return p;
}

// ---- validation (src/io.cpp:381-454, src/main.cpp:88-106) ------------------------------------------------------
std::string base_mode(const char *evol) {
  std::string m(evol);
  if (m.size() > 3 && strcasecmp(m.c_str() + m.size() - 3, "GPU") == 0) m.resize(m.size() - 3);
  return m;
}

void derive_and_validate(Params &p) {
  p.flipMove = (is(p.potential, "pear") || p.elecP != 0) ? 1 : 0;
  if (p.MCQ < 0) p.MCQ = p.MCT;
  if (p.radial[0] == '\0') strcpy(p.radial, is(p.geometry, "sphere") ? "sphere" : "none");
  if (!is(p.radial, "sphere") && !is(p.radial, "cylinder") && !is(p.radial, "both") && !is(p.radial, "none"))
    input_fail("radial must be sphere, cylinder, both or none (got '%s')", p.radial);
  if (p.elecA != 0 || p.elecP != 0) {
    float norm = sqrtf(p.elecX * p.elecX + p.elecY * p.elecY + p.elecZ * p.elecZ);
    if (norm == 0) input_fail("elecA or elecP is set but the field direction (elecX, elecY, elecZ) is zero");
    p.elecX /= norm;
    p.elecY /= norm;
    p.elecZ /= norm;
  }
  std::vector<std::string> errs;
  char msg[400];
  const std::string mode = base_mode(p.evol);
  const char *m = mode.c_str();
  if (p.Nx < 1 || p.Ny < 1 || p.Nz < 1) {
    snprintf(msg, sizeof msg, "Grid sizes must be >= 1 (got %d x %d x %d).", p.Nx, p.Ny, p.Nz);
    errs.push_back(msg);
  }
  if (p.MCS < 1) {
    snprintf(msg, sizeof msg, "MCS must be >= 1 (got %d): averages are taken over the MCS steps.", p.MCS);
    errs.push_back(msg);
  }
  if (p.MCT < 0) {
    snprintf(msg, sizeof msg, "MCT must be >= 0 (got %d).", p.MCT);
    errs.push_back(msg);
  }
  if ((is(m, "step") || is(m, "quench")) && p.fn < 1) {
    snprintf(msg, sizeof msg, "fn must be >= 1 in %s mode (got %d).", m, p.fn);
    errs.push_back(msg);
  }
  if (p.Ti < 0) {
    snprintf(msg, sizeof msg, "Ti must be >= 0 (got %g).", p.Ti);
    errs.push_back(msg);
  }
  if ((is(m, "thermal") || is(m, "quench")) && p.Tf < 0) {
    snprintf(msg, sizeof msg, "Tf must be >= 0 (got %g).", p.Tf);
    errs.push_back(msg);
  }
  if (is(m, "thermal")) {
    if (p.dT == 0)
      errs.push_back("dT must be nonzero in thermal mode.");
    else if ((p.Tf - p.Ti) * p.dT < 0) {
      snprintf(msg, sizeof msg, "dT = %g does not lead from Ti = %g to Tf = %g (use dT < 0 to cool, dT > 0 to heat).",
               p.dT, p.Ti, p.Tf);
      errs.push_back(msg);
    }
  }
  if (is(m, "electric")) {
    if (p.elecdE == 0)
      errs.push_back("dE must be nonzero in electric mode.");
    else if ((p.elecEf - p.elecEi) * p.elecdE < 0) {
      snprintf(msg, sizeof msg, "dE = %g does not lead from Ei = %g to Ef = %g.", p.elecdE, p.elecEi, p.elecEf);
      errs.push_back(msg);
    }
  }
  if (is(p.potential, "ghrl") || is(p.potential, "gruhn-hess")) {
    if (p.k11 <= 0 || p.k22 <= 0 || p.k33 <= 0) {
      snprintf(msg, sizeof msg, "k11, k22 and k33 must be > 0 (got %g, %g, %g).", p.k11, p.k22, p.k33);
      errs.push_back(msg);
    } else if (p.k11 - 3 * p.k22 - p.k33 >= -1e-6 * p.k22) {
      snprintf(msg, sizeof msg,
               "The GHRL potential needs k11 < 3 k22 + k33 (got k11 = %g, k22 = %g, k33 = %g): otherwise its energy "
               "scale nu is not negative and the pair potential is not nematic.",
               p.k11, p.k22, p.k33);
      errs.push_back(msg);
    }
    if (p.p0 != 0 && fabs(p.p0) < 2 * M_PI)
      fprintf(stderr,
              "  [WARNING] |p0| = %g < 2 pi: the twist per lattice bond exceeds 90 degrees and the lattice has no\n"
              "            equilibrium helix (sin(phi) = 2 pi / p0 > 1).\n",
              fabs(p.p0));
  }
  if (is(p.ic, "cholesteric") && p.p0_i == 0 && p.p0 == 0)
    errs.push_back("ic cholesteric needs a nonzero pitch: set p0_i (or p0).");
  if (!errs.empty()) {
    for (auto &s : errs) fprintf(stderr, "  [ERROR] %s\n", s.c_str());
    fprintf(stderr, "  %zu error(s) in the input file. Nothing was run and no file was changed.\n", errs.size());
    fail(MCL_ERR_INPUT, "%s", errs[0].c_str());
    throw InputError{MCL_ERR_INPUT};
  }
}

// ---- set-up: geometry, boundaries, anchoring, initial condition, potential ---------------------------------------
struct Setup {
  int geometry = MCL_GEOM_BULK;
  int periodic[3] = {0, 0, 0};
  int nSurfaces = 0;
  std::vector<int> pt;
  std::vector<float> ns;
  std::vector<float> ni;
  mcl_model model;
  bool pear = false, sph = false, cyl = false;
};

std::vector<std::string> split_csv(const std::string &line) {
  std::vector<std::string> out;
  std::string f;
  for (size_t k = 0; k <= line.size(); k++) {
    if (k == line.size() || line[k] == ',') {
      size_t a = f.find_first_not_of(" \t\r"), b = f.find_last_not_of(" \t\r");
      out.push_back(a == std::string::npos ? "" : f.substr(a, b - a + 1));
      f.clear();
    } else {
      f += line[k];
    }
  }
  return out;
}

// Columns by name from the header of a CSV (geometry and IC files); missing ones are an error.
std::vector<int> csv_columns(const std::vector<std::string> &header, const std::vector<const char *> &names,
                             const char *file, const char *required, int code) {
  std::vector<int> col(names.size(), -1);
  std::string missing;
  for (size_t c = 0; c < names.size(); c++) {
    for (size_t h = 0; h < header.size(); h++)
      if (is(header[h].c_str(), names[c])) col[c] = (int)h;
    if (col[c] < 0) missing += std::string(missing.empty() ? "" : ", ") + names[c];
  }
  if (!missing.empty()) {
    fprintf(stderr, "  [ERROR] %s, line 1: missing column(s) in the header: %s (required: %s).\n", file,
            missing.c_str(), required);
    fail(code, "missing columns in %s", file);
    throw InputError{code};
  }
  return col;
}

[[noreturn]] void file_fail(int code, const char *file, int line, const char *msg) {
  fprintf(stderr, "  [ERROR] %s, line %d: %s\n", file, line, msg);
  fail(code, "%s, line %d: %s", file, line, msg);
  throw InputError{code};
}

// src/geometry_custom.cpp:70-163
void custom_geometry(const Params &p, Setup &s) {
  const char *fname = p.bound_file;
  std::ifstream in(fname);
  if (!in) {
    perror(fname);
    fail(MCL_ERR_IO, "cannot open boundary file %s", fname);
    throw InputError{MCL_ERR_IO};
  }
  std::string line;
  if (!std::getline(in, line)) file_fail(MCL_ERR_INPUT, fname, 1, "empty file (a header line is expected).");
  std::vector<std::string> header = split_csv(line);
  std::vector<int> col = csv_columns(header, {"x", "y", "z", "nx", "ny", "nz", "pt"}, fname, "x,y,z,nx,ny,nz,pt",
                                     MCL_ERR_INPUT);
  const long long Nt = (long long)p.Nx * p.Ny * p.Nz;
  std::vector<char> seen(Nt, 0);
  std::fill(s.pt.begin(), s.pt.end(), 1);
  int maxk = 0, ln = 1, renorm = 0;
  long long listed = 0;
  char msg[300];
  static const char *names[7] = {"x", "y", "z", "nx", "ny", "nz", "pt"};
  while (std::getline(in, line)) {
    ln++;
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    std::vector<std::string> f = split_csv(line);
    if (f.size() != header.size()) {
      snprintf(msg, sizeof msg, "%zu fields, but the header has %zu.", f.size(), header.size());
      file_fail(MCL_ERR_INPUT, fname, ln, msg);
    }
    double v[7];
    for (int c = 0; c < 7; c++) {
      char *end;
      v[c] = strtod(f[col[c]].c_str(), &end);
      if (f[col[c]].empty() || *end != '\0') {
        snprintf(msg, sizeof msg, "column %s is not a number: '%s'.", names[c], f[col[c]].c_str());
        file_fail(MCL_ERR_INPUT, fname, ln, msg);
      }
    }
    int i = (int)v[0], j = (int)v[1], k = (int)v[2], type = (int)v[6];
    if (v[0] != i || v[1] != j || v[2] != k || v[6] != type)
      file_fail(MCL_ERR_INPUT, fname, ln, "x, y, z and pt must be integers.");
    if (i < 0 || i >= p.Nx || j < 0 || j >= p.Ny || k < 0 || k >= p.Nz) {
      snprintf(msg, sizeof msg, "point (%d, %d, %d) outside the %d x %d x %d grid.", i, j, k, p.Nx, p.Ny, p.Nz);
      file_fail(MCL_ERR_INPUT, fname, ln, msg);
    }
    if (type < 0) file_fail(MCL_ERR_INPUT, fname, ln, "negative point type (use 0 empty, 1 bulk, 2+ surface).");
    long long idx = ((long long)k * p.Ny + j) * p.Nx + i;
    if (seen[idx]) {
      snprintf(msg, sizeof msg, "point (%d, %d, %d) is listed twice.", i, j, k);
      file_fail(MCL_ERR_INPUT, fname, ln, msg);
    }
    seen[idx] = 1;
    listed++;
    double nx = v[3], ny = v[4], nz = v[5], norm = sqrt(nx * nx + ny * ny + nz * nz);
    if (type >= 2) {
      if (norm < 1e-6) file_fail(MCL_ERR_INPUT, fname, ln, "surface point with a zero normal vector.");
      if (fabs(norm - 1) > 1e-3) {
        renorm++;
        nx /= norm;
        ny /= norm;
        nz /= norm;
      }
    }
    s.ns[3 * idx] = (float)nx;
    s.ns[3 * idx + 1] = (float)ny;
    s.ns[3 * idx + 2] = (float)nz;
    s.pt[idx] = type;
    if (type > maxk) maxk = type;
  }
  if (listed < Nt)
    fprintf(stderr, "  [WARNING] %lld of the %lld grid points are not listed in %s; they were set to bulk (pt = 1).\n",
            Nt - listed, Nt, fname);
  if (renorm > 0)
    fprintf(stderr, "  [WARNING] %d surface normal(s) in %s did not have unit length and were normalized.\n", renorm,
            fname);
  s.nSurfaces = maxk > 1 ? maxk - 1 : 0;
}

void set_boundary(const char *axis, const char *type, int &periodic) {
  if (is(type, "free"))
    periodic = 0;
  else if (is(type, "periodic"))
    periodic = 1;
  else
    input_fail("%s boundary '%s' not implemented. Options: free | periodic", axis, type);
}

int anchoring_code(const std::string &a) {
  const char *n = a.c_str();
  if (is(n, "homeotropic")) return MCL_ANCH_HOMEOTROPIC;
  if (is(n, "rp")) return MCL_ANCH_RP;
  if (is(n, "rp_tangent")) return MCL_ANCH_RP_TANGENT;
  if (is(n, "fg")) return MCL_ANCH_FG;
  if (is(n, "homeotropic_ghrl")) return MCL_ANCH_HOMEOTROPIC_GHRL;
  if (is(n, "rp_ghrl")) return MCL_ANCH_RP_GHRL;
  if (is(n, "fg_ghrl")) return MCL_ANCH_FG_GHRL;
  return -1;
}

// Philox stream 2 of (seed, site): isotropic unit vector (z uniform in [-1, 1), azimuth uniform).
void random_unit(unsigned long long seed, uint32_t site, float out[3]) {
  mcl::U4 r = mcl::site_draws(seed, 0, site, 2);
  double z = 2.0 * ((r.x >> 8) * (1.0 / 16777216.0)) - 1.0;
  double phi = 2.0 * M_PI * ((r.y >> 8) * (1.0 / 16777216.0));
  double rho = sqrt(fmax(0.0, 1.0 - z * z));
  out[0] = (float)(rho * cos(phi));
  out[1] = (float)(rho * sin(phi));
  out[2] = (float)z;
}

// src/ic.cpp:103-200
void read_ic_file(const Params &p, Setup &s) {
  const char *fname = p.ic_file;
  std::ifstream in(fname);
  if (!in) {
    perror(fname);
    fail(MCL_ERR_IO, "cannot open initial-condition file %s", fname);
    throw InputError{MCL_ERR_IO};
  }
  std::string line;
  if (!std::getline(in, line)) file_fail(MCL_ERR_INPUT, fname, 1, "empty file (a header line is expected).");
  std::vector<std::string> header = split_csv(line);
  std::vector<int> col = csv_columns(header, {"x", "y", "z", "nx", "ny", "nz"}, fname, "x,y,z,nx,ny,nz", MCL_ERR_INPUT);
  const long long Nt = (long long)p.Nx * p.Ny * p.Nz;
  std::vector<char> seen(Nt, 0);
  int ln = 1, normalized = 0;
  char msg[300];
  static const char *names[6] = {"x", "y", "z", "nx", "ny", "nz"};
  while (std::getline(in, line)) {
    ln++;
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    std::vector<std::string> f = split_csv(line);
    if (f.size() != header.size()) {
      snprintf(msg, sizeof msg, "%zu fields, but the header has %zu.", f.size(), header.size());
      file_fail(MCL_ERR_INPUT, fname, ln, msg);
    }
    double v[6];
    for (int c = 0; c < 6; c++) {
      char *end;
      v[c] = strtod(f[col[c]].c_str(), &end);
      if (f[col[c]].empty() || *end != '\0') {
        snprintf(msg, sizeof msg, "column %s is not a number: '%s'.", names[c], f[col[c]].c_str());
        file_fail(MCL_ERR_INPUT, fname, ln, msg);
      }
    }
    int i = (int)v[0], j = (int)v[1], k = (int)v[2];
    if (v[0] != i || v[1] != j || v[2] != k) file_fail(MCL_ERR_INPUT, fname, ln, "x, y and z must be integers.");
    if (i < 0 || i >= p.Nx || j < 0 || j >= p.Ny || k < 0 || k >= p.Nz) {
      snprintf(msg, sizeof msg, "point (%d, %d, %d) outside the %d x %d x %d grid.", i, j, k, p.Nx, p.Ny, p.Nz);
      file_fail(MCL_ERR_INPUT, fname, ln, msg);
    }
    long long idx = i + (long long)p.Nx * (j + (long long)p.Ny * k);
    if (seen[idx]) {
      snprintf(msg, sizeof msg, "point (%d, %d, %d) is listed twice.", i, j, k);
      file_fail(MCL_ERR_INPUT, fname, ln, msg);
    }
    seen[idx] = 1;
    double nx = v[3], ny = v[4], nz = v[5], norm = sqrt(nx * nx + ny * ny + nz * nz);
    if (s.pt[idx]) {
      if (norm < 1e-6) file_fail(MCL_ERR_INPUT, fname, ln, "zero director on a non-empty site.");
      if (fabs(norm - 1) > 1e-3) {
        normalized++;
        nx /= norm;
        ny /= norm;
        nz /= norm;
      }
    } else {
      nx = 0;
      ny = 0;
      nz = 1;
    }
    s.ni[3 * idx] = (float)nx;
    s.ni[3 * idx + 1] = (float)ny;
    s.ni[3 * idx + 2] = (float)nz;
  }
  long long unlisted = 0;
  for (long long idx = 0; idx < Nt; idx++) {
    if (seen[idx]) continue;
    if (s.pt[idx]) unlisted++;
    s.ni[3 * idx] = 0;
    s.ni[3 * idx + 1] = 0;
    s.ni[3 * idx + 2] = 1;
  }
  if (unlisted > 0) {
    fprintf(stderr, "  [ERROR] %s: %lld non-empty grid point(s) are not listed (the grid is %d x %d x %d).\n", fname,
            unlisted, p.Nx, p.Ny, p.Nz);
    fail(MCL_ERR_INPUT, "unlisted points in %s", fname);
    throw InputError{MCL_ERR_INPUT};
  }
  if (normalized > 0)
    fprintf(stderr, "  [WARNING] %d director(s) in %s did not have unit length and were normalized.\n", normalized,
            fname);
}

void initial_condition(const Params &p, Setup &s) {
  const long long Nt = (long long)p.Nx * p.Ny * p.Nz;
  s.ni.assign(3 * Nt, 0.f);
  if (is(p.ic, "ic_file")) {
    read_ic_file(p, s);
    return;
  }
  const bool rnd = is(p.ic, "random"), hom = is(p.ic, "homogeneous"), chol = is(p.ic, "cholesteric");
  if (!rnd && !hom && !chol)
    input_fail("Initial condition '%s' not implemented. Options: random | homogeneous | ic_file | cholesteric", p.ic);
  const float p0 = p.p0_i ? p.p0_i : p.p0;
  for (int i = 0; i < p.Nx; i++)
    for (int j = 0; j < p.Ny; j++)
      for (int k = 0; k < p.Nz; k++) {
        const long long idx = i + (long long)p.Nx * (j + (long long)p.Ny * k);
        float *n = &s.ni[3 * idx];
        if (!s.pt[idx]) {
          n[0] = 0;
          n[1] = 0;
          n[2] = 1;
        } else if (rnd) {
          random_unit((unsigned long long)(long long)p.seed, (uint32_t)idx, n);
        } else if (hom) {  // src/ic.cpp:67-92
          n[0] = (float)(sin(p.theta_0 * M_PI / 180) * cos(p.phi_0 * M_PI / 180));
          n[1] = (float)(sin(p.theta_0 * M_PI / 180) * sin(p.phi_0 * M_PI / 180));
          n[2] = (float)cos(p.theta_0 * M_PI / 180);
        } else {  // src/ic.cpp:202-232
          float phi = (float)(p.phi_0 * M_PI / 180 - 2 * M_PI * k / p0);
          n[0] = (float)(sin(p.theta_0 * M_PI / 180) * cos(phi));
          n[1] = (float)(sin(p.theta_0 * M_PI / 180) * sin(phi));
          n[2] = (float)cos(p.theta_0 * M_PI / 180);
        }
      }
}

// src/io.cpp:346-371 (float inputs, double Scale expression as in the reference)
void set_ghrl(Params &p) {
  float k11 = p.k11, k22 = p.k22, k33 = p.k33, p0 = p.p0;
  float Scale = fabs((9.0) / (k11 - 3 * k22 - k33));
  p.ghrl_sigma = p0 ? -Scale * k22 * (2 * M_PI / p0) : 0;
  p.ghrl_lambda = (Scale / 9) * (2 * k11 - 3 * k22 + k33);
  p.ghrl_mu = Scale * (k22 - k11);
  p.ghrl_rho = (Scale / 9) * (k11 - k33);
  p.ghrl_nu = (Scale / 9) * (k11 - 3 * k22 - k33);
}

Setup build_setup(Params &p) {
  Setup s;
  const long long Nt = (long long)p.Nx * p.Ny * p.Nz;
  s.pt.assign(Nt, 1);
  s.ns.assign(3 * Nt, 0.f);
  const std::string mode = base_mode(p.evol);
  if (!is(mode.c_str(), "thermal") && !is(mode.c_str(), "step") && !is(mode.c_str(), "quench") &&
      !is(mode.c_str(), "electric"))
    input_fail("Evol mode '%s' not implemented. Options: thermal | step | quench | electric, or the same with the GPU "
               "suffix (thermalGPU, ...)", p.evol);
  if (is(p.geometry, "bulk")) {
    s.geometry = MCL_GEOM_BULK;
    s.nSurfaces = 0;
  } else if (is(p.geometry, "slab")) {
    s.geometry = MCL_GEOM_SLAB;
    s.nSurfaces = 2;
    strcpy(p.ZB, "free");
    for (int i = 0; i < p.Nx; i++)
      for (int j = 0; j < p.Ny; j++) {
        long long a = i + (long long)p.Nx * j, b = i + (long long)p.Nx * (j + (long long)p.Ny * (p.Nz - 1));
        s.pt[a] = 2;
        s.ns[3 * a + 2] = -1;
        for (int k = 1; k < p.Nz - 1; k++) s.pt[i + (long long)p.Nx * (j + (long long)p.Ny * k)] = 1;
        s.pt[b] = 3;
        s.ns[3 * b + 0] = 0;
        s.ns[3 * b + 1] = 0;
        s.ns[3 * b + 2] = 1;
      }
  } else if (is(p.geometry, "sphere")) {
    s.geometry = MCL_GEOM_SPHERE;
    s.nSurfaces = 1;
    strcpy(p.XB, "free");
    strcpy(p.YB, "free");
    strcpy(p.ZB, "free");
    const float Hx = p.Nx / 2, Hy = p.Ny / 2, Hz = p.Nz / 2;
    for (int i = 0; i < p.Nx; i++)
      for (int j = 0; j < p.Ny; j++)
        for (int k = 0; k < p.Nz; k++) {
          long long idx = i + (long long)p.Nx * (j + (long long)p.Ny * k);
          float Rx = i - Hx, Ry = j - Hy, Rz = k - Hz;
          float r = sqrt(Rx * Rx + Ry * Ry + Rz * Rz);
          if (r < Hz - 1)
            s.pt[idx] = 1;
          else if (r < Hz + 1) {
            s.pt[idx] = 2;
            s.ns[3 * idx] = Rx / r;
            s.ns[3 * idx + 1] = Ry / r;
            s.ns[3 * idx + 2] = Rz / r;
          } else
            s.pt[idx] = 0;
        }
  } else if (is(p.geometry, "custom")) {
    s.geometry = MCL_GEOM_CUSTOM;
    custom_geometry(p, s);
  } else {
    input_fail("Geometry '%s' not implemented. Options: bulk | slab | sphere | custom", p.geometry);
  }
  set_boundary("X", p.XB, s.periodic[0]);
  set_boundary("Y", p.YB, s.periodic[1]);
  set_boundary("Z", p.ZB, s.periodic[2]);
  // src/io.cpp:462-475
  const int n[3] = {p.Nx, p.Ny, p.Nz};
  for (int a = 0; a < 3; a++)
    if (s.periodic[a] && n[a] % 2) {
      fprintf(stderr,
              "  [ERROR] Periodic boundary along %c requires an even number of sites (N%c = %d).\n"
              "          The checkerboard update needs it; use an even size or a free boundary.\n",
              "xyz"[a], "xyz"[a], n[a]);
      fail(MCL_ERR_INPUT, "periodic boundary along %c requires an even number of sites", "xyz"[a]);
      throw InputError{MCL_ERR_INPUT};
    }
  // anchorings, src/geometry.cpp:78-107 and the constructors' parameter checks
  mcl_model &m = s.model;
  memset(&m, 0, sizeof m);
  if (s.nSurfaces > MCL_MAX_SURFACES) input_fail("at most %d surfaces are supported (got %d)", MCL_MAX_SURFACES, s.nSurfaces);
  m.n_surfaces = s.nSurfaces;
  for (int sid = 0; sid < s.nSurfaces; sid++) {
    auto it = p.anchoring_type.find(sid);
    if (it == p.anchoring_type.end())
      input_fail("The geometry has %d surface(s), but anchoring_type %d is not defined in the input file.",
                 s.nSurfaces, sid);
    int code = anchoring_code(it->second);
    if (code < 0)
      input_fail("Anchoring type '%s' not implemented. Options: homeotropic | rp | rp_tangent | fg | homeotropic_ghrl |"
                 " rp_ghrl | fg_ghrl", it->second.c_str());
    m.anch_type[sid] = code;
    if (!p.W.count(sid)) input_fail("Parameter W not defined for the boundary condition #%d.", sid);
    m.anch_W[sid] = p.W[sid];
    if (code == MCL_ANCH_RP || code == MCL_ANCH_RP_TANGENT || code == MCL_ANCH_RP_GHRL) {
      if (!p.phi_s.count(sid)) input_fail("Parameter phi_s not defined for the boundary condition #%d.", sid);
      if (!p.theta_s.count(sid)) input_fail("Parameter theta_s not defined for the boundary condition #%d.", sid);
      m.anch_theta[sid] = p.theta_s[sid];
      m.anch_phi[sid] = p.phi_s[sid];
    }
  }
  initial_condition(p, s);
  if (is(p.potential, "ll") || is(p.potential, "lebwohl-lasher")) {
    m.potential = MCL_POT_LL;
  } else if (is(p.potential, "ghrl") || is(p.potential, "gruhn-hess")) {
    m.potential = MCL_POT_GHRL;
    set_ghrl(p);
  } else if (is(p.potential, "pear")) {
    m.potential = MCL_POT_PEAR;
  } else {
    input_fail("Potential '%s' not implemented. Options: ll | ghrl | pear", p.potential);
  }
  m.A = p.A;
  m.B1 = p.B1;
  m.C = p.C;
  m.ghrl_lambda = p.ghrl_lambda;
  m.ghrl_mu = p.ghrl_mu;
  m.ghrl_nu = p.ghrl_nu;
  m.ghrl_rho = p.ghrl_rho;
  m.ghrl_sigma = p.ghrl_sigma;
  m.field_dir[0] = p.elecX;
  m.field_dir[1] = p.elecY;
  m.field_dir[2] = p.elecZ;
  m.elecA = p.elecA;
  m.elecP = p.elecP;
  m.flip_move = p.flipMove;
  s.pear = is(p.potential, "pear");
  s.sph = is(p.radial, "sphere") || is(p.radial, "both");
  s.cyl = is(p.radial, "cylinder") || is(p.radial, "both");
  return s;
}

// ---- outputs ------------------------------------------------------------------------------------------------
inline int sweep_points(double a, double b, double d) { return (int)floor((b - a) / d + 1e-3) + 1; }
inline double sweep_value(double a, double b, double d, int n, int np) {
  if (n == np - 1 && fabs((b - a) / d - (np - 1)) < 1e-3) return b;
  return a + n * d;
}
inline int snapshot_scale(double step) {
  int S = 100;
  while (S * fabs(step) < 1 - 1e-3 && S < 100000000) S *= 10;
  return S;
}
inline long snapshot_index(double x, int S) { return (long)(S * (x + 1e-3 / S)); }

bool bnd(int periodic, int &v, int N) {
  if (periodic) {
    v = (v + N) % N;
    return true;
  }
  return !(v == -1 || v == N);
}

// Local S of a site: largest eigenvalue of Q over the site and its existing non-empty neighbours
// (src/parameter_order.cpp:75-127, float accumulation as there).
float local_S(const Params &p, const Setup &s, const float *ni, int i, int j, int k) {
  float Q[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int points = 0;
  for (int di = -1; di < 2; di++)
    for (int dj = -1; dj < 2; dj++)
      for (int dk = -1; dk < 2; dk++) {
        if (abs(di) + abs(dj) + abs(dk) > 1) continue;
        int ii = i + di, jj = j + dj, kk = k + dk;
        if (!bnd(s.periodic[0], ii, p.Nx) || !bnd(s.periodic[1], jj, p.Ny) || !bnd(s.periodic[2], kk, p.Nz)) continue;
        long long q = ii + (long long)p.Nx * (jj + (long long)p.Ny * kk);
        if (!s.pt[q]) continue;
        for (int l = 0; l < 3; l++) {
          for (int mm = 0; mm <= l; mm++) Q[3 * mm + l] = (float)(Q[3 * mm + l] + 3.0 * (ni[3 * q + l] * ni[3 * q + mm]));
          Q[4 * l] -= 1;
        }
        points++;
      }
  double q6[6] = {Q[0] / (2.0 * points), Q[1] / (2.0 * points), Q[2] / (2.0 * points),
                  Q[4] / (2.0 * points), Q[5] / (2.0 * points), Q[8] / (2.0 * points)};
  float qf[6];
  for (int c = 0; c < 6; c++) qf[c] = (float)q6[c];
  double qd[6] = {qf[0], qf[1], qf[2], qf[3], qf[4], qf[5]}, v[3];
  return (float)mcl::largest_eigen3(qd, v);
}

// Snapshot / ic.csv (src/io.cpp:59-89). S: the local order parameters from the device (mcl_local_order), or null
// to compute them here (ic.csv, written before the engine exists).
int print_n(const char *fname, const Params &p, const Setup &s, const float *ni, const float *S = nullptr) {
  FILE *f = fopen(fname, "w");
  if (!f) {
    perror(fname);
    return fail(MCL_ERR_IO, "cannot write %s", fname);
  }
  fprintf(f, "x,y,z,nx,ny,nz,S,pt\n");
  for (int k = 0; k < p.Nz; k++)
    for (int j = 0; j < p.Ny; j++)
      for (int i = 0; i < p.Nx; i++) {
        long long q = i + (long long)p.Nx * (j + (long long)p.Ny * k);
        const float Sq = s.pt[q] ? (S ? S[q] : local_S(p, s, ni, i, j, k)) : NAN;
        fprintf(f, "%d,%d,%d,%g,%g,%g,%g,%d\n", i, j, k, ni[3 * q], ni[3 * q + 1], ni[3 * q + 2], Sq, s.pt[q]);
      }
  fclose(f);
  printf("  Snapshot -> %s\n", fname);
  fflush(stdout);
  return MCL_OK;
}

// Extra po.dat columns (src/parameter_order.cpp:129-295), computed on the device after every measurement sweep
// (mcl_measure_extras) and accumulated as ExtraObservables::accumulate does (P, dtheta, divn rounded to float, the
// radial orders in double).
struct Extras {
  bool pear, sph, cyl;
  double P = 0, dTheta = 0, divN = 0, SrS = 0, PrS = 0, SrC = 0, PrC = 0;
  void reset() { P = dTheta = divN = SrS = PrS = SrC = PrC = 0; }
  bool any() const { return pear || sph || cyl; }
  void add(const mcl_extras &x) {
    if (pear) {
      P += (float)x.P;
      dTheta += (float)x.dtheta;
      divN += (float)x.divn;
    }
    if (sph) {
      SrS += x.Sr_sph;
      PrS += x.Pr_sph;
    }
    if (cyl) {
      SrC += x.Sr_cyl;
      PrC += x.Pr_cyl;
    }
  }
  void header(FILE *f) const {
    if (pear) fprintf(f, " P dtheta divn");
    if (sph) fprintf(f, pear ? " Sr_sph Pr_sph" : " Sr_sph");
    if (cyl) fprintf(f, pear ? " Sr_cyl Pr_cyl" : " Sr_cyl");
    fprintf(f, "\n");
  }
  void values(FILE *f, int n) const {
    if (pear) fprintf(f, " %g %g %g", P / n, dTheta / n, divN / n);
    if (sph) {
      fprintf(f, " %g", SrS / n);
      if (pear) fprintf(f, " %g", PrS / n);
    }
    if (cyl) {
      fprintf(f, " %g", SrC / n);
      if (pear) fprintf(f, " %g", PrC / n);
    }
    fprintf(f, "\n");
  }
};

void clean_previous_output() {
  printf("  Removing output files from previous run... ");
  int removed = 0;
  DIR *dir = opendir(".");
  if (dir) {
    struct dirent *ent;
    while ((ent = readdir(dir)) != NULL) {
      const char *n = ent->d_name;
      size_t L = strlen(n);
      if (!strcmp(n, "ic.csv") || !strcmp(n, "po.dat") ||
          (!strncmp(n, "director_field_", 15) && L > 4 && !strcmp(n + L - 4, ".csv"))) {
        remove(n);
        removed++;
      }
    }
    closedir(dir);
  }
  printf("%d file(s) removed.\n\n", removed);
}

// One measured block: MCS sweeps with observables after each (the inner loops of src/evolve_*.cu).
struct BlockResult {
  double S1 = 0, S2 = 0, E = 0, E2 = 0;
};

#define RUN_CK(call)                   \
  do {                                 \
    int rc_ = (call);                  \
    if (rc_ != MCL_OK) return rc_;     \
  } while (0)

int measure_block(mcl_engine *e, const Params &p, const Setup &s, Extras &ex, std::vector<float> &host_ni,
                  BlockResult &r) {
  RUN_CK(mcl_clear_series(e));
  std::vector<mcl_observables> obs;
  if (ex.any()) {
    // the extra observables of the state after every measurement sweep, as in the reference
    for (int step = 0; step < p.MCS; step++) {
      RUN_CK(mcl_sweeps(e, 1, 1));
      mcl_observables o;
      RUN_CK(mcl_read_series(e, 0, step, 1, &o));
      mcl_extras x;
      RUN_CK(mcl_measure_extras(e, 0, o.director, &x));
      ex.add(x);
      obs.push_back(o);
    }
  } else {
    RUN_CK(mcl_sweeps(e, p.MCS, 1));
    obs.resize(p.MCS);
    RUN_CK(mcl_read_series(e, 0, 0, p.MCS, obs.data()));
  }
  for (const auto &o : obs) {
    const float tempE = (float)o.energy;  // energy_calculator_GPU returns float
    r.E2 += tempE * tempE;
    r.E += tempE;
    const float sTemp = (float)o.S;
    r.S1 += sTemp;
    r.S2 += sTemp * sTemp;
  }
  r.E /= p.MCS;
  r.E2 /= p.MCS;
  r.S1 /= p.MCS;
  r.S2 /= p.MCS;
  return MCL_OK;
}

int run_modes(Params &p, Setup &s) {
  mcl_replica rep;
  memset(&rep, 0, sizeof rep);
  rep.nx = p.Nx;
  rep.ny = p.Ny;
  rep.nz = p.Nz;
  rep.geometry = s.geometry;
  for (int a = 0; a < 3; a++) rep.periodic[a] = s.periodic[a];
  rep.T = p.Ti;
  rep.elecE = 1.f;
  rep.ang_var = 0.5f;  // src/evolve_thermal.cu:43
  rep.seed = (unsigned long long)(long long)p.seed;
  mcl_engine *e = nullptr;
  RUN_CK(mcl_create(&s.model, &rep, 1, MCL_SCHED_CHECKER2, &e));
  struct Guard {
    mcl_engine *e;
    ~Guard() { mcl_destroy(e); }
  } guard{e};
  if (s.geometry == MCL_GEOM_CUSTOM || s.geometry == MCL_GEOM_SPHERE)
    RUN_CK(mcl_set_geometry(e, 0, s.pt.data(), s.ns.data()));
  RUN_CK(mcl_upload_directors(e, 0, s.ni.data()));
  Extras ex;
  ex.pear = s.pear;
  ex.sph = s.sph;
  ex.cyl = s.cyl;
  std::vector<float> host(s.ni.size()), localS(s.ni.size() / 3);
  const std::string mode = base_mode(p.evol);
  FILE *po = fopen("po.dat", "a");
  if (!po) return fail(MCL_ERR_IO, "cannot write po.dat");
  char fname[1000];
  int rc = MCL_OK;
  if (is(mode.c_str(), "thermal")) {  // src/evolve_thermal.cu:37-112
    fprintf(po, "T S varS E varE");
    ex.header(po);
    fflush(po);
    const int snapS = snapshot_scale(p.dT);
    if (snapS != 100) printf("  Snapshot names: director_field_<int(%d T)>.csv (|dT| < 0.01)\n", snapS);
    const int nT = sweep_points(p.Ti, p.Tf, p.dT);
    for (int it = 0; it < nT && rc == MCL_OK; it++) {
      p.T = (float)sweep_value(p.Ti, p.Tf, p.dT, it, nT);
      if ((rc = mcl_set_temperature(e, 0, p.T))) break;
      if ((rc = mcl_sweeps(e, p.MCT, 0))) break;
      ex.reset();
      BlockResult r;
      if ((rc = measure_block(e, p, s, ex, host, r))) break;
      if ((rc = mcl_download_directors(e, 0, host.data()))) break;
      if ((rc = mcl_local_order(e, 0, localS.data()))) break;
      snprintf(fname, sizeof fname, "director_field_%ld.csv", snapshot_index(p.T, snapS));
      if ((rc = print_n(fname, p, s, host.data(), localS.data()))) break;
      fprintf(po, "%g %g %g %g %g", p.T, r.S1, r.S2 - r.S1 * r.S1, r.E, r.E2 - r.E * r.E);
      ex.values(po, p.MCS);
      fflush(po);
    }
  } else if (is(mode.c_str(), "step") || is(mode.c_str(), "quench")) {
    const bool quench = is(mode.c_str(), "quench");  // src/evolve_step.cu:34-109, src/evolve_quench.cu:36-115
    fprintf(po, "ii S varS E varE");
    ex.header(po);
    fflush(po);
    p.T = p.Ti;
    rc = mcl_set_temperature(e, 0, p.T);
    for (int ii = p.first_file; ii < p.fn + p.first_file && rc == MCL_OK; ii++) {
      if (quench && (rc = mcl_set_temperature(e, 0, p.Ti))) break;
      if ((rc = mcl_sweeps(e, p.MCT, 0))) break;
      if (quench) {
        p.T = p.Tf;
        if ((rc = mcl_set_temperature(e, 0, p.Tf))) break;
        if ((rc = mcl_sweeps(e, p.MCQ, 0))) break;
      }
      ex.reset();
      BlockResult r;
      if ((rc = measure_block(e, p, s, ex, host, r))) break;
      if ((rc = mcl_download_directors(e, 0, host.data()))) break;
      if ((rc = mcl_local_order(e, 0, localS.data()))) break;
      snprintf(fname, sizeof fname, "director_field_%d.csv", ii);
      if ((rc = print_n(fname, p, s, host.data(), localS.data()))) break;
      fprintf(po, "%d %g %g %g %g", ii, r.S1, r.S2 - r.S1 * r.S1, r.E, r.E2 - r.E * r.E);
      ex.values(po, p.MCS);
      fflush(po);
    }
  } else {  // electric, src/evolve_electric.cu:37-115
    fprintf(po, "field S varS E varE");
    ex.header(po);
    fflush(po);
    p.T = p.Ti;
    rc = mcl_set_temperature(e, 0, p.T);
    const int snapS = snapshot_scale(p.elecdE);
    printf("  Snapshot names: director_field_<int(%d E)>.csv\n", snapS);
    const int nE = sweep_points(p.elecEi, p.elecEf, p.elecdE);
    for (int ie = 0; ie < nE && rc == MCL_OK; ie++) {
      p.elecE = (float)sweep_value(p.elecEi, p.elecEf, p.elecdE, ie, nE);
      if ((rc = mcl_set_field(e, 0, p.elecE))) break;
      if ((rc = mcl_sweeps(e, p.MCT, 0))) break;
      ex.reset();
      BlockResult r;
      if ((rc = measure_block(e, p, s, ex, host, r))) break;
      if ((rc = mcl_download_directors(e, 0, host.data()))) break;
      if ((rc = mcl_local_order(e, 0, localS.data()))) break;
      snprintf(fname, sizeof fname, "director_field_%ld.csv", snapshot_index(p.elecE, snapS));
      if ((rc = print_n(fname, p, s, host.data(), localS.data()))) break;
      fprintf(po, "%g %g %g %g %g", p.elecE, r.S1, r.S2 - r.S1 * r.S1, r.E, r.E2 - r.E * r.E);
      ex.values(po, p.MCS);
      fflush(po);
    }
  }
  fclose(po);
  return rc;
}

}  // namespace

extern "C" int mcl_run_input_file(const char *path) {
  try {
    if (!path) return fail(MCL_ERR_ARG, "no input file");
    printf("  Parameter file : %s\n\n", path);
    Params p = read_input(path);
    derive_and_validate(p);
    Setup s = build_setup(p);
    printf("  Grid %dx%dx%d, geometry %s, potential %s, mode %s, MCT %d, MCS %d, seed %d\n\n", p.Nx, p.Ny, p.Nz,
           p.geometry, p.potential, p.evol, p.MCT, p.MCS, p.seed);
    clean_previous_output();
    int rc = print_n("ic.csv", p, s, s.ni.data());
    if (rc) return rc;
    return run_modes(p, s);
  } catch (const InputError &err) {
    return err.code;
  } catch (const std::exception &ex) {
    return fail(MCL_ERR_NOMEM, "host exception: %s", ex.what());
  }
}
