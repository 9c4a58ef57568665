// The reference's file front end in C++: model_mesh (MEDIT .mesh,
// src/FETD_FWD.f90:112-166), model_ctl (keyword .cntl, :284-497), the .field
// and .field2 rows of solution_output (:1623, :1625-1640), and the driver of
// `./FETD -f ROOT` (FETD_MAIN + time_solver): read, load the context the way
// mesh_process does, run adap_euler, write the outputs.  Host code only; the
// work goes through the library's C ABI.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/temf_b200.h"
#include "element.cuh"

namespace {

constexpr double kMu0 = 3.141592653589793238462643383279502884197 * 4.0e-7;  // src/FETD_FWD.f90:15

struct AnisoDomain {
  int phys = 0;
  double sv[3], sa[3], ev[3], ea[3], mv[3], ma[3];
};

struct Case {
  // mesh
  std::vector<double> nod;  // (nodes, 3) row-major
  std::vector<int> tet;     // (tets, 4) row-major, 1-based
  std::vector<int> tet_phy;
  std::vector<int> src;     // (segments, 2) row-major, 1-based
  std::vector<int> src_phy;
  // control
  std::vector<double> rec;  // (receivers, 3) row-major
  double rec_charac = 10.0;
  std::vector<int> dom_phys;
  std::vector<double> dom_sig, dom_eps, dom_mu;
  std::vector<AnisoDomain> aniso;
  int bound_cond = 0, src_num = 0, source_type = 1, pulse_type = 1;
  double t0 = 0.0, current = 1.0;
  int sp_mthd = 0, sp_division = 0, sp_double = 0, sp_dblesize = 2, vtkout = 0;
  double time_maximum = 0.0;
  bool output[9] = {false, false, false, false, false, false, false, false, false};
  std::vector<double> time_points;
  bool have_time_points = false;
  std::vector<double> vtk_times;  // whole-mesh field dumps (vtkout)
  // set by load
  std::vector<int> edg_vex;  // (edges, 2) column-major, 1-based
  int n_edges = 0;
};

[[noreturn]] void fail(const std::string& s) { throw std::runtime_error(s); }

double num(std::string t) {
  for (char& ch : t)
    if (ch == 'd' || ch == 'D') ch = 'e';
  char* end = nullptr;
  const double v = std::strtod(t.c_str(), &end);
  if (end == t.c_str()) fail("not a number: '" + t + "'");
  return v;
}

int inum(const std::string& t) {
  char* end = nullptr;
  const long v = std::strtol(t.c_str(), &end, 10);
  if (end == t.c_str()) fail("not an integer: '" + t + "'");
  return (int)v;
}

std::vector<std::string> split(const std::string& s) {
  std::istringstream is(s);
  std::vector<std::string> t;
  std::string w;
  while (is >> w) t.push_back(w);
  return t;
}

std::vector<std::string> read_lines(const std::string& path) {
  std::ifstream f(path);
  if (!f) fail("cannot open " + path);
  std::vector<std::string> L;
  std::string s;
  while (std::getline(f, s)) {
    if (!s.empty() && s.back() == '\r') s.pop_back();
    L.push_back(s);
  }
  return L;
}

// model_mesh: sections keyed by the first five letters of their first word
void read_mesh(const std::string& path, Case& c) {
  const std::vector<std::string> L = read_lines(path);
  bool have_nod = false, have_tet = false;
  for (size_t i = 0; i < L.size();) {
    const std::vector<std::string> t = split(L[i]);
    const std::string w = t.empty() ? "" : t[0].substr(0, 5);
    if (w != "Verti" && w != "Edges" && w != "Trian" && w != "Tetra") {
      ++i;
      continue;
    }
    if (i + 1 >= L.size()) fail(path + ": section " + t[0] + " without a count");
    const std::vector<std::string> tc = split(L[i + 1]);
    if (tc.empty()) fail(path + ": section " + t[0] + " without a count");
    const int cnt = inum(tc[0]);
    if (cnt < 0 || i + 2 + (size_t)cnt > L.size()) fail(path + ": section " + t[0] + " is truncated");
    for (int q = 0; q < cnt; ++q) {
      const std::vector<std::string> r = split(L[i + 2 + q]);
      if (w == "Verti") {
        if (r.size() < 3) fail(path + ": short vertex line");
        for (int a = 0; a < 3; ++a) c.nod.push_back(num(r[a]));
      } else if (w == "Edges") {
        if (r.size() < 3) fail(path + ": short edge line");
        const int tag = inum(r[2]);
        if (tag != 0) {  // tagged edges are the source segments
          c.src.push_back(inum(r[0]));
          c.src.push_back(inum(r[1]));
          c.src_phy.push_back(tag);
        }
      } else if (w == "Tetra") {
        if (r.size() < 5) fail(path + ": short tetrahedron line");
        for (int a = 0; a < 4; ++a) c.tet.push_back(inum(r[a]));
        c.tet_phy.push_back(inum(r[4]));
      }
    }
    if (w == "Verti") have_nod = true;
    if (w == "Tetra") have_tet = true;
    i += 2 + cnt;
  }
  if (!have_nod || !have_tet) fail(path + ": no Vertices/Tetrahedra section");
}

// one keyword line: (key, value) with the key lower-cased and the value cut at
// a comment; false for blank and comment lines
bool parse_line(std::string s, std::string& key, std::string& val) {
  std::replace(s.begin(), s.end(), '\t', ' ');
  const size_t b = s.find_first_not_of(' ');
  if (b == std::string::npos || s[b] == '%' || s[b] == '!') return false;
  const size_t k = s.find(':');
  if (k == std::string::npos) {
    key.clear();
    val.clear();
    return true;
  }
  key = s.substr(0, k);
  val = s.substr(k + 1);
  const size_t cut = val.find_first_of("%!");
  if (cut != std::string::npos && cut > 0) val = val.substr(0, cut);
  auto trim = [](std::string& x) {
    const size_t p = x.find_first_not_of(' '), q = x.find_last_not_of(' ');
    x = p == std::string::npos ? "" : x.substr(p, q - p + 1);
  };
  trim(key);
  trim(val);
  for (char& ch : key) ch = (char)std::tolower((unsigned char)ch);
  return true;
}

// model_ctl
void read_cntl(const std::string& path, Case& c) {
  const std::vector<std::string> L = read_lines(path);
  auto line = [&](size_t i) -> std::vector<std::string> {
    if (i >= L.size()) fail(path + ": file ends inside a section");
    return split(L[i]);
  };
  auto first = [&](const std::string& v) -> std::string {
    const std::vector<std::string> t = split(v);
    if (t.empty()) fail(path + ": keyword without a value");
    return t[0];
  };
  bool have_rec = false;
  for (size_t i = 0; i < L.size();) {
    std::string k, v;
    const bool kv = parse_line(L[i], k, v);
    ++i;
    if (!kv) continue;
    if (k == "receivers") {
      const int n = inum(first(v));
      for (int q = 0; q < n; ++q) {
        const std::vector<std::string> t = line(i + q);
        if (t.size() < 3) fail(path + ": short receiver line");
        for (int a = 0; a < 3; ++a) c.rec.push_back(num(t[a]));
      }
      i += n;
      have_rec = n > 0;
    } else if (k == "rec_charac") {
      c.rec_charac = num(first(v));
    } else if (k == "isotropic") {
      const int n = inum(first(v));
      for (int q = 0; q < n; ++q) {
        const std::vector<std::string> t = line(i + q);
        if (t.size() < 4) fail(path + ": short isotropic domain line");
        c.dom_phys.push_back(inum(t[0]));
        c.dom_sig.push_back(num(t[1]));
        c.dom_eps.push_back(num(t[2]));
        c.dom_mu.push_back(num(t[3]));
      }
      i += n;
    } else if (k == "anisotropic") {
      const int n = inum(first(v));
      for (int q = 0; q < n; ++q) {
        AnisoDomain d;
        double* vals[3] = {d.sv, d.ev, d.mv};
        double* angs[3] = {d.sa, d.ea, d.ma};
        for (int part = 0; part < 3; ++part) {  // sigma, eps_r, mu_r lines
          const std::vector<std::string> t = line(i + 3 * q + part);
          if (t.size() < 7) fail(path + ": short anisotropic domain line");
          if (part == 0) d.phys = (int)num(t[0]);
          for (int a = 0; a < 3; ++a) {
            vals[part][a] = num(t[1 + a]);
            angs[part][a] = num(t[4 + a]);
          }
        }
        c.aniso.push_back(d);
      }
      i += 3 * (size_t)n;
    } else if (k == "boundary condition") {
      c.bound_cond = inum(first(v));
    } else if (k == "source") {
      c.src_num = inum(first(v));
      const std::vector<std::string> t = line(i);
      if (t.size() < 4) fail(path + ": short source line");
      c.source_type = inum(t[0]);
      c.pulse_type = inum(t[1]);
      c.t0 = num(t[2]);
      c.current = num(t[3]);
      i += 1;
    } else if (k == "sp_mthd") {
      c.sp_mthd = inum(first(v));
    } else if (k == "sp_division") {
      c.sp_division = inum(first(v));
    } else if (k == "time_maximum") {
      c.time_maximum = num(first(v));
    } else if (k == "sp_double") {
      c.sp_double = inum(first(v));
    } else if (k == "sp_dblesize") {
      c.sp_dblesize = inum(first(v));
    } else if (k == "output") {
      const std::vector<std::string> t = line(i);
      if (t.size() < 9) fail(path + ": the output line needs 9 flags");
      for (int a = 0; a < 9; ++a) c.output[a] = inum(t[a]) == 1;
      i += 1;
    } else if (k == "time_points") {
      const int n = inum(first(v));
      for (int q = 0; q < n; ++q) c.time_points.push_back(num(line(i + q).at(0)));
      c.have_time_points = true;
      i += n;
    } else if (k == "vtkout") {
      c.vtkout = inum(first(v));
      for (int q = 0; q < c.vtkout; ++q) c.vtk_times.push_back(num(line(i + q).at(0)));
      i += std::max(c.vtkout, 0);
    }
  }
  bool any_out = false;
  for (bool b : c.output) any_out |= b;
  // the completeness test of model_ctl (src/FETD_FWD.f90:490-497)
  if (!have_rec || (c.dom_phys.empty() && c.aniso.empty()) || c.src_num == 0 || c.sp_mthd == 0 ||
      c.sp_division == 0 || std::fabs(c.time_maximum) < 1e-20 || c.sp_double == 0 || !any_out)
    fail(path + ": incomplete control file (src/FETD_FWD.f90:490-497)");
}

// the rotation dm = dx dy dz of the anisotropic media (src/FETD_FWD.f90:387-390),
// angles in degrees; the z factor carries cos of the second angle at (2,2) as
// the reference's does
void rotation(const double* ang, double dm[3][3]) {
  const double d2r = 3.141592653589793238462643383279502884197 / 180.0;
  const double a1 = ang[0] * d2r, a2 = ang[1] * d2r, a3 = ang[2] * d2r;
  const double dx[3][3] = {{1, 0, 0}, {0, std::cos(a1), -std::sin(a1)}, {0, std::sin(a1), std::cos(a1)}};
  const double dy[3][3] = {{std::cos(a2), 0, std::sin(a2)}, {0, 1, 0}, {-std::sin(a2), 0, std::cos(a2)}};
  const double dz[3][3] = {{std::cos(a3), -std::sin(a3), 0}, {std::sin(a3), std::cos(a2), 0}, {0, 0, 1}};
  double t[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      t[i][j] = 0;
      for (int k = 0; k < 3; ++k) t[i][j] += dx[i][k] * dy[k][j];
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      dm[i][j] = 0;
      for (int k = 0; k < 3; ++k) dm[i][j] += t[i][k] * dz[k][j];
    }
}

// dm diag(v) dm^T, row-major into out[9]
void tensor(const double* v, const double* ang, double scale, double* out) {
  double dm[3][3];
  rotation(ang, dm);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += dm[i][k] * v[k] * dm[j][k];
      out[3 * i + j] = s * scale;
    }
}

// per-tet media (src/FETD_FWD.f90:347-409): isotropic sig/mu, or row-major
// 3 x 3 tensors per tet
void media(const Case& c, std::vector<double>& sig, std::vector<double>& mu) {
  const size_t T = c.tet_phy.size();
  if (c.aniso.empty()) {
    sig.assign(T, 0.0);
    mu.assign(T, 0.0);
    for (size_t t = 0; t < T; ++t) {
      size_t j = 0;
      while (j < c.dom_phys.size() && c.dom_phys[j] != c.tet_phy[t]) ++j;
      if (j == c.dom_phys.size()) fail("error - physical domain not found!");
      sig[t] = c.dom_sig[j];
      mu[t] = c.dom_mu[j] * kMu0;
    }
    return;
  }
  sig.assign(9 * T, 0.0);
  mu.assign(9 * T, 0.0);
  for (size_t t = 0; t < T; ++t) {
    size_t j = 0;
    while (j < c.aniso.size() && c.aniso[j].phys != c.tet_phy[t]) ++j;
    if (j == c.aniso.size()) fail("error - physical domain not found!");
    tensor(c.aniso[j].sv, c.aniso[j].sa, 1.0, &sig[9 * t]);
    tensor(c.aniso[j].mv, c.aniso[j].ma, kMu0, &mu[9 * t]);
  }
}

// Fortran Ew.d with d significant digits after "0.": [-]0.ddddd E+ee,
// right-justified in w columns (three-digit exponents drop the E)
std::string fortran_e(double v, int w, int d) {
  char buf[64];
  std::string s;
  if (std::isnan(v)) {
    s = "NaN";
  } else if (std::isinf(v)) {
    s = v < 0 ? "-Infinity" : "Infinity";
  } else if (v == 0.0) {
    s = "0." + std::string(d, '0') + "E+00";
  } else {
    std::snprintf(buf, sizeof buf, "%.*E", d - 1, std::fabs(v));  // m.mmmmE+xx, m != 0
    const std::string t(buf);
    const size_t e = t.find('E');
    const std::string digits = t.substr(0, 1) + t.substr(2, e - 2);
    const int ex = std::atoi(t.c_str() + e + 1) + 1;
    char eb[16];
    if (std::abs(ex) < 100) std::snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else std::snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    s = std::string(v < 0 ? "-" : "") + "0." + digits + eb;
  }
  if ((int)s.size() < w) s = std::string(w - s.size(), ' ') + s;
  return s;
}

// one output row: i6, e15.5, 2x, then per receiver the selected columns
// (e15.5 each) and 2x; trailing blanks dropped
void write_rows(const std::string& path, int rows, int nrec, const int* steps, const double* times,
                const double* fields, const int* mask) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) fail("cannot write " + path);
  for (int i = 0; i < rows; ++i) {
    char head[32];
    std::snprintf(head, sizeof head, "%6d", steps[i]);
    std::string line = std::string(head) + fortran_e(times[i], 15, 5) + "  ";
    for (int r = 0; r < nrec; ++r) {
      for (int k = 0; k < 9; ++k)
        if (mask[k]) line += fortran_e(fields[(size_t)k + 9 * ((size_t)r + (size_t)nrec * i)], 15, 5);
      line += "  ";
    }
    while (!line.empty() && line.back() == ' ') line.pop_back();
    line += "\n";
    std::fputs(line.c_str(), f);
  }
  if (std::fclose(f) != 0) fail("writing " + path + " failed");
}

void check(int rc, temf_ctx* ctx, const char* what) {
  if (rc < 0) fail(std::string(what) + ": " + (ctx ? temf_last_error(ctx) : "error"));
}

// mesh_process + the source and receiver set-up of model_ctl / model_mesh
void load(Case& c, temf_ctx* ctx) {
  const int N = (int)(c.nod.size() / 3), T = (int)c.tet_phy.size();
  std::vector<int> tv(4 * (size_t)T);  // Fortran tet_vex(T,4)
  for (int t = 0; t < T; ++t)
    for (int a = 0; a < 4; ++a) tv[(size_t)a * T + t] = c.tet[4 * (size_t)t + a];
  std::vector<double> nod(3 * (size_t)N);
  for (int i = 0; i < N; ++i)
    for (int a = 0; a < 3; ++a) nod[(size_t)a * N + i] = c.nod[3 * (size_t)i + a];
  int ne = 0;
  check(temf_mesh_count_edges(T, tv.data(), &ne), nullptr, "temf_mesh_count_edges");
  c.n_edges = ne;
  c.edg_vex.assign(2 * (size_t)ne, 0);
  std::vector<int> te(6 * (size_t)T), td(6 * (size_t)T);
  check(temf_mesh_topology(T, tv.data(), ne, c.edg_vex.data(), te.data(), td.data()), nullptr, "temf_mesh_topology");
  check(temf_set_mesh(ctx, N, nod.data(), T, tv.data(), ne, c.edg_vex.data(), te.data(), td.data()), ctx,
        "temf_set_mesh");
  std::vector<double> sig, mu;
  media(c, sig, mu);
  if (c.aniso.empty()) check(temf_set_media(ctx, sig.data(), mu.data()), ctx, "temf_set_media");
  else check(temf_set_media_tensor(ctx, sig.data(), mu.data()), ctx, "temf_set_media_tensor");
  check(temf_set_boundary(ctx, c.bound_cond, nullptr), ctx, "temf_set_boundary");
  check(temf_analyse(ctx), ctx, "temf_analyse");
  check(temf_assemble(ctx), ctx, "temf_assemble");
  // src_edg / src_drc (src/FETD_FWD.f90:435-448): the edge of each segment;
  // +1 for every segment but the last, which gets -1
  const int S = (int)c.src_phy.size();
  std::vector<long long> key(ne);
  for (int e = 0; e < ne; ++e) key[e] = ((long long)c.edg_vex[e] << 32) | (long long)c.edg_vex[(size_t)ne + e];
  std::vector<int> se(std::max(S, 1), 0), sd(std::max(S, 1), 0);
  for (int s = 0; s < S; ++s) {
    const long long a = std::min(c.src[2 * s], c.src[2 * s + 1]), b = std::max(c.src[2 * s], c.src[2 * s + 1]);
    const long long k = (a << 32) | b;
    const auto p = std::lower_bound(key.begin(), key.end(), k);
    if (p == key.end() || *p != k) fail("source segment " + std::to_string(s + 1) + " is not an edge of the mesh");
    se[s] = (int)(p - key.begin()) + 1;
    sd[s] = s == S - 1 ? -1 : 1;
  }
  const int col_ptr[2] = {0, S};
  check(temf_set_sources(ctx, 1, col_ptr, se.data(), sd.data(), c.source_type, c.pulse_type, c.t0, c.current), ctx,
        "temf_set_sources");
  // receivers: p_in_tet (src/FETD_FWD.f90:1009-1049) on the GPU
  const int R = (int)(c.rec.size() / 3);
  std::vector<double> rc(3 * (size_t)R);
  for (int r = 0; r < R; ++r)
    for (int a = 0; a < 3; ++a) rc[(size_t)a * R + r] = c.rec[3 * (size_t)r + a];
  std::vector<int> rt(std::max(R, 1), 0);
  check(temf_locate_points(ctx, R, rc.data(), c.rec_charac, rt.data()), ctx, "temf_locate_points");
  for (int r = 0; r < R; ++r)
    if (rt[r] == 0) fail("no rec tet No. " + std::to_string(r + 1));
  check(temf_set_receivers(ctx, R, rt.data(), rc.data(), nullptr), ctx, "temf_set_receivers");
}

void write_outputs(const Case& c, temf_ctx* ctx, const std::string& root) {
  int rows = 0;
  check(temf_result_rows(ctx, &rows), ctx, "temf_result_rows");
  const int R = (int)(c.rec.size() / 3);
  std::vector<int> steps(std::max(rows, 1));
  std::vector<double> times(std::max(rows, 1)), fields(9 * (size_t)std::max(R, 1) * std::max(rows, 1));
  check(temf_result_get(ctx, steps.data(), times.data(), nullptr, fields.data()), ctx, "temf_result_get");
  int mask[9];
  for (int k = 0; k < 9; ++k) mask[k] = c.output[k] ? 1 : 0;
  write_rows(root + ".field", rows, R, steps.data(), times.data(), fields.data(), mask);
  if (!c.have_time_points) return;
  const int G = (int)c.time_points.size();
  std::vector<double> g(9 * (size_t)std::max(R, 1) * std::max(G, 1));
  std::vector<int> done(std::max(G, 1));
  check(temf_result_gates(ctx, G, c.time_points.data(), g.data(), done.data()), ctx, "temf_result_gates");
  // rows for the channels the run reached, numbered as the reference numbers them
  std::vector<int> idx;
  std::vector<double> t2, f2;
  for (int i = 0; i < G; ++i) {
    if (!done[i]) continue;
    idx.push_back(i + 1);
    t2.push_back(c.time_points[i]);
    f2.insert(f2.end(), g.begin() + 9 * (size_t)R * i, g.begin() + 9 * (size_t)R * (i + 1));
  }
  write_rows(root + ".field2", (int)idx.size(), R, idx.data(), t2.data(), f2.data(), mask);
}

// msh_output (src/FETD_FWD.f90:1713-1864): the tetrahedron (type 4) element
// tags of a Gmsh 4.1 file in file order ...
std::vector<long long> msh_tet_tags(const std::string& path) {
  const std::vector<std::string> L = read_lines(path);
  size_t i = 0;
  while (i < L.size() && L[i].compare(0, 9, "$Elements") != 0) ++i;
  if (i == L.size()) fail(path + ": no $Elements section");
  ++i;
  auto fields = [&](size_t k) -> std::vector<std::string> {
    if (k >= L.size()) fail(path + ": $Elements is truncated");
    return split(L[k]);
  };
  const int nblk = inum(fields(i).at(0));
  ++i;
  std::vector<long long> tags;
  for (int b = 0; b < nblk; ++b) {
    const std::vector<std::string> h = fields(i);
    if (h.size() < 4) fail(path + ": short element block header");
    const int type = inum(h[2]), cnt = inum(h[3]);
    ++i;
    if (type == 4)
      for (int q = 0; q < cnt; ++q) tags.push_back(std::atoll(fields(i + q).at(0).c_str()));
    i += cnt;
  }
  return tags;
}

// ... then a copy of the file with one $ElementData block per selected column
// of fields (tets x 9: E, D, B), absolute values, format (i10, e16.8)
void write_msh(const Case& c, const std::string& src, const std::string& dst, const double* fields) {
  static const char* names[9] = {"Ex", "Ey", "Ez", "Dx", "Dy", "Dz", "Bx", "By", "Bz"};
  const std::vector<long long> tags = msh_tet_tags(src);
  if (tags.size() != c.tet_phy.size())
    fail(src + ": " + std::to_string(tags.size()) + " tetrahedra, the mesh has " + std::to_string(c.tet_phy.size()));
  std::ifstream in(src, std::ios::binary);
  std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  if (!text.empty() && text.back() != '\n') text += '\n';
  FILE* f = std::fopen(dst.c_str(), "w");
  if (!f) fail("cannot write " + dst);
  std::fputs(text.c_str(), f);
  char buf[64];
  for (int k = 0; k < 9; ++k) {
    if (!c.output[k]) continue;
    std::fprintf(f, "$ElementData\n1\n\"%s data\"\n1\n0.0\n3\n0\n1\n%12d\n", names[k], (int)tags.size());
    for (size_t t = 0; t < tags.size(); ++t) {
      std::snprintf(buf, sizeof buf, "%10lld", tags[t]);
      std::fputs((std::string(buf) + fortran_e(std::fabs(fields[9 * t + k]), 16, 8) + "\n").c_str(), f);
    }
    std::fputs("$EndElementData\n", f);
  }
  if (std::fclose(f) != 0) fail("writing " + dst + " failed");
}

void copy_msg(const std::string& s, char* msg, int len) {
  if (msg && len > 0) {
    std::strncpy(msg, s.c_str(), len - 1);
    msg[len - 1] = 0;
  }
}

}  // namespace

struct temf_case : Case {};

extern "C" {

int temf_case_read(const char* root, temf_case** out, char* msg, int msg_len) {
  if (!root || !out) return TEMF_EARG;
  *out = nullptr;
  temf_case* c = new temf_case();
  try {
    read_mesh(std::string(root) + ".mesh", *c);
    read_cntl(std::string(root) + ".cntl", *c);
    *out = c;
    copy_msg("", msg, msg_len);
    return TEMF_OK;
  } catch (const std::exception& e) {
    delete c;
    copy_msg(e.what(), msg, msg_len);
    return TEMF_EARG;
  }
}

int temf_case_free(temf_case* c) {
  delete c;
  return TEMF_OK;
}

int temf_case_sizes(const temf_case* c, int* sizes) {
  if (!c || !sizes) return TEMF_EARG;
  sizes[0] = (int)(c->nod.size() / 3);
  sizes[1] = (int)c->tet_phy.size();
  sizes[2] = (int)c->src_phy.size();
  sizes[3] = (int)(c->rec.size() / 3);
  sizes[4] = (int)c->dom_phys.size();
  sizes[5] = (int)c->aniso.size();
  sizes[6] = c->have_time_points ? (int)c->time_points.size() : -1;
  return TEMF_OK;
}

int temf_case_mesh(const temf_case* c, double* nod_cor, int* tet_vex, int* tet_phy, int* src_vex, int* src_phy) {
  if (!c) return TEMF_EARG;
  const size_t N = c->nod.size() / 3, T = c->tet_phy.size(), S = c->src_phy.size();
  if (nod_cor)
    for (size_t i = 0; i < N; ++i)
      for (int a = 0; a < 3; ++a) nod_cor[a * N + i] = c->nod[3 * i + a];
  if (tet_vex)
    for (size_t t = 0; t < T; ++t)
      for (int a = 0; a < 4; ++a) tet_vex[a * T + t] = c->tet[4 * t + a];
  if (tet_phy) std::copy(c->tet_phy.begin(), c->tet_phy.end(), tet_phy);
  if (src_vex)
    for (size_t s = 0; s < S; ++s)
      for (int a = 0; a < 2; ++a) src_vex[a * S + s] = c->src[2 * s + a];
  if (src_phy) std::copy(c->src_phy.begin(), c->src_phy.end(), src_phy);
  return TEMF_OK;
}

int temf_case_control(const temf_case* c, int* ints, double* reals, double* rec_cor, double* time_points) {
  if (!c) return TEMF_EARG;
  if (ints) {
    const int v[10] = {c->bound_cond, c->src_num, c->source_type, c->pulse_type, c->sp_mthd,
                       c->sp_division, c->sp_double, c->sp_dblesize, c->vtkout, 0};
    std::copy(v, v + 10, ints);
    for (int k = 0; k < 9; ++k) ints[9] |= (c->output[k] ? 1 : 0) << k;
  }
  if (reals) {
    reals[0] = c->rec_charac;
    reals[1] = c->t0;
    reals[2] = c->current;
    reals[3] = c->time_maximum;
  }
  const size_t R = c->rec.size() / 3;
  if (rec_cor)
    for (size_t r = 0; r < R; ++r)
      for (int a = 0; a < 3; ++a) rec_cor[a * R + r] = c->rec[3 * r + a];
  if (time_points) std::copy(c->time_points.begin(), c->time_points.end(), time_points);
  return TEMF_OK;
}

int temf_case_media(const temf_case* c, double* sig, double* mu, int* aniso) {
  if (!c) return TEMF_EARG;
  try {
    std::vector<double> s, m;
    media(*c, s, m);
    if (aniso) *aniso = c->aniso.empty() ? 0 : 1;
    if (sig) std::copy(s.begin(), s.end(), sig);
    if (mu) std::copy(m.begin(), m.end(), mu);
    return TEMF_OK;
  } catch (const std::exception&) {
    return TEMF_EARG;
  }
}

int temf_case_write_rows(const char* path, int rows, int nrec, const int* steps, const double* times,
                         const double* fields, const int* output_mask) {
  if (!path || rows < 0 || nrec < 0 || (rows > 0 && (!steps || !times || !fields)) || !output_mask) return TEMF_EARG;
  try {
    write_rows(path, rows, nrec, steps, times, fields, output_mask);
    return TEMF_OK;
  } catch (const std::exception&) {
    return TEMF_EINTERNAL;
  }
}

int temf_case_vtk_times(const temf_case* c, int* n, double* times) {
  if (!c || !n) return TEMF_EARG;
  *n = (int)c->vtk_times.size();
  if (times) std::copy(c->vtk_times.begin(), c->vtk_times.end(), times);
  return TEMF_OK;
}

int temf_case_write_msh(const temf_case* c, const char* src_msh, const char* dst_msh, const double* fields, char* msg,
                        int msg_len) {
  if (!c || !src_msh || !dst_msh || !fields) return TEMF_EARG;
  try {
    write_msh(*c, src_msh, dst_msh, fields);
    copy_msg("", msg, msg_len);
    return TEMF_OK;
  } catch (const std::exception& e) {
    copy_msg(e.what(), msg, msg_len);
    return TEMF_EARG;
  }
}

int temf_mesh_fields_host(int n_nodes, const double* nod_cor, int n_tets, const int* tet_vex, const int* tet_edg,
                          const int* tet_drc, int n_edges, const double* e, double* fields) {
  if (n_nodes <= 0 || n_tets <= 0 || n_edges <= 0 || !nod_cor || !tet_vex || !tet_edg || !tet_drc || !e || !fields)
    return TEMF_EARG;
  for (int64_t q = 0; q < 4LL * n_tets; ++q)
    if (tet_vex[q] < 1 || tet_vex[q] > n_nodes) return TEMF_EARG;
  for (int64_t q = 0; q < 6LL * n_tets; ++q)
    if (tet_edg[q] < 1 || tet_edg[q] > n_edges) return TEMF_EARG;
  for (int t = 0; t < n_tets; ++t) {
    double X[4][3], ev[6], E[3], D[3];
    for (int k = 0; k < 4; ++k)
      for (int a = 0; a < 3; ++a) X[k][a] = nod_cor[(int64_t)a * n_nodes + tet_vex[(int64_t)k * n_tets + t] - 1];
    for (int j = 0; j < 6; ++j)
      ev[j] = tet_drc[(int64_t)j * n_tets + t] * e[tet_edg[(int64_t)j * n_tets + t] - 1];
    temf::centroid_fields(X, ev, E, D);
    for (int a = 0; a < 3; ++a) {
      fields[6LL * t + a] = E[a];
      fields[6LL * t + 3 + a] = D[a];
    }
  }
  return TEMF_OK;
}

int temf_case_load(temf_case* c, temf_ctx* ctx, char* msg, int msg_len) {
  if (!c || !ctx) return TEMF_EARG;
  try {
    load(*c, ctx);
    copy_msg("", msg, msg_len);
    return TEMF_OK;
  } catch (const std::exception& e) {
    copy_msg(e.what(), msg, msg_len);
    return TEMF_EARG;
  }
}

int temf_case_write(const temf_case* c, temf_ctx* ctx, const char* root, char* msg, int msg_len) {
  if (!c || !ctx || !root) return TEMF_EARG;
  try {
    write_outputs(*c, ctx, root);
    copy_msg("", msg, msg_len);
    return TEMF_OK;
  } catch (const std::exception& e) {
    copy_msg(e.what(), msg, msg_len);
    return TEMF_EINTERNAL;
  }
}

int temf_case_run(const char* root, int device, int flags, char* msg, int msg_len) {
  if (!root) return TEMF_EARG;
  temf_case* c = nullptr;
  int rc = temf_case_read(root, &c, msg, msg_len);
  if (rc != TEMF_OK) return rc;
  temf_ctx* ctx = nullptr;
  try {
    check(temf_create(device, &ctx), nullptr, "temf_create");
    load(*c, ctx);
    // whole-mesh dumps need the model's Gmsh file next to it (msh_output copies ROOT.msh)
    const std::string msh = std::string(root) + ".msh";
    const bool dumps = !c->vtk_times.empty() && std::ifstream(msh).good();
    if (dumps)
      check(temf_set_mesh_fields(ctx, (int)c->vtk_times.size(), c->vtk_times.data()), ctx, "temf_set_mesh_fields");
    check(temf_run(ctx, c->sp_division, c->sp_double, c->sp_dblesize, c->time_maximum, flags, nullptr, 0, 0), ctx,
          "temf_run");
    write_outputs(*c, ctx, root);
    if (dumps) {
      std::vector<double> f(9 * c->tet_phy.size());
      for (int i = 0; i < (int)c->vtk_times.size(); ++i) {
        int done = 0;
        check(temf_result_mesh_fields(ctx, i, f.data(), &done), ctx, "temf_result_mesh_fields");
        if (done) write_msh(*c, msh, std::string(root) + "_" + std::to_string(i + 1) + ".msh", f.data());
      }
    }
    copy_msg("", msg, msg_len);
    rc = TEMF_OK;
  } catch (const std::exception& e) {
    copy_msg(e.what(), msg, msg_len);
    rc = TEMF_EINTERNAL;
  }
  if (ctx) temf_destroy(ctx);
  temf_case_free(c);
  return rc;
}

}  // extern "C"
