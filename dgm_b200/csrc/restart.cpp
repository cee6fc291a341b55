// Restart files in DGM's format, and the Domain::diff comparison.
//
// Layout (src/Domain.cpp:1721-1785 header, src/vField.cpp:1082-1200 data):
// ten text lines, each a value left-justified in 40 columns and a label
// (Session, Created, Name, "Nel, Nsd, Lmax", Step, Time, Time step,
// Viscosity, Field names, Format "Normalized"), then per field: the global
// length (int32), the number of modes of every element (int32), their
// displacements (int32), and the orthonormal modal coefficients (float64,
// element by element, index c + L*(b + L*a)).  This text header is what is
// written; the reader also takes the newer JSON header (a JSON object, then
// the rest of its closing line, src/Domain.cpp:1368-1466) with int32 sizes,
// float64 scalars, little-endian byte order and the normalized basis.
//
// Domain::diff (src/Domain.cpp:1000-1066) reads two restart files, takes the
// Linf / L2 / H1 norms (Field::norm, src/Field.cpp:4675-4697; Hex::norm_*,
// src/Hex.cpp:2356-2450) of the first and of their difference at the GLL
// points, and fails a field when an absolute norm exceeds aeps, or a norm
// relative to the first file's exceeds reps where that norm is above
// sqrt(machine epsilon).  Everything here runs on the host.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "dgmx_internal.hpp"

using namespace dgmx;

namespace {

thread_local std::string g_restart_error;

const char *field_names(int physics, int k) {
  static const char *e2[] = {"R", "U", "V", "E"};
  static const char *e3[] = {"R", "U", "V", "W", "E"};
  static const char *sw[] = {"H", "U", "V"};
  if (physics == DGMX_SHALLOW) return sw[k];
  return dim_of(physics) == 3 ? e3[k] : e2[k];
}

std::string pad(const std::string &s, size_t w) {
  return s.size() >= w ? s : s + std::string(w - s.size(), ' ');
}

template <class V>
std::string str(V v) {
  std::ostringstream o;
  o << v;
  return o.str();
}

struct Header {
  int ne = 0, nsd = 0, lmax = 0, step = 0;
  double t = 0, dt = 0, vis = 0;
  size_t bytes = 0;   // header length
};

// Value of "key" in a JSON object text (keys are unique in DGM's restart
// header, nested ones included); strings come back without quotes.
bool json_value(const std::string &js, const std::string &key, std::string &out) {
  const std::string q = "\"" + key + "\"";
  size_t at = 0;
  while ((at = js.find(q, at)) != std::string::npos) {
    size_t c = js.find_first_not_of(" \t\r\n", at + q.size());
    if (c == std::string::npos || js[c] != ':') { at += q.size(); continue; }
    c = js.find_first_not_of(" \t\r\n", c + 1);
    if (c == std::string::npos) return false;
    if (js[c] == '"') {
      const size_t e = js.find('"', c + 1);
      if (e == std::string::npos) return false;
      out = js.substr(c + 1, e - c - 1);
    } else {
      const size_t e = js.find_first_of(",}\r\n", c);
      out = js.substr(c, e == std::string::npos ? std::string::npos : e - c);
      while (!out.empty() && std::isspace((unsigned char)out.back())) out.pop_back();
    }
    return true;
  }
  return false;
}

bool read_json_header(std::ifstream &f, Header &h) {
  std::string js;
  int depth = 0;
  bool instr = false;
  char c;
  while (f.get(c)) {
    js.push_back(c);
    if (instr) { if (c == '"') instr = false; continue; }
    if (c == '"') instr = true;
    else if (c == '{') ++depth;
    else if (c == '}' && --depth == 0) break;
  }
  std::string rest;
  if (depth != 0 || !std::getline(f, rest)) { g_restart_error = "restart: unterminated JSON header"; return false; }
  std::string v;
  auto num = [&](const char *k, double &x, bool need) {
    if (!json_value(js, k, v)) {
      if (need) g_restart_error = std::string("restart: JSON header has no \"") + k + "\"";
      return !need;
    }
    x = std::stod(v);
    return true;
  };
  double ne = 0, nsd = 0, lmax = 0, step = 0;
  if (!num("Nel", ne, true) || !num("Nsd", nsd, true) || !num("Lmax", lmax, true) || !num("Step", step, true) ||
      !num("Time", h.t, true) || !num("Time step", h.dt, false) || !num("Viscosity", h.vis, false))
    return false;
  h.ne = (int)ne; h.nsd = (int)nsd; h.lmax = (int)lmax; h.step = (int)step;
  std::string basis;
  if (!json_value(js, "Basis type", basis) || (basis != "Normalized" && basis != "normalized")) {
    g_restart_error = "restart: only the normalized (orthonormal) basis is supported";
    return false;
  }
  const char *want[][2] = {{"GlobalSize", "int32"}, {"LocalSize", "int32"}, {"Scalar", "float64"},
                           {"ByteOrder", "LittleEndian"}};
  for (auto &w : want)
    if (json_value(js, w[0], v) && v != w[1]) {
      g_restart_error = std::string("restart: ") + w[0] + " = " + v + " is not supported (" + w[1] + " is)";
      return false;
    }
  h.bytes = (size_t)f.tellg();
  return true;
}

bool read_header(std::ifstream &f, Header &h) {
  if (f.peek() == '{') return read_json_header(f, h);
  std::vector<std::string> lines(10);
  for (auto &l : lines)
    if (!std::getline(f, l)) { g_restart_error = "restart: header is shorter than ten lines"; return false; }
  std::istringstream a(lines[3]);
  if (!(a >> h.ne >> h.nsd >> h.lmax) || lines[3].find("Nel") == std::string::npos) {
    g_restart_error = "restart: malformed 'Nel, Nsd, Lmax' line";
    return false;
  }
  std::istringstream s4(lines[4]), s5(lines[5]), s6(lines[6]), s7(lines[7]);
  s4 >> h.step;
  s5 >> h.t;
  s6 >> h.dt;
  s7 >> h.vis;
  if (lines[9].find("Normalized") == std::string::npos || lines[9].find("Unnormalized") != std::string::npos) {
    g_restart_error = "restart: only the normalized (orthonormal) basis is supported";
    return false;
  }
  h.bytes = (size_t)f.tellg();
  return true;
}

// Reads nf fields; nmodes gets ne entries (of field 0), modes the data in
// restart layout [field][element modes].
bool read_fields(std::ifstream &f, const Header &h, int nf, std::vector<int> &nmodes, std::vector<double> &modes) {
  modes.clear();
  for (int n = 0; n < nf; ++n) {
    int32_t glen = 0;
    f.read(reinterpret_cast<char *>(&glen), 4);
    std::vector<int32_t> nm(h.ne), disp(h.ne);
    f.read(reinterpret_cast<char *>(nm.data()), 4 * (std::streamsize)h.ne);
    f.read(reinterpret_cast<char *>(disp.data()), 4 * (std::streamsize)h.ne);
    if (!f) { g_restart_error = "restart: truncated field header"; return false; }
    long long tot = 0;
    for (int e = 0; e < h.ne; ++e) {
      if (nm[e] <= 0 || disp[e] != tot) { g_restart_error = "restart: inconsistent mode counts"; return false; }
      tot += nm[e];
    }
    if (tot != glen) { g_restart_error = "restart: global length does not match the mode counts"; return false; }
    if (n == 0) nmodes.assign(nm.begin(), nm.end());
    else if (!std::equal(nmodes.begin(), nmodes.end(), nm.begin())) {
      g_restart_error = "restart: fields have different mode counts";
      return false;
    }
    const size_t at = modes.size();
    modes.resize(at + (size_t)tot);
    f.read(reinterpret_cast<char *>(modes.data() + at), 8 * (std::streamsize)tot);
    if (!f) { g_restart_error = "restart: truncated field data"; return false; }
  }
  return true;
}

bool read_file(const char *path, int nf, Header &h, std::vector<int> &nmodes, std::vector<double> &modes) {
  std::ifstream f(path, std::ios::binary);
  if (!f) { g_restart_error = std::string("restart: cannot open ") + path; return false; }
  return read_header(f, h) && read_fields(f, h, nf, nmodes, modes);
}

// GLL values and their physical gradient of one element from its modes
// (sum-factorised backward transform and collocation derivative, host FP64).
void element_values(const Tables1D &t, int dim, const double *uh, const double *metric, double *u, double *gx,
                    double *gy, double *gz) {
  const int L = t.L, Q = t.Q;
  if (dim == 2) {
    std::vector<double> s((size_t)Q * L, 0.0);
    for (int i = 0; i < Q; ++i)
      for (int b = 0; b < L; ++b) {
        double acc = 0.0;
        for (int a = 0; a < L; ++a) acc += t.B[(size_t)a * Q + i] * uh[a * L + b];
        s[(size_t)i * L + b] = acc;
      }
    for (int i = 0; i < Q; ++i)
      for (int j = 0; j < Q; ++j) {
        double acc = 0.0;
        for (int b = 0; b < L; ++b) acc += t.B[(size_t)b * Q + j] * s[(size_t)i * L + b];
        u[i * Q + j] = acc;
      }
    for (int i = 0; i < Q; ++i)
      for (int j = 0; j < Q; ++j) {
        double dr = 0.0, ds = 0.0;
        for (int m = 0; m < Q; ++m) {
          dr += t.D[(size_t)i * Q + m] * u[m * Q + j];
          ds += t.D[(size_t)j * Q + m] * u[i * Q + m];
        }
        gx[i * Q + j] = metric[0] * dr + metric[3] * ds;
        gy[i * Q + j] = metric[1] * dr + metric[4] * ds;
      }
    return;
  }
  std::vector<double> s1((size_t)Q * L * L, 0.0), s2((size_t)Q * Q * L, 0.0);
  for (int i = 0; i < Q; ++i)
    for (int bc = 0; bc < L * L; ++bc) {
      double acc = 0.0;
      for (int a = 0; a < L; ++a) acc += t.B[(size_t)a * Q + i] * uh[a * L * L + bc];
      s1[(size_t)i * L * L + bc] = acc;
    }
  for (int i = 0; i < Q; ++i)
    for (int j = 0; j < Q; ++j)
      for (int c = 0; c < L; ++c) {
        double acc = 0.0;
        for (int b = 0; b < L; ++b) acc += t.B[(size_t)b * Q + j] * s1[((size_t)i * L + b) * L + c];
        s2[((size_t)i * Q + j) * L + c] = acc;
      }
  for (int ij = 0; ij < Q * Q; ++ij)
    for (int k = 0; k < Q; ++k) {
      double acc = 0.0;
      for (int c = 0; c < L; ++c) acc += t.B[(size_t)c * Q + k] * s2[(size_t)ij * L + c];
      u[ij * Q + k] = acc;
    }
  for (int i = 0; i < Q; ++i)
    for (int j = 0; j < Q; ++j)
      for (int k = 0; k < Q; ++k) {
        double dr = 0.0, ds = 0.0, dt = 0.0;
        for (int m = 0; m < Q; ++m) {
          dr += t.D[(size_t)i * Q + m] * u[(m * Q + j) * Q + k];
          ds += t.D[(size_t)j * Q + m] * u[(i * Q + m) * Q + k];
          dt += t.D[(size_t)k * Q + m] * u[(i * Q + j) * Q + m];
        }
        const int p = (i * Q + j) * Q + k;
        gx[p] = metric[0] * dr + metric[3] * ds + metric[6] * dt;
        gy[p] = metric[1] * dr + metric[4] * ds + metric[7] * dt;
        gz[p] = metric[2] * dr + metric[5] * ds + metric[8] * dt;
      }
}

// Field::norm of each field: Linf, L2, H1 (area-normalised).
void field_norms(const HostMesh &hm, const Tables1D &t, int nf, const double *modes, double *out /* nf x 3 */) {
  const int dim = hm.dim, L = t.L, Q = t.Q, ld = dim == 2 ? L * L : L * L * L, qd = dim == 2 ? Q * Q : Q * Q * Q;
  std::vector<double> u(qd), gx(qd), gy(qd), gz(qd, 0.0), wq(qd);
  for (int p = 0; p < qd; ++p) {
    const int i = dim == 2 ? p / Q : p / (Q * Q), j = dim == 2 ? p % Q : (p / Q) % Q, k = p % Q;
    wq[p] = t.w[i] * t.w[j] * (dim == 3 ? t.w[k] : 1.0);
  }
  for (int n = 0; n < nf; ++n) {
    double linf = 0.0, l2 = 0.0, h1 = 0.0, area = 0.0;
    for (int e = 0; e < hm.ne; ++e) {
      const GeomClass &gc = hm.classes[hm.gclass[e]];
      element_values(t, dim, modes + ((size_t)n * hm.ne + e) * ld, gc.metric, u.data(), gx.data(), gy.data(),
                     gz.data());
      for (int p = 0; p < qd; ++p) {
        const double wj = wq[p] * gc.J;
        linf = std::max(linf, std::fabs(u[p]));
        l2 += wj * u[p] * u[p];
        h1 += wj * (u[p] * u[p] + gx[p] * gx[p] + gy[p] * gy[p] + (dim == 3 ? gz[p] * gz[p] : 0.0));
        area += wj;
      }
    }
    out[3 * n + 0] = linf;
    out[3 * n + 1] = std::sqrt(std::fabs(l2 / area));
    out[3 * n + 2] = std::sqrt(std::fabs(h1 / area));
  }
}

}  // namespace

extern "C" {

dgmx_status dgmx_restart_write(const char *path, int physics, int ne, int nmodes, int step, double t, double dt,
                               double vis, const double *modes) {
  if (!path || !modes || ne <= 0 || nmodes <= 0) return DGMX_ERR_ARGUMENT;
  const int nf = nfields_of(physics), nsd = dim_of(physics);
  if (nf <= 0) return DGMX_ERR_ARGUMENT;
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) { g_restart_error = std::string("restart: cannot create ") + path; return DGMX_ERR_IO; }
  const size_t W = 40;
  char now[64];
  const std::time_t tp = std::time(nullptr);
  std::strftime(now, sizeof(now), "%a %b %d %H:%M:%S %Y", std::localtime(&tp));
  std::string name(path);
  const size_t slash = name.find_last_of('/');
  if (slash != std::string::npos) name = name.substr(slash + 1);
  if (name.size() > W) name = name.substr(name.size() - W);
  f << pad("dgmx", W) << " Session\n";
  f << pad(now, W) << " Created\n";
  f << pad(name, W) << " Name\n";
  f << pad(str(ne), W / 3) << pad(str(nsd), W / 3) << pad(str(nmodes), W / 3) << " Nel, Nsd, Lmax\n";
  f << pad(str(step), W) << " Step\n";
  f << pad(str(t), W) << " Time\n";
  f << pad(str(dt), W) << " Time step\n";
  f << pad(str(vis), W) << " Viscosity\n";
  std::string names;
  for (int k = 0; k < nf; ++k) names += pad(field_names(physics, k), std::max<size_t>(W / nf, 2));
  if ((W / nf) * nf < W) names += " ";
  f << names << " Field names\n";
  f << pad("Normalized", W) << " Format\n";
  for (int n = 0; n < nf; ++n) {
    const int32_t glen = (int32_t)((long long)ne * nmodes);
    f.write(reinterpret_cast<const char *>(&glen), 4);
    std::vector<int32_t> nm(ne, nmodes), disp(ne);
    for (int e = 0; e < ne; ++e) disp[e] = e * nmodes;
    f.write(reinterpret_cast<const char *>(nm.data()), 4 * (std::streamsize)ne);
    f.write(reinterpret_cast<const char *>(disp.data()), 4 * (std::streamsize)ne);
    f.write(reinterpret_cast<const char *>(modes + (size_t)n * ne * nmodes), 8 * (std::streamsize)ne * nmodes);
  }
  if (!f) { g_restart_error = std::string("restart: write failed on ") + path; return DGMX_ERR_IO; }
  return DGMX_OK;
}

dgmx_status dgmx_restart_info(const char *path, int *ne, int *nsd, int *lmax, int *step, double *t, double *dt,
                              double *vis) {
  if (!path) return DGMX_ERR_ARGUMENT;
  std::ifstream f(path, std::ios::binary);
  if (!f) { g_restart_error = std::string("restart: cannot open ") + path; return DGMX_ERR_IO; }
  Header h;
  if (!read_header(f, h)) return DGMX_ERR_IO;
  if (ne) *ne = h.ne;
  if (nsd) *nsd = h.nsd;
  if (lmax) *lmax = h.lmax;
  if (step) *step = h.step;
  if (t) *t = h.t;
  if (dt) *dt = h.dt;
  if (vis) *vis = h.vis;
  return DGMX_OK;
}

dgmx_status dgmx_restart_read(const char *path, int nf, int ne, int *nmodes, double *modes, long long cap) {
  if (!path || !nmodes || !modes || nf <= 0 || ne <= 0) return DGMX_ERR_ARGUMENT;
  Header h;
  std::vector<int> nm;
  std::vector<double> m;
  if (!read_file(path, nf, h, nm, m)) return DGMX_ERR_IO;
  if (h.ne != ne) { g_restart_error = "restart: element count differs from the caller's"; return DGMX_ERR_ARGUMENT; }
  if ((long long)m.size() > cap) { g_restart_error = "restart: output array too small"; return DGMX_ERR_ARGUMENT; }
  std::copy(nm.begin(), nm.end(), nmodes);
  std::copy(m.begin(), m.end(), modes);
  return DGMX_OK;
}

dgmx_status dgmx_restart_diff(const dgmx_mesh *mesh, int physics, const char *rst1, const char *rst2, double aeps,
                              double reps, double *norms, int *status) {
  if (!mesh || !rst1 || !rst2 || !status || !mesh->porder) return DGMX_ERR_ARGUMENT;
  if (aeps < 0 && reps < 0) { g_restart_error = "diff: no tests requested"; return DGMX_ERR_ARGUMENT; }
  try {
    const int nf = nfields_of(physics);
    const int p = mesh->porder[0], q = (mesh->qorder && mesh->qorder[0]) ? mesh->qorder[0] : p + 2;
    for (int e = 0; e < mesh->ne; ++e)
      if (mesh->porder[e] != p || ((mesh->qorder && mesh->qorder[e]) ? mesh->qorder[e] : mesh->porder[e] + 2) != q) {
        g_restart_error = "diff: one polynomial order per mesh";
        return DGMX_ERR_UNSUPPORTED;
      }
    const Tables1D tab = make_tables(p + 1, q, q - 1);
    HostMesh hm;
    std::string err;
    if (!build_mesh(*mesh, tab, hm, err)) { g_restart_error = err; return DGMX_ERR_ARGUMENT; }
    const int ld = mesh->dim == 2 ? (p + 1) * (p + 1) : (p + 1) * (p + 1) * (p + 1);
    Header h1, h2;
    std::vector<int> n1, n2;
    std::vector<double> m1, m2;
    if (!read_file(rst1, nf, h1, n1, m1) || !read_file(rst2, nf, h2, n2, m2)) return DGMX_ERR_IO;
    if (h1.ne != mesh->ne || h2.ne != mesh->ne) { g_restart_error = "diff: element count differs from the mesh"; return DGMX_ERR_ARGUMENT; }
    for (int e = 0; e < mesh->ne; ++e)
      if (n1[e] != ld || n2[e] != ld) { g_restart_error = "diff: mode count differs from the mesh order"; return DGMX_ERR_ARGUMENT; }
    std::vector<double> d(m1.size());
    for (size_t k = 0; k < d.size(); ++k) d[k] = m1[k] - m2[k];
    std::vector<double> r(3 * nf), x(3 * nf);
    field_norms(hm, tab, nf, m1.data(), r.data());
    field_norms(hm, tab, nf, d.data(), x.data());
    const double repsM = std::sqrt(std::numeric_limits<double>::epsilon());
    int st = 0;
    for (int n = 0; n < nf; ++n) {
      const double *a = &x[3 * n], *b = &r[3 * n];
      if (aeps >= 0)
        for (int k = 0; k < 3; ++k)
          if (a[k] > aeps || std::isnan(a[k])) st |= 1 << k;            // Linf, L2, H1 failed
      if (reps >= 0)
        for (int k = 0; k < 3; ++k)
          if (b[k] > repsM || std::isnan(b[k]))
            if (a[k] / b[k] > reps || std::isnan(a[k] / b[k])) st |= 8 << k;   // relative
      if (norms)
        for (int k = 0; k < 3; ++k) { norms[6 * n + k] = a[k]; norms[6 * n + 3 + k] = b[k]; }
    }
    *status = st;
    return DGMX_OK;
  } catch (...) {
    g_restart_error = "diff: host allocation failed";
    return DGMX_ERR_MEMORY;
  }
}

const char *dgmx_restart_last_error(void) { return g_restart_error.c_str(); }

}  // extern "C"
