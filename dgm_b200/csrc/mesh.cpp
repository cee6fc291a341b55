// Host mesh processing for the B200 engine: connectivity, side orientation,
// affine geometry and geometry classes; readers for DGM's input files.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "dgmx_internal.hpp"

namespace dgmx {
namespace {

// Quad edge-flip table (src/Field.cpp:87-90): flip when the linked edges
// run in the same local sense.
const int kQuadFlip[4][4] = {{1, 1, 0, 0}, {1, 1, 0, 0}, {0, 0, 1, 1}, {0, 0, 1, 1}};
// Hex face vertices (src/Hex.cpp:68-69)
const int kHexFace[6][4] = {{0, 1, 2, 3}, {0, 1, 5, 4}, {1, 2, 6, 5},
                            {3, 2, 6, 7}, {0, 3, 7, 4}, {4, 5, 6, 7}};

struct SideInfo {
  bool master = false;
  int le = -1, ls = -1;
  bool flip_a = false, flip_b = false, transp = false;
  int bc = 0;           // boundary type (0: interior side)
};

// Side point index map with flips and transpose (src/BaseQuad.hpp:53-57,
// src/BaseHex.hpp:291-308); n1 x n2 Gauss points on the side.
int side_map(int dim, const SideInfo &s, int n1, int n2, int q) {
  if (dim == 2) return s.flip_a ? (n1 - 1) - q : q;
  const int il = q / n2, jl = q % n2;
  int i, j;
  if (s.transp) {
    j = il; i = jl;
    if (s.flip_a) j = (n1 - 1) - j;
    if (s.flip_b) i = (n2 - 1) - i;
  } else {
    i = il; j = jl;
    if (s.flip_a) i = (n1 - 1) - i;
    if (s.flip_b) j = (n2 - 1) - j;
  }
  return j + n2 * i;
}

void unit_diff(const double *p, const double *q, double *o) {
  o[0] = p[0] - q[0]; o[1] = p[1] - q[1]; o[2] = p[2] - q[2];
  const double n = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
  o[0] /= n; o[1] /= n; o[2] /= n;
}
double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

}  // namespace

bool build_mesh(const dgmx_mesh &m, const Tables1D &t, HostMesh &out, std::string &err,
                const std::vector<BoundarySide> *bcs) {
  const int dim = m.dim, ne = m.ne;
  if ((dim != 2 && dim != 3) || ne <= 0 || !m.verts || !m.con || m.ncon <= 0) {
    err = "mesh: dim must be 2 or 3 and verts/con must be given";
    return false;
  }
  const int nv = dim == 2 ? 4 : 8, nfaces = dim == 2 ? 4 : 6;
  out.dim = dim; out.ne = ne; out.nfaces = nfaces;
  out.L = t.L; out.Q = t.Q; out.G = t.G; out.p = t.L - 1;
  out.gf = dim == 2 ? t.G : t.G * t.G;
  const int Q = t.Q, gf = out.gf;

  // --- connectivity: the first record naming a pair makes its side master
  std::vector<SideInfo> side((size_t)ne * nfaces);
  for (int c = 0; c < m.ncon; ++c) {
    const int e = m.con[4 * c], s = m.con[4 * c + 1], le = m.con[4 * c + 2], ls = m.con[4 * c + 3];
    if (e < 0 || e >= ne || le < 0 || le >= ne || s < 0 || s >= nfaces || ls < 0 || ls >= nfaces) {
      err = "mesh: connectivity record " + std::to_string(c) + " out of range";
      return false;
    }
    SideInfo &nb = side[(size_t)le * nfaces + ls];
    if (nb.master) {
      if (nb.le != e || nb.ls != s) { err = "mesh: contradictory side links"; return false; }
      continue;
    }
    SideInfo &me = side[(size_t)e * nfaces + s];
    me.master = true; me.le = le; me.ls = ls;
    nb.master = false; nb.le = e; nb.ls = s;
  }
  // --- boundary sides (src/Field.cpp:4440-4460): the record replaces the
  // side's link; the side becomes master with no flips
  if (bcs && !bcs->empty()) {
    for (const BoundarySide &b : *bcs) {
      if (b.e < 0 || b.e >= ne || b.s < 0 || b.s >= nfaces || b.type < 1 || b.type > kMaxBcTypes) {
        err = "mesh: boundary record out of range";
        return false;
      }
      SideInfo &S = side[(size_t)b.e * nfaces + b.s];
      if (S.bc) { err = "mesh: element " + std::to_string(b.e) + " side " + std::to_string(b.s) + " named twice"; return false; }
      S.bc = b.type;
    }
    for (const BoundarySide &b : *bcs) {
      const SideInfo &S = side[(size_t)b.e * nfaces + b.s];
      if (S.le >= 0 && !side[(size_t)S.le * nfaces + S.ls].bc) {
        err = "mesh: boundary side " + std::to_string(b.e) + ":" + std::to_string(b.s) +
              " is linked to an interior side";
        return false;
      }
    }
    for (const BoundarySide &b : *bcs) {
      SideInfo &S = side[(size_t)b.e * nfaces + b.s];
      S.master = true; S.le = -1; S.ls = -1;
      S.flip_a = S.flip_b = S.transp = false;
    }
  }
  for (size_t i = 0; i < side.size(); ++i)
    if (side[i].le < 0 && !side[i].bc) {
      err = "mesh: element " + std::to_string(i / nfaces) + " side " + std::to_string(i % nfaces) +
            " has no neighbour and no boundary condition";
      return false;
    }

  auto X = [&](int e, int v, int c) { return m.verts[((size_t)e * nv + v) * 3 + c]; };

  // --- orientation flags on master sides (src/Field.cpp:416-680)
  for (int e = 0; e < ne; ++e)
    for (int s = 0; s < nfaces; ++s) {
      SideInfo &S = side[(size_t)e * nfaces + s];
      if (!S.master || S.bc) continue;
      if (dim == 2) { S.flip_a = kQuadFlip[s][S.ls] != 0; continue; }
      const int *f0 = kHexFace[s], *f1 = kHexFace[S.ls];
      double A[4][3], B[4][3];
      for (int v = 0; v < 4; ++v)
        for (int c = 0; c < 3; ++c) { A[v][c] = X(e, f0[v], c); B[v][c] = X(S.le, f1[v], c); }
      double a0[3], b0[3], a1[3], b1[3], a1p[3];
      unit_diff(A[1], A[0], a0); unit_diff(A[3], A[0], b0);
      unit_diff(B[1], B[0], a1); unit_diff(B[3], B[0], b1); unit_diff(B[2], B[3], a1p);
      const double a0a1 = dot3(a0, a1), a0a1p = dot3(a0, a1p);
      auto unit = [](double v) { return std::fabs(std::fabs(v) - 1.0) < 1e-8; };
      if (unit(a0a1) || unit(a0a1p)) {
        S.flip_a = a0a1 < 0; S.flip_b = dot3(b0, b1) < 0;
      } else {
        S.transp = true; S.flip_a = dot3(b0, a1) < 0; S.flip_b = dot3(a0, b1) < 0;
      }
    }

  // --- per-element affine geometry
  struct ElemGeo { double metric[9]; double J; double nrm[6][3]; double jr[6]; };
  std::vector<ElemGeo> geo(ne);
  out.J.resize(ne);
  const size_t qd = dim == 2 ? (size_t)Q * Q : (size_t)Q * Q * Q;
  out.cx.assign(qd * ne, 0.0); out.cy.assign(qd * ne, 0.0); out.cz.assign(qd * ne, 0.0);
  for (int e = 0; e < ne; ++e) {
    ElemGeo &g = geo[e];
    std::memset(&g, 0, sizeof(g));
    if (dim == 2) {
      const double xr = (X(e, 1, 0) - X(e, 0, 0)) * 0.5, xs = (X(e, 3, 0) - X(e, 0, 0)) * 0.5;
      const double yr = (X(e, 1, 1) - X(e, 0, 1)) * 0.5, ys = (X(e, 3, 1) - X(e, 0, 1)) * 0.5;
      const double J = xr * ys - xs * yr;
      if (!(J > 0.0)) { err = "mesh: element " + std::to_string(e) + " has a non-positive Jacobian"; return false; }
      g.J = J;
      g.metric[0] = ys / J; g.metric[1] = -xs / J;     // rx ry
      g.metric[3] = -yr / J; g.metric[4] = xr / J;     // sx sy
      // edges: 0 y-, 1 x+, 2 y+, 3 x-  (src/Quad.cpp:1367-1455)
      const double *rowr = &g.metric[0], *rows = &g.metric[3];
      for (int s = 0; s < 4; ++s) {
        const double *row = (s == 0 || s == 2) ? rows : rowr;
        const double sg = (s == 0 || s == 3) ? -1.0 : 1.0;
        const double len = std::sqrt(row[0] * row[0] + row[1] * row[1]);
        g.nrm[s][0] = sg * row[0] / len; g.nrm[s][1] = sg * row[1] / len;
        const double tx = (s == 0 || s == 2) ? xr : xs, ty = (s == 0 || s == 2) ? yr : ys;
        g.jr[s] = std::sqrt(tx * tx + ty * ty) / J;
      }
      for (int i = 0; i < Q; ++i)
        for (int j = 0; j < Q; ++j) {
          const double pa0 = 0.5 * (1.0 - t.z[i]), pa1 = 0.5 * (1.0 + t.z[i]);
          const double pb0 = 0.5 * (1.0 - t.z[j]), pb1 = 0.5 * (1.0 + t.z[j]);
          const double w[4] = {pa0 * pb0, pa1 * pb0, pa1 * pb1, pa0 * pb1};
          double x = 0, y = 0;
          for (int v = 0; v < 4; ++v) { x += X(e, v, 0) * w[v]; y += X(e, v, 1) * w[v]; }
          out.cx[(size_t)e * qd + i * Q + j] = x;
          out.cy[(size_t)e * qd + i * Q + j] = y;
        }
    } else {
      double d[3][3];  // d[c][0]=x_r-ish: d[c][k] = (X(v_k) - X(v_0))/2 for k = r,s,t
      const int vk[3] = {1, 3, 4};
      for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) d[c][k] = (X(e, vk[k], c) - X(e, 0, c)) * 0.5;
      const double xr = d[0][0], xs = d[0][1], xt = d[0][2];
      const double yr = d[1][0], ys = d[1][1], yt = d[1][2];
      const double zr = d[2][0], zs = d[2][1], zt = d[2][2];
      const double J = xr * ys * zt + yr * zs * xt + zr * xs * yt - xt * ys * zr - zt * xs * yr - xr * zs * yt;
      if (!(J > 0.0)) { err = "mesh: element " + std::to_string(e) + " has a non-positive Jacobian"; return false; }
      g.J = J;
      g.metric[0] = (ys * zt - yt * zs) / J;  g.metric[1] = -(xs * zt - xt * zs) / J; g.metric[2] = (xs * yt - xt * ys) / J;
      g.metric[3] = -(yr * zt - yt * zr) / J; g.metric[4] = (xr * zt - xt * zr) / J;  g.metric[5] = -(xr * yt - xt * yr) / J;
      g.metric[6] = (yr * zs - ys * zr) / J;  g.metric[7] = -(xr * zs - xs * zr) / J; g.metric[8] = (xr * ys - xs * yr) / J;
      // faces: 0 t-, 1 s-, 2 r+, 3 s+, 4 r-, 5 t+  (src/Hex.cpp:1385-1497)
      const int row_of[6] = {2, 1, 0, 1, 0, 2};
      const double sgn[6] = {-1, -1, 1, 1, -1, 1};
      const double tr[3][3] = {{xr, yr, zr}, {xs, ys, zs}, {xt, yt, zt}};
      const int ta[6][2] = {{0, 1}, {0, 2}, {1, 2}, {0, 2}, {1, 2}, {0, 1}};
      for (int s = 0; s < 6; ++s) {
        const double *row = &g.metric[3 * row_of[s]];
        const double len = std::sqrt(row[0] * row[0] + row[1] * row[1] + row[2] * row[2]);
        for (int c = 0; c < 3; ++c) g.nrm[s][c] = sgn[s] * row[c] / len;
        const double *u = tr[ta[s][0]], *v = tr[ta[s][1]];
        const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
        g.jr[s] = std::sqrt(cx * cx + cy * cy + cz * cz) / J;
      }
      for (int i = 0; i < Q; ++i)
        for (int j = 0; j < Q; ++j)
          for (int k = 0; k < Q; ++k) {
            const double pa[2] = {0.5 * (1.0 - t.z[i]), 0.5 * (1.0 + t.z[i])};
            const double pb[2] = {0.5 * (1.0 - t.z[j]), 0.5 * (1.0 + t.z[j])};
            const double pc[2] = {0.5 * (1.0 - t.z[k]), 0.5 * (1.0 + t.z[k])};
            static const int va[8] = {0, 1, 1, 0, 0, 1, 1, 0}, vb[8] = {0, 0, 1, 1, 0, 0, 1, 1},
                             vc[8] = {0, 0, 0, 0, 1, 1, 1, 1};
            double x = 0, y = 0, z = 0;
            for (int v = 0; v < 8; ++v) {
              const double w = pa[va[v]] * pb[vb[v]] * pc[vc[v]];
              x += X(e, v, 0) * w; y += X(e, v, 1) * w; z += X(e, v, 2) * w;
            }
            const size_t q = (size_t)e * qd + (i * Q + j) * Q + k;
            out.cx[q] = x; out.cy[q] = y; out.cz[q] = z;
          }
    }
    out.J[e] = g.J;
  }

  // --- links and point permutations
  out.links.assign((size_t)ne * nfaces, FaceLink{0, 0, 0, 0});
  out.perm.clear();
  std::map<std::vector<int>, int> perm_ids;
  const int n1 = t.G, n2 = dim == 2 ? 1 : t.G;
  for (int e = 0; e < ne; ++e)
    for (int s = 0; s < nfaces; ++s) {
      const SideInfo &S = side[(size_t)e * nfaces + s];
      std::vector<int> p(gf);
      if (S.master) {
        // master point side_map(S, q) pairs with the slave's point q
        for (int q = 0; q < gf; ++q) p[side_map(dim, S, n1, n2, q)] = q;
      } else {
        const SideInfo &M = side[(size_t)S.le * nfaces + S.ls];
        for (int q = 0; q < gf; ++q) p[q] = side_map(dim, M, n1, n2, q);
      }
      auto it = perm_ids.find(p);
      int off;
      if (it == perm_ids.end()) {
        off = (int)out.perm.size();
        out.perm.insert(out.perm.end(), p.begin(), p.end());
        perm_ids[p] = off;
      } else {
        off = it->second;
      }
      // a boundary side points at itself (identity order); its neighbour
      // state is made from its own trace
      out.links[(size_t)e * nfaces + s] = S.bc ? FaceLink{e, s, off, 0} : FaceLink{S.le, S.ls, off, 0};
    }

  // --- geometry classes
  std::map<std::string, int> class_ids;
  out.gclass.resize(ne);
  out.classes.clear();
  for (int e = 0; e < ne; ++e) {
    GeomClass c;
    std::memset(&c, 0, sizeof(c));
    std::memcpy(c.metric, geo[e].metric, sizeof(c.metric));
    c.J = geo[e].J;
    for (int s = 0; s < nfaces; ++s) {
      const SideInfo &S = side[(size_t)e * nfaces + s];
      const double *n = S.master ? geo[e].nrm[s] : geo[S.le].nrm[S.ls];
      c.bc |= S.bc << (4 * s);
      for (int k = 0; k < 3; ++k) c.nrm[s][k] = n[k];
      for (int k = 0; k < 3; ++k) c.onrm[s][k] = geo[e].nrm[s][k];
      c.jr[s] = geo[e].jr[s];
      if (dim == 3) face_frame(c.nrm[s], c.fr[s]);
      if (S.master) c.master |= 1 << s;
    }
    std::string key(reinterpret_cast<const char *>(&c), sizeof(c));
    auto it = class_ids.find(key);
    if (it == class_ids.end()) {
      const int id = (int)out.classes.size();
      out.classes.push_back(c);
      class_ids[key] = id;
      out.gclass[e] = id;
    } else {
      out.gclass[e] = it->second;
    }
    out.links[(size_t)e * nfaces].cls = out.gclass[e];
  }
  return true;
}

// ---------------------------------------------------------------- partitions
bool partition_mesh(const HostMesh &g, const int *part, int nranks, int rank, HostMesh &local, PartitionPlan &plan,
                    std::string &err) {
  const int ne = g.ne, nf = g.nfaces;
  if (nranks < 1 || rank < 0 || rank >= nranks) { err = "partition: rank out of range"; return false; }
  for (int e = 0; e < ne; ++e)
    if (part[e] < 0 || part[e] >= nranks) { err = "partition: element " + std::to_string(e) + " has no rank"; return false; }
  plan = PartitionPlan();
  plan.nranks = nranks; plan.rank = rank;
  std::vector<int> local_of(ne, -1), ghost_of(ne, -1);
  for (int e = 0; e < ne; ++e)
    if (part[e] == rank) { local_of[e] = (int)plan.global_of_local.size(); plan.global_of_local.push_back(e); }
  plan.ne_local = (int)plan.global_of_local.size();
  if (!plan.ne_local) { err = "partition: rank " + std::to_string(rank) + " owns no element"; return false; }
  // ghosts: remote neighbours of local faces, in global order
  std::vector<char> need(ne, 0);
  for (int e : plan.global_of_local)
    for (int f = 0; f < nf; ++f) {
      const FaceLink &l = g.links[(size_t)e * nf + f];
      if (part[l.elem] != rank) need[l.elem] = 1;
    }
  for (int e = 0; e < ne; ++e)
    if (need[e]) { ghost_of[e] = plan.ne_local + (int)plan.global_of_ghost.size(); plan.global_of_ghost.push_back(e); }
  plan.nghost = (int)plan.global_of_ghost.size();
  // local mesh: the rank's elements, links remapped to local indices or ghost slots
  local = HostMesh();
  local.dim = g.dim; local.ne = plan.ne_local; local.p = g.p; local.L = g.L; local.Q = g.Q; local.G = g.G;
  local.nfaces = nf; local.gf = g.gf;
  local.classes = g.classes;
  local.perm = g.perm;
  const size_t qd = g.cx.size() / (size_t)ne;
  for (int e : plan.global_of_local) {
    local.gclass.push_back(g.gclass[e]);
    local.J.push_back(g.J[e]);
    local.cx.insert(local.cx.end(), g.cx.begin() + (size_t)e * qd, g.cx.begin() + (size_t)(e + 1) * qd);
    local.cy.insert(local.cy.end(), g.cy.begin() + (size_t)e * qd, g.cy.begin() + (size_t)(e + 1) * qd);
    local.cz.insert(local.cz.end(), g.cz.begin() + (size_t)e * qd, g.cz.begin() + (size_t)(e + 1) * qd);
    for (int f = 0; f < nf; ++f) {
      FaceLink l = g.links[(size_t)e * nf + f];
      l.elem = part[l.elem] == rank ? local_of[l.elem] : ghost_of[l.elem];
      l.cls = f == 0 ? g.gclass[e] : 0;
      local.links.push_back(l);
    }
  }
  // exchange lists, ordered by the global (element, face) of the block
  plan.send.assign(nranks, {});
  plan.recv.assign(nranks, {});
  for (int e : plan.global_of_local)
    for (int f = 0; f < nf; ++f) {
      const FaceLink &l = g.links[(size_t)e * nf + f];
      const int q = part[l.elem];
      if (q == rank) continue;
      // q needs this face's trace (the neighbour side of its face l)
      plan.send[q].push_back(local_of[e] * nf + f);
      plan.recv[q].push_back(ghost_of[l.elem] * nf + l.face);
    }
  auto gkey = [&](int v, bool ghost) {
    const int slot = v / nf, f = v % nf;
    const int ge = ghost ? plan.global_of_ghost[slot - plan.ne_local] : plan.global_of_local[slot];
    return (long long)ge * nf + f;
  };
  for (int q = 0; q < nranks; ++q) {
    std::sort(plan.send[q].begin(), plan.send[q].end(),
              [&](int a, int b) { return gkey(a, false) < gkey(b, false); });
    std::sort(plan.recv[q].begin(), plan.recv[q].end(),
              [&](int a, int b) { return gkey(a, true) < gkey(b, true); });
  }
  return true;
}

// ---------------------------------------------------------------- file input
namespace {
std::string lower(std::string s) {
  for (auto &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}
}  // namespace

bool read_case_files(const std::string &root, FileCase &fc, std::string &err) {
  // root.inp: "key = value" lines, '#' comments (src/Domain.cpp:294)
  {
    std::ifstream in(root + ".inp");
    if (!in) { err = "cannot open " + root + ".inp"; return false; }
    std::string line;
    while (std::getline(in, line)) {
      line = line.substr(0, line.find('#'));
      const size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      std::string k = line.substr(0, eq), v = line.substr(eq + 1);
      std::stringstream ks(k), vs(v);
      ks >> k;
      vs >> v;
      if (k == "eqntype") fc.eqntype = std::stoi(v);
      else if (k == "inttype") fc.inttype = std::stoi(v);
      else if (k == "p") fc.p = std::stoi(v);
      else if (k == "q") fc.q = std::stoi(v);
      else if (k == "gamma") fc.gamma = std::stod(v);
      else if (k == "vis") fc.vis = std::stod(v);
      else if (k == "Pr") fc.Pr = std::stod(v);
      else if (k == "flux") fc.flux = lower(v);
    }
    if (fc.p < 0) { err = root + ".inp: no polynomial order p"; return false; }
  }
  // root.msh (src/Field.cpp:2271-2600)
  {
    std::ifstream in(root + ".msh");
    if (!in) { err = "cannot open " + root + ".msh"; return false; }
    std::string line;
    std::getline(in, line);
    if (!(in >> fc.ne >> fc.dim)) { err = root + ".msh: cannot read ne nsd"; return false; }
    std::getline(in, line);
    if (fc.dim != 2 && fc.dim != 3) { err = root + ".msh: nsd must be 2 or 3"; return false; }
    const int nv = fc.dim == 2 ? 4 : 8;
    fc.verts.assign((size_t)fc.ne * nv * 3, 0.0);
    for (int e = 0; e < fc.ne; ++e) {
      std::string type;
      std::getline(in, type);
      const std::string lt = lower(type);
      const bool ok = fc.dim == 2 ? (lt.find("quad") != std::string::npos && lt.find("nodal") == std::string::npos &&
                                     lt.find("spectral") == std::string::npos)
                                  : (lt.find("hex") != std::string::npos && lt.find("nodal") == std::string::npos &&
                                     lt.find("spectral") == std::string::npos);
      if (!ok) { err = root + ".msh: element type '" + type + "' is not a modal Quad/Hex"; return false; }
      for (int c = 0; c < fc.dim; ++c) {
        for (int v = 0; v < nv; ++v)
          if (!(in >> fc.verts[((size_t)e * nv + v) * 3 + c])) { err = root + ".msh: short element"; return false; }
        std::getline(in, line);
      }
    }
  }
  // root.con (src/Field.cpp:3478-3540)
  {
    std::ifstream in(root + ".con");
    if (!in) { err = "cannot open " + root + ".con"; return false; }
    std::string line;
    std::getline(in, line);
    std::getline(in, line);
    char type;
    int e, s, le, ls;
    while (in >> type >> e >> s >> le >> ls) {
      fc.con.insert(fc.con.end(), {e, s, le, ls});
      std::getline(in, line);
    }
  }
  // root.ord (optional, src/Field.cpp:2295-2322)
  fc.porder.assign(fc.ne, fc.p);
  fc.qorder.assign(fc.ne, fc.q ? fc.q : fc.p + 2);
  {
    std::ifstream in(root + ".ord");
    if (in) {
      std::string line;
      std::getline(in, line);
      int e, pl, ql;
      while (in >> e >> pl >> ql) {
        if (e < 0 || e >= fc.ne) { err = root + ".ord: bad element id"; return false; }
        fc.porder[e] = pl;
        fc.qorder[e] = ql ? ql : pl + 2;
        std::getline(in, line);
      }
    }
  }
  // root.bc (optional): a header line, the count, then `type eid sid`
  // records (src/Field.cpp:4469-4490, src/Boundary.cpp:83-87)
  {
    std::ifstream in(root + ".bc");
    if (in) {
      std::string line;
      std::getline(in, line);
      int nbc = 0;
      while (std::getline(in, line)) {
        std::stringstream ls(line);
        if (ls >> nbc) break;
      }
      for (int i = 0; i < nbc; ++i) {
        FileCase::BcRecord r;
        if (!(in >> r.tag >> r.e >> r.s)) { err = root + ".bc: short record"; return false; }
        if (r.e < 0 || r.e >= fc.ne) { err = root + ".bc: bad element id"; return false; }
        std::getline(in, line);
        fc.bcs.push_back(r);
      }
    }
  }
  // root.bct (optional): `Code Tag { values }` blocks
  // (src/Navier_Stokes3d.cpp:416-455; braces scanned as src/BC.hpp:159)
  {
    std::ifstream in(root + ".bct");
    if (in) {
      std::string code, tag, tok;
      while (in >> code >> tag) {
        std::vector<double> vals;
        if (in >> tok && tok == "{") {
          while (in >> tok && tok != "}") vals.push_back(std::stod(tok));
        }
        fc.bct[tag] = {lower(code), vals};
      }
    }
  }
  // root.chn (optional): its presence makes Euler3d build a Channel
  // (src/Euler3d.cpp:75-77, src/Channel.hpp:40-70)
  fc.channel = static_cast<bool>(std::ifstream(root + ".chn"));
  return true;
}

}  // namespace dgmx
