// Element pools: many independent DG solves advanced together on one GPU.
//
// Solves of equal (physics, p, q) live in one arena: one set of
// element-major device arrays (modal registers, double-buffered face traces,
// geometry classes, face links) in which each solve owns a contiguous,
// tile-aligned range of element slots.  Face links of a solve point inside
// its own range, so the ordinary stage kernel advances every solve of the
// arena at once; a device-side tile list selects the live tiles, and the
// kernel runs persistently over it, so the per-step CUDA graph of an arena
// (14 LSRK stages) stays valid while solves join and leave.  Each solve
// carries its own step (dts[solve]) and, in the mixed form, its own
// reference state (uref[solve]).
//
// The 2-D arenas (Euler 2-D and shallow water, p = 1..7, q = p + 2) are
// advanced together by default: one persistent launch of the fused
// multi-order stage kernel (fused.cuh) per LSRK stage walks a device-side
// list of (arena, tile) work items, so a step of any mix of orders is 14
// launches, replayed from one CUDA graph.  Other arenas (3-D Euler, other q)
// keep their own per-arena launches.
//
// Per solve the arithmetic is exactly dgmx_advance's with inttype 14
// (src/TimeInt.cpp:1989-2013); the last step is shortened to end on t_end.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/dgmx_pool.h"
#include "dgmx_internal.hpp"

using namespace dgmx;

namespace {

template <class T>
cudaError_t dalloc(T **p, size_t n) {
  return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * (n ? n : 1));
}

// ---------------------------------------------------------------- autotuning
// Tile variant per (kernel key, L, Q), chosen once per process by timing the
// stage kernel of every registered variant on a periodic box of ~4k
// elements in a uniform flow.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tuned;

void box_mesh(int dim, int n, std::vector<double> &verts, std::vector<int> &con) {
  const int ne = dim == 2 ? n * n : n * n * n, nv = dim == 2 ? 4 : 8, nf = 2 * dim;
  verts.assign((size_t)ne * nv * 3, 0.0);
  con.assign((size_t)ne * nf * 4, 0);
  const double h = 1.0 / n;
  static const int c2[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
  static const int c3[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  auto wrap = [n](int a) { return (a + n) % n; };
  for (int e = 0; e < ne; ++e) {
    const int i = e % n, j = (e / n) % n, k = dim == 3 ? e / (n * n) : 0;
    for (int v = 0; v < nv; ++v) {
      const int *c = dim == 2 ? c2[v] : c3[v];
      verts[((size_t)e * nv + v) * 3 + 0] = (i + c[0]) * h;
      verts[((size_t)e * nv + v) * 3 + 1] = (j + c[1]) * h;
      if (dim == 3) verts[((size_t)e * nv + v) * 3 + 2] = (k + c[2]) * h;
    }
    int nb[6], opp[6];
    if (dim == 2) {
      // Quad sides 0 y-, 1 x+, 2 y+, 3 x- (src/Quad.cpp:767-790)
      nb[0] = i + n * wrap(j - 1); nb[1] = wrap(i + 1) + n * j; nb[2] = i + n * wrap(j + 1); nb[3] = wrap(i - 1) + n * j;
      opp[0] = 2; opp[1] = 3; opp[2] = 0; opp[3] = 1;
    } else {
      // Hex sides 0 z-, 1 y-, 2 x+, 3 y+, 4 x-, 5 z+ (src/Hex.cpp:68-69)
      auto id = [&](int a, int b, int c) { return wrap(a) + n * (wrap(b) + n * wrap(c)); };
      nb[0] = id(i, j, k - 1); nb[1] = id(i, j - 1, k); nb[2] = id(i + 1, j, k);
      nb[3] = id(i, j + 1, k); nb[4] = id(i - 1, j, k); nb[5] = id(i, j, k + 1);
      opp[0] = 5; opp[1] = 3; opp[2] = 4; opp[3] = 1; opp[4] = 2; opp[5] = 0;
    }
    for (int s = 0; s < nf; ++s) {
      int *r = &con[((size_t)e * nf + s) * 4];
      r[0] = e; r[1] = s; r[2] = nb[s]; r[3] = opp[s];
    }
  }
}

// Returns the index into find_variants(key, L, Q) of the fastest tile, or
// -1 when timing failed (the default variant is used then).
int tuned_variant(int physics, bool mixed, int L, int Q, double gamma, int flux, int device) {
  const int key = physics + (mixed ? kMixedKey : 0);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find({key, L, Q});
  if (it != g_tuned.end()) return it->second;
  const int dim = dim_of(physics), nf = nfields_of(physics);
  const int n = dim == 2 ? 64 : 16;
  std::vector<double> verts;
  std::vector<int> con;
  box_mesh(dim, n, verts, con);
  const int ne = dim == 2 ? n * n : n * n * n;
  std::vector<int> po(ne, L - 1), qo(ne, Q);
  dgmx_mesh m{dim, ne, verts.data(), ne * 2 * dim, con.data(), po.data(), qo.data()};
  dgmx_params prm{physics, flux, DGMX_LSRK14, mixed ? DGMX_MIXED : DGMX_FP64, 0, device, gamma, 0.0, 0.72};
  dgmx_domain *d = nullptr;
  int chosen = -1;
  if (dgmx_create(&m, &prm, &d) == DGMX_OK) {
    long nfo = 0, nq = 0, nm = 0;
    dgmx_sizes(d, &nfo, &nq, &nm);
    std::vector<double> U((size_t)nf * nq);
    // uniform flow: rho 1, velocity (0.3, 0.2, 0.1), p 1 (shallow water: phi 1)
    const double st[5] = {1.0, 0.3, 0.2, dim == 3 ? 0.1 : 1.0 / (gamma - 1.0) + 0.5 * 0.13,
                          1.0 / (gamma - 1.0) + 0.5 * 0.14};
    for (int k = 0; k < nf; ++k) {
      const double v = physics == DGMX_SHALLOW ? (k == 0 ? 1.0 : 0.1 * k) : st[k];
      std::fill(U.begin() + (size_t)k * nq, U.begin() + (size_t)(k + 1) * nq, v);
    }
    int nv = 0;
    if (dgmx_set_state(d, U.data()) != DGMX_OK || dgmx_autotune(d, 10, nullptr, 0, &nv, &chosen) != DGMX_OK)
      chosen = -1;
    dgmx_destroy(d);
  }
  g_tuned[{key, L, Q}] = chosen;
  return chosen;
}

struct PoolSolve {
  int id = -1, arena = -1, slot = -1;
  int e0 = 0, ne = 0, nalloc = 0;    // elements [e0, e0 + ne) live, nalloc slots held
  double dt = 0.0, t = 0.0, t_end = 0.0;
  long steps = 0;
  bool finished = false;
};

struct Arena {
  int phys = 0, L = 0, Q = 0, dim = 0, nf = 0, nfaces = 0, gf = 0, ld = 0, qd = 0;
  bool mixed = false;
  int body = -1;                      // fused multi-order kernel body, -1: own launches
  Tables1D tab;
  const KernelOps *fops = nullptr;   // FP64 tile: projections
  const KernelOps *sops = nullptr;   // stage tile (FP64 or mixed)
  int epb = 1, grid = 1;
  int cap = 0, slot_cap = 0, class_cap = 0, perm_cap = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t uploaded = nullptr;
  double *U = nullptr, *Ut = nullptr, *T[2] = {nullptr, nullptr};
  float *Utf = nullptr, *Tf[2] = {nullptr, nullptr};
  int *gclass = nullptr, *esolve = nullptr, *perm = nullptr, *tiles = nullptr, *err = nullptr;
  GeomClass *classes = nullptr;
  FaceLink *links = nullptr;
  double *uref = nullptr, *dts = nullptr;
  // host side
  std::vector<GeomClass> classes_h;
  std::map<std::string, int> class_index;
  std::vector<int> perm_h;
  std::map<std::vector<int>, int> perm_index;
  std::map<int, int> free_ranges;     // start -> length, in elements (tile aligned)
  std::vector<int> free_slots;
  int next_slot = 0;
  std::vector<int> live;              // solve ids stepping in this arena
  bool tiles_dirty = true, dts_dirty = true;
  int *tiles_pin = nullptr;           // pinned: [0] = count, then tiles
  double *dts_pin = nullptr;          // pinned: one step per solve slot
  double *uref_pin = nullptr;         // pinned: kUrefStride doubles per solve slot
  cudaGraphExec_t graph = nullptr;
  int tcur = 0;

  size_t elem_bytes() const {
    const size_t m = (size_t)nf * ld, tr = (size_t)nfaces * nf * gf;
    size_t b = m * 8 + 4 + 4 + sizeof(FaceLink) * nfaces;
    b += mixed ? m * 4 + 2 * tr * 4 : m * 8 + 2 * tr * 8;
    return b;
  }
};

}  // namespace

struct dgmx_pool {
  dgmx_pool_params prm{};
  std::vector<std::unique_ptr<Arena>> arenas;
  std::map<int, PoolSolve> solves;
  std::vector<int> finished_queue;
  int next_id = 0;
  int nsm = 148;
  size_t bytes = 0;
  double *scratch = nullptr;          // nodal staging for projections
  size_t scratch_n = 0;
  long launches = 0;
  std::string errmsg;
  // fused multi-order stage kernel for the 2-D arenas
  bool fused_on = true, fused_ready = false, args_dirty = true, items_dirty = true;
  const FusedOps *fops = nullptr;
  cudaStream_t fstream = nullptr;
  cudaEvent_t fuploaded = nullptr;
  StageArgs *args_dev = nullptr, *args_pin = nullptr;   // [14][arenas]
  int args_cap = 0;                                     // arenas the table holds
  int *bodies_dev = nullptr, *bodies_pin = nullptr;
  int2 *items_dev = nullptr, *items_pin = nullptr;      // (arena, tile)
  int *nitems_dev = nullptr, *nitems_pin = nullptr;
  int items_cap = 0, fgrid = 1;
  cudaGraphExec_t fgraph = nullptr;
  bool unsynced = false;              // steps enqueued since the last sync

  dgmx_status fail(dgmx_status s, const std::string &m) { errmsg = m; return s; }
  dgmx_status cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return DGMX_OK;
    errmsg = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? DGMX_ERR_MEMORY : DGMX_ERR_CUDA;
  }
  bool fits(size_t more) const { return prm.budget_bytes == 0 || bytes + more <= prm.budget_bytes; }
};

namespace {

constexpr int kSlotCap = 16384;       // solves per arena
constexpr int kClassCap = 4096;       // geometry classes per arena
constexpr int kPermCap = 1 << 16;     // permutation entries per arena

void free_arena(Arena &a) {
  if (a.graph) cudaGraphExecDestroy(a.graph);
  a.graph = nullptr;
  void *dev[] = {a.U, a.Ut, a.T[0], a.T[1], a.Utf, a.Tf[0], a.Tf[1], a.gclass, a.esolve, a.perm,
                 a.tiles, a.err, a.classes, a.links, a.uref, a.dts};
  for (void *p : dev) if (p) cudaFree(p);
  void *pin[] = {a.tiles_pin, a.dts_pin, a.uref_pin};
  for (void *p : pin) if (p) cudaFreeHost(p);
  if (a.uploaded) cudaEventDestroy(a.uploaded);
  if (a.stream) cudaStreamDestroy(a.stream);
}

// Element-slot arrays of an arena at a given capacity.
struct ElemArrays {
  double *U = nullptr, *Ut = nullptr, *T[2] = {nullptr, nullptr};
  float *Utf = nullptr, *Tf[2] = {nullptr, nullptr};
  int *gclass = nullptr, *esolve = nullptr, *tiles = nullptr;
  FaceLink *links = nullptr;
  void release() {
    void *p[] = {U, Ut, T[0], T[1], Utf, Tf[0], Tf[1], gclass, esolve, tiles, links};
    for (void *q : p) if (q) cudaFree(q);
    *this = ElemArrays{};
  }
};

cudaError_t alloc_elems(const Arena &a, int cap, ElemArrays &x) {
  const size_t m = (size_t)cap * a.nf * a.ld, tr = (size_t)cap * a.nfaces * a.nf * a.gf;
  cudaError_t e = dalloc(&x.U, m);
  if (e == cudaSuccess) e = dalloc(&x.gclass, (size_t)cap);
  if (e == cudaSuccess) e = dalloc(&x.esolve, (size_t)cap);
  if (e == cudaSuccess) e = dalloc(&x.tiles, (size_t)cap / a.epb + 1);
  if (e == cudaSuccess) e = dalloc(&x.links, (size_t)cap * a.nfaces);
  if (a.mixed) {
    if (e == cudaSuccess) e = dalloc(&x.Utf, m);
    if (e == cudaSuccess) e = dalloc(&x.Tf[0], tr);
    if (e == cudaSuccess) e = dalloc(&x.Tf[1], tr);
  } else {
    if (e == cudaSuccess) e = dalloc(&x.Ut, m);
    if (e == cudaSuccess) e = dalloc(&x.T[0], tr);
    if (e == cudaSuccess) e = dalloc(&x.T[1], tr);
  }
  if (e != cudaSuccess) x.release();
  return e;
}

// Grows (or first allocates) the element arrays of an arena to new_cap
// slots, keeping the contents of the old ones.
dgmx_status grow(dgmx_pool *P, Arena &a, int new_cap) {
  const size_t more = (size_t)(new_cap - a.cap) * a.elem_bytes();
  if (!P->fits(more)) return P->fail(DGMX_ERR_MEMORY, "pool budget exceeded");
  // the arrays are copied and freed: no step may be reading them
  if (P->fstream) {
    const cudaError_t q = cudaStreamSynchronize(P->fstream);
    if (q != cudaSuccess) return P->cuda(q, "arena growth");
  }
  ElemArrays x;
  cudaError_t e = alloc_elems(a, new_cap, x);
  if (e != cudaSuccess) return P->cuda(e, "arena allocation");
  const size_t m = (size_t)a.nf * a.ld, tr = (size_t)a.nfaces * a.nf * a.gf;
  auto cp = [&](void *dst, const void *src, size_t bytes) {
    if (e == cudaSuccess && src && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, a.stream);
  };
  cp(x.U, a.U, sizeof(double) * m * a.cap);
  cp(x.Ut, a.Ut, sizeof(double) * m * a.cap);
  cp(x.Utf, a.Utf, sizeof(float) * m * a.cap);
  for (int k = 0; k < 2; ++k) {
    cp(x.T[k], a.T[k], sizeof(double) * tr * a.cap);
    cp(x.Tf[k], a.Tf[k], sizeof(float) * tr * a.cap);
  }
  cp(x.esolve, a.esolve, sizeof(int) * a.cap);
  cp(x.links, a.links, sizeof(FaceLink) * a.nfaces * a.cap);
  cp(x.gclass, a.gclass, sizeof(int) * a.cap);
  // new slots are unallocated: class -1
  if (e == cudaSuccess)
    e = cudaMemsetAsync(x.gclass + a.cap, 0xff, sizeof(int) * (size_t)(new_cap - a.cap), a.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a.stream);
  int *pin = nullptr;
  if (e == cudaSuccess)
    e = cudaHostAlloc(reinterpret_cast<void **>(&pin), sizeof(int) * ((size_t)new_cap / a.epb + 2),
                      cudaHostAllocDefault);
  if (e != cudaSuccess) {
    x.release();
    return P->cuda(e, "arena growth");
  }
  ElemArrays old;
  old.U = a.U; old.Ut = a.Ut; old.T[0] = a.T[0]; old.T[1] = a.T[1];
  old.Utf = a.Utf; old.Tf[0] = a.Tf[0]; old.Tf[1] = a.Tf[1];
  old.gclass = a.gclass; old.esolve = a.esolve; old.tiles = a.tiles; old.links = a.links;
  old.release();
  a.U = x.U; a.Ut = x.Ut; a.T[0] = x.T[0]; a.T[1] = x.T[1];
  a.Utf = x.Utf; a.Tf[0] = x.Tf[0]; a.Tf[1] = x.Tf[1];
  a.gclass = x.gclass; a.esolve = x.esolve; a.tiles = x.tiles; a.links = x.links;
  if (a.tiles_pin) cudaFreeHost(a.tiles_pin);
  a.tiles_pin = pin;
  // the free range at the old end grows, or a new one starts there
  int start = a.cap, len = new_cap - a.cap;
  for (auto it = a.free_ranges.begin(); it != a.free_ranges.end(); ++it)
    if (it->first + it->second == a.cap) { start = it->first; len += it->second; a.free_ranges.erase(it); break; }
  a.free_ranges[start] = len;
  P->bytes += more;
  a.cap = new_cap;
  a.grid = std::max(1, std::min(new_cap / a.epb, P->nsm * a.sops->blocks_per_sm()));
  if (a.graph) { cudaGraphExecDestroy(a.graph); a.graph = nullptr; }
  a.tiles_dirty = true;
  P->args_dirty = true;   // the fused kernel's stage arguments hold these pointers
  return DGMX_OK;
}

// The fused kernel's stream finishes its work before a caller touches an
// arena's buffers from the arena stream.
cudaError_t fused_quiesce(dgmx_pool *P) {
  return P->fstream ? cudaStreamSynchronize(P->fstream) : cudaSuccess;
}

// First use of the fused multi-order kernel: its tables and attributes, its
// stream and the counters of its work list.
dgmx_status fused_setup(dgmx_pool *P) {
  if (P->fused_ready) return DGMX_OK;
  P->fops = P->prm.precision == DGMX_MIXED ? &fused_ops_mixed() : &fused_ops_fp64();
  cudaError_t e = P->fops->init();
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P->fstream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->fuploaded, cudaEventDisableTiming);
  if (e == cudaSuccess) e = dalloc(&P->nitems_dev, (size_t)1);
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&P->nitems_pin), sizeof(int), cudaHostAllocDefault);
  if (e != cudaSuccess) return P->cuda(e, "fused kernel setup");
  P->fgrid = std::max(1, P->nsm * P->fops->blocks_per_sm());
  P->fused_ready = true;
  return DGMX_OK;
}

dgmx_status get_arena(dgmx_pool *P, int phys, int L, int Q, Arena **out) {
  for (auto &a : P->arenas)
    if (a->phys == phys && a->L == L && a->Q == Q) { *out = a.get(); return DGMX_OK; }
  const bool mixed = P->prm.precision == DGMX_MIXED;
  auto a = std::make_unique<Arena>();
  a->phys = phys; a->L = L; a->Q = Q; a->mixed = mixed;
  a->dim = dim_of(phys); a->nf = nfields_of(phys); a->nfaces = 2 * a->dim;
  a->gf = a->dim == 2 ? Q - 1 : (Q - 1) * (Q - 1);
  a->ld = a->dim == 2 ? L * L : L * L * L;
  a->qd = a->dim == 2 ? Q * Q : Q * Q * Q;
  a->fops = find_ops(phys, L, Q);
  const int key = phys + (mixed ? kMixedKey : 0);
  const std::vector<KernelOps> *vs = find_variants(key, L, Q);
  if (!a->fops || !vs || vs->empty())
    return P->fail(DGMX_ERR_UNSUPPORTED, "no kernels built for physics " + std::to_string(phys) + ", p=" +
                                             std::to_string(L - 1) + ", q=" + std::to_string(Q));
  const size_t fixed = sizeof(GeomClass) * kClassCap + sizeof(int) * kPermCap +
                       sizeof(double) * (kUrefStride + 1) * kSlotCap + 8;
  if (!P->fits(fixed)) return P->fail(DGMX_ERR_MEMORY, "pool budget exceeded");
  a->body = P->fused_on ? fused_body(phys, L, Q) : -1;
  if (a->body >= 0) {
    // the fused kernel's body of this (physics, p, q) steps the arena; the
    // plain default tile supplies its trace and projection kernels
    dgmx_status st = fused_setup(P);
    if (st != DGMX_OK) return st;
    a->sops = &(*vs)[0];
    a->epb = P->fops->epb(a->body);
  } else {
    const int v = P->prm.autotune ? tuned_variant(phys, mixed, L, Q, P->prm.gamma, P->prm.flux, P->prm.device) : -1;
    a->sops = (v >= 0 && v < (int)vs->size()) ? &(*vs)[v] : &(*vs)[0];
    a->epb = a->sops->epb;
  }
  a->tab = make_tables(L, Q, Q - 1);
  cudaError_t e = a->fops->init(a->tab);
  if (e == cudaSuccess) e = a->sops->init(a->tab);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&a->uploaded, cudaEventDisableTiming);
  if (e == cudaSuccess) e = dalloc(&a->classes, (size_t)kClassCap);
  if (e == cudaSuccess) e = dalloc(&a->perm, (size_t)kPermCap);
  if (e == cudaSuccess) e = dalloc(&a->uref, (size_t)kUrefStride * kSlotCap);
  if (e == cudaSuccess) e = dalloc(&a->dts, (size_t)kSlotCap);
  if (e == cudaSuccess) e = dalloc(&a->err, (size_t)2);
  if (e == cudaSuccess) e = cudaMemsetAsync(a->uref, 0, sizeof(double) * kUrefStride * kSlotCap, a->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a->dts, 0, sizeof(double) * kSlotCap, a->stream);
  if (e == cudaSuccess)
    e = cudaHostAlloc(reinterpret_cast<void **>(&a->dts_pin), sizeof(double) * kSlotCap, cudaHostAllocDefault);
  if (e == cudaSuccess)
    e = cudaHostAlloc(reinterpret_cast<void **>(&a->uref_pin), sizeof(double) * kUrefStride * kSlotCap,
                      cudaHostAllocDefault);
  const int init[2] = {0, 0x7fffffff};
  if (e == cudaSuccess) e = cudaMemcpyAsync(a->err, init, sizeof(init), cudaMemcpyHostToDevice, a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) { free_arena(*a); return P->cuda(e, "arena setup"); }
  std::memset(a->dts_pin, 0, sizeof(double) * kSlotCap);
  std::memset(a->uref_pin, 0, sizeof(double) * kUrefStride * kSlotCap);
  a->slot_cap = kSlotCap; a->class_cap = kClassCap; a->perm_cap = kPermCap;
  P->bytes += fixed;
  *out = a.get();
  P->arenas.push_back(std::move(a));
  return DGMX_OK;
}

// First-fit range of n tile-aligned slots; grows the arena when none fits.
dgmx_status take_range(dgmx_pool *P, Arena &a, int n, int *e0) {
  for (auto it = a.free_ranges.begin(); it != a.free_ranges.end(); ++it) {
    if (it->second >= n) {
      *e0 = it->first;
      const int rest = it->second - n, at = it->first + n;
      a.free_ranges.erase(it);
      if (rest > 0) a.free_ranges[at] = rest;
      return DGMX_OK;
    }
  }
  // grow: double, or at least enough for this solve (within the budget)
  int tail = 0;
  for (auto &r : a.free_ranges) if (r.first + r.second == a.cap) tail = r.second;
  const int need = a.cap + (n - tail);
  int want = std::max(need, 2 * a.cap);
  want = (want + a.epb - 1) / a.epb * a.epb;
  dgmx_status st = grow(P, a, want);
  if (st == DGMX_ERR_MEMORY && want > need) st = grow(P, a, (need + a.epb - 1) / a.epb * a.epb);
  if (st != DGMX_OK) return st;
  return take_range(P, a, n, e0);
}

void give_range(Arena &a, int e0, int n) {
  a.free_ranges[e0] = n;
  auto it = a.free_ranges.find(e0);
  if (it != a.free_ranges.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) { pv->second += it->second; a.free_ranges.erase(it); it = pv; }
  }
  auto nx = std::next(it);
  if (nx != a.free_ranges.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    a.free_ranges.erase(nx);
  }
}

dgmx_status ensure_scratch(dgmx_pool *P, size_t n) {
  if (P->scratch_n >= n) return DGMX_OK;
  if (P->scratch) { cudaFree(P->scratch); P->bytes -= sizeof(double) * P->scratch_n; }
  P->scratch = nullptr; P->scratch_n = 0;
  cudaError_t e = dalloc(&P->scratch, n);
  if (e != cudaSuccess) return P->cuda(e, "pool scratch");
  P->scratch_n = n;
  P->bytes += sizeof(double) * n;
  return DGMX_OK;
}

StageArgs arena_args(const dgmx_pool *P, const Arena &a) {
  StageArgs s;
  std::memset(&s, 0, sizeof(s));
  s.gclass = a.gclass; s.classes = a.classes; s.links = a.links; s.perm = a.perm;
  s.ne = a.cap; s.gamma = P->prm.gamma; s.flux = P->prm.flux; s.err = a.err;
  s.uref = a.mixed ? a.uref : nullptr;
  s.esolve = a.esolve;
  s.wait_tries = kWaitTries;
  return s;
}

// Captures one LSRK14 step of the whole arena: 14 persistent stage launches.
dgmx_status capture(dgmx_pool *P, Arena &a) {
  if (a.graph) { cudaGraphExecDestroy(a.graph); a.graph = nullptr; }
  StageArgs s = arena_args(P, a);
  s.kind = kLSRK; s.X = a.U; s.U = a.U; s.Ut = a.Ut; s.Utf = a.Utf;
  s.tiles = a.tiles + 1; s.ntiles = a.tiles; s.dts = a.dts;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(a.stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return P->cuda(e, "graph capture");
  int tc = a.tcur;
  for (int k = 0; k < 14 && e == cudaSuccess; ++k) {
    s.c0 = kLsrkA[k]; s.c1 = kLsrkB[k];
    s.Tin = a.T[tc]; s.Tout = a.T[tc ^ 1]; s.Tinf = a.Tf[tc]; s.Toutf = a.Tf[tc ^ 1];
    e = a.sops->stage_grid(s, a.grid, a.stream);
    tc ^= 1;
  }
  const cudaError_t e2 = cudaStreamEndCapture(a.stream, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&a.graph, g, 0);
  if (g) cudaGraphDestroy(g);
  return P->cuda(e, "graph capture");
}

dgmx_status check_arena_error(dgmx_pool *P, int ai) {
  Arena &a = *P->arenas[ai];
  int h[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(h, a.err, sizeof(h), cudaMemcpyDeviceToHost, a.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a.stream);
  if (e != cudaSuccess) return P->cuda(e, "error word readback");
  if (h[0] & 2) return P->fail(DGMX_ERR_CUDA, "a stage kernel's copy pipeline did not complete in time");
  if (!(h[0] & 1)) return DGMX_OK;
  int sid = -1;
  for (auto &kv : P->solves)
    if (kv.second.arena == ai && h[1] >= kv.second.e0 && h[1] < kv.second.e0 + kv.second.ne) sid = kv.first;
  const int init[2] = {0, 0x7fffffff};
  cudaMemcpyAsync(a.err, init, sizeof(init), cudaMemcpyHostToDevice, a.stream);
  cudaStreamSynchronize(a.stream);
  return P->fail(DGMX_ERR_NONPHYSICAL, "non-physical state (density or pressure below eps^(2/3)) in solve " +
                                           std::to_string(sid) + ", element " + std::to_string(h[1] - (sid >= 0 ? P->solves[sid].e0 : 0)));
}

int arena_index(const dgmx_pool *P, const Arena *a) {
  for (size_t i = 0; i < P->arenas.size(); ++i) if (P->arenas[i].get() == a) return (int)i;
  return -1;
}

dgmx_status add_impl(dgmx_pool *P, const dgmx_mesh *m, int phys, const double *U0, double dt, double t_end,
                     int *id) {
  if (!m || !U0 || !id || !(dt > 0.0) || !(t_end > 0.0)) return P->fail(DGMX_ERR_ARGUMENT, "bad argument");
  if (phys != DGMX_EULER2D && phys != DGMX_EULER3D && phys != DGMX_SHALLOW)
    return P->fail(DGMX_ERR_UNSUPPORTED, "pools run Euler 2-D/3-D and shallow water");
  if (phys == DGMX_SHALLOW && P->prm.flux != DGMX_FLUX_LF)
    return P->fail(DGMX_ERR_UNSUPPORTED, "shallow water supports Lax-Friedrichs only");
  if (m->dim != dim_of(phys) || m->ne <= 0 || !m->porder) return P->fail(DGMX_ERR_ARGUMENT, "mesh does not match");
  const int p = m->porder[0], q = (m->qorder && m->qorder[0]) ? m->qorder[0] : p + 2;
  for (int e = 0; e < m->ne; ++e) {
    const int qe = (m->qorder && m->qorder[e]) ? m->qorder[e] : m->porder[e] + 2;
    if (m->porder[e] != p || qe != q) return P->fail(DGMX_ERR_UNSUPPORTED, "one polynomial order per solve");
  }
  Arena *ap = nullptr;
  dgmx_status st = get_arena(P, phys, p + 1, q, &ap);
  if (st != DGMX_OK) return st;
  Arena &a = *ap;
  HostMesh hm;
  std::string err;
  if (!build_mesh(*m, a.tab, hm, err)) return P->fail(DGMX_ERR_ARGUMENT, err);
  const int ne = m->ne, nalloc = (ne + a.epb - 1) / a.epb * a.epb;
  // admission against the budget: element slots (unless a free range
  // fits) and nodal staging
  bool have_range = false;
  for (auto &r : a.free_ranges) if (r.second >= nalloc) have_range = true;
  const size_t nodal = (size_t)a.nf * ne * a.qd;
  size_t need = nodal > P->scratch_n ? sizeof(double) * (nodal - P->scratch_n) : 0;
  if (!have_range) need += (size_t)nalloc * a.elem_bytes();
  if (!P->fits(need)) return P->fail(DGMX_ERR_MEMORY, "pool budget exceeded");
  if (a.free_slots.empty() && a.next_slot >= a.slot_cap) return P->fail(DGMX_ERR_MEMORY, "too many solves in one arena");
  // geometry classes and permutations, deduplicated across the arena
  std::vector<int> cmap(hm.classes.size());
  std::vector<GeomClass> new_classes;
  for (size_t c = 0; c < hm.classes.size(); ++c) {
    std::string key(reinterpret_cast<const char *>(&hm.classes[c]), sizeof(GeomClass));
    auto it = a.class_index.find(key);
    if (it != a.class_index.end()) { cmap[c] = it->second; continue; }
    const int nid = (int)(a.classes_h.size() + new_classes.size());
    if (nid >= a.class_cap) return P->fail(DGMX_ERR_MEMORY, "too many geometry classes in one arena");
    cmap[c] = nid;
    new_classes.push_back(hm.classes[c]);
  }
  std::map<int, int> pmap;   // solve's perm offset -> arena offset
  std::vector<int> new_perm;
  std::map<std::vector<int>, int> new_perm_keys;
  for (const FaceLink &lk : hm.links) {
    if (pmap.count(lk.perm)) continue;
    std::vector<int> key(hm.perm.begin() + lk.perm, hm.perm.begin() + lk.perm + a.gf);
    int off;
    auto it = a.perm_index.find(key);
    auto jt = new_perm_keys.find(key);
    if (it != a.perm_index.end()) {
      off = it->second;
    } else if (jt != new_perm_keys.end()) {
      off = jt->second;
    } else {
      off = (int)(a.perm_h.size() + new_perm.size());
      if (off + a.gf > a.perm_cap) return P->fail(DGMX_ERR_MEMORY, "too many face permutations in one arena");
      new_perm.insert(new_perm.end(), key.begin(), key.end());
      new_perm_keys[key] = off;
    }
    pmap[lk.perm] = off;
  }
  if ((st = ensure_scratch(P, nodal)) != DGMX_OK) return st;
  int e0 = 0;
  if ((st = take_range(P, a, nalloc, &e0)) != DGMX_OK) return st;
  int slot;
  if (a.free_slots.empty()) {
    slot = a.next_slot++;
  } else {
    slot = a.free_slots.back();
    a.free_slots.pop_back();
  }
  // host records of the range; padding slots keep class -1
  std::vector<int> gcl(nalloc, -1), es(nalloc, slot);
  std::vector<FaceLink> lks((size_t)nalloc * a.nfaces, FaceLink{0, 0, 0, -1});
  for (int e = 0; e < ne; ++e) {
    gcl[e] = cmap[hm.gclass[e]];
    for (int f = 0; f < a.nfaces; ++f) {
      FaceLink lk = hm.links[(size_t)e * a.nfaces + f];
      lk.elem += e0;
      lk.perm = pmap[lk.perm];
      lks[(size_t)e * a.nfaces + f] = lk;
    }
    lks[(size_t)e * a.nfaces].cls = gcl[e];
  }
  // reference state of the mixed form: the J- and GLL-weighted mean of U0
  double ref[kUrefStride] = {};
  {
    std::vector<double> wq(a.qd);
    for (int i = 0; i < a.qd; ++i) {
      const int ix = i % a.Q, iy = (i / a.Q) % a.Q, iz = i / (a.Q * a.Q);
      wq[i] = a.tab.w[ix] * a.tab.w[iy] * (a.dim == 3 ? a.tab.w[iz] : 1.0);
    }
    double vol = 0.0;
    for (int e = 0; e < ne; ++e)
      for (int i = 0; i < a.qd; ++i) vol += hm.J[e] * wq[i];
    for (int n = 0; n < a.nf; ++n) {
      double s = 0.0;
      for (int e = 0; e < ne; ++e)
        for (int i = 0; i < a.qd; ++i) s += hm.J[e] * wq[i] * U0[((size_t)n * ne + e) * a.qd + i];
      ref[n] = s / vol;
    }
    fill_reference_row(phys, P->prm.gamma, std::pow(a.tab.B[0], a.dim), ref);
  }
  // uploads on the arena stream.  A fused step in flight does not touch the
  // slots, classes, permutations and solve rows written here (none of them
  // is on its work list yet), so admission overlaps it; a per-arena step in
  // flight finishes first (it runs on this stream).
  cudaError_t e = cudaStreamSynchronize(a.stream);
  auto up = [&](void *dst, const void *src, size_t bytes) {
    if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, a.stream);
  };
  up(a.classes + a.classes_h.size(), new_classes.data(), sizeof(GeomClass) * new_classes.size());
  up(a.perm + a.perm_h.size(), new_perm.data(), sizeof(int) * new_perm.size());
  up(a.gclass + e0, gcl.data(), sizeof(int) * nalloc);
  up(a.esolve + e0, es.data(), sizeof(int) * nalloc);
  up(a.links + (size_t)e0 * a.nfaces, lks.data(), sizeof(FaceLink) * lks.size());
  std::memcpy(a.uref_pin + (size_t)kUrefStride * slot, ref, sizeof(ref));
  up(a.uref + (size_t)kUrefStride * slot, a.uref_pin + (size_t)kUrefStride * slot, sizeof(ref));
  up(P->scratch, U0, sizeof(double) * nodal);
  // projection of U0 into the range, zero second register, traces
  StageArgs s = arena_args(P, a);
  s.ne = ne; s.gclass = a.gclass + e0; s.esolve = a.esolve + e0;
  const size_t m0 = (size_t)e0 * a.nf * a.ld, t0 = (size_t)e0 * a.nfaces * a.nf * a.gf;
  if (e == cudaSuccess) e = a.fops->forward(s, P->scratch, a.U + m0, a.stream);
  if (e == cudaSuccess) {
    if (a.mixed) e = cudaMemsetAsync(a.Utf + m0, 0, sizeof(float) * (size_t)nalloc * a.nf * a.ld, a.stream);
    else e = cudaMemsetAsync(a.Ut + m0, 0, sizeof(double) * (size_t)nalloc * a.nf * a.ld, a.stream);
  }
  if (e == cudaSuccess) {
    if (a.mixed) e = a.sops->traces_modal(s, a.U + m0, a.Tf[a.tcur] + t0, a.stream);
    else e = a.sops->traces_modal(s, a.U + m0, a.T[a.tcur] + t0, a.stream);
  }
  P->launches += 2;
  if (e == cudaSuccess) e = cudaStreamSynchronize(a.stream);
  if (e != cudaSuccess) {
    give_range(a, e0, nalloc);
    a.free_slots.push_back(slot);
    return P->cuda(e, "solve admission");
  }
  for (size_t c = 0; c < new_classes.size(); ++c) {
    a.class_index[std::string(reinterpret_cast<const char *>(&new_classes[c]), sizeof(GeomClass))] =
        (int)a.classes_h.size();
    a.classes_h.push_back(new_classes[c]);
  }
  for (auto &kv : new_perm_keys) a.perm_index[kv.first] = kv.second;
  a.perm_h.insert(a.perm_h.end(), new_perm.begin(), new_perm.end());
  PoolSolve sv;
  sv.id = P->next_id++; sv.arena = arena_index(P, &a); sv.slot = slot;
  sv.e0 = e0; sv.ne = ne; sv.nalloc = nalloc;
  sv.dt = dt; sv.t = 0.0; sv.t_end = t_end;
  P->solves[sv.id] = sv;
  a.live.push_back(sv.id);
  a.tiles_dirty = true;
  if (a.body >= 0) P->items_dirty = true;
  *id = sv.id;
  return DGMX_OK;
}

// The step a live solve takes next (shortened to land on t_end).
double next_dt(const PoolSolve &s) { return std::min(s.dt, s.t_end - s.t); }

// Work list and stage arguments of the fused kernel, uploaded on its stream
// when the fused arenas' membership or buffers changed.
dgmx_status fused_upload(dgmx_pool *P) {
  cudaError_t e = cudaSuccess;
  const int narena = (int)P->arenas.size();
  if (P->items_dirty) {
    cudaEventSynchronize(P->fuploaded);
    // arenas of higher order (more work per tile) first, so the short tiles
    // fill the end of each stage
    std::vector<int> order;
    for (int ai = 0; ai < narena; ++ai) if (P->arenas[ai]->body >= 0) order.push_back(ai);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
      return (size_t)P->arenas[x]->nf * P->arenas[x]->qd * P->arenas[x]->epb >
             (size_t)P->arenas[y]->nf * P->arenas[y]->qd * P->arenas[y]->epb;
    });
    std::vector<int2> items;
    for (int ai : order) {
      const Arena &a = *P->arenas[ai];
      for (int id : a.live) {
        const PoolSolve &sv = P->solves[id];
        for (int t = sv.e0 / a.epb; t < (sv.e0 + sv.nalloc) / a.epb; ++t) items.push_back(make_int2(ai, t));
      }
    }
    if ((int)items.size() > P->items_cap) {
      const int cap = std::max<int>((int)items.size(), 2 * P->items_cap);
      if (P->items_dev) cudaFree(P->items_dev);
      if (P->items_pin) cudaFreeHost(P->items_pin);
      P->items_dev = nullptr; P->items_pin = nullptr; P->items_cap = 0;
      e = dalloc(&P->items_dev, (size_t)cap);
      if (e == cudaSuccess)
        e = cudaHostAlloc(reinterpret_cast<void **>(&P->items_pin), sizeof(int2) * cap, cudaHostAllocDefault);
      if (e != cudaSuccess) return P->cuda(e, "fused work list");
      P->items_cap = cap;
      if (P->fgraph) { cudaGraphExecDestroy(P->fgraph); P->fgraph = nullptr; }
    }
    std::copy(items.begin(), items.end(), P->items_pin);
    *P->nitems_pin = (int)items.size();
    if (!items.empty())
      e = cudaMemcpyAsync(P->items_dev, P->items_pin, sizeof(int2) * items.size(), cudaMemcpyHostToDevice, P->fstream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(P->nitems_dev, P->nitems_pin, sizeof(int), cudaMemcpyHostToDevice, P->fstream);
    if (e != cudaSuccess) return P->cuda(e, "fused work list");
    P->items_dirty = false;
  }
  if (P->args_dirty) {
    cudaEventSynchronize(P->fuploaded);
    if (narena > P->args_cap) {
      const int cap = std::max(narena, 2 * P->args_cap);
      void *old[] = {P->args_dev, P->bodies_dev};
      for (void *q : old) if (q) cudaFree(q);
      if (P->args_pin) cudaFreeHost(P->args_pin);
      if (P->bodies_pin) cudaFreeHost(P->bodies_pin);
      P->args_dev = nullptr; P->bodies_dev = nullptr; P->args_pin = nullptr; P->bodies_pin = nullptr; P->args_cap = 0;
      e = dalloc(&P->args_dev, (size_t)14 * cap);
      if (e == cudaSuccess) e = dalloc(&P->bodies_dev, (size_t)cap);
      if (e == cudaSuccess)
        e = cudaHostAlloc(reinterpret_cast<void **>(&P->args_pin), sizeof(StageArgs) * 14 * cap, cudaHostAllocDefault);
      if (e == cudaSuccess)
        e = cudaHostAlloc(reinterpret_cast<void **>(&P->bodies_pin), sizeof(int) * cap, cudaHostAllocDefault);
      if (e != cudaSuccess) return P->cuda(e, "fused stage arguments");
      P->args_cap = cap;
      if (P->fgraph) { cudaGraphExecDestroy(P->fgraph); P->fgraph = nullptr; }
    }
    std::memset(P->args_pin, 0, sizeof(StageArgs) * 14 * P->args_cap);
    for (int ai = 0; ai < P->args_cap; ++ai) P->bodies_pin[ai] = -1;
    for (int ai = 0; ai < narena; ++ai) {
      const Arena &a = *P->arenas[ai];
      if (a.body < 0) continue;
      P->bodies_pin[ai] = a.body;
      StageArgs g = arena_args(P, a);
      g.kind = kLSRK; g.X = a.U; g.U = a.U; g.Ut = a.Ut; g.Utf = a.Utf; g.dts = a.dts;
      for (int k = 0; k < 14; ++k) {
        const int tc = (a.tcur + k) & 1;
        g.c0 = kLsrkA[k]; g.c1 = kLsrkB[k];
        g.Tin = a.T[tc]; g.Tout = a.T[tc ^ 1]; g.Tinf = a.Tf[tc]; g.Toutf = a.Tf[tc ^ 1];
        P->args_pin[(size_t)k * P->args_cap + ai] = g;
      }
    }
    e = cudaMemcpyAsync(P->args_dev, P->args_pin, sizeof(StageArgs) * 14 * P->args_cap, cudaMemcpyHostToDevice,
                        P->fstream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(P->bodies_dev, P->bodies_pin, sizeof(int) * P->args_cap, cudaMemcpyHostToDevice, P->fstream);
    if (e != cudaSuccess) return P->cuda(e, "fused stage arguments");
    P->args_dirty = false;
  }
  return DGMX_OK;
}

// One LSRK14 step of every fused arena: 14 launches of the fused kernel.
dgmx_status fused_capture(dgmx_pool *P) {
  if (P->fgraph) { cudaGraphExecDestroy(P->fgraph); P->fgraph = nullptr; }
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(P->fstream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return P->cuda(e, "graph capture");
  for (int k = 0; k < 14 && e == cudaSuccess; ++k)
    e = P->fops->launch(P->args_dev, P->args_cap, P->bodies_dev, P->items_dev, P->nitems_dev, k, P->fgrid, P->fstream);
  const cudaError_t e2 = cudaStreamEndCapture(P->fstream, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&P->fgraph, g, 0);
  if (g) cudaGraphDestroy(g);
  return P->cuda(e, "graph capture");
}

// Waits for every enqueued step and reads the arenas' error words.
dgmx_status sync_impl(dgmx_pool *P) {
  dgmx_status st = DGMX_OK;
  if (P->fstream) {
    const cudaError_t e = cudaStreamSynchronize(P->fstream);
    if (e != cudaSuccess) return P->cuda(e, "pool step");
  }
  for (size_t i = 0; i < P->arenas.size(); ++i) {
    cudaError_t e = cudaStreamSynchronize(P->arenas[i]->stream);
    if (e != cudaSuccess) return P->cuda(e, "pool step");
    const dgmx_status s2 = check_arena_error(P, (int)i);
    if (s2 != DGMX_OK && st == DGMX_OK) st = s2;
  }
  P->unsynced = false;
  return st;
}

dgmx_status step_impl(dgmx_pool *P, int nsteps, bool sync) {
  P->unsynced = true;
  for (int k = 0; k < nsteps; ++k) {
    bool any = false, fused_any = false;
    for (auto &ap : P->arenas) {
      Arena &a = *ap;
      const bool fz = a.body >= 0;
      // a fused arena whose membership changed (solves finished, joined or
      // left, possibly all of them) changes the fused kernel's work list
      if (fz && a.tiles_dirty) { P->items_dirty = true; a.tiles_dirty = false; }
      if (a.live.empty()) continue;
      any = true;
      cudaEvent_t up_ev = fz ? P->fuploaded : a.uploaded;
      // per-solve steps, and the tile list when membership changed; the
      // pinned staging is rewritten only after its last copy has run
      for (int id : a.live) {
        const PoolSolve &s = P->solves[id];
        const double h = next_dt(s);
        if (a.dts_pin[s.slot] != h) {
          if (!a.dts_dirty) cudaEventSynchronize(up_ev);
          a.dts_dirty = true;
          a.dts_pin[s.slot] = h;
        }
      }
      cudaError_t e = cudaSuccess;
      if (fz) {
        // stepped below by the fused kernel, from its own work list
        if (a.dts_dirty) {
          e = cudaMemcpyAsync(a.dts, a.dts_pin, sizeof(double) * a.next_slot, cudaMemcpyHostToDevice, P->fstream);
          a.dts_dirty = false;
        }
        if (e != cudaSuccess) return P->cuda(e, "pool upload");
        fused_any = true;
        continue;
      }
      if (a.tiles_dirty) {
        cudaEventSynchronize(a.uploaded);
        std::vector<int> tl;
        for (int id : a.live) {
          const PoolSolve &s = P->solves[id];
          for (int t = s.e0 / a.epb; t < (s.e0 + s.nalloc) / a.epb; ++t) tl.push_back(t);
        }
        std::sort(tl.begin(), tl.end());
        a.tiles_pin[0] = (int)tl.size();
        std::copy(tl.begin(), tl.end(), a.tiles_pin + 1);
        e = cudaMemcpyAsync(a.tiles, a.tiles_pin, sizeof(int) * (tl.size() + 1), cudaMemcpyHostToDevice, a.stream);
        a.tiles_dirty = false;
      }
      if (a.dts_dirty && e == cudaSuccess) {
        e = cudaMemcpyAsync(a.dts, a.dts_pin, sizeof(double) * a.next_slot, cudaMemcpyHostToDevice, a.stream);
        a.dts_dirty = false;
      }
      if (e == cudaSuccess) e = cudaEventRecord(a.uploaded, a.stream);
      if (e != cudaSuccess) return P->cuda(e, "pool upload");
      if (!a.graph) {
        const dgmx_status st = capture(P, a);
        if (st != DGMX_OK) return st;
      }
      if ((e = cudaGraphLaunch(a.graph, a.stream)) != cudaSuccess) return P->cuda(e, "graph launch");
      P->launches += 14;
    }
    if (fused_any) {
      dgmx_status st = fused_upload(P);
      if (st != DGMX_OK) return st;
      cudaError_t e = cudaEventRecord(P->fuploaded, P->fstream);
      if (e != cudaSuccess) return P->cuda(e, "pool upload");
      if (!P->fgraph && (st = fused_capture(P)) != DGMX_OK) return st;
      if ((e = cudaGraphLaunch(P->fgraph, P->fstream)) != cudaSuccess) return P->cuda(e, "graph launch");
      P->launches += 14;
    }
    if (!any) break;
    // host time keeping; solves that reach t_end leave the tile list
    for (auto &ap : P->arenas) {
      Arena &a = *ap;
      std::vector<int> keep;
      for (int id : a.live) {
        PoolSolve &s = P->solves[id];
        const double h = next_dt(s);
        s.t = (h < s.dt) ? s.t_end : s.t + h;
        ++s.steps;
        if (s.t_end - s.t <= 1e-12 * std::max(std::fabs(s.t_end), s.dt)) {
          s.t = s.t_end;
          s.finished = true;
          P->finished_queue.push_back(id);
          a.tiles_dirty = true;
        } else {
          keep.push_back(id);
        }
      }
      a.live.swap(keep);
    }
  }
  return sync ? sync_impl(P) : DGMX_OK;
}

}  // namespace

extern "C" {

dgmx_status dgmx_pool_create(const dgmx_pool_params *params, dgmx_pool **out) {
  if (!params || !out) return DGMX_ERR_ARGUMENT;
  *out = nullptr;
  if (params->precision != DGMX_FP64 && params->precision != DGMX_MIXED) return DGMX_ERR_ARGUMENT;
  if (params->flux != DGMX_FLUX_LF && params->flux != DGMX_FLUX_ROE) return DGMX_ERR_UNSUPPORTED;
  try {
    auto P = std::make_unique<dgmx_pool>();
    P->prm = *params;
    if (P->prm.gamma <= 0) P->prm.gamma = 1.4;
    cudaError_t e = cudaSetDevice(params->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&P->nsm, cudaDevAttrMultiProcessorCount, params->device);
    if (e != cudaSuccess) return DGMX_ERR_CUDA;
    *out = P.release();
    return DGMX_OK;
  } catch (...) {
    return DGMX_ERR_MEMORY;
  }
}

dgmx_status dgmx_pool_destroy(dgmx_pool *p) {
  if (!p) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(p->prm.device);
  if (p->fstream) cudaStreamSynchronize(p->fstream);
  for (auto &a : p->arenas) free_arena(*a);
  if (p->scratch) cudaFree(p->scratch);
  if (p->fgraph) cudaGraphExecDestroy(p->fgraph);
  void *dev[] = {p->args_dev, p->bodies_dev, p->items_dev, p->nitems_dev};
  for (void *q : dev) if (q) cudaFree(q);
  void *pin[] = {p->args_pin, p->bodies_pin, p->items_pin, p->nitems_pin};
  for (void *q : pin) if (q) cudaFreeHost(q);
  if (p->fuploaded) cudaEventDestroy(p->fuploaded);
  if (p->fstream) cudaStreamDestroy(p->fstream);
  delete p;
  return DGMX_OK;
}

dgmx_status dgmx_pool_prepare(dgmx_pool *p, int physics, int porder, int qorder, int elements) {
  if (!p || porder < 1 || elements < 0) return DGMX_ERR_ARGUMENT;
  try {
    cudaSetDevice(p->prm.device);
    if (physics != DGMX_EULER2D && physics != DGMX_EULER3D && physics != DGMX_SHALLOW)
      return p->fail(DGMX_ERR_UNSUPPORTED, "pools run Euler 2-D/3-D and shallow water");
    Arena *a = nullptr;
    dgmx_status st = get_arena(p, physics, porder + 1, qorder ? qorder : porder + 2, &a);
    if (st != DGMX_OK) return st;
    const int want = (elements + a->epb - 1) / a->epb * a->epb;
    if (want > a->cap) st = grow(p, *a, want);
    return st;
  } catch (...) {
    return p->fail(DGMX_ERR_MEMORY, "host allocation failed");
  }
}

dgmx_status dgmx_pool_add(dgmx_pool *p, const dgmx_mesh *mesh, int physics, const double *U0, double dt,
                          double t_end, int *id) {
  if (!p) return DGMX_ERR_ARGUMENT;
  try {
    cudaSetDevice(p->prm.device);
    return add_impl(p, mesh, physics, U0, dt, t_end, id);
  } catch (...) {
    return p->fail(DGMX_ERR_MEMORY, "host allocation failed");
  }
}

dgmx_status dgmx_pool_step(dgmx_pool *p, int nsteps) {
  if (!p || nsteps < 0) return DGMX_ERR_ARGUMENT;
  try {
    cudaSetDevice(p->prm.device);
    return step_impl(p, nsteps, true);
  } catch (...) {
    return p->fail(DGMX_ERR_MEMORY, "host allocation failed");
  }
}

dgmx_status dgmx_pool_step_async(dgmx_pool *p, int nsteps) {
  if (!p || nsteps < 0) return DGMX_ERR_ARGUMENT;
  try {
    cudaSetDevice(p->prm.device);
    return step_impl(p, nsteps, false);
  } catch (...) {
    return p->fail(DGMX_ERR_MEMORY, "host allocation failed");
  }
}

dgmx_status dgmx_pool_sync(dgmx_pool *p) {
  if (!p) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(p->prm.device);
  return sync_impl(p);
}

dgmx_status dgmx_pool_finished(dgmx_pool *p, int *ids, int cap, int *n) {
  if (!p || !n || (cap > 0 && !ids)) return DGMX_ERR_ARGUMENT;
  if (p->unsynced) return p->fail(DGMX_ERR_ARGUMENT, "steps are still in flight: call dgmx_pool_sync first");
  const int k = std::max(0, std::min(cap, (int)p->finished_queue.size()));
  for (int i = 0; i < k; ++i) ids[i] = p->finished_queue[i];
  p->finished_queue.erase(p->finished_queue.begin(), p->finished_queue.begin() + k);
  *n = k;
  return DGMX_OK;
}

dgmx_status dgmx_pool_get_state(dgmx_pool *p, int id, double *U) {
  if (!p || !U) return DGMX_ERR_ARGUMENT;
  auto it = p->solves.find(id);
  if (it == p->solves.end()) return p->fail(DGMX_ERR_ARGUMENT, "no such solve");
  cudaSetDevice(p->prm.device);
  const PoolSolve &s = it->second;
  Arena &a = *p->arenas[s.arena];
  const size_t nodal = (size_t)a.nf * s.ne * a.qd;
  dgmx_status st = ensure_scratch(p, nodal);
  if (st != DGMX_OK) return st;
  StageArgs g = arena_args(p, a);
  g.ne = s.ne; g.gclass = a.gclass + s.e0; g.esolve = a.esolve + s.e0;
  cudaError_t e = fused_quiesce(p);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a.stream);
  if (e == cudaSuccess) e = a.fops->backward(g, a.U + (size_t)s.e0 * a.nf * a.ld, p->scratch, a.stream);
  ++p->launches;
  if (e == cudaSuccess) e = cudaMemcpyAsync(U, p->scratch, sizeof(double) * nodal, cudaMemcpyDeviceToHost, a.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a.stream);
  return p->cuda(e, "get_state");
}

dgmx_status dgmx_pool_solve_info(dgmx_pool *p, int id, double *t, long *steps, int *finished) {
  if (!p) return DGMX_ERR_ARGUMENT;
  auto it = p->solves.find(id);
  if (it == p->solves.end()) return p->fail(DGMX_ERR_ARGUMENT, "no such solve");
  if (t) *t = it->second.t;
  if (steps) *steps = it->second.steps;
  if (finished) *finished = it->second.finished ? 1 : 0;
  return DGMX_OK;
}

dgmx_status dgmx_pool_remove(dgmx_pool *p, int id) {
  if (!p) return DGMX_ERR_ARGUMENT;
  auto it = p->solves.find(id);
  if (it == p->solves.end()) return p->fail(DGMX_ERR_ARGUMENT, "no such solve");
  cudaSetDevice(p->prm.device);
  const PoolSolve s = it->second;
  Arena &a = *p->arenas[s.arena];
  cudaError_t e = fused_quiesce(p);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.gclass + s.e0, 0xff, sizeof(int) * (size_t)s.nalloc, a.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a.stream);
  if (e != cudaSuccess) return p->cuda(e, "remove");
  give_range(a, s.e0, s.nalloc);
  a.free_slots.push_back(s.slot);
  auto lv = std::find(a.live.begin(), a.live.end(), id);
  if (lv != a.live.end()) { a.live.erase(lv); a.tiles_dirty = true; if (a.body >= 0) p->items_dirty = true; }
  p->solves.erase(it);
  return DGMX_OK;
}

dgmx_status dgmx_pool_stats(dgmx_pool *p, size_t *bytes, int *resident, int *active, long long *dof_active) {
  if (!p) return DGMX_ERR_ARGUMENT;
  int act = 0;
  long long dof = 0;
  for (auto &kv : p->solves) {
    if (kv.second.finished) continue;
    ++act;
    const Arena &a = *p->arenas[kv.second.arena];
    dof += (long long)a.nf * kv.second.ne * a.ld;
  }
  if (bytes) *bytes = p->bytes;
  if (resident) *resident = (int)p->solves.size();
  if (active) *active = act;
  if (dof_active) *dof_active = dof;
  return DGMX_OK;
}

long dgmx_pool_launch_count(const dgmx_pool *p) { return p ? p->launches : 0; }

dgmx_status dgmx_pool_set_fused(dgmx_pool *p, int on) {
  if (!p) return DGMX_ERR_ARGUMENT;
  if (!p->arenas.empty()) return p->fail(DGMX_ERR_ARGUMENT, "the stepping path is chosen before the first solve");
  p->fused_on = on != 0;
  return DGMX_OK;
}

const char *dgmx_pool_last_error(const dgmx_pool *p) { return p ? p->errmsg.c_str() : "null pool"; }

}  // extern "C"
