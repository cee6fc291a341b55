// C ABI of the B200 DG engine (include/dgmx.h): handle management, device
// buffers, and the integrator stage sequences replayed from CUDA graphs.
#include <cuda_runtime.h>

#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "dgmx_internal.hpp"

using namespace dgmx;

namespace {

thread_local std::string g_create_error;

// TVD-RK3 (src/TimeInt.cpp:738-740), RK4 (:204-209); LSRK14 is in dgmx_internal.hpp
const double kTvdA[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};
const double kTvdB[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
const double kRk4A[3] = {0.5, 0.5, 1.0};
const double kRk4B[4] = {0.16666666666666667, 0.33333333333333333, 0.33333333333333333, 0.16666666666666667};
template <class T>
cudaError_t dalloc(T **p, size_t n) {
  return cudaMalloc(reinterpret_cast<void **>(p), sizeof(T) * (n ? n : 1));
}

// NCCL entry points, resolved at first use so the library has no link-time
// dependency on NCCL: the file named by DGMX_NCCL_LIBRARY, else the
// libnccl.so.2 the process already has, else the one on the library path.
// Only one libnccl.so.2 can live in a process: a host that also uses another
// NCCL user (PyTorch) loads that one first.
struct NcclApi {
  bool ok = false;
  std::string why;
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
};
const NcclApi &nccl_api() {
  static NcclApi api = [] {
    NcclApi a;
    void *h = nullptr;
    if (const char *path = std::getenv("DGMX_NCCL_LIBRARY")) h = dlopen(path, RTLD_NOW);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW);
    if (!h) { a.why = "libnccl.so.2 not found"; return a; }
    auto sym = [&](const char *n) { return dlsym(h, n); };
    a.GetUniqueId = reinterpret_cast<decltype(a.GetUniqueId)>(sym("ncclGetUniqueId"));
    a.CommInitRank = reinterpret_cast<decltype(a.CommInitRank)>(sym("ncclCommInitRank"));
    a.CommDestroy = reinterpret_cast<decltype(a.CommDestroy)>(sym("ncclCommDestroy"));
    a.GroupStart = reinterpret_cast<decltype(a.GroupStart)>(sym("ncclGroupStart"));
    a.GroupEnd = reinterpret_cast<decltype(a.GroupEnd)>(sym("ncclGroupEnd"));
    a.Send = reinterpret_cast<decltype(a.Send)>(sym("ncclSend"));
    a.Recv = reinterpret_cast<decltype(a.Recv)>(sym("ncclRecv"));
    a.GetErrorString = reinterpret_cast<decltype(a.GetErrorString)>(sym("ncclGetErrorString"));
    a.ok = a.GetUniqueId && a.CommInitRank && a.CommDestroy && a.GroupStart && a.GroupEnd && a.Send && a.Recv &&
           a.GetErrorString;
    if (!a.ok) a.why = "libnccl.so.2 lacks a needed symbol";
    return a;
  }();
  return api;
}

// true if p is page-locked host memory the copy engines can read directly
bool is_pinned(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) { cudaGetLastError(); return false; }
  return at.type == cudaMemoryTypeHost;
}

}  // namespace

struct dgmx_domain {
  dgmx_params prm{};
  int dim = 0, nf = 0, ne = 0, L = 0, Q = 0, G = 0, nfaces = 0, gf = 0, ld = 0, qd = 0;
  HostMesh mesh;
  Tables1D tab;
  const KernelOps *ops = nullptr;     // FP64 tiles (also the nodal path)
  const KernelOps *ops_m = nullptr;   // mixed-precision stage tiles (precision = DGMX_MIXED)
  cudaStream_t stream = nullptr;
  // device state
  double *U = nullptr, *Ut = nullptr, *Acc = nullptr;   // modal registers [e][n][ld]
  double *T[2] = {nullptr, nullptr};                     // traces [e][f][n][gf]
  double *Rsw = nullptr;                                 // shallow-water first RHS (modal)
  double *Ssrc = nullptr;                                // projected source field (modal), 2-D physics
  double *Ghat = nullptr, *Vtr = nullptr, *Pv = nullptr; // Navier-Stokes BR1 work
  float *Utf = nullptr, *Tf[2] = {nullptr, nullptr};     // mixed form: FP32 register and traces
  double *uref = nullptr;                                // mixed form: reference state row (kUrefStride)
  double *nod_in = nullptr, *nod_out = nullptr;          // Field-layout staging
  double *Jdev = nullptr, *integ = nullptr;
  int *gclass = nullptr, *perm = nullptr, *err = nullptr;
  GeomClass *classes = nullptr;
  FaceLink *links = nullptr;
  double *host_pinned = nullptr;                         // pinned staging for host I/O
  // boundary types 1..nbct (kind, two parameters) and the bulk-flow hold
  int nbct = 0;
  int bckind[kMaxBcTypes + 1] = {};
  double bcpar[kMaxBcTypes + 1][5] = {};
  bool hold = false;
  double *R0 = nullptr, *cbar = nullptr;                 // hold: [e][n] constant coefficients, [n] means
  // Navier-Stokes with precision = DGMX_MIXED: the BR1 viscous kernels run in
  // FP32 (from the uncapped tile vops); stage, registers and traces stay FP64
  bool visc32 = false;
  bool visc_tc = false;     // the FP32 viscous kernels' contractions on the tensor cores (3xTF32)
  const KernelOps *vops = nullptr;
  // element partition: ghost slots in the trace buffers and the halo
  // exchange lists (plan.nranks == 1: the whole mesh, no exchange)
  PartitionPlan plan;
  int ne_global = 0, max_ne = 0;                         // whole mesh; most elements of one rank
  // bulk-flow hold on a partition: every rank's constant coefficients in
  // the whole mesh's order, so cbar is the unpartitioned domain's
  double *R0g = nullptr, *Jg = nullptr;                  // [ne_global][nf], [ne_global]
  double *hold_rows = nullptr;                           // [nranks][max_ne][nf] as received
  int *gid_all = nullptr;                                // [nranks][max_ne] global ids (-1: padding)
  int nslot = 0;                                         // ne + ghost slots
  int *x_send = nullptr, *x_recv = nullptr;              // concatenated block lists (device)
  std::vector<int> x_cnt, x_off;                         // per peer block counts and offsets
  int x_total = 0;
  double *x_sbuf = nullptr, *x_rbuf = nullptr;           // nf*gf doubles per block
  ncclComm_t nccl = nullptr;                             // multi-rank transport
  // host-staged transport (alternative to NCCL): packed blocks are copied to
  // pinned host buffers and handed to the caller's function
  dgmx_exchange_fn xhost = nullptr;
  void *xhost_ctx = nullptr;
  double *xh_send = nullptr, *xh_recv = nullptr;
  bool in_group = false;                                 // in-process partitions: the group exchanges
  // overlap: tiles with a face on a ghost slot run first, the exchange of
  // their traces then runs on xstream while the interior tiles run
  cudaStream_t xstream = nullptr;
  cudaEvent_t ev_b = nullptr, ev_x = nullptr;
  int *tiles = nullptr;                                  // [boundary tiles | interior tiles], then the two counts
  int tiles_epb = 0, ntiles_b = 0, ntiles_i = 0;
  int *vtiles = nullptr;                                 // the same split at the viscous kernel's tile size
  int vtiles_epb = 0, nvt_b = 0, nvt_i = 0;
  int tcur = 0;
  bool sw_captured = false;
  long launches = 0;
  // bound of the copy pipeline's first wait per tile (dgmx_set_wait_limit)
  int wait_tries = kWaitTries;
  // graph of one whole step
  cudaGraphExec_t graph = nullptr;
  double graph_dt = 0.0;
  int graph_tcur = -1;
  // time (Domain::t) and the source's time factor exp(-(t - t0)^2 / (2 sigma_t^2))
  // of Shallow::GaussianSource (src/Shallow.hpp:666-735); pulse off: factor 1
  double t = 0.0;
  bool pulse = false;
  double pulse_t0 = 0.0, pulse_s2t2i = 0.0;
  double source_factor(double tt) const {
    if (!pulse) return 1.0;
    const double d = tt - pulse_t0;
    return std::exp(-(d * d * pulse_s2t2i));
  }
  std::string errmsg;

  size_t nmodal() const { return (size_t)ne * nf * ld; }
  size_t nnodal() const { return (size_t)ne * nf * qd; }
  size_t ntrace() const { return (size_t)nslot * nfaces * nf * gf; }
  bool partitioned() const { return plan.nranks > 1; }

  dgmx_status fail(dgmx_status s, const std::string &m) {
    errmsg = m;
    return s;
  }
  dgmx_status cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return DGMX_OK;
    errmsg = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? DGMX_ERR_MEMORY : DGMX_ERR_CUDA;
  }

  StageArgs base_args() const {
    StageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.gclass = gclass; a.classes = classes; a.links = links; a.perm = perm;
    a.ne = ne; a.gamma = prm.gamma; a.vis = prm.vis; a.Pr = prm.Pr; a.flux = prm.flux;
    a.err = err;
    a.Ghat = Ghat; a.V = Vtr; a.Pv = Pv;
    a.uref = uref;
    a.Ssrc = Ssrc;
    a.src_scale = source_factor(t);
    a.wait_tries = wait_tries;
    for (int t = 0; t <= kMaxBcTypes; ++t) {
      a.bckind[t] = bckind[t];
      for (int k = 0; k < 5; ++k) a.bcpar[t][k] = bcpar[t][k];
    }
    return a;
  }
  // bulk-flow hold after a stage of kind a.kind (hold.cu) over this
  // handle's elements; Fn: nodal RHS
  HoldArgs hold_args(const StageArgs &a, double *Tout, double *Fn) const {
    HoldArgs h;
    h.ne = ne; h.nf = nf; h.ld = ld; h.gf = gf; h.qd = qd; h.nfaces = nfaces;
    h.R0 = R0; h.J = Jdev; h.cbar = cbar;
    h.kind = a.kind; h.c0 = a.c0; h.c1 = a.c1; h.dt = a.dt;
    h.U = a.U; h.Ut = a.Ut; h.A = a.A; h.Tout = Tout; h.Fn = Fn;
    return h;
  }
  cudaError_t hold_after(const StageArgs &a, double *Tout, double *Fn) {
    launches += 2;
    return launch_hold(hold_args(a, Tout, Fn), stream);
  }
  // the same with the means taken over the whole mesh: R0g / Jg in global
  // element order (filled by the caller), cbar then applied here
  cudaError_t hold_after_global(const StageArgs &a, double *Tout, double *Fn, double *cb) {
    HoldArgs g = hold_args(a, Tout, Fn);
    g.ne = ne_global; g.R0 = R0g; g.J = Jg; g.cbar = cb;
    cudaError_t e = launch_hold_reduce(g, stream);
    HoldArgs h = hold_args(a, Tout, Fn);
    h.cbar = cb;
    if (e == cudaSuccess) e = launch_hold_apply(h, stream);
    launches += 2;
    return e;
  }
  bool ns() const { return prm.physics == DGMX_NS2D || prm.physics == DGMX_NS3D; }
  cudaError_t ns_grad(const StageArgs &a, bool nodal, cudaStream_t s) const {
    if (visc32 && visc_tc) return vops->ns_grad32tc(a, nodal, s);
    return visc32 ? vops->ns_grad32(a, nodal, s) : ops->ns_grad(a, nodal, s);
  }
  cudaError_t ns_visc(const StageArgs &a, bool nodal, cudaStream_t s) const {
    if (visc32 && visc_tc) return vops->ns_visc32tc(a, nodal, s);
    return visc32 ? vops->ns_visc32(a, nodal, s) : ops->ns_visc(a, nodal, s);
  }
  int visc_epb() const { return (visc32 ? vops : ops)->epb; }
  // the viscous flux kernel over tile list which (0 boundary, 1 interior);
  // no launch for an empty list
  cudaError_t ns_visc_tiles(StageArgs a, int which, cudaStream_t s) const {
    a.nvtiles = which == 0 ? nvt_b : nvt_i;
    if (!a.nvtiles) return cudaSuccess;
    a.vtiles = vtiles + (which == 0 ? 0 : nvt_b);
    return ns_visc(a, false, s);
  }
  bool mixed() const { return prm.precision == DGMX_MIXED; }
  const KernelOps *stage_ops() const { return mixed() ? ops_m : ops; }

  void release() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    void *ptrs[] = {U, Ut, Acc, T[0], T[1], Rsw, nod_in, nod_out, Jdev, integ, gclass, perm, err, classes, links,
                    Ghat, Vtr, Pv, Utf, Tf[0], Tf[1], uref, R0, cbar, x_send, x_recv, x_sbuf, x_rbuf, tiles, Ssrc,
                    R0g, Jg, hold_rows, gid_all, vtiles};
    for (void *p : ptrs) if (p) cudaFree(p);
    if (host_pinned) cudaFreeHost(host_pinned);
    if (xh_send) cudaFreeHost(xh_send);
    if (xh_recv) cudaFreeHost(xh_recv);
    xh_send = xh_recv = nullptr;
    if (nccl && nccl_api().ok) nccl_api().CommDestroy(nccl);
    nccl = nullptr;
    if (stream) cudaStreamDestroy(stream);
    U = Ut = Acc = Rsw = nod_in = nod_out = Jdev = integ = host_pinned = nullptr;
    Ghat = Vtr = Pv = nullptr;
    Utf = Tf[0] = Tf[1] = nullptr;
    uref = nullptr;
    R0 = cbar = Ssrc = nullptr;
    R0g = Jg = hold_rows = nullptr; gid_all = nullptr;
    x_send = x_recv = nullptr; x_sbuf = x_rbuf = nullptr; tiles = nullptr; tiles_epb = 0;
    vtiles = nullptr; vtiles_epb = 0;
    if (ev_b) cudaEventDestroy(ev_b);
    if (ev_x) cudaEventDestroy(ev_x);
    if (xstream) cudaStreamDestroy(xstream);
    ev_b = ev_x = nullptr; xstream = nullptr;
    T[0] = T[1] = nullptr; gclass = perm = err = nullptr; classes = nullptr; links = nullptr; stream = nullptr;
  }
};

namespace {

// One buffer the halo exchange moves: FP64 blocks of blk values, or the
// mixed form's FP32 trace blocks, packed at an even stride so that a block
// is wire() whole doubles in the send and receive buffers.
struct Halo {
  double *T = nullptr;
  float *Tf = nullptr;
  int blk = 0;
  int wire() const { return Tf ? (blk + 1) / 2 : blk; }   // doubles per block in x_sbuf / x_rbuf
  cudaError_t pack(const dgmx_domain *d, cudaStream_t s) const {
    return Tf ? launch_pack(Tf, d->x_send, d->x_total, blk, 2 * wire(), reinterpret_cast<float *>(d->x_sbuf), s)
              : launch_pack(T, d->x_send, d->x_total, blk, d->x_sbuf, s);
  }
  cudaError_t unpack(const dgmx_domain *d, cudaStream_t s) const {
    return Tf ? launch_unpack(reinterpret_cast<const float *>(d->x_rbuf), d->x_recv, d->x_total, blk, 2 * wire(), Tf, s)
              : launch_unpack(d->x_rbuf, d->x_recv, d->x_total, blk, T, s);
  }
};
Halo fp64_halo(double *T, int blk) { Halo h; h.T = T; h.blk = blk; return h; }
// the stage traces of slot k (FP32 in the mixed form)
Halo trace_halo(const dgmx_domain *d, int k) {
  Halo h;
  if (d->mixed()) h.Tf = d->Tf[k]; else h.T = d->T[k];
  h.blk = d->nf * d->gf;
  return h;
}
Halo visc_halo(const dgmx_domain *d) { return fp64_halo(d->Vtr, (d->nf - 1) * d->gf); }

// Halo exchange of one buffer between the ranks of a partitioned domain
// over NCCL (or the caller's host transport): pack, grouped send/receive
// with every peer, unpack into the ghost slots.  A no-op when the domain is
// not partitioned or belongs to an in-process group (the group exchanges).
dgmx_status exchange(dgmx_domain *d, const Halo &h) {
  if (!d->partitioned() || d->in_group) return DGMX_OK;
  if (!d->nccl && !d->xhost)
    return d->fail(DGMX_ERR_ARGUMENT, "partitioned domain without an exchange (dgmx_set_exchange_nccl)");
  const int blk = h.wire();
  cudaError_t e = h.pack(d, d->stream);
  if (e != cudaSuccess) return d->cuda(e, "halo pack");
  if (d->xhost) {
    // host-staged: blocks to the host, the caller's transport, back, unpack
    const size_t n = (size_t)d->x_total * blk;
    if (n) e = cudaMemcpyAsync(d->xh_send, d->x_sbuf, sizeof(double) * n, cudaMemcpyDeviceToHost, d->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) return d->cuda(e, "halo download");
    if (d->xhost(d->xhost_ctx, d->xh_send, d->xh_recv, d->x_cnt.data(), d->x_off.data(), blk, d->plan.nranks) != 0)
      return d->fail(DGMX_ERR_CUDA, "host halo transport reported a failure");
    if (n) e = cudaMemcpyAsync(d->x_rbuf, d->xh_recv, sizeof(double) * n, cudaMemcpyHostToDevice, d->stream);
    if (e == cudaSuccess) e = h.unpack(d, d->stream);
    d->launches += 2;
    return d->cuda(e, "halo unpack");
  }
  const NcclApi &nc = nccl_api();
  ncclResult_t r = nc.GroupStart();
  for (int q = 0; q < d->plan.nranks && r == ncclSuccess; ++q) {
    if (!d->x_cnt[q]) continue;
    const size_t off = (size_t)d->x_off[q] * blk, n = (size_t)d->x_cnt[q] * blk;
    r = nc.Send(d->x_sbuf + off, n, ncclFloat64, q, d->nccl, d->stream);
    if (r == ncclSuccess) r = nc.Recv(d->x_rbuf + off, n, ncclFloat64, q, d->nccl, d->stream);
  }
  const ncclResult_t r2 = nc.GroupEnd();
  if (r == ncclSuccess) r = r2;
  if (r != ncclSuccess) return d->fail(DGMX_ERR_CUDA, std::string("halo exchange: ") + nc.GetErrorString(r));
  e = h.unpack(d, d->stream);
  d->launches += 2;
  return d->cuda(e, "halo unpack");
}

dgmx_status allgather_blocks(dgmx_domain *d, const std::vector<double> &mine, int cap, int blk,
                             std::vector<double> &all);

// Bulk-flow hold on a rank of a partition: this rank's constant
// coefficients go to every peer (NCCL sends on the stream, or the host
// transport), all ranks' rows are scattered into the whole mesh's order
// (R0g), and the means over R0g / Jg, the unpartitioned domain's cbar, are
// applied to this rank's elements.  Elsewhere: the handle's own hold.
dgmx_status hold_stage(dgmx_domain *d, const StageArgs &a, double *Tout, double *Fn) {
  if (!d->partitioned() || d->in_group) return d->cuda(d->hold_after(a, Tout, Fn), "bulk-flow hold");
  const int nr = d->plan.nranks, me = d->plan.rank, nf = d->nf;
  const size_t per = (size_t)d->max_ne * nf;
  double *mine = d->hold_rows + (size_t)me * per;
  cudaError_t e = cudaMemcpyAsync(mine, d->R0, sizeof(double) * d->ne * nf, cudaMemcpyDeviceToDevice, d->stream);
  if (e != cudaSuccess) return d->cuda(e, "bulk-flow hold rows");
  if (d->xhost) {
    std::vector<double> h(per, 0.0), all;
    e = cudaMemcpyAsync(h.data(), mine, sizeof(double) * d->ne * nf, cudaMemcpyDeviceToHost, d->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) return d->cuda(e, "bulk-flow hold rows");
    const dgmx_status st = allgather_blocks(d, h, d->max_ne, nf, all);
    if (st != DGMX_OK) return st;
    e = cudaMemcpyAsync(d->hold_rows, all.data(), sizeof(double) * all.size(), cudaMemcpyHostToDevice, d->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) return d->cuda(e, "bulk-flow hold rows");
  } else {
    if (!d->nccl) return d->fail(DGMX_ERR_ARGUMENT, "partitioned domain without an exchange (dgmx_set_exchange_nccl)");
    const NcclApi &nc = nccl_api();
    ncclResult_t r = nc.GroupStart();
    for (int q = 0; q < nr && r == ncclSuccess; ++q) {
      if (q == me) continue;
      r = nc.Send(mine, per, ncclFloat64, q, d->nccl, d->stream);
      if (r == ncclSuccess) r = nc.Recv(d->hold_rows + (size_t)q * per, per, ncclFloat64, q, d->nccl, d->stream);
    }
    const ncclResult_t r2 = nc.GroupEnd();
    if (r == ncclSuccess) r = r2;
    if (r != ncclSuccess) return d->fail(DGMX_ERR_CUDA, std::string("bulk-flow hold rows: ") + nc.GetErrorString(r));
  }
  e = launch_scatter_rows(d->hold_rows, d->gid_all, nr * d->max_ne, nf, d->R0g, d->stream);
  ++d->launches;
  if (e == cudaSuccess) e = d->hold_after_global(a, Tout, Fn, d->cbar);
  return d->cuda(e, "bulk-flow hold");
}

// The stages of one step: kind, whether the RHS is evaluated on Ut (else U)
// and the two stage coefficients.
struct StageSpec { int kind; bool on_ut; double c0, c1, ct = 0.0; };   // ct: stage time / dt
std::vector<StageSpec> stage_specs(int inttype, double dt) {
  std::vector<StageSpec> v;
  switch (inttype) {
    case DGMX_LSRK14:
      for (int s = 0; s < 14; ++s) v.push_back({kLSRK, false, kLsrkA[s], kLsrkB[s], kLsrkC[s]});
      break;
    case DGMX_TVD3:
      v.push_back({kTVD0, false, 0.0, 0.0});
      v.push_back({kTVD1, true, kTvdA[1], kTvdB[1], 1.0});
      v.push_back({kTVD2, true, kTvdA[2], kTvdB[2], 0.5});
      break;
    case DGMX_RK4:
      v.push_back({kRK40, false, -kRk4A[0] * dt, -kRk4B[0]});
      v.push_back({kRK41, true, -kRk4A[1] * dt, -kRk4B[1], 0.5});
      v.push_back({kRK41, true, -kRk4A[2] * dt, -kRk4B[2], 0.5});
      v.push_back({kRK43, true, dt, -kRk4B[3], 1.0});
      break;
    default:
      break;
  }
  return v;
}

// Arguments of one stage of d (traces T[tcur] in, T[tcur^1] out).
StageArgs stage_args(const dgmx_domain *d, const StageSpec &sp, double dt) {
  StageArgs a = d->base_args();
  a.dt = dt;
  a.U = d->U; a.Ut = d->Ut; a.A = d->Acc;
  if (d->prm.physics == DGMX_SHALLOW && d->prm.sw_balance) a.Rsub = d->Rsw;
  a.kind = sp.kind; a.X = sp.on_ut ? d->Ut : d->U; a.c0 = sp.c0; a.c1 = sp.c1;
  a.src_scale = d->source_factor(d->t + sp.ct * dt);   // Domain::t at this stage
  a.Tin = d->T[d->tcur]; a.Tout = d->T[d->tcur ^ 1];
  if (d->mixed()) { a.Utf = d->Utf; a.Tinf = d->Tf[d->tcur]; a.Toutf = d->Tf[d->tcur ^ 1]; }
  a.R0 = d->hold ? d->R0 : nullptr;
  return a;
}

// Tile lists of a partitioned handle for the stage kernel's tile size:
// boundary tiles (an element with a face on a ghost slot) first, then the
// interior ones; the two counts follow the lists (read on the device).
dgmx_status build_tiles(dgmx_domain *d) {
  const int epb = d->stage_ops()->epb;
  if (d->tiles && d->tiles_epb == epb) return DGMX_OK;
  const int nt = (d->ne + epb - 1) / epb, nf = d->nfaces;
  std::vector<int> b, in;
  for (int t = 0; t < nt; ++t) {
    bool bnd = false;
    for (int e = t * epb; e < std::min(d->ne, (t + 1) * epb) && !bnd; ++e)
      for (int f = 0; f < nf; ++f)
        if (d->mesh.links[(size_t)e * nf + f].elem >= d->ne) { bnd = true; break; }
    (bnd ? b : in).push_back(t);
  }
  std::vector<int> h(b);
  h.insert(h.end(), in.begin(), in.end());
  h.push_back((int)b.size());
  h.push_back((int)in.size());
  if (d->tiles) { cudaFree(d->tiles); d->tiles = nullptr; }
  cudaError_t e = dalloc(&d->tiles, h.size());
  if (e == cudaSuccess) e = cudaMemcpy(d->tiles, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return d->cuda(e, "tile lists");
  d->tiles_epb = epb; d->ntiles_b = (int)b.size(); d->ntiles_i = (int)in.size();
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  return DGMX_OK;
}

// The boundary / interior split of build_tiles at the viscous flux
// kernel's tile size (Navier-Stokes), for its launch over a list.
dgmx_status build_vtiles(dgmx_domain *d) {
  if (!d->ns()) return DGMX_OK;
  const int epb = d->visc_epb();
  if (d->vtiles && d->vtiles_epb == epb) return DGMX_OK;
  const int nt = (d->ne + epb - 1) / epb, nf = d->nfaces;
  std::vector<int> b, in;
  for (int t = 0; t < nt; ++t) {
    bool bnd = false;
    for (int e = t * epb; e < std::min(d->ne, (t + 1) * epb) && !bnd; ++e)
      for (int f = 0; f < nf; ++f)
        if (d->mesh.links[(size_t)e * nf + f].elem >= d->ne) { bnd = true; break; }
    (bnd ? b : in).push_back(t);
  }
  b.insert(b.end(), in.begin(), in.end());
  if (d->vtiles) { cudaFree(d->vtiles); d->vtiles = nullptr; }
  cudaError_t e = dalloc(&d->vtiles, b.size());
  if (e == cudaSuccess) e = cudaMemcpy(d->vtiles, b.data(), sizeof(int) * b.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return d->cuda(e, "viscous tile lists");
  d->vtiles_epb = epb; d->nvt_b = (int)(b.size() - in.size()); d->nvt_i = (int)in.size();
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  return DGMX_OK;
}

// The stage kernel over one of the two tile lists (0 boundary, 1 interior).
cudaError_t stage_tiles(const dgmx_domain *d, StageArgs a, int which, cudaStream_t s) {
  const int n = which == 0 ? d->ntiles_b : d->ntiles_i;
  if (!n) return cudaSuccess;
  const int nt = d->ntiles_b + d->ntiles_i;
  a.tiles = d->tiles + (which == 0 ? 0 : d->ntiles_b);
  a.ntiles = d->tiles + nt + which;
  const KernelOps *o = d->stage_ops();
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->prm.device) != cudaSuccess || sms < 1) sms = 1;
  const int cap = sms * (o->blocks_per_sm ? o->blocks_per_sm() : 1);
  return o->stage_grid(a, n < cap ? n : cap, s);
}

// The NCCL halo exchange of one buffer enqueued on stream s (pack, grouped
// send / receive with every peer, unpack), without a host wait.
dgmx_status exchange_on(dgmx_domain *d, const Halo &h, cudaStream_t s) {
  const int blk = h.wire();
  cudaError_t e = h.pack(d, s);
  if (e != cudaSuccess) return d->cuda(e, "halo pack");
  const NcclApi &nc = nccl_api();
  ncclResult_t r = nc.GroupStart();
  for (int q = 0; q < d->plan.nranks && r == ncclSuccess; ++q) {
    if (!d->x_cnt[q]) continue;
    const size_t off = (size_t)d->x_off[q] * blk, n = (size_t)d->x_cnt[q] * blk;
    r = nc.Send(d->x_sbuf + off, n, ncclFloat64, q, d->nccl, s);
    if (r == ncclSuccess) r = nc.Recv(d->x_rbuf + off, n, ncclFloat64, q, d->nccl, s);
  }
  const ncclResult_t r2 = nc.GroupEnd();
  if (r == ncclSuccess) r = r2;
  if (r != ncclSuccess) return d->fail(DGMX_ERR_CUDA, std::string("halo exchange: ") + nc.GetErrorString(r));
  d->launches += 2;
  return d->cuda(h.unpack(d, s), "halo unpack");
}

bool overlaps(const dgmx_domain *d) { return d->partitioned() && d->nccl && !d->xhost && d->xstream; }

// One stage of an NCCL rank with the exchange overlapped: boundary tiles,
// then the exchange on xstream while the interior tiles run on stream.
dgmx_status stage_overlapped(dgmx_domain *d, const StageArgs &a) {
  cudaError_t e = stage_tiles(d, a, 0, d->stream);
  if (e == cudaSuccess) e = cudaEventRecord(d->ev_b, d->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(d->xstream, d->ev_b, 0);
  if (e != cudaSuccess) return d->cuda(e, "boundary tiles");
  const dgmx_status xs = exchange_on(d, trace_halo(d, d->tcur ^ 1), d->xstream);
  if (xs != DGMX_OK) return xs;
  e = cudaEventRecord(d->ev_x, d->xstream);
  if (e == cudaSuccess) e = stage_tiles(d, a, 1, d->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(d->stream, d->ev_x, 0);
  d->launches += 2;
  return d->cuda(e, "overlapped stage");
}

// Navier-Stokes viscous flux of an NCCL rank with its trace exchange
// overlapped: boundary tiles, then the exchange of their viscous traces on
// xstream while the interior tiles run on stream.
dgmx_status visc_overlapped(dgmx_domain *d, const StageArgs &a) {
  cudaError_t e = d->ns_visc_tiles(a, 0, d->stream);
  if (e == cudaSuccess) e = cudaEventRecord(d->ev_b, d->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(d->xstream, d->ev_b, 0);
  if (e != cudaSuccess) return d->cuda(e, "viscous boundary tiles");
  const dgmx_status xs = exchange_on(d, visc_halo(d), d->xstream);
  if (xs != DGMX_OK) return xs;
  e = cudaEventRecord(d->ev_x, d->xstream);
  if (e == cudaSuccess) e = d->ns_visc_tiles(a, 1, d->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(d->stream, d->ev_x, 0);
  d->launches += 2;
  return d->cuda(e, "overlapped viscous flux");
}

// enqueue the stages of one time step on d->stream
dgmx_status enqueue_step(dgmx_domain *d, double dt) {
  const std::vector<StageSpec> specs = stage_specs(d->prm.inttype, dt);
  if (specs.empty()) return d->fail(DGMX_ERR_UNSUPPORTED, "inttype must be 3, 4 or 14");
  for (const StageSpec &sp : specs) {
    const StageArgs a = stage_args(d, sp, dt);
    cudaError_t e;
    if (d->ns()) {
      if ((e = d->ns_grad(a, false, d->stream)) != cudaSuccess) return d->cuda(e, "viscous gradient kernel");
      ++d->launches;
      if (overlaps(d)) {
        const dgmx_status xs = visc_overlapped(d, a);
        if (xs != DGMX_OK) return xs;
      } else {
        if ((e = d->ns_visc(a, false, d->stream)) != cudaSuccess) return d->cuda(e, "viscous flux kernel");
        ++d->launches;
        const dgmx_status xs = exchange(d, visc_halo(d));
        if (xs != DGMX_OK) return xs;
      }
    }
    if (overlaps(d) && !d->hold) {   // the hold needs all tiles first
      const dgmx_status xs = stage_overlapped(d, a);
      if (xs != DGMX_OK) return xs;
      d->tcur ^= 1;
      continue;
    }
    e = d->stage_ops()->stage(a, d->stream);
    if (e != cudaSuccess) return d->cuda(e, "stage kernel launch");
    ++d->launches;
    if (d->hold) {
      const dgmx_status hs = hold_stage(d, a, d->T[d->tcur ^ 1], nullptr);
      if (hs != DGMX_OK) return hs;
    }
    dgmx_status xs = exchange(d, trace_halo(d, d->tcur ^ 1));
    if (xs != DGMX_OK) return xs;
    d->tcur ^= 1;
  }
  return DGMX_OK;
}

int stages_per_step(int inttype) { return inttype == DGMX_LSRK14 ? 14 : (inttype == DGMX_TVD3 ? 3 : 4); }
int launches_per_stage(const dgmx_domain *d) {
  const bool rank = d->partitioned() && !d->in_group;
  const int halo = rank ? (d->ns() ? 4 : 2) : 0;   // pack + unpack per exchange
  // boundary and interior tiles: the stage kernel (not with the hold) and
  // the viscous flux kernel
  const int split = (overlaps(d) && !d->hold ? 1 : 0) + (overlaps(d) && d->ns() ? 1 : 0);
  const int hold = d->hold ? (rank ? 3 : 2) : 0;   // (scatter,) reduce, apply
  return (d->ns() ? 3 : 1) + split + hold + halo;
}

// Host repeat of launch_reference_integrals' summation order over the
// products rows[e][n] of ne elements in global element order: lane
// l = e mod kRefLanes in increasing e, lanes pairwise with halving strides,
// then times c_d.  Bit-identical to the kernel (every product and sum
// rounded on its own there, IEEE double here).
void reference_sum(const double *rows, int ne, int nf, double c_d, double *out) {
  std::vector<double> red(kRefLanes);
  for (int n = 0; n < nf; ++n) {
    for (int l = 0; l < kRefLanes; ++l) {
      double acc = 0.0;
      for (int e = l; e < ne; e += kRefLanes) acc += rows[(size_t)e * nf + n];
      red[l] = acc;
    }
    for (int s = kRefLanes / 2; s > 0; s >>= 1)
      for (int l = 0; l < s; ++l) red[l] += red[l + s];
    out[n] = c_d * red[0];
  }
}

// The mixed form's reference row from the field integrals tot[0 .. nf) and
// the sum of the element Jacobians, uploaded to d->uref.
dgmx_status upload_reference(dgmx_domain *d, const double *tot, double jsum) {
  const double vol = jsum * std::pow(2.0, d->dim);
  const double phi0 = std::pow(d->tab.B[0], d->dim);   // constant mode's value
  double h[kUrefStride] = {};
  for (int n = 0; n < d->nf; ++n) h[n] = tot[n] / vol;
  fill_reference_row(d->prm.physics, d->prm.gamma, phi0, h);
  cudaError_t e = cudaMemcpyAsync(d->uref, h, sizeof(h), cudaMemcpyHostToDevice, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  return d->cuda(e, "reference state upload");
}

// This domain's per-element integrands J_e * Um[e][n][0] ([e][n], local
// order) on the host; d->nod_out (nf * ne * qd doubles) is the scratch.
dgmx_status element_integrands(dgmx_domain *d, std::vector<double> &rows) {
  rows.assign((size_t)d->ne * d->nf, 0.0);
  cudaError_t e = launch_element_integrands(d->nf, d->ne, d->ld, d->U, d->Jdev, d->nod_out, d->stream);
  ++d->launches;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(rows.data(), d->nod_out, sizeof(double) * rows.size(), cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  return d->cuda(e, "element integrands");
}

// Every rank's cap blocks of blk doubles to every rank through the
// domain's transport (NCCL sends between device buffers, or the caller's
// host function): all[q * cap * blk ...] = rank q's blocks.  Collective.
dgmx_status allgather_blocks(dgmx_domain *d, const std::vector<double> &mine, int cap, int blk,
                             std::vector<double> &all) {
  const int nr = d->plan.nranks, me = d->plan.rank;
  const size_t per = (size_t)cap * blk;
  all.assign((size_t)nr * per, 0.0);
  std::copy(mine.begin(), mine.begin() + per, all.begin() + (size_t)me * per);
  if (d->xhost) {
    // the halo's conventions: peers in rank order, none to this rank itself
    std::vector<double> snd((size_t)(nr - 1) * per), rcv((size_t)(nr - 1) * per);
    std::vector<int> cnt(nr, cap), off(nr);
    for (int q = 0; q < nr; ++q) {
      off[q] = (q < me ? q : (q > me ? q - 1 : 0)) * cap;
      if (q == me) cnt[q] = 0;
      else std::copy(mine.begin(), mine.begin() + per, snd.begin() + (size_t)off[q] * blk);
    }
    if (d->xhost(d->xhost_ctx, snd.data(), rcv.data(), cnt.data(), off.data(), blk, nr) != 0)
      return d->fail(DGMX_ERR_CUDA, "host transport reported a failure (reference state)");
    for (int q = 0; q < nr; ++q)
      if (q != me) std::copy(rcv.begin() + (size_t)off[q] * blk, rcv.begin() + (size_t)off[q] * blk + per,
                             all.begin() + (size_t)q * per);
    return DGMX_OK;
  }
  if (!d->nccl) return d->fail(DGMX_ERR_ARGUMENT, "partitioned domain without an exchange (dgmx_set_exchange_nccl)");
  double *sb = nullptr, *rb = nullptr;
  cudaError_t e = dalloc(&sb, per);
  if (e == cudaSuccess) e = dalloc(&rb, (size_t)nr * per);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sb, mine.data(), sizeof(double) * per, cudaMemcpyHostToDevice, d->stream);
  ncclResult_t r = ncclSuccess;
  if (e == cudaSuccess) {
    const NcclApi &nc = nccl_api();
    r = nc.GroupStart();
    for (int q = 0; q < nr && r == ncclSuccess; ++q) {
      if (q == me) continue;
      r = nc.Send(sb, per, ncclFloat64, q, d->nccl, d->stream);
      if (r == ncclSuccess) r = nc.Recv(rb + (size_t)q * per, per, ncclFloat64, q, d->nccl, d->stream);
    }
    const ncclResult_t r2 = nc.GroupEnd();
    if (r == ncclSuccess) r = r2;
    if (r == ncclSuccess) {
      for (int q = 0; q < nr && e == cudaSuccess; ++q)
        if (q != me)
          e = cudaMemcpyAsync(all.data() + (size_t)q * per, rb + (size_t)q * per, sizeof(double) * per,
                              cudaMemcpyDeviceToHost, d->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    }
  }
  if (sb) cudaFree(sb);
  if (rb) cudaFree(rb);
  if (r != ncclSuccess) return d->fail(DGMX_ERR_CUDA, std::string("reference state gather: ") + nccl_api().GetErrorString(r));
  return d->cuda(e, "reference state gather");
}

// Mixed form: the reference state the FP32 working copies are perturbations
// about is the domain mean of U (any constant gives the same scheme; the
// mean keeps the perturbations small); one row, see fill_reference_row.
// Its integrals follow one fixed summation order over the whole mesh
// (launch_reference_integrals), so a partitioned domain (its ranks gather
// every element's integrands) gets the row of the unpartitioned one, on
// every rank.
dgmx_status update_reference(dgmx_domain *d) {
  const double c = std::pow(std::sqrt(2.0), d->dim);
  double tot[5] = {0, 0, 0, 0, 0};
  double jsum = 0.0;
  if (!d->partitioned()) {
    cudaError_t e = launch_reference_integrals(d->nf, d->ne, d->ld, c, d->U, d->Jdev, d->integ, d->stream);
    ++d->launches;
    if (e == cudaSuccess) e = cudaMemcpyAsync(tot, d->integ, sizeof(double) * d->nf, cudaMemcpyDeviceToHost, d->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) return d->cuda(e, "reference state");
    for (int k = 0; k < d->ne; ++k) jsum += d->mesh.J[k];
    return upload_reference(d, tot, jsum);
  }
  // ranks: blocks (global id, J, integrands) padded to max_ne per rank
  std::vector<double> rows, all;
  dgmx_status st = element_integrands(d, rows);
  if (st != DGMX_OK) return st;
  const int nf = d->nf, blk = nf + 2;
  std::vector<double> mine((size_t)d->max_ne * blk, -1.0);
  for (int e = 0; e < d->ne; ++e) {
    double *b = &mine[(size_t)e * blk];
    b[0] = d->plan.global_of_local[e];
    b[1] = d->mesh.J[e];
    for (int n = 0; n < nf; ++n) b[2 + n] = rows[(size_t)e * nf + n];
  }
  if ((st = allgather_blocks(d, mine, d->max_ne, blk, all)) != DGMX_OK) return st;
  std::vector<double> R((size_t)d->ne_global * nf, 0.0), J(d->ne_global, 0.0);
  for (size_t i = 0; i < all.size() / blk; ++i) {
    const double *b = &all[i * blk];
    const long g = (long)b[0];
    if (g < 0 || g >= d->ne_global) continue;   // padding
    J[g] = b[1];
    for (int n = 0; n < nf; ++n) R[(size_t)g * nf + n] = b[2 + n];
  }
  reference_sum(R.data(), d->ne_global, nf, c, tot);
  for (int k = 0; k < d->ne_global; ++k) jsum += J[k];
  return upload_reference(d, tot, jsum);
}

// traces of U into T[tcur] (Tf[tcur] in the mixed form)
dgmx_status refresh_traces(dgmx_domain *d) {
  if (d->mixed()) {
    if (d->in_group) return DGMX_OK;   // the group sets its parts' reference state and traces
    const dgmx_status st = update_reference(d);
    if (st != DGMX_OK) return st;
  }
  StageArgs a = d->base_args();
  cudaError_t e = d->mixed() ? d->ops_m->traces_modal(a, d->U, d->Tf[d->tcur], d->stream)
                             : d->ops->traces_modal(a, d->U, d->T[d->tcur], d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "trace kernel launch");
  return exchange(d, trace_halo(d, d->tcur));
}

// Shallow-water balance: the first RHS ever evaluated is subtracted from all
// later ones (src/Shallow.cpp:255-267).  Captured from the current state.
dgmx_status capture_sw_source(dgmx_domain *d) {
  StageArgs a = d->base_args();
  a.kind = kRHS; a.X = d->U; a.U = d->U; a.Ut = d->Ut; a.A = d->Rsw;
  a.Tin = d->T[d->tcur]; a.Tout = d->T[d->tcur ^ 1];
  if (d->mixed()) { a.Utf = d->Utf; a.Tinf = d->Tf[d->tcur]; a.Toutf = d->Tf[d->tcur ^ 1]; }
  cudaError_t e = d->stage_ops()->stage(a, d->stream);
  ++d->launches;
  d->tcur ^= 1;
  d->sw_captured = true;
  if (e != cudaSuccess) return d->cuda(e, "shallow-water source capture");
  return exchange(d, trace_halo(d, d->tcur));
}

dgmx_status check_error_word(dgmx_domain *d) {
  int h[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(h, d->err, sizeof(h), cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return d->cuda(e, "error word readback");
  if (h[0] & 2) return d->fail(DGMX_ERR_CUDA, "a stage kernel's copy pipeline did not complete in time");
  if (h[0] & 1) {
    char buf[160];
    std::snprintf(buf, sizeof(buf), "non-physical state (density or pressure below eps^(2/3)) on element %d", h[1]);
    return d->fail(DGMX_ERR_NONPHYSICAL, buf);
  }
  return DGMX_OK;
}

dgmx_status reset_error_word(dgmx_domain *d) {
  const int init[2] = {0, 0x7fffffff};
  return d->cuda(cudaMemcpyAsync(d->err, init, sizeof(init), cudaMemcpyHostToDevice, d->stream), "error reset");
}

// Boundary sides and their (kind, parameter) types, and the bulk-flow hold.
struct BoundarySpec {
  std::vector<BoundarySide> sides;
  int ntypes = 0;
  int kind[kMaxBcTypes + 1] = {};
  double par[kMaxBcTypes + 1][5] = {};
  bool hold = false;
  // type index of (kind, parameters), added on first use; 0 when the table is full
  int type_of(int k, const double *v) {
    double w[5] = {0, 0, 0, 0, 0};
    const int np = k == DGMX_BC_ISOTHERMAL_WALL ? 2 : (k == DGMX_BC_STATE ? 5 : (k == DGMX_BC_SUBSONIC_OUTFLOW ? 1 : 0));
    for (int i = 0; i < np; ++i) w[i] = v[i];
    for (int t = 1; t <= ntypes; ++t)
      if (kind[t] == k && std::equal(w, w + 5, par[t])) return t;
    if (ntypes == kMaxBcTypes) return 0;
    ++ntypes;
    kind[ntypes] = k;
    std::copy(w, w + 5, par[ntypes]);
    return ntypes;
  }
};

// The rank's part of an element partition (part[e] = owning rank).
struct PartitionSpec {
  const int *part = nullptr;
  int nranks = 1, rank = 0;
  bool group = false;     // in-process partitions: the group performs the exchange
};

dgmx_status create_impl(const dgmx_mesh *m, const dgmx_params *p, dgmx_domain **out,
                        const BoundarySpec *bspec = nullptr, const PartitionSpec *pspec = nullptr) {
  if (!m || !p || !out) { g_create_error = "null argument"; return DGMX_ERR_ARGUMENT; }
  *out = nullptr;
  auto d = std::make_unique<dgmx_domain>();
  d->prm = *p;
  const bool ns_phys = p->physics == DGMX_NS2D || p->physics == DGMX_NS3D;
  if (bspec && !bspec->sides.empty()) {
    if (p->precision != DGMX_FP64 && !ns_phys) {
      g_create_error = "boundary sides are supported in FP64 (and with the FP32 viscous form of Navier-Stokes)";
      return DGMX_ERR_UNSUPPORTED;
    }
    for (int t = 1; t <= bspec->ntypes; ++t) {
      const int k = bspec->kind[t];
      const bool euler = p->physics == DGMX_EULER3D || p->physics == DGMX_EULER2D;
      const bool ns = p->physics == DGMX_NS3D || p->physics == DGMX_NS2D;
      const bool outflow = k == DGMX_BC_SUBSONIC_OUTFLOW || k == DGMX_BC_SUPERSONIC_OUTFLOW;
      const bool sw = p->physics == DGMX_SHALLOW;
      if (!(k == DGMX_BC_SLIP_WALL && (euler || sw)) && !(k == DGMX_BC_ISOTHERMAL_WALL && ns) &&
          !(k == DGMX_BC_STATE && (euler || ns)) && !(outflow && (euler || ns) && m->dim == 2)) {
        g_create_error = "boundary kind " + std::to_string(k) +
                         " is not built for this physics (Euler and shallow water: slip wall; Navier-Stokes:"
                         " isothermal wall; Euler and Navier-Stokes: fixed state, and the outflows in 2-D)";
        return DGMX_ERR_UNSUPPORTED;
      }
    }
    d->nbct = bspec->ntypes;
    for (int t = 0; t <= kMaxBcTypes; ++t) {
      d->bckind[t] = bspec->kind[t];
      for (int k = 0; k < 5; ++k) d->bcpar[t][k] = bspec->par[t][k];
    }
  }
  if (bspec && bspec->hold) {
    if (p->physics != DGMX_NS3D) { g_create_error = "the bulk-flow hold is a Navier-Stokes 3-D option"; return DGMX_ERR_UNSUPPORTED; }
    d->hold = true;
  }
  if (d->prm.gamma <= 0) d->prm.gamma = 1.4;
  if (d->prm.Pr <= 0) d->prm.Pr = 0.72;
  const int phys = p->physics;
  if (phys != DGMX_EULER2D && phys != DGMX_EULER3D && phys != DGMX_SHALLOW && phys != DGMX_NS2D &&
      phys != DGMX_NS3D) {
    g_create_error = "unknown physics " + std::to_string(phys);
    return DGMX_ERR_ARGUMENT;
  }
  if (m->dim != dim_of(phys)) { g_create_error = "mesh dimension does not match the physics"; return DGMX_ERR_ARGUMENT; }
  if (p->inttype != DGMX_TVD3 && p->inttype != DGMX_RK4 && p->inttype != DGMX_LSRK14) {
    g_create_error = "inttype must be 3 (TVD), 4 (RK4) or 14 (LSRK14)";
    return DGMX_ERR_UNSUPPORTED;
  }
  if (p->flux < DGMX_FLUX_LF || p->flux > DGMX_FLUX_VAN_LEER) {
    g_create_error = "flux must be LF, Roe, Steger-Warming or van Leer";
    return DGMX_ERR_UNSUPPORTED;
  }
  if ((p->flux == DGMX_FLUX_STEGER_WARMING || p->flux == DGMX_FLUX_VAN_LEER) &&
      (phys != DGMX_EULER2D && phys != DGMX_NS2D)) {
    g_create_error = "Steger-Warming and van Leer are 2-D Euler/Navier-Stokes fluxes (Euler3d computes Lax-Friedrichs only)";
    return DGMX_ERR_UNSUPPORTED;
  }
  if ((p->flux == DGMX_FLUX_STEGER_WARMING || p->flux == DGMX_FLUX_VAN_LEER) && p->precision == DGMX_MIXED) {
    g_create_error = "the mixed-precision form is built for the Lax-Friedrichs and Roe fluxes";
    return DGMX_ERR_UNSUPPORTED;
  }
  if (phys == DGMX_SHALLOW && p->flux != DGMX_FLUX_LF) { g_create_error = "shallow water supports Lax-Friedrichs only"; return DGMX_ERR_UNSUPPORTED; }
  if (p->precision != DGMX_FP64 && p->precision != DGMX_MIXED) { g_create_error = "precision must be FP64 or MIXED"; return DGMX_ERR_ARGUMENT; }
  if (p->precision == DGMX_MIXED && p->inttype != DGMX_LSRK14 && !ns_phys) {
    g_create_error = "the mixed-precision form is built for LSRK14 with Euler and shallow water";
    return DGMX_ERR_UNSUPPORTED;
  }
  if (p->precision == DGMX_MIXED && ns_phys) {
    // Navier-Stokes: FP32 viscous kernels, FP64 everything else
    d->visc32 = true;
    d->prm.precision = DGMX_FP64;
  }
  if (!m->porder || m->ne <= 0) { g_create_error = "mesh needs porder"; return DGMX_ERR_ARGUMENT; }
  const int pp = m->porder[0];
  const int qq = (m->qorder && m->qorder[0]) ? m->qorder[0] : pp + 2;
  for (int e = 0; e < m->ne; ++e) {
    const int qe = (m->qorder && m->qorder[e]) ? m->qorder[e] : m->porder[e] + 2;
    if (m->porder[e] != pp || qe != qq) {
      g_create_error = "the GPU path needs one polynomial order for all elements";
      return DGMX_ERR_UNSUPPORTED;
    }
  }
  d->ops = find_ops(phys, pp + 1, qq);
  if (d->visc32) {
    d->vops = d->ops;
    if (!d->vops || !d->vops->ns_grad32) {
      g_create_error = "no FP32 viscous kernels built for p=" + std::to_string(pp) + ", q=" + std::to_string(qq);
      return DGMX_ERR_UNSUPPORTED;
    }
  }
  if (d->ops && d->prm.precision == DGMX_MIXED) {
    d->ops_m = find_ops(phys + kMixedKey, pp + 1, qq);
    if (!d->ops_m) {
      g_create_error = "no mixed-precision kernels built for p=" + std::to_string(pp) + ", q=" + std::to_string(qq);
      return DGMX_ERR_UNSUPPORTED;
    }
  }
  if (!d->ops) {
    g_create_error = "no kernels built for physics " + std::to_string(phys) + ", p=" + std::to_string(pp) +
                     ", q=" + std::to_string(qq);
    return DGMX_ERR_UNSUPPORTED;
  }
  d->dim = m->dim; d->nf = nfields_of(phys); d->ne = m->ne;
  d->L = pp + 1; d->Q = qq; d->G = qq - 1;
  d->nfaces = 2 * d->dim;
  d->gf = d->dim == 2 ? d->G : d->G * d->G;
  d->ld = d->dim == 2 ? d->L * d->L : d->L * d->L * d->L;
  d->qd = d->dim == 2 ? d->Q * d->Q : d->Q * d->Q * d->Q;
  d->tab = make_tables(d->L, d->Q, d->G);
  std::string err;
  if (!build_mesh(*m, d->tab, d->mesh, err, bspec ? &bspec->sides : nullptr)) {
    g_create_error = err;
    return DGMX_ERR_ARGUMENT;
  }
  std::vector<double> Jglob;   // partitions of Navier-Stokes 3-D: the whole mesh's Jacobians and
  std::vector<int> gid_host;   // every rank's global ids, for the bulk-flow hold
  if (pspec && pspec->nranks > 1) {
    if (pspec->group && phys == DGMX_SHALLOW && p->sw_balance) {
      g_create_error = "in-process partitions of shallow water need sw_balance = 0";
      return DGMX_ERR_UNSUPPORTED;
    }
    HostMesh local;
    if (!partition_mesh(d->mesh, pspec->part, pspec->nranks, pspec->rank, local, d->plan, err)) {
      g_create_error = err;
      return DGMX_ERR_ARGUMENT;
    }
    d->ne_global = d->mesh.ne;
    std::vector<int> per(pspec->nranks, 0);
    for (int e = 0; e < d->ne_global; ++e) ++per[pspec->part[e]];
    d->max_ne = *std::max_element(per.begin(), per.end());
    if (phys == DGMX_NS3D) {
      Jglob = d->mesh.J;
      gid_host.assign((size_t)pspec->nranks * d->max_ne, -1);
      std::vector<int> fill(pspec->nranks, 0);
      for (int e = 0; e < d->ne_global; ++e) {
        const int q = pspec->part[e];
        gid_host[(size_t)q * d->max_ne + fill[q]++] = e;
      }
    }
    d->mesh = std::move(local);
    d->ne = d->plan.ne_local;
    d->in_group = pspec->group;
  }
  d->nslot = d->ne + d->plan.nghost;

  cudaError_t e = cudaSetDevice(p->device);
  if (e != cudaSuccess) { g_create_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e); return DGMX_ERR_CUDA; }
  dgmx_status st;
  auto chk = [&](cudaError_t ce, const char *what) {
    if (ce != cudaSuccess) { st = d->cuda(ce, what); return false; }
    return true;
  };
  st = DGMX_OK;
  if (!chk(d->ops->init(d->tab), "kernel table upload")) { g_create_error = d->errmsg; d->release(); return st; }
  if (d->ops_m && !chk(d->ops_m->init(d->tab), "kernel table upload")) { g_create_error = d->errmsg; d->release(); return st; }
  if (!chk(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking), "stream")) { g_create_error = d->errmsg; d->release(); return st; }
  bool ok = chk(dalloc(&d->U, d->nmodal()), "alloc U") && chk(dalloc(&d->Ut, d->nmodal()), "alloc Ut") &&
            chk(dalloc(&d->Acc, d->nmodal()), "alloc Acc") && chk(dalloc(&d->T[0], d->ntrace()), "alloc T0") &&
            chk(dalloc(&d->T[1], d->ntrace()), "alloc T1") && chk(dalloc(&d->nod_in, d->nnodal()), "alloc nodal") &&
            chk(dalloc(&d->nod_out, d->nnodal()), "alloc nodal") && chk(dalloc(&d->Jdev, (size_t)d->ne), "alloc J") &&
            chk(dalloc(&d->integ, (size_t)d->nf), "alloc integrals") &&
            chk(dalloc(&d->gclass, (size_t)d->ne), "alloc gclass") &&
            chk(dalloc(&d->classes, d->mesh.classes.size()), "alloc classes") &&
            chk(dalloc(&d->links, d->mesh.links.size()), "alloc links") &&
            chk(dalloc(&d->perm, d->mesh.perm.size()), "alloc perm") && chk(dalloc(&d->err, (size_t)2), "alloc err") &&
            (phys != DGMX_SHALLOW || chk(dalloc(&d->Rsw, d->nmodal()), "alloc sw source")) &&
            (!d->mixed() || (chk(dalloc(&d->Utf, d->nmodal()), "alloc Ut (FP32)") &&
                             chk(dalloc(&d->Tf[0], d->ntrace()), "alloc T0 (FP32)") &&
                             chk(dalloc(&d->Tf[1], d->ntrace()), "alloc T1 (FP32)") &&
                             chk(dalloc(&d->uref, (size_t)kUrefStride), "alloc reference state"))) &&
            (!d->ns() || (chk(dalloc(&d->Ghat, (size_t)d->ne * (d->dim + 1) * d->dim * d->ld), "alloc gradients") &&
                          chk(dalloc(&d->Vtr, (size_t)d->nslot * d->nfaces * (d->nf - 1) * d->gf), "alloc viscous traces") &&
                          chk(dalloc(&d->Pv, (size_t)d->ne * (d->nf - 1) * d->ld), "alloc viscous divergence"))) &&
            (!d->ns() || d->dim != 3 || (chk(dalloc(&d->R0, (size_t)d->ne * d->nf), "alloc hold coefficients") &&
                                          chk(dalloc(&d->cbar, (size_t)d->nf), "alloc hold means"))) &&
            (gid_host.empty() ||
             (chk(dalloc(&d->R0g, (size_t)d->ne_global * d->nf), "alloc hold coefficients (whole mesh)") &&
              chk(dalloc(&d->Jg, (size_t)d->ne_global), "alloc Jacobians (whole mesh)") &&
              chk(dalloc(&d->hold_rows, gid_host.size() * d->nf), "alloc hold rows") &&
              chk(dalloc(&d->gid_all, gid_host.size()), "alloc global ids") &&
              chk(cudaMemcpy(d->Jg, Jglob.data(), sizeof(double) * Jglob.size(), cudaMemcpyHostToDevice), "upload") &&
              chk(cudaMemcpy(d->gid_all, gid_host.data(), sizeof(int) * gid_host.size(), cudaMemcpyHostToDevice),
                  "upload")));
  if (ok) {
    ok = chk(cudaMemcpy(d->gclass, d->mesh.gclass.data(), sizeof(int) * d->ne, cudaMemcpyHostToDevice), "upload") &&
         chk(cudaMemcpy(d->classes, d->mesh.classes.data(), sizeof(GeomClass) * d->mesh.classes.size(),
                        cudaMemcpyHostToDevice), "upload") &&
         chk(cudaMemcpy(d->links, d->mesh.links.data(), sizeof(FaceLink) * d->mesh.links.size(),
                        cudaMemcpyHostToDevice), "upload") &&
         chk(cudaMemcpy(d->perm, d->mesh.perm.data(), sizeof(int) * d->mesh.perm.size(), cudaMemcpyHostToDevice),
             "upload") &&
         chk(cudaMemcpy(d->Jdev, d->mesh.J.data(), sizeof(double) * d->ne, cudaMemcpyHostToDevice), "upload") &&
         chk(cudaMemset(d->U, 0, sizeof(double) * d->nmodal()), "memset") &&
         chk(cudaMemset(d->Ut, 0, sizeof(double) * d->nmodal()), "memset") &&
         chk(cudaMemset(d->Acc, 0, sizeof(double) * d->nmodal()), "memset") &&
         chk(cudaMemset(d->T[0], 0, sizeof(double) * d->ntrace()), "memset") &&
         chk(cudaMemset(d->T[1], 0, sizeof(double) * d->ntrace()), "memset") &&
         chk(cudaHostAlloc(reinterpret_cast<void **>(&d->host_pinned), sizeof(double) * d->nnodal() * 2,
                           cudaHostAllocDefault), "pinned staging");
  }
  if (ok && d->partitioned()) {
    // exchange lists, concatenated over peers in rank order
    std::vector<int> snd, rcv;
    d->x_cnt.assign(d->plan.nranks, 0);
    d->x_off.assign(d->plan.nranks, 0);
    for (int q = 0; q < d->plan.nranks; ++q) {
      d->x_off[q] = (int)snd.size();
      d->x_cnt[q] = (int)d->plan.send[q].size();
      snd.insert(snd.end(), d->plan.send[q].begin(), d->plan.send[q].end());
      rcv.insert(rcv.end(), d->plan.recv[q].begin(), d->plan.recv[q].end());
    }
    d->x_total = (int)snd.size();
    const size_t blk = (size_t)d->nf * d->gf;
    ok = chk(dalloc(&d->x_send, snd.size()), "alloc halo lists") && chk(dalloc(&d->x_recv, rcv.size()), "alloc halo lists") &&
         chk(dalloc(&d->x_sbuf, snd.size() * blk), "alloc halo buffers") &&
         chk(dalloc(&d->x_rbuf, rcv.size() * blk), "alloc halo buffers") &&
         (snd.empty() || (chk(cudaMemcpy(d->x_send, snd.data(), sizeof(int) * snd.size(), cudaMemcpyHostToDevice), "upload") &&
                          chk(cudaMemcpy(d->x_recv, rcv.data(), sizeof(int) * rcv.size(), cudaMemcpyHostToDevice), "upload")));
  }
  if (!ok) { g_create_error = d->errmsg; d->release(); return st; }
  if ((st = reset_error_word(d.get())) != DGMX_OK) { g_create_error = d->errmsg; d->release(); return st; }
  cudaStreamSynchronize(d->stream);
  *out = d.release();
  return DGMX_OK;
}

dgmx_status set_state_from_device_nodal(dgmx_domain *d, const double *Un_dev) {
  StageArgs a = d->base_args();
  cudaError_t e = d->ops->forward(a, Un_dev, d->U, d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "forward kernel");
  if ((e = cudaMemsetAsync(d->Ut, 0, sizeof(double) * d->nmodal(), d->stream))) return d->cuda(e, "memset");
  if ((e = cudaMemsetAsync(d->Acc, 0, sizeof(double) * d->nmodal(), d->stream))) return d->cuda(e, "memset");
  if (d->Utf && (e = cudaMemsetAsync(d->Utf, 0, sizeof(float) * d->nmodal(), d->stream))) return d->cuda(e, "memset");
  d->tcur = 0;
  d->sw_captured = false;
  dgmx_status st = refresh_traces(d);
  if (st != DGMX_OK) return st;
  return d->cuda(cudaStreamSynchronize(d->stream), "set_state");
}

// set_state_from_device_nodal without a host wait: the projection, the
// registers' reset, the mixed form's reference state (integrals and the
// reference row on the stream) and the traces, all enqueued on d->stream.
dgmx_status enqueue_state_from_device_nodal(dgmx_domain *d, const double *Un_dev) {
  StageArgs a = d->base_args();
  cudaError_t e = d->ops->forward(a, Un_dev, d->U, d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "forward kernel");
  if ((e = cudaMemsetAsync(d->Ut, 0, sizeof(double) * d->nmodal(), d->stream))) return d->cuda(e, "memset");
  if ((e = cudaMemsetAsync(d->Acc, 0, sizeof(double) * d->nmodal(), d->stream))) return d->cuda(e, "memset");
  if (d->Utf && (e = cudaMemsetAsync(d->Utf, 0, sizeof(float) * d->nmodal(), d->stream))) return d->cuda(e, "memset");
  d->tcur = 0;
  d->sw_captured = false;
  if (d->mixed()) {
    double vol = 0.0;
    for (int k = 0; k < d->ne; ++k) vol += d->mesh.J[k];
    vol *= std::pow(2.0, d->dim);
    e = launch_reference_integrals(d->nf, d->ne, d->ld, std::pow(std::sqrt(2.0), d->dim), d->U, d->Jdev, d->integ,
                                   d->stream);
    if (e == cudaSuccess)
      e = launch_reference_row(d->prm.physics, d->nf, d->prm.gamma, std::pow(d->tab.B[0], d->dim), vol, d->integ,
                               d->uref, d->stream);
    d->launches += 2;
    if (e != cudaSuccess) return d->cuda(e, "reference state");
  }
  a = d->base_args();
  e = d->mixed() ? d->ops_m->traces_modal(a, d->U, d->Tf[d->tcur], d->stream)
                 : d->ops->traces_modal(a, d->U, d->T[d->tcur], d->stream);
  ++d->launches;
  return d->cuda(e, "trace kernel launch");
}

}  // namespace

extern "C" {

dgmx_status dgmx_set_state_async(dgmx_domain *d, const double *U) {
  if (!d || !U) return DGMX_ERR_ARGUMENT;
  if (d->partitioned()) return d->fail(DGMX_ERR_UNSUPPORTED, "the asynchronous state calls are not built for partitions");
  if (!is_pinned(U)) return d->fail(DGMX_ERR_ARGUMENT, "dgmx_set_state_async needs page-locked host memory");
  cudaSetDevice(d->prm.device);
  cudaError_t e = cudaMemcpyAsync(d->nod_in, U, sizeof(double) * d->nnodal(), cudaMemcpyHostToDevice, d->stream);
  if (e != cudaSuccess) return d->cuda(e, "state upload");
  return enqueue_state_from_device_nodal(d, d->nod_in);
}

dgmx_status dgmx_get_state_async(dgmx_domain *d, double *U) {
  if (!d || !U) return DGMX_ERR_ARGUMENT;
  if (d->partitioned()) return d->fail(DGMX_ERR_UNSUPPORTED, "the asynchronous state calls are not built for partitions");
  if (!is_pinned(U)) return d->fail(DGMX_ERR_ARGUMENT, "dgmx_get_state_async needs page-locked host memory");
  cudaSetDevice(d->prm.device);
  StageArgs a = d->base_args();
  cudaError_t e = d->ops->backward(a, d->U, d->nod_out, d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "backward kernel");
  e = cudaMemcpyAsync(U, d->nod_out, sizeof(double) * d->nnodal(), cudaMemcpyDeviceToHost, d->stream);
  return d->cuda(e, "state download");
}

dgmx_status dgmx_create(const dgmx_mesh *mesh, const dgmx_params *params, dgmx_domain **out) {
  try {
    return create_impl(mesh, params, out);
  } catch (const std::exception &ex) {
    g_create_error = ex.what();
    return DGMX_ERR_ARGUMENT;
  }
}

}  // extern "C"

namespace {
// (element, side, kind) records with five parameters each into a BoundarySpec
dgmx_status parse_boundaries(int nbc, const int *bc_sides, const double *bc_params, BoundarySpec &b) {
  if (nbc < 0 || (nbc > 0 && (!bc_sides || !bc_params))) { g_create_error = "null argument"; return DGMX_ERR_ARGUMENT; }
  for (int i = 0; i < nbc; ++i) {
    const int k = bc_sides[3 * i + 2];
    if (k < DGMX_BC_SLIP_WALL || k > DGMX_BC_SUPERSONIC_OUTFLOW) {
      g_create_error = "unknown boundary kind " + std::to_string(k);
      return DGMX_ERR_ARGUMENT;
    }
    const int t = b.type_of(k, bc_params + 5 * i);
    if (!t) { g_create_error = "more than 15 distinct boundary types"; return DGMX_ERR_UNSUPPORTED; }
    b.sides.push_back(BoundarySide{bc_sides[3 * i], bc_sides[3 * i + 1], t});
  }
  return DGMX_OK;
}
}  // namespace

extern "C" {

dgmx_status dgmx_create_with_boundaries(const dgmx_mesh *mesh, const dgmx_params *params, int nbc,
                                        const int *bc_sides, const double *bc_params, dgmx_domain **out) {
  if (!mesh || !params || !out) { g_create_error = "null argument"; return DGMX_ERR_ARGUMENT; }
  try {
    BoundarySpec b;
    const dgmx_status st = parse_boundaries(nbc, bc_sides, bc_params, b);
    if (st != DGMX_OK) return st;
    return create_impl(mesh, params, out, &b);
  } catch (const std::exception &ex) {
    g_create_error = ex.what();
    return DGMX_ERR_ARGUMENT;
  }
}

dgmx_status dgmx_create_partition(const dgmx_mesh *mesh, const dgmx_params *params, const int *part, int nranks,
                                  int rank, dgmx_domain **out) {
  return dgmx_create_partition_with_boundaries(mesh, params, part, nranks, rank, 0, nullptr, nullptr, out);
}

dgmx_status dgmx_create_partition_with_boundaries(const dgmx_mesh *mesh, const dgmx_params *params, const int *part,
                                                  int nranks, int rank, int nbc, const int *bc_sides,
                                                  const double *bc_params, dgmx_domain **out) {
  if (!mesh || !params || !part || !out || nranks < 1) { g_create_error = "null argument"; return DGMX_ERR_ARGUMENT; }
  try {
    BoundarySpec b;
    const dgmx_status st = parse_boundaries(nbc, bc_sides, bc_params, b);
    if (st != DGMX_OK) return st;
    PartitionSpec ps;
    ps.part = part; ps.nranks = nranks; ps.rank = rank;
    return create_impl(mesh, params, out, nbc > 0 ? &b : nullptr, &ps);
  } catch (const std::exception &ex) {
    g_create_error = ex.what();
    return DGMX_ERR_ARGUMENT;
  }
}

dgmx_status dgmx_nccl_unique_id(unsigned char *id) {
  if (!id) return DGMX_ERR_ARGUMENT;
  const NcclApi &nc = nccl_api();
  if (!nc.ok) { g_create_error = nc.why; return DGMX_ERR_UNSUPPORTED; }
  ncclUniqueId u;
  const ncclResult_t r = nc.GetUniqueId(&u);
  if (r != ncclSuccess) { g_create_error = nc.GetErrorString(r); return DGMX_ERR_CUDA; }
  static_assert(sizeof(u.internal) == DGMX_NCCL_ID_BYTES, "NCCL unique id size");
  std::memcpy(id, u.internal, DGMX_NCCL_ID_BYTES);
  return DGMX_OK;
}

dgmx_status dgmx_set_exchange_nccl(dgmx_domain *d, const unsigned char *id) {
  if (!d || !id) return DGMX_ERR_ARGUMENT;
  if (!d->partitioned() || d->in_group) return d->fail(DGMX_ERR_ARGUMENT, "not a rank of a partitioned domain");
  const NcclApi &nc = nccl_api();
  if (!nc.ok) return d->fail(DGMX_ERR_UNSUPPORTED, nc.why);
  cudaSetDevice(d->prm.device);
  ncclUniqueId u;
  std::memcpy(u.internal, id, DGMX_NCCL_ID_BYTES);
  if (d->nccl) { nc.CommDestroy(d->nccl); d->nccl = nullptr; }
  const ncclResult_t r = nc.CommInitRank(&d->nccl, d->plan.nranks, u, d->plan.rank);
  if (r != ncclSuccess) { d->nccl = nullptr; return d->fail(DGMX_ERR_CUDA, std::string("ncclCommInitRank: ") + nc.GetErrorString(r)); }
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  // exchange overlapped with the interior tiles
  cudaError_t e = cudaSuccess;
  if (!d->xstream) e = cudaStreamCreateWithFlags(&d->xstream, cudaStreamNonBlocking);
  if (e == cudaSuccess && !d->ev_b) e = cudaEventCreateWithFlags(&d->ev_b, cudaEventDisableTiming);
  if (e == cudaSuccess && !d->ev_x) e = cudaEventCreateWithFlags(&d->ev_x, cudaEventDisableTiming);
  if (e != cudaSuccess) return d->cuda(e, "exchange stream");
  return build_tiles(d);
}

dgmx_status dgmx_set_exchange_host(dgmx_domain *d, dgmx_exchange_fn fn, void *ctx) {
  if (!d || !fn) return DGMX_ERR_ARGUMENT;
  if (!d->partitioned() || d->in_group) return d->fail(DGMX_ERR_ARGUMENT, "not a rank of a partitioned domain");
  cudaSetDevice(d->prm.device);
  const size_t n = (size_t)std::max(1, d->x_total) * d->nf * d->gf;
  cudaError_t e = cudaSuccess;
  if (!d->xh_send) e = cudaHostAlloc(reinterpret_cast<void **>(&d->xh_send), sizeof(double) * n, cudaHostAllocDefault);
  if (e == cudaSuccess && !d->xh_recv)
    e = cudaHostAlloc(reinterpret_cast<void **>(&d->xh_recv), sizeof(double) * n, cudaHostAllocDefault);
  if (e != cudaSuccess) return d->cuda(e, "host halo buffers");
  d->xhost = fn; d->xhost_ctx = ctx;
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  return DGMX_OK;
}

dgmx_status dgmx_partition_info(const dgmx_domain *d, int *ne_local, int *nghost, int *global_of_local) {
  if (!d) return DGMX_ERR_ARGUMENT;
  if (ne_local) *ne_local = d->ne;
  if (nghost) *nghost = d->plan.nghost;
  if (global_of_local) {
    if (d->partitioned()) std::memcpy(global_of_local, d->plan.global_of_local.data(), sizeof(int) * d->ne);
    else for (int e = 0; e < d->ne; ++e) global_of_local[e] = e;
  }
  return DGMX_OK;
}

dgmx_status dgmx_set_source(dgmx_domain *d, const double *S) {
  if (!d) return DGMX_ERR_ARGUMENT;
  if (d->dim == 3)
    return d->fail(DGMX_ERR_UNSUPPORTED, "source terms are a 2-D feature: Euler3d and Navier_Stokes3d::time_derivative "
                                         "apply none");
  cudaSetDevice(d->prm.device);
  if (!S) {   // clear
    if (d->Ssrc) {
      cudaError_t e = cudaStreamSynchronize(d->stream);
      cudaFree(d->Ssrc);
      d->Ssrc = nullptr;
      if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
      if (e != cudaSuccess) return d->cuda(e, "source clear");
    }
    return DGMX_OK;
  }
  if (!d->Ssrc) {
    cudaError_t e = dalloc(&d->Ssrc, d->nmodal());
    if (e != cudaSuccess) { d->Ssrc = nullptr; return d->cuda(e, "alloc source"); }
    if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  }
  // upload the GLL values and project them once (Field layout in, register layout out)
  const size_t n = d->nnodal();
  const double *src = S;
  if (!is_pinned(S)) { std::memcpy(d->host_pinned, S, sizeof(double) * n); src = d->host_pinned; }
  cudaError_t e = cudaMemcpyAsync(d->nod_in, src, sizeof(double) * n, cudaMemcpyHostToDevice, d->stream);
  if (e != cudaSuccess) return d->cuda(e, "source upload");
  StageArgs a = d->base_args();
  e = d->ops->forward(a, d->nod_in, d->Ssrc, d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "forward kernel");
  return d->cuda(cudaStreamSynchronize(d->stream), "set_source");
}

dgmx_status dgmx_set_time(dgmx_domain *d, double t) {
  if (!d) return DGMX_ERR_ARGUMENT;
  d->t = t;
  return DGMX_OK;
}

dgmx_status dgmx_get_time(const dgmx_domain *d, double *t) {
  if (!d || !t) return DGMX_ERR_ARGUMENT;
  *t = d->t;
  return DGMX_OK;
}

dgmx_status dgmx_set_source_pulse(dgmx_domain *d, double t0, double sigma_t) {
  if (!d) return DGMX_ERR_ARGUMENT;
  if (d->dim == 3) return d->fail(DGMX_ERR_UNSUPPORTED, "source terms are a 2-D feature");
  if (sigma_t > 0.0 && d->partitioned())
    return d->fail(DGMX_ERR_UNSUPPORTED, "the source pulse is not built for partitions");
  d->pulse = sigma_t > 0.0;
  d->pulse_t0 = t0;
  d->pulse_s2t2i = d->pulse ? 1.0 / (2.0 * sigma_t * sigma_t) : 0.0;
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  return DGMX_OK;
}

dgmx_status dgmx_set_bulk_hold(dgmx_domain *d, int on) {
  if (!d) return DGMX_ERR_ARGUMENT;
  if (on && !d->R0) return d->fail(DGMX_ERR_UNSUPPORTED, "the bulk-flow hold is a Navier-Stokes 3-D option");
  if (on && d->partitioned() && !d->R0g) return d->fail(DGMX_ERR_UNSUPPORTED, "partition without the whole-mesh hold buffers");
  if (d->hold != (on != 0)) {
    d->hold = on != 0;
    if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  }
  return DGMX_OK;
}

dgmx_status dgmx_create_from_files(const char *root, const dgmx_params *params, dgmx_domain **out) {
  if (!root || !params || !out) { g_create_error = "null argument"; return DGMX_ERR_ARGUMENT; }
  try {
    FileCase fc;
    std::string err;
    if (!read_case_files(root, fc, err)) { g_create_error = err; return DGMX_ERR_IO; }
    dgmx_params p = *params;
    if (fc.eqntype >= 0) p.physics = fc.eqntype;
    if (fc.inttype >= 0) p.inttype = fc.inttype;
    if (fc.gamma > 0) p.gamma = fc.gamma;
    if (fc.vis >= 0) p.vis = fc.vis;
    if (fc.Pr > 0) p.Pr = fc.Pr;
    if (!fc.flux.empty())
      p.flux = fc.flux == "roe" ? DGMX_FLUX_ROE
               : fc.flux == "stegerwarming" ? DGMX_FLUX_STEGER_WARMING
               : fc.flux == "vanleer" ? DGMX_FLUX_VAN_LEER : DGMX_FLUX_LF;
    dgmx_mesh m;
    m.dim = fc.dim; m.ne = fc.ne; m.verts = fc.verts.data();
    m.ncon = (int)(fc.con.size() / 4); m.con = fc.con.data();
    m.porder = fc.porder.data(); m.qorder = fc.qorder.data();
    // boundary sides: root.bc records typed by root.bct blocks; the kind
    // follows the physics' BC databases (src/Euler3d.cpp:855-870,
    // src/Navier_Stokes3d.cpp:430-455)
    BoundarySpec b;
    b.hold = p.physics == DGMX_NS3D && fc.channel;
    for (const auto &r : fc.bcs) {
      auto it = fc.bct.find(r.tag);
      std::string code;
      std::vector<double> vals;
      if (it != fc.bct.end()) { code = it->second.first; vals = it->second.second; }
      int k = 0;
      double pa = 0.0, pb = 0.0, st[5] = {0, 0, 0, 0, 0};
      const bool euler = p.physics == DGMX_EULER3D || p.physics == DGMX_EULER2D;
      const bool ns = p.physics == DGMX_NS3D || p.physics == DGMX_NS2D;
      const int nfp = nfields_of(p.physics);
      if ((euler || ns) && code == "state" && (int)vals.size() == nfp) {
        k = DGMX_BC_STATE;                     // StateBC(tag, in, nf): src/BC.hpp:184-193
        for (int i = 0; i < nfp; ++i) st[i] = vals[i];
      } else if ((euler || ns) && code.empty() && r.tag == "S") {
        // default "S": Ma 0.3 uniform flow (src/Euler.cpp:1202-1207, src/Euler3d.cpp:828-834,
        // src/Navier_Stokes.cpp:263-269, src/Navier_Stokes3d.cpp:402-409)
        k = DGMX_BC_STATE;
        st[0] = 1.0; st[1] = 1.0; st[nfp - 1] = 20.34126984126985;
      } else if (fc.dim == 2 && (euler || ns) && code.find("outflow") != std::string::npos && vals.size() >= 1 &&
                 (code.find("subsonicoutflow") != std::string::npos ||
                  code.find("supersonicoutflow") != std::string::npos)) {
        // both codes build SubsonicOutflowBC (src/Euler.cpp:1253-1258, src/Navier_Stokes.cpp:348-354)
        k = DGMX_BC_SUBSONIC_OUTFLOW; st[0] = vals[0];
      } else if (fc.dim == 2 && euler && code.empty() && r.tag == "O") {
        k = DGMX_BC_SUPERSONIC_OUTFLOW;        // default "O" (src/Euler.cpp:1209)
      } else if ((euler || p.physics == DGMX_SHALLOW) && code.find("wall") != std::string::npos) {
        k = DGMX_BC_SLIP_WALL;   // src/Euler.cpp:1241-1243, src/Euler3d.cpp:862-866, src/Shallow.cpp:782-785
      } else if ((euler || p.physics == DGMX_SHALLOW) && code.empty() && r.tag == "W") {
        k = DGMX_BC_SLIP_WALL;                 // default "W" (src/Euler.cpp:1208, src/Euler3d.cpp:835)
      } else if (ns && code == "isothermal_wall" && vals.size() >= 2) {
        k = DGMX_BC_ISOTHERMAL_WALL; pa = vals[0]; pb = vals[1];
      } else if (ns && code.empty() && r.tag == "W") {
        // default "W" (src/Navier_Stokes.cpp:263-270, src/Navier_Stokes3d.cpp:403-410)
        k = DGMX_BC_ISOTHERMAL_WALL; pa = 1.0; pb = 20.34126984126985;
      } else {
        g_create_error = std::string(root) + ".bc: boundary type '" + r.tag + "' (" +
                         (code.empty() ? "no .bct entry" : code) + ") is not built for this physics";
        return DGMX_ERR_UNSUPPORTED;
      }
      if (k == DGMX_BC_ISOTHERMAL_WALL) { st[0] = pa; st[1] = pb; }
      const int t = b.type_of(k, st);
      if (!t) { g_create_error = "more than 15 distinct boundary types"; return DGMX_ERR_UNSUPPORTED; }
      b.sides.push_back(BoundarySide{r.e, r.s, t});
    }
    return create_impl(&m, &p, out, &b);
  } catch (const std::exception &ex) {
    g_create_error = ex.what();
    return DGMX_ERR_IO;
  }
}

dgmx_status dgmx_destroy(dgmx_domain *d) {
  if (!d) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  if (d->stream) cudaStreamSynchronize(d->stream);
  d->release();
  delete d;
  return DGMX_OK;
}

dgmx_status dgmx_sizes(const dgmx_domain *d, long *nf, long *nq, long *nm) {
  if (!d) return DGMX_ERR_ARGUMENT;
  if (nf) *nf = d->nf;
  if (nq) *nq = (long)d->ne * d->qd;
  if (nm) *nm = (long)d->ne * d->ld;
  return DGMX_OK;
}

dgmx_status dgmx_coordinates(const dgmx_domain *d, double *x, double *y, double *z) {
  if (!d) return DGMX_ERR_ARGUMENT;
  const size_t n = d->mesh.cx.size();
  if (x) std::memcpy(x, d->mesh.cx.data(), sizeof(double) * n);
  if (y) std::memcpy(y, d->mesh.cy.data(), sizeof(double) * n);
  if (z) std::memcpy(z, d->mesh.cz.data(), sizeof(double) * n);
  return DGMX_OK;
}

dgmx_status dgmx_set_state_device(dgmx_domain *d, const double *U_dev) {
  if (!d || !U_dev) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  return set_state_from_device_nodal(d, U_dev);
}

dgmx_status dgmx_set_state(dgmx_domain *d, const double *U) {
  if (!d || !U) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  const size_t n = d->nnodal();
  const double *src = U;
  if (!is_pinned(U)) { std::memcpy(d->host_pinned, U, sizeof(double) * n); src = d->host_pinned; }
  cudaError_t e = cudaMemcpyAsync(d->nod_in, src, sizeof(double) * n, cudaMemcpyHostToDevice, d->stream);
  if (e != cudaSuccess) return d->cuda(e, "state upload");
  return set_state_from_device_nodal(d, d->nod_in);
}

dgmx_status dgmx_get_state_device(dgmx_domain *d, double *U_dev) {
  if (!d || !U_dev) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  StageArgs a = d->base_args();
  cudaError_t e = d->ops->backward(a, d->U, U_dev, d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "backward kernel");
  return d->cuda(cudaStreamSynchronize(d->stream), "get_state");
}

dgmx_status dgmx_get_state(dgmx_domain *d, double *U) {
  if (!d || !U) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  StageArgs a = d->base_args();
  cudaError_t e = d->ops->backward(a, d->U, d->nod_out, d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "backward kernel");
  const size_t n = d->nnodal();
  const bool direct = is_pinned(U);
  if ((e = cudaMemcpyAsync(direct ? U : d->host_pinned, d->nod_out, sizeof(double) * n, cudaMemcpyDeviceToHost,
                           d->stream)))
    return d->cuda(e, "state download");
  if ((e = cudaStreamSynchronize(d->stream))) return d->cuda(e, "get_state");
  if (!direct) std::memcpy(U, d->host_pinned, sizeof(double) * n);
  return DGMX_OK;
}

dgmx_status dgmx_get_modes(dgmx_domain *d, double *Uh) {
  if (!d || !Uh) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  std::vector<double> em(d->nmodal());
  cudaError_t e = cudaMemcpyAsync(em.data(), d->U, sizeof(double) * em.size(), cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return d->cuda(e, "modes download");
  // element-major [e][n][m] -> restart layout [n][e][m]
  for (int el = 0; el < d->ne; ++el)
    for (int n = 0; n < d->nf; ++n)
      std::memcpy(Uh + ((size_t)n * d->ne + el) * d->ld, em.data() + ((size_t)el * d->nf + n) * d->ld,
                  sizeof(double) * d->ld);
  return DGMX_OK;
}

dgmx_status dgmx_set_modes(dgmx_domain *d, const double *Uh) {
  if (!d || !Uh) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  // restart layout [n][e][m] -> element-major [e][n][m]
  std::vector<double> em(d->nmodal());
  for (int el = 0; el < d->ne; ++el)
    for (int n = 0; n < d->nf; ++n)
      std::memcpy(em.data() + ((size_t)el * d->nf + n) * d->ld, Uh + ((size_t)n * d->ne + el) * d->ld,
                  sizeof(double) * d->ld);
  cudaError_t e = cudaMemcpyAsync(d->U, em.data(), sizeof(double) * em.size(), cudaMemcpyHostToDevice, d->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d->Ut, 0, sizeof(double) * d->nmodal(), d->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(d->Acc, 0, sizeof(double) * d->nmodal(), d->stream);
  if (e == cudaSuccess && d->Utf) e = cudaMemsetAsync(d->Utf, 0, sizeof(float) * d->nmodal(), d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return d->cuda(e, "set_modes");
  d->tcur = 0;
  d->sw_captured = false;
  const dgmx_status st = refresh_traces(d);
  if (st != DGMX_OK) return st;
  return d->cuda(cudaStreamSynchronize(d->stream), "set_modes");
}

dgmx_status dgmx_write_restart(dgmx_domain *d, const char *path, int step, double t, double dt) {
  if (!d || !path) return DGMX_ERR_ARGUMENT;
  std::vector<double> Uh((size_t)d->nf * d->ne * d->ld);
  dgmx_status st = dgmx_get_modes(d, Uh.data());
  if (st != DGMX_OK) return st;
  st = dgmx_restart_write(path, d->prm.physics, d->ne, d->ld, step, t, dt, d->prm.vis, Uh.data());
  if (st != DGMX_OK) d->errmsg = dgmx_restart_last_error();
  return st;
}

dgmx_status dgmx_read_restart(dgmx_domain *d, const char *path, int *step, double *t) {
  if (!d || !path) return DGMX_ERR_ARGUMENT;
  int ne = 0, nsd = 0, lmax = 0, stp = 0;
  double tt = 0, dt = 0, vis = 0;
  dgmx_status st = dgmx_restart_info(path, &ne, &nsd, &lmax, &stp, &tt, &dt, &vis);
  if (st != DGMX_OK) { d->errmsg = dgmx_restart_last_error(); return st; }
  if (ne != d->ne || nsd != d->dim) return d->fail(DGMX_ERR_ARGUMENT, "restart: mesh size or dimension differs");
  std::vector<int> nm(ne);
  std::vector<double> Uh((size_t)d->nf * d->ne * d->ld);
  st = dgmx_restart_read(path, d->nf, ne, nm.data(), Uh.data(), (long long)Uh.size());
  if (st != DGMX_OK) { d->errmsg = dgmx_restart_last_error(); return st; }
  for (int e = 0; e < ne; ++e)
    if (nm[e] != d->ld) return d->fail(DGMX_ERR_ARGUMENT, "restart: mode count differs from this domain's order");
  st = dgmx_set_modes(d, Uh.data());
  if (st != DGMX_OK) return st;
  if (step) *step = stp;
  if (t) *t = tt;
  return DGMX_OK;
}

dgmx_status dgmx_time_derivative_device(dgmx_domain *d, const double *U_dev, double *F_dev) {
  if (!d || !U_dev || !F_dev) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  StageArgs a = d->base_args();
  a.Xn = U_dev; a.Fn = F_dev;
  a.Tout = d->T[d->tcur ^ 1];
  cudaError_t e = d->ops->traces_nodal(a, d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "nodal trace kernel");
  dgmx_status xs = exchange(d, fp64_halo(d->T[d->tcur ^ 1], d->nf * d->gf));
  if (xs != DGMX_OK) return xs;
  a.Tin = d->T[d->tcur ^ 1];
  if (d->prm.physics == DGMX_SHALLOW && d->prm.sw_balance) {
    if (!d->sw_captured) { a.Rcap = d->Rsw; d->sw_captured = true; }
    a.Rsub = d->Rsw;
  }
  if (d->ns()) {
    if ((e = d->ns_grad(a, true, d->stream)) != cudaSuccess) return d->cuda(e, "viscous gradient kernel");
    if ((e = d->ns_visc(a, true, d->stream)) != cudaSuccess) return d->cuda(e, "viscous flux kernel");
    d->launches += 2;
    if ((xs = exchange(d, visc_halo(d))) != DGMX_OK) return xs;
  }
  a.R0 = d->hold ? d->R0 : nullptr;
  e = d->ops->rhs_nodal(a, d->stream);
  ++d->launches;
  if (e != cudaSuccess) return d->cuda(e, "nodal rhs kernel");
  if (d->hold) {
    a.kind = kRHS; a.A = nullptr;
    if ((xs = hold_stage(d, a, nullptr, F_dev)) != DGMX_OK) return xs;
  }
  // the traces of the current modal register live in T[tcur]; T[tcur^1]
  // was used as scratch and is rewritten by the next stage.
  return DGMX_OK;
}

dgmx_status dgmx_time_derivative(dgmx_domain *d, const double *U, double *F) {
  if (!d || !U || !F) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  const size_t n = d->nnodal();
  dgmx_status st = reset_error_word(d);
  if (st != DGMX_OK) return st;
  const bool pin_in = is_pinned(U), pin_out = is_pinned(F);
  if (!pin_in) std::memcpy(d->host_pinned, U, sizeof(double) * n);
  cudaError_t e = cudaMemcpyAsync(d->nod_in, pin_in ? U : d->host_pinned, sizeof(double) * n,
                                  cudaMemcpyHostToDevice, d->stream);
  if (e != cudaSuccess) return d->cuda(e, "upload");
  if ((st = dgmx_time_derivative_device(d, d->nod_in, d->nod_out)) != DGMX_OK) return st;
  if ((e = cudaMemcpyAsync(pin_out ? F : d->host_pinned + n, d->nod_out, sizeof(double) * n,
                           cudaMemcpyDeviceToHost, d->stream)))
    return d->cuda(e, "download");
  if ((st = check_error_word(d)) != DGMX_OK) return st;
  if (!pin_out) std::memcpy(F, d->host_pinned + n, sizeof(double) * n);
  return DGMX_OK;
}

dgmx_status dgmx_advance_async(dgmx_domain *d, double dt, int nsteps) {
  if (!d || nsteps < 0) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  if (nsteps == 0) return DGMX_OK;
  dgmx_status st;
  if (d->prm.physics == DGMX_SHALLOW && d->prm.sw_balance && !d->sw_captured)
    if ((st = capture_sw_source(d)) != DGMX_OK) return st;
  // The trace buffers swap once per stage, so a graph holds two steps when a
  // step has an odd stage count (TVD3) and the buffer parity repeats.  The
  // graph is rebuilt when dt or the starting parity changes.
  if (overlaps(d) && ((st = build_tiles(d)) != DGMX_OK || (st = build_vtiles(d)) != DGMX_OK)) return st;
  const int nst = stages_per_step(d->prm.inttype);
  const int reps = (nst & 1) ? 2 : 1;
  // no graph: host-staged exchanges synchronise every stage, a source pulse
  // changes its factor every stage, and NCCL ranks enqueue their sends and
  // receives directly (a step is a few dozen launches, well under its time)
  if (d->xhost || d->pulse || d->nccl) {
    for (int s = 0; s < nsteps; ++s) {
      if ((st = enqueue_step(d, dt)) != DGMX_OK) return st;
      d->t += dt;
    }
    return DGMX_OK;
  }
  if (nsteps >= reps && (!d->graph || d->graph_dt != dt || d->graph_tcur != d->tcur)) {
    if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
    const int t0 = d->tcur;
    const long l0 = d->launches;
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return d->cuda(e, "graph capture");
    st = DGMX_OK;
    for (int r = 0; r < reps && st == DGMX_OK; ++r) st = enqueue_step(d, dt);
    e = cudaStreamEndCapture(d->stream, &g);
    d->tcur = t0;               // capture recorded the launches, ran nothing
    d->launches = l0;
    if (st != DGMX_OK) return st;
    if (e != cudaSuccess) return d->cuda(e, "graph capture");
    e = cudaGraphInstantiate(&d->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return d->cuda(e, "graph instantiate");
    d->graph_dt = dt;
    d->graph_tcur = t0;
  }
  int s = 0;
  for (; d->graph && s + reps <= nsteps; s += reps) {
    cudaError_t e = cudaGraphLaunch(d->graph, d->stream);
    if (e != cudaSuccess) return d->cuda(e, "graph launch");
    d->launches += (long)nst * reps * launches_per_stage(d);
    for (int r = 0; r < reps; ++r) d->t += dt;
  }
  for (; s < nsteps; ++s) {
    if ((st = enqueue_step(d, dt)) != DGMX_OK) return st;
    d->t += dt;
  }
  return DGMX_OK;
}

dgmx_status dgmx_sync(dgmx_domain *d) {
  if (!d) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  dgmx_status st = check_error_word(d);
  if (st != DGMX_OK) { reset_error_word(d); return st; }
  return DGMX_OK;
}

dgmx_status dgmx_advance(dgmx_domain *d, double dt, int nsteps) {
  dgmx_status st = dgmx_advance_async(d, dt, nsteps);
  if (st != DGMX_OK) return st;
  return dgmx_sync(d);
}

dgmx_status dgmx_integrals(dgmx_domain *d, double *totals) {
  if (!d || !totals) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  // integral of the orthonormal mode 0 over the reference element: 2^d/sqrt(2)^d
  const double c = std::pow(std::sqrt(2.0), d->dim);
  cudaError_t e = launch_integrals(d->nf, d->ne, d->ld, c, d->U, d->Jdev, d->integ, d->stream);
  ++d->launches;
  if (e == cudaSuccess) e = cudaMemcpyAsync(totals, d->integ, sizeof(double) * d->nf, cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  return d->cuda(e, "integrals");
}

const char *dgmx_last_error(const dgmx_domain *d) {
  return d ? d->errmsg.c_str() : g_create_error.c_str();
}

long dgmx_launch_count(const dgmx_domain *d) { return d ? d->launches : 0; }

void *dgmx_stream(const dgmx_domain *d) { return d ? (void *)d->stream : nullptr; }

// Kernel instantiations compiled into this library: rows of (physics, L, Q,
// elements per CTA, threads per CTA, shared memory bytes).  Returns the row
// count; writes at most cap rows.
int dgmx_kernel_list(int *rows, int cap) {
  std::vector<std::vector<int>> v;
  list_ops(v);
  for (int i = 0; i < (int)v.size() && i < cap; ++i)
    for (int k = 0; k < 7; ++k) rows[i * 7 + k] = v[i][k];
  return (int)v.size();
}

// Autotuner: times every compiled tile variant (elements per CTA, register
// cap) of this handle's (physics, L, Q) on the handle's own mesh with
// right-hand-side-only stage launches (the state is not modified) and keeps
// the fastest.  rows (optional, cap rows of 4 doubles): epb, minb, threads,
// microseconds per launch.  Returns the variant count in *nvariants and the
// chosen index in *chosen.
dgmx_status dgmx_autotune(dgmx_domain *d, int reps, double *rows, int cap, int *nvariants, int *chosen) {
  if (!d || reps <= 0) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  const std::vector<KernelOps> *vs =
      find_variants(d->prm.physics + (d->mixed() ? kMixedKey : 0), d->L, d->Q);
  if (!vs || vs->empty()) return d->fail(DGMX_ERR_UNSUPPORTED, "no kernel variants");
  double *scratch = nullptr;
  cudaError_t e = dalloc(&scratch, d->nmodal());
  if (e != cudaSuccess) return d->cuda(e, "autotune scratch");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = -1;
  float best_ms = 0.f;
  dgmx_status st = DGMX_OK;
  for (size_t i = 0; i < vs->size() && st == DGMX_OK; ++i) {
    const KernelOps &v = (*vs)[i];
    if (d->nbct && v.warp != 0) {   // the prefetching kernel has no boundary sides
      if ((int)i < cap && rows) {
        rows[4 * i + 0] = v.epb; rows[4 * i + 1] = v.minb; rows[4 * i + 2] = v.nt; rows[4 * i + 3] = 0.0;
      }
      continue;
    }
    if ((e = v.init(d->tab)) != cudaSuccess) { st = d->cuda(e, "variant init"); break; }
    StageArgs a = d->base_args();
    a.kind = kRHS; a.X = d->U; a.U = d->U; a.Ut = d->Ut; a.A = scratch;
    a.Tin = d->T[d->tcur]; a.Tout = d->T[d->tcur ^ 1];
    if (d->mixed()) { a.Utf = d->Utf; a.Tinf = d->Tf[d->tcur]; a.Toutf = d->Tf[d->tcur ^ 1]; }
    for (int w = 0; w < 2; ++w) e = v.stage(a, d->stream);
    cudaEventRecord(e0, d->stream);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = v.stage(a, d->stream);
    cudaEventRecord(e1, d->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) { st = d->cuda(e, "autotune launch"); break; }
    d->launches += 2 + reps;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= reps;
    if ((int)i < cap && rows) {
      rows[4 * i + 0] = v.epb; rows[4 * i + 1] = v.minb; rows[4 * i + 2] = v.nt; rows[4 * i + 3] = 1e3 * ms;
    }
    if (best < 0 || ms < best_ms) { best = (int)i; best_ms = ms; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(scratch);
  if (st != DGMX_OK) return st;
  // the timing launches evaluate whatever state the handle holds (possibly
  // none yet): what they flagged says nothing about the caller's next call
  if ((st = reset_error_word(d)) != DGMX_OK) return st;
  const KernelOps &chosen_ops = (*vs)[best];
  if ((e = chosen_ops.init(d->tab)) != cudaSuccess) return d->cuda(e, "variant init");
  if (d->mixed()) d->ops_m = &chosen_ops; else d->ops = &chosen_ops;
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  if (nvariants) *nvariants = (int)vs->size();
  if (chosen) *chosen = best;
  return DGMX_OK;
}

dgmx_status dgmx_set_tensor_contractions(dgmx_domain *d, int on) {
  if (!d) return DGMX_ERR_ARGUMENT;
  if (on && (!d->visc32 || !d->vops || !d->vops->ns_grad32tc))
    return d->fail(DGMX_ERR_UNSUPPORTED, "tensor-core contractions run in the FP32 viscous form (precision "
                                         "DGMX_MIXED) of Navier-Stokes 3-D at p >= 5");
  d->visc_tc = on != 0;
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  return DGMX_OK;
}

dgmx_status dgmx_set_wait_limit(dgmx_domain *d, int tries) {
  if (!d) return DGMX_ERR_ARGUMENT;
  d->wait_tries = tries < 0 ? kWaitTries : tries;
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  return DGMX_OK;
}

dgmx_status dgmx_set_variant(dgmx_domain *d, int index, int *count, int *warp) {
  if (!d) return DGMX_ERR_ARGUMENT;
  cudaSetDevice(d->prm.device);
  const std::vector<KernelOps> *vs = find_variants(d->prm.physics + (d->mixed() ? kMixedKey : 0), d->L, d->Q);
  if (!vs || vs->empty()) return d->fail(DGMX_ERR_UNSUPPORTED, "no kernel variants");
  if (count) *count = (int)vs->size();
  if (index < 0 || index >= (int)vs->size()) return d->fail(DGMX_ERR_ARGUMENT, "no such variant");
  const KernelOps &v = (*vs)[index];
  if (d->nbct && v.warp != 0) {
    if (warp) *warp = v.warp;
    return d->fail(DGMX_ERR_UNSUPPORTED, "the prefetching kernel does not handle boundary sides");
  }
  const cudaError_t e = v.init(d->tab);
  if (e != cudaSuccess) return d->cuda(e, "variant init");
  if (d->mixed()) d->ops_m = &v; else d->ops = &v;
  if (d->graph) { cudaGraphExecDestroy(d->graph); d->graph = nullptr; }
  if (warp) *warp = v.warp;
  return DGMX_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// In-process partitions: every part of an element partition as its own
// handle on one device, stepped in lockstep on one stream with the halo
// exchange done by device copies between the parts' buffers (pack on the
// owner, copy, unpack into the receiver's ghost slots: the same lists and
// kernels the NCCL path uses).  It runs the partitioned path where only one
// GPU is present.
struct dgmx_group {
  std::vector<dgmx_domain *> parts;
  std::vector<int> part;
  int ne = 0;
  std::string errmsg;
  cudaStream_t xs = nullptr;                 // the exchange, overlapped with the interior tiles
  cudaEvent_t ev_b = nullptr, ev_x = nullptr;
  ~dgmx_group() {
    if (ev_b) cudaEventDestroy(ev_b);
    if (ev_x) cudaEventDestroy(ev_x);
    if (xs) cudaStreamDestroy(xs);
    for (dgmx_domain *d : parts) {
      if (!d) continue;
      cudaSetDevice(d->prm.device);
      if (d->stream) cudaStreamSynchronize(d->stream);
      d->release();
      delete d;
    }
  }
  cudaStream_t stream() const { return parts[0]->stream; }
};

namespace {

// which = 0: stage traces T[tcur], 1: T[tcur ^ 1] (Tf in the mixed form),
// 2: viscous traces; on stream s
dgmx_status group_exchange(dgmx_group *g, int which, cudaStream_t s) {
  auto halo = [&](dgmx_domain *d) { return which == 2 ? visc_halo(d) : trace_halo(d, which == 0 ? d->tcur : d->tcur ^ 1); };
  const int blk = halo(g->parts[0]).wire();   // doubles per block in the send and receive buffers
  cudaError_t e = cudaSuccess;
  for (dgmx_domain *d : g->parts) {
    if (e == cudaSuccess) e = halo(d).pack(d, s);
    ++d->launches;
  }
  const int n = (int)g->parts.size();
  for (int r = 0; r < n && e == cudaSuccess; ++r)
    for (int q = 0; q < n && e == cudaSuccess; ++q) {
      dgmx_domain *dr = g->parts[r], *dq = g->parts[q];
      if (!dr->x_cnt[q]) continue;
      e = cudaMemcpyAsync(dr->x_rbuf + (size_t)dr->x_off[q] * blk, dq->x_sbuf + (size_t)dq->x_off[r] * blk,
                          sizeof(double) * blk * dr->x_cnt[q], cudaMemcpyDeviceToDevice, s);
    }
  for (dgmx_domain *d : g->parts) {
    if (e == cudaSuccess) e = halo(d).unpack(d, s);
    ++d->launches;
  }
  if (e != cudaSuccess) { g->errmsg = std::string("group halo exchange: ") + cudaGetErrorString(e); return DGMX_ERR_CUDA; }
  return DGMX_OK;
}

// Mixed form: one reference row for every part, the unpartitioned
// domain's (the integrands of all parts in global element order, summed as
// launch_reference_integrals does), then each part's FP32 traces.
dgmx_status group_reference(dgmx_group *g) {
  dgmx_domain *d0 = g->parts[0];
  const int nf = d0->nf, ne = g->ne;
  std::vector<double> R((size_t)ne * nf, 0.0), J(ne, 0.0), rows;
  for (dgmx_domain *d : g->parts) {
    dgmx_status st = element_integrands(d, rows);
    if (st != DGMX_OK) { g->errmsg = d->errmsg; return st; }
    for (int e = 0; e < d->ne; ++e) {
      const int gid = d->plan.global_of_local[e];
      J[gid] = d->mesh.J[e];
      for (int n = 0; n < nf; ++n) R[(size_t)gid * nf + n] = rows[(size_t)e * nf + n];
    }
  }
  double tot[5] = {0, 0, 0, 0, 0}, jsum = 0.0;
  reference_sum(R.data(), ne, nf, std::pow(std::sqrt(2.0), d0->dim), tot);
  for (int k = 0; k < ne; ++k) jsum += J[k];
  for (dgmx_domain *d : g->parts) {
    dgmx_status st = upload_reference(d, tot, jsum);
    if (st != DGMX_OK) { g->errmsg = d->errmsg; return st; }
    const StageArgs a = d->base_args();
    cudaError_t e = d->ops_m->traces_modal(a, d->U, d->Tf[d->tcur], d->stream);
    ++d->launches;
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) { g->errmsg = std::string("group traces: ") + cudaGetErrorString(e); return DGMX_ERR_CUDA; }
  }
  return DGMX_OK;
}

dgmx_status group_fail(dgmx_group *g, dgmx_domain *d, dgmx_status st) {
  g->errmsg = d->errmsg;
  return st;
}

}  // namespace

extern "C" {

dgmx_status dgmx_group_create(const dgmx_mesh *mesh, const dgmx_params *params, const int *part, int nparts,
                              dgmx_group **out) {
  return dgmx_group_create_with_boundaries(mesh, params, part, nparts, 0, nullptr, nullptr, out);
}

dgmx_status dgmx_group_create_with_boundaries(const dgmx_mesh *mesh, const dgmx_params *params, const int *part,
                                              int nparts, int nbc, const int *bc_sides, const double *bc_params,
                                              dgmx_group **out) {
  if (!mesh || !params || !part || !out || nparts < 2) { g_create_error = "group: null argument or nparts < 2"; return DGMX_ERR_ARGUMENT; }
  *out = nullptr;
  auto g = std::make_unique<dgmx_group>();
  g->ne = mesh->ne;
  g->part.assign(part, part + mesh->ne);
  for (int r = 0; r < nparts; ++r) {
    PartitionSpec ps;
    ps.part = part; ps.nranks = nparts; ps.rank = r; ps.group = true;
    dgmx_domain *d = nullptr;
    dgmx_status st;
    try {
      BoundarySpec b;
      st = parse_boundaries(nbc, bc_sides, bc_params, b);
      if (st == DGMX_OK) st = create_impl(mesh, params, &d, nbc > 0 ? &b : nullptr, &ps);
    } catch (const std::exception &ex) {
      g_create_error = ex.what();
      st = DGMX_ERR_ARGUMENT;
    }
    if (st != DGMX_OK) return st;
    g->parts.push_back(d);
  }
  *out = g.release();
  return DGMX_OK;
}

dgmx_status dgmx_group_set_bulk_hold(dgmx_group *g, int on) {
  if (!g) return DGMX_ERR_ARGUMENT;
  for (dgmx_domain *d : g->parts) {
    const dgmx_status st = dgmx_set_bulk_hold(d, on);
    if (st != DGMX_OK) return group_fail(g, d, st);
  }
  return DGMX_OK;
}

dgmx_status dgmx_group_destroy(dgmx_group *g) {
  if (!g) return DGMX_ERR_ARGUMENT;
  delete g;
  return DGMX_OK;
}

dgmx_domain *dgmx_group_part(dgmx_group *g, int r) {
  return g && r >= 0 && r < (int)g->parts.size() ? g->parts[r] : nullptr;
}

const char *dgmx_group_last_error(const dgmx_group *g) { return g ? g->errmsg.c_str() : g_create_error.c_str(); }

dgmx_status dgmx_group_set_state(dgmx_group *g, const double *U) {
  if (!g || !U) return DGMX_ERR_ARGUMENT;
  dgmx_domain *d0 = g->parts[0];
  const size_t qd = d0->qd;
  for (dgmx_domain *d : g->parts) {
    std::vector<double> loc((size_t)d->nf * d->ne * qd);
    for (int n = 0; n < d->nf; ++n)
      for (int e = 0; e < d->ne; ++e)
        std::memcpy(&loc[((size_t)n * d->ne + e) * qd], U + ((size_t)n * g->ne + d->plan.global_of_local[e]) * qd,
                    sizeof(double) * qd);
    const dgmx_status st = dgmx_set_state(d, loc.data());
    if (st != DGMX_OK) return group_fail(g, d, st);
  }
  cudaSetDevice(d0->prm.device);
  dgmx_status st = d0->mixed() ? group_reference(g) : DGMX_OK;
  if (st != DGMX_OK) return st;
  st = group_exchange(g, 0, g->stream());
  if (st != DGMX_OK) return st;
  return cudaStreamSynchronize(g->stream()) == cudaSuccess ? DGMX_OK : DGMX_ERR_CUDA;
}

dgmx_status dgmx_group_get_state(dgmx_group *g, double *U) {
  if (!g || !U) return DGMX_ERR_ARGUMENT;
  const size_t qd = g->parts[0]->qd;
  for (dgmx_domain *d : g->parts) {
    std::vector<double> loc((size_t)d->nf * d->ne * qd);
    const dgmx_status st = dgmx_get_state(d, loc.data());
    if (st != DGMX_OK) return group_fail(g, d, st);
    for (int n = 0; n < d->nf; ++n)
      for (int e = 0; e < d->ne; ++e)
        std::memcpy(U + ((size_t)n * g->ne + d->plan.global_of_local[e]) * qd, &loc[((size_t)n * d->ne + e) * qd],
                    sizeof(double) * qd);
  }
  return DGMX_OK;
}

dgmx_status dgmx_group_advance(dgmx_group *g, double dt, int nsteps) {
  if (!g || nsteps < 0) return DGMX_ERR_ARGUMENT;
  dgmx_domain *d0 = g->parts[0];
  cudaSetDevice(d0->prm.device);
  const cudaStream_t s = g->stream();
  const std::vector<StageSpec> specs = stage_specs(d0->prm.inttype, dt);
  if (specs.empty()) { g->errmsg = "inttype must be 3, 4 or 14"; return DGMX_ERR_UNSUPPORTED; }
  for (dgmx_domain *d : g->parts) {
    if (d->prm.physics == DGMX_SHALLOW && d->prm.sw_balance) { g->errmsg = "shallow-water balance is off in groups"; return DGMX_ERR_UNSUPPORTED; }
    if (reset_error_word(d) != DGMX_OK || cudaStreamSynchronize(d->stream) != cudaSuccess) return group_fail(g, d, DGMX_ERR_CUDA);
    if (build_tiles(d) != DGMX_OK || build_vtiles(d) != DGMX_OK) return group_fail(g, d, DGMX_ERR_CUDA);
  }
  if (!g->xs) {
    cudaError_t ce = cudaStreamCreateWithFlags(&g->xs, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&g->ev_b, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&g->ev_x, cudaEventDisableTiming);
    if (ce != cudaSuccess) { g->errmsg = std::string("group streams: ") + cudaGetErrorString(ce); return DGMX_ERR_CUDA; }
  }
  cudaError_t e = cudaSuccess;
  dgmx_status st = DGMX_OK;
  for (int step = 0; step < nsteps && st == DGMX_OK; ++step)
    for (const StageSpec &sp : specs) {
      if (d0->ns()) {
        // gradients, the viscous flux of the boundary tiles, then the
        // exchange of their viscous traces on the side stream while the
        // interior tiles' viscous flux runs
        for (dgmx_domain *d : g->parts) {
          const StageArgs a = stage_args(d, sp, dt);
          if (e == cudaSuccess) e = d->ns_grad(a, false, s);
          if (e == cudaSuccess) e = d->ns_visc_tiles(a, 0, s);
          d->launches += 2;
        }
        if (e == cudaSuccess) e = cudaEventRecord(g->ev_b, s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(g->xs, g->ev_b, 0);
        if (e == cudaSuccess && (st = group_exchange(g, 2, g->xs)) != DGMX_OK) return st;
        if (e == cudaSuccess) e = cudaEventRecord(g->ev_x, g->xs);
        for (dgmx_domain *d : g->parts) {
          const StageArgs a = stage_args(d, sp, dt);
          if (e == cudaSuccess) e = d->ns_visc_tiles(a, 1, s);
          ++d->launches;
        }
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, g->ev_x, 0);
      }
      if (d0->hold) {
        // bulk-flow hold: every part's tiles, the parts' constant
        // coefficients into the whole mesh's order, the unpartitioned
        // domain's means (part 0's buffers), applied to every part, then
        // the exchange of the held traces
        for (dgmx_domain *d : g->parts) {
          const StageArgs a = stage_args(d, sp, dt);
          if (e == cudaSuccess) e = stage_tiles(d, a, 0, s);
          if (e == cudaSuccess) e = stage_tiles(d, a, 1, s);
          if (e == cudaSuccess)
            e = launch_scatter_rows(d->R0, d->gid_all + (size_t)d->plan.rank * d->max_ne, d->ne, d->nf, d0->R0g, s);
          d->launches += 3;
        }
        if (e == cudaSuccess) {
          HoldArgs h = d0->hold_args(stage_args(d0, sp, dt), nullptr, nullptr);
          h.ne = d0->ne_global; h.R0 = d0->R0g; h.J = d0->Jg;
          e = launch_hold_reduce(h, s);
          ++d0->launches;
        }
        for (dgmx_domain *d : g->parts) {
          HoldArgs h = d->hold_args(stage_args(d, sp, dt), d->T[d->tcur ^ 1], nullptr);
          h.cbar = d0->cbar;
          if (e == cudaSuccess) e = launch_hold_apply(h, s);
          ++d->launches;
        }
        if (e == cudaSuccess && (st = group_exchange(g, 1, s)) != DGMX_OK) return st;
        for (dgmx_domain *d : g->parts) d->tcur ^= 1;
        if (e != cudaSuccess) break;
        continue;
      }
      // boundary tiles of every part, then their exchange on the side
      // stream while the interior tiles run
      for (dgmx_domain *d : g->parts) {
        const StageArgs a = stage_args(d, sp, dt);
        if (e == cudaSuccess) e = stage_tiles(d, a, 0, s);
        ++d->launches;
      }
      if (e == cudaSuccess) e = cudaEventRecord(g->ev_b, s);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(g->xs, g->ev_b, 0);
      if (e == cudaSuccess && (st = group_exchange(g, 1, g->xs)) != DGMX_OK) return st;
      if (e == cudaSuccess) e = cudaEventRecord(g->ev_x, g->xs);
      for (dgmx_domain *d : g->parts) {
        const StageArgs a = stage_args(d, sp, dt);
        if (e == cudaSuccess) e = stage_tiles(d, a, 1, s);
        ++d->launches;
      }
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s, g->ev_x, 0);
      for (dgmx_domain *d : g->parts) d->tcur ^= 1;
      if (e != cudaSuccess) break;
    }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) { g->errmsg = std::string("group advance: ") + cudaGetErrorString(e); return DGMX_ERR_CUDA; }
  for (dgmx_domain *d : g->parts) {
    st = check_error_word(d);
    if (st != DGMX_OK) return group_fail(g, d, st);
  }
  return DGMX_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// Host-only inspection entry points (no CUDA calls): the 1-D tables and the
// processed connectivity, so the setup can be checked on machines without a
// GPU.
extern "C" {

dgmx_status dgmx_tables(int L, int Q, double *z, double *w, double *D, double *B, double *Bg, double *gl2g,
                        double *g2gl) {
  if (L < 1 || Q < 2 || !z || !w || !D || !B || !Bg || !gl2g || !g2gl) return DGMX_ERR_ARGUMENT;
  const Tables1D t = make_tables(L, Q, Q - 1);
  std::memcpy(z, t.z.data(), sizeof(double) * Q);
  std::memcpy(w, t.w.data(), sizeof(double) * Q);
  std::memcpy(D, t.D.data(), sizeof(double) * Q * Q);
  std::memcpy(B, t.B.data(), sizeof(double) * L * Q);
  std::memcpy(Bg, t.Bg.data(), sizeof(double) * L * (Q - 1));
  std::memcpy(gl2g, t.gl2g.data(), sizeof(double) * (Q - 1) * Q);
  std::memcpy(g2gl, t.g2gl.data(), sizeof(double) * Q * (Q - 1));
  return DGMX_OK;
}

// The partition plan of one rank (host only).  sizes[0..2] = local
// elements, ghost slots, exchanged blocks; the arrays (each may be NULL, e.g.
// on a first call for the sizes) get the global ids of the local elements
// and of the ghosts, the per-peer block counts (nranks) and the concatenated
// send blocks (local element * nfaces + face) and receive blocks (slot *
// nfaces + face), peers in rank order.
dgmx_status dgmx_partition_plan(const dgmx_mesh *m, const int *part, int nranks, int rank, int *sizes,
                                int *global_of_local, int *global_of_ghost, int *peer_counts, int *send, int *recv) {
  if (!m || !part || !sizes || !m->porder) return DGMX_ERR_ARGUMENT;
  try {
    const int p = m->porder[0], q = (m->qorder && m->qorder[0]) ? m->qorder[0] : p + 2;
    const Tables1D t = make_tables(p + 1, q, q - 1);
    HostMesh hm, loc;
    PartitionPlan plan;
    std::string err;
    if (!build_mesh(*m, t, hm, err) || !partition_mesh(hm, part, nranks, rank, loc, plan, err)) {
      g_create_error = err;
      return DGMX_ERR_ARGUMENT;
    }
    int nb = 0;
    for (int r = 0; r < nranks; ++r) nb += (int)plan.send[r].size();
    sizes[0] = plan.ne_local; sizes[1] = plan.nghost; sizes[2] = nb;
    if (global_of_local) std::copy(plan.global_of_local.begin(), plan.global_of_local.end(), global_of_local);
    if (global_of_ghost) std::copy(plan.global_of_ghost.begin(), plan.global_of_ghost.end(), global_of_ghost);
    for (int r = 0, at = 0; r < nranks; ++r) {
      if (peer_counts) peer_counts[r] = (int)plan.send[r].size();
      if (send) std::copy(plan.send[r].begin(), plan.send[r].end(), send + at);
      if (recv) std::copy(plan.recv[r].begin(), plan.recv[r].end(), recv + at);
      at += (int)plan.send[r].size();
    }
    return DGMX_OK;
  } catch (const std::exception &ex) {
    g_create_error = ex.what();
    return DGMX_ERR_ARGUMENT;
  }
}

// links: ne*nfaces*4 ints (neighbour, neighbour face, master flag, class id);
// perm_pairs: ne*nfaces*gf ints, the neighbour's point index for each own
// face point.  Uses mesh->porder[0]/qorder[0].
dgmx_status dgmx_mesh_links(const dgmx_mesh *m, int *links, int *perm_pairs) {
  if (!m || !links || !perm_pairs || !m->porder) return DGMX_ERR_ARGUMENT;
  try {
    const int p = m->porder[0], q = (m->qorder && m->qorder[0]) ? m->qorder[0] : p + 2;
    const Tables1D t = make_tables(p + 1, q, q - 1);
    HostMesh hm;
    std::string err;
    if (!build_mesh(*m, t, hm, err)) { g_create_error = err; return DGMX_ERR_ARGUMENT; }
    for (int e = 0; e < hm.ne; ++e)
      for (int f = 0; f < hm.nfaces; ++f) {
        const FaceLink &l = hm.links[(size_t)e * hm.nfaces + f];
        const GeomClass &c = hm.classes[hm.gclass[e]];
        int *o = links + ((size_t)e * hm.nfaces + f) * 4;
        o[0] = l.elem; o[1] = l.face; o[2] = (c.master >> f) & 1; o[3] = hm.gclass[e];
        for (int g = 0; g < hm.gf; ++g) perm_pairs[((size_t)e * hm.nfaces + f) * hm.gf + g] = hm.perm[l.perm + g];
      }
    return DGMX_OK;
  } catch (const std::exception &ex) {
    g_create_error = ex.what();
    return DGMX_ERR_ARGUMENT;
  }
}

}  // extern "C"

// ------------------------------------------------------------------------
// Read-only view of a handle for entry points compiled in other units.
namespace dgmx {
bool domain_view(dgmx_domain *d, DomainView *v, bool *partitioned, std::string **errmsg) {
  if (partitioned) *partitioned = d && d->partitioned();
  if (errmsg) *errmsg = d ? &d->errmsg : nullptr;
  if (!d || !v || d->partitioned()) return false;
  v->ops = d->ops;
  v->stream = d->stream;
  v->base = d->base_args();
  v->ntrace = d->ntrace();
  v->device = d->prm.device;
  v->sw_balance = d->prm.physics == DGMX_SHALLOW && d->prm.sw_balance;
  v->Rsw = d->Rsw;
  v->sw_captured = &d->sw_captured;
  v->errmsg = &d->errmsg;
  v->launches = &d->launches;
  return true;
}
}  // namespace dgmx
