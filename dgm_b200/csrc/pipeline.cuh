// Persistent stage kernel with an asynchronous copy pipeline (sm_100a).
//
// The plain stage kernel spends most of its time waiting on global memory:
// each tile loads its geometry, modal register and traces, then (after the
// compute) reads the neighbour traces and the second register, each a
// round trip of latency with little else in flight.  Here every CTA walks
// its tiles in order and, while it computes tile i, the copy engine brings
// tile i+1's inputs into a second shared-memory buffer with bulk
// asynchronous copies (cp.async.bulk, completion counted in bytes on an
// mbarrier):
//   the modal register U and the second register Ut of each element,
//   its own face traces (written by the previous stage),
//   the six neighbour face-trace blocks (addresses from the face links,
//   which arrive one tile earlier, with the buffer before),
//   the face links of tile i+2 (whose first entry carries the geometry class).
// Every copy is a contiguous block whose size and addresses are multiples of
// 16 bytes (a static condition selects the configurations that qualify).
// Waits are bounded: a wait that does not complete sets bit 1 of the error
// word and the CTA leaves after a second bounded wait for its copies.
// Arithmetic per element is that of stage_tile (LSRK and right-hand-side
// stages; the other stage kinds use the plain kernel).
#pragma once

#include "stage.cuh"

namespace dgmx {

template <class C>
struct Pipe {
  using T = typename C::R;
  using TT = T;                       // trace storage type = working precision
  using UT = T;                       // second register storage type
  static constexpr int NF = C::NF, LD = C::LD, NFACE = C::NFACE, GF = C::GF, EPB = C::EPB;
  static constexpr int U_B = NF * LD * (int)sizeof(double);
  static constexpr int UT_B = NF * LD * (int)sizeof(UT);
  static constexpr int OWN_B = NFACE * NF * GF * (int)sizeof(TT);
  static constexpr int NBF_B = NF * GF * (int)sizeof(TT);    // one neighbour face block
  static constexpr int LNK_B = NFACE * (int)sizeof(FaceLink);
  static constexpr int SLOT_B = U_B + UT_B + 2 * OWN_B + LNK_B;
  static constexpr int BUF_B = EPB * SLOT_B;
  static constexpr bool OK = !is_ns(C::PHYSICS) && U_B % 16 == 0 && UT_B % 16 == 0 && NBF_B % 16 == 0 &&
                             LNK_B % 16 == 0;
  // shared-memory layout after the tile's own regions: 2 buffers, 2 barriers
  static constexpr size_t OFF = (C::SMEM + 15) / 16 * 16;
  static constexpr size_t SMEM = OFF + 2 * (size_t)BUF_B + 16;
  // offsets inside one buffer, per slot s
  static __device__ __forceinline__ int u_off(int s) { return s * SLOT_B; }
  static __device__ __forceinline__ int ut_off(int s) { return s * SLOT_B + U_B; }
  static __device__ __forceinline__ int own_off(int s) { return s * SLOT_B + U_B + UT_B; }
  static __device__ __forceinline__ int nbr_off(int s) { return s * SLOT_B + U_B + UT_B + OWN_B; }
  static __device__ __forceinline__ int lnk_off(int s) { return s * SLOT_B + U_B + UT_B + 2 * OWN_B; }
};

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait (each try suspends for at most a few microseconds).
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, int tries = kWaitTries) {
  for (int it = 0; it < tries; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Bulk copy global -> shared, completion counted on bar (bytes, 16-aligned).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Issues the copies of tile `e0` (elements e0 .. e0+EPB-1) into buffer `buf`,
// with the links of tile `e1` (or none when e1 < 0).  The links of tile e0
// are read from `lnk` (shared, arrived with the previous buffer).  Run by
// one thread.
template <class C>
__device__ __forceinline__ void pipe_issue(unsigned char *buf, unsigned long long *bar, const StageArgs &a,
                                           int e0, int e1, const FaceLink *lnk) {
  using P = Pipe<C>;
  const typename P::TT *Tin = trace_in<C>(a);
  const typename P::UT *Ut = nullptr;
  if constexpr (C::MIXED) Ut = a.Utf; else Ut = a.Ut;
  unsigned bytes = 0;
  int n_el = 0, n_nx = 0;
  for (int s = 0; s < P::EPB; ++s) {
    const int e = e0 + s;
    if (e < a.ne && lnk[s * P::NFACE].cls >= 0) ++n_el;
    if (e1 >= 0 && e1 + s < a.ne) ++n_nx;
  }
  bytes = n_el * (P::U_B + P::UT_B + 2 * P::OWN_B) + n_nx * P::LNK_B;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(bar, bytes);
  for (int s = 0; s < P::EPB; ++s) {
    const int e = e0 + s;
    if (e < a.ne && lnk[s * P::NFACE].cls >= 0) {
      bulk_g2s(buf + P::u_off(s), a.X + (size_t)e * P::NF * P::LD, P::U_B, bar);
      bulk_g2s(buf + P::ut_off(s), Ut + (size_t)e * P::NF * P::LD, P::UT_B, bar);
      bulk_g2s(buf + P::own_off(s), Tin + (size_t)e * P::NFACE * P::NF * P::GF, P::OWN_B, bar);
      for (int f = 0; f < P::NFACE; ++f) {
        const FaceLink &lk = lnk[s * P::NFACE + f];
        bulk_g2s(buf + P::nbr_off(s) + f * P::NBF_B, Tin + (size_t)(lk.elem * P::NFACE + lk.face) * P::NF * P::GF,
                 P::NBF_B, bar);
      }
    }
    if (e1 >= 0 && e1 + s < a.ne)
      bulk_g2s(buf + P::lnk_off(s), a.links + (size_t)(e1 + s) * P::NFACE, P::LNK_B, bar);
  }
}

// Numerical fluxes with the neighbour traces taken from the pipeline buffer
// (face_fluxes with a different source for Un).
template <class C, int PHYS>
__device__ __forceinline__ void face_fluxes_pipe(const Smem<C> &sm, const StageArgs &a, const unsigned char *buf,
                                                 int tid) {
  using T = typename C::R;
  using P = Pipe<C>;
  constexpr int NF = C::NF, GF = C::GF, NFACE = C::NFACE, EPB = C::EPB, EB = C::EB;
  for (int w = tid; w < NFACE * EPB * GF; w += C::NT) {
    const int f = w / (EPB * GF), rem = w - f * EPB * GF, slot = rem / GF, g = rem - slot * GF;
    const int e = sm.eid[slot];
    if (e < 0) continue;
    const FaceLink lk = sm.lnk[slot * NFACE + f];
    const GeomClass &gc = sm.geo[slot];
    const int gn = a.perm[lk.perm + g];
    T Uo[5], Un[5], Fh[5], FL[5], FR[5];
    T *eo = sm.E + ((f * EPB + slot) * NF) * EB + epos<C>(g);
    const T *tn = reinterpret_cast<const T *>(buf + P::nbr_off(slot) + f * P::NBF_B) + gn;
    const T nm[3] = {T(gc.nrm[f][0]), T(gc.nrm[f][1]), T(gc.nrm[f][2])};
#pragma unroll
    for (int n = 0; n < NF; ++n) { Uo[n] = eo[n * EB]; Un[n] = tn[n * GF]; }
    const bool master = (gc.master >> f) & 1;
    const T jr = T(gc.jr[f]);
    bool ok;
    if constexpr (C::MIXED) {
      if (master) ok = face_flux_pert<PHYS, T>(sm.ref[slot], Uo, Un, nm, T(a.gamma), a.flux, Fh, FR, gc.fr[f]);
      else ok = face_flux_pert<PHYS, T>(sm.ref[slot], Un, Uo, nm, T(a.gamma), a.flux, Fh, FR, gc.fr[f]);
#pragma unroll
      for (int n = 0; n < NF; ++n) eo[n * EB] = master ? Fh[n] * jr : (FR[n] - Fh[n]) * jr;
    } else {
      if (master) ok = face_flux<PHYS, T>(Uo, Un, nm, T(a.gamma), a.flux, Fh, FL, FR, gc.fr[f]);
      else ok = face_flux<PHYS, T>(Un, Uo, nm, T(a.gamma), a.flux, Fh, FL, FR, gc.fr[f]);
#pragma unroll
      for (int n = 0; n < NF; ++n) eo[n * EB] = master ? (Fh[n] - FL[n]) * jr : (FR[n] - Fh[n]) * jr;
    }
    if (!ok) {
      atomicOr(a.err, 1);
      atomicMin(a.err + 1, e);
    }
  }
  csync<C>();
}

// One LSRK (or right-hand-side) stage of tile e0 whose inputs are in `buf`.
template <class C, int PHYS>
__device__ __forceinline__ void stage_tile_pipe(const Smem<C> &sm, const StageArgs &a, int e0,
                                                const unsigned char *buf, int tid) {
  using T = typename C::R;
  using P = Pipe<C>;
  constexpr int NF = C::NF, LD = C::LD, NFACE = C::NFACE, GF = C::GF, G = C::G, EPB = C::EPB, L = C::L;
  constexpr int RPF = LD / L, RPS = NF * RPF;                  // modal rows
  constexpr int TPF = GF / G, TPS = NFACE * NF * TPF;          // trace rows
  // geometry (class from the first face link), and the reference state
  constexpr int GW = (int)(sizeof(GeomClass) / sizeof(double));
  for (int k = tid; k < EPB * GW; k += C::NT) {
    const int s = k / GW, j = k - s * GW, e = e0 + s;
    const int gc = e < a.ne ? sm.lnk[s * NFACE].cls : -1;
    reinterpret_cast<double *>(sm.geo + s)[j] = reinterpret_cast<const double *>(a.classes + (gc >= 0 ? gc : 0))[j];
    if (j == 0) {
      sm.eid[s] = gc >= 0 ? e : -1;
      if constexpr (C::MIXED)
        sm.ref[s] = *reinterpret_cast<const RefState<float> *>(a.uref + kUrefStride * solve_of(a, gc >= 0 ? e : -1) + 10);
    }
  }
  // modal register (padded, perturbation form when mixed), a row per thread
  for (int r = tid; r < EPB * RPS; r += C::NT) {
    const int s = r / RPS, rr = r - s * RPS, e = e0 + s;
    const double *src = reinterpret_cast<const double *>(buf + P::u_off(s)) + rr * L;
    const bool live = e < a.ne && sm.lnk[s * NFACE].cls >= 0;
    double ref0 = 0.0;
    if constexpr (C::MIXED)
      if (live && rr % RPF == 0) ref0 = a.uref[kUrefStride * solve_of(a, e) + 5 + rr / RPF];
#pragma unroll
    for (int k = 0; k < L; ++k)
      sm.A[r * C::PL + k] = live ? T(k == 0 ? src[k] - ref0 : src[k]) : T(k == 0 && rr % RPF == 0 ? 1.0 : 0.0);
  }
  // own traces, a row of G per thread
  for (int r = tid; r < EPB * TPS; r += C::NT) {
    const int s = r / TPS, rr = r - s * TPS, fn = rr / TPF, g1 = rr - fn * TPF, f = fn / NF, n = fn - f * NF;
    const int e = e0 + s;
    const bool live = e < a.ne && sm.lnk[s * NFACE].cls >= 0;
    const T *src = reinterpret_cast<const T *>(buf + P::own_off(s)) + rr * G;
    T *dst = sm.E + ((f * EPB + s) * NF + n) * C::EB + g1 * C::PG;
#pragma unroll
    for (int k = 0; k < G; ++k) dst[k] = live ? src[k] : T(n == 0 ? 1.0 : 0.0);
  }
  csync<C>();
  backward<C>(sm.A, sm.B, sm.S, sm.C, tid, C::NT);
  volume<C, PHYS>(sm, a.gamma, tid);
  face_fluxes_pipe<C, PHYS>(sm, a, buf, tid);
  lift<C>(sm, tid);
  forward<C>(sm.D, sm.R, sm.C, sm.B, tid, C::NT);
  // LSRK update, a row of L modes per thread (U and Ut from the buffer)
  for (int r = tid; r < EPB * RPS; r += C::NT) {
    const int s = r / RPS, rr = r - s * RPS, e = e0 + s;
    if (sm.eid[s] < 0) continue;
    const size_t gi = ((size_t)e0 * RPS + r) * L;
    const double dt = a.dts ? a.dts[solve_of(a, e)] : a.dt;
    const double *u0 = reinterpret_cast<const double *>(buf + P::u_off(s)) + rr * L;
    const typename P::UT *ut0 = reinterpret_cast<const typename P::UT *>(buf + P::ut_off(s)) + rr * L;
    T *Ar = sm.A + r * C::PL;
    const T *Rr = sm.R + r * L;
    if constexpr (C::MIXED) {
      float q[L];
#pragma unroll
      for (int k = 0; k < L; ++k) q[k] = Rr[k];
      if (a.Ssrc)
#pragma unroll
        for (int k = 0; k < L; ++k) q[k] -= float(a.src_scale * a.Ssrc[gi + k]);
      if (a.Rsub)
#pragma unroll
        for (int k = 0; k < L; ++k) q[k] -= float(a.Rsub[gi + k]);
      if (a.kind == kRHS) {
#pragma unroll
        for (int k = 0; k < L; ++k) a.A[gi + k] = q[k];
        continue;
      }
      float ut[L];
      double u[L];
      const float c0 = float(a.c0), mdt = -float(dt);
#pragma unroll
      for (int k = 0; k < L; ++k) {
        ut[k] = fmaf(mdt, q[k], c0 * ut0[k]);
        u[k] = fma(a.c1, double(ut[k]), u0[k]);
      }
      st_row<L>(a.Utf + gi, ut);
      st_row<L>(a.U + gi, u);
      const double ref0 = rr % RPF == 0 ? a.uref[kUrefStride * solve_of(a, e) + 5 + rr / RPF] : 0.0;
#pragma unroll
      for (int k = 0; k < L; ++k) Ar[k] = float(k == 0 ? u[k] - ref0 : u[k]);
    } else {
      double q[L];
#pragma unroll
      for (int k = 0; k < L; ++k) q[k] = Rr[k];
      if (a.Ssrc)
#pragma unroll
        for (int k = 0; k < L; ++k) q[k] -= a.src_scale * a.Ssrc[gi + k];
      if (a.Rcap)
#pragma unroll
        for (int k = 0; k < L; ++k) a.Rcap[gi + k] = q[k];
      if (a.Rsub)
#pragma unroll
        for (int k = 0; k < L; ++k) q[k] -= a.Rsub[gi + k];
      if (a.kind == kRHS) {
#pragma unroll
        for (int k = 0; k < L; ++k) a.A[gi + k] = q[k];
        continue;
      }
      double ut[L], u[L];
#pragma unroll
      for (int k = 0; k < L; ++k) {
        ut[k] = fma(-dt, q[k], a.c0 * ut0[k]);
        u[k] = fma(a.c1, ut[k], u0[k]);
        Ar[k] = u[k];
      }
      st_row<L>(a.Ut + gi, ut);
      st_row<L>(a.U + gi, u);
    }
  }
  csync<C>();
  modal_traces<C>(sm.A, sm.E, sm.S, sm.B, tid, C::NT);
  store_traces<C>(sm.E, trace_out<C>(a), e0, a.ne, tid);
}

// Persistent pipelined stage kernel: grid <= tiles; CTA b takes tiles
// b, b + grid, b + 2 grid, ...
template <class C, int PHYS>
__global__ void __launch_bounds__(C::NT, C::MINB) stage_pipe_kernel(StageArgs a) {
  using P = Pipe<C>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<C> sm(smem_raw);
  unsigned char *bufs = smem_raw + P::OFF;
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(bufs + 2 * P::BUF_B);
  const int tid = threadIdx.x;
  const int ntile = a.tiles ? *a.ntiles : (a.ne + C::EPB - 1) / C::EPB;
  auto tile_e0 = [&](int i) -> int {
    const int t = blockIdx.x + i * (int)gridDim.x;
    if (t >= ntile) return -1;
    return (a.tiles ? a.tiles[t] : t) * C::EPB;
  };
  if ((int)blockIdx.x >= ntile) return;
  // prologue: barriers, links of tile 0 (plain loads into buffer 1's link
  // slots, which are not used before tile 1), then tile 0's copies
  const int e00 = tile_e0(0);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int k = tid; k < C::EPB * C::NFACE; k += C::NT) {
    const int s = k / C::NFACE, f = k - s * C::NFACE, e = e00 + s;
    reinterpret_cast<FaceLink *>(bufs + P::BUF_B + P::lnk_off(s))[f] =
        e < a.ne ? a.links[(size_t)e * C::NFACE + f] : FaceLink{0, 0, 0, -1};
  }
  __syncthreads();
  if (tid == 0) {
    // gather tile 0's links from the strided slots into a compact list
    FaceLink l0[C::EPB * C::NFACE];
    for (int s = 0; s < C::EPB; ++s)
      for (int f = 0; f < C::NFACE; ++f)
        l0[s * C::NFACE + f] = reinterpret_cast<const FaceLink *>(bufs + P::BUF_B + P::lnk_off(s))[f];
    pipe_issue<C>(bufs, &bar[0], a, e00, tile_e0(1), l0);
  }
  for (int i = 0;; ++i) {
    const int e0 = tile_e0(i);
    if (e0 < 0) break;
    const int b = i & 1;
    unsigned char *buf = bufs + b * P::BUF_B;
    const bool ok = mbar_wait(&bar[b], (unsigned)((i >> 1) & 1), a.wait_tries);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(a.err, 2);
      // let copies still in flight land before the CTA leaves (with the
      // full bound, whatever bound the first wait had)
      mbar_wait(&bar[b], (unsigned)((i >> 1) & 1));
      return;
    }
    // this tile's links arrived with the previous buffer (or the prologue)
    for (int k = tid; k < C::EPB * C::NFACE; k += C::NT) {
      const int s = k / C::NFACE, f = k - s * C::NFACE;
      sm.lnk[k] = reinterpret_cast<const FaceLink *>(bufs + (b ^ 1) * P::BUF_B + P::lnk_off(s))[f];
    }
    __syncthreads();
    // next tile's copies into the other buffer, with the links after it
    const int e1 = tile_e0(i + 1);
    if (tid == 0 && e1 >= 0) {
      FaceLink l1[C::EPB * C::NFACE];
      for (int s = 0; s < C::EPB; ++s)
        for (int f = 0; f < C::NFACE; ++f)
          l1[s * C::NFACE + f] = reinterpret_cast<const FaceLink *>(buf + P::lnk_off(s))[f];
      pipe_issue<C>(bufs + (b ^ 1) * P::BUF_B, &bar[b ^ 1], a, e1, tile_e0(i + 2), l1);
    }
    stage_tile_pipe<C, PHYS>(sm, a, e0, buf, tid);
    __syncthreads();
  }
}

}  // namespace dgmx
