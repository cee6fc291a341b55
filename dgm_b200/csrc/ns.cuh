// Navier-Stokes (BR1) viscous kernels for sm_100a, FP64.
//
// The viscous part of Navier_Stokes[3d]::diffusion (src/Navier_Stokes3d.cpp:
// 182-391, src/Navier_Stokes.cpp:113-252) needs two face exchanges per
// stage, so it runs as two launches before the fused stage kernel:
//   ns_grad_kernel : primitive traces (src/Euler3d.cpp:1162-1199), BR1
//     averages (src/Domain.cpp:1883-1937, '+'), collocation gradients of
//     u, v, w, e, the lift of ({{q}} - q) n J, and the L2 projection of each
//     gradient component (src/Euler3d.cpp:1144-1159); writes the projected
//     gradients as modal coefficients.
//   ns_visc_kernel : stresses and heat flux at the GLL points from the
//     projected gradients, the viscous normal-flux traces g.n of every
//     element side (fill_sides(fx,fy,fz), src/Hex.cpp:950-972), and the
//     projected collocation divergence of g.
// The stage kernel then adds the viscous lift ('-' averages of the traces)
// and subtracts the projected divergence (projection is linear, so
// proj(conv) - proj(div g + lift) equals the reference's single projection).
#pragma once

#include "stage.cuh"

namespace dgmx {

constexpr bool is_ns(int p) { return p == DGMX_NS2D || p == DGMX_NS3D; }

template <class C>
struct NsCfg {
  static constexpr int DIM = C::DIM, NF = C::NF, L = C::L, Q = C::Q, G = C::G;
  static constexpr int EPB = C::EPB, NFACE = C::NFACE, NT = C::NT;
  static constexpr int QD = C::QD, LD = C::LD, GF = C::GF, QF = C::QF, LF = C::LF;
  static constexpr int NVC = DIM + 1;       // primitive components u, v, (w), e
  static constexpr int NG = NVC * DIM;      // gradient components
  static constexpr int NV = NF - 1;         // viscous fields
  static_assert(NV * DIM == NG, "viscous flux components reuse the gradient slots");
  static constexpr int P1 = DIM == 3 ? Q * L * L : Q * L;     // backward pass-1 size
  static constexpr int P2 = DIM == 3 ? Q * Q * L : 0;         // backward pass-2 size
  static constexpr int F1 = DIM == 3 ? L * Q * Q : L * Q;     // forward pass-1 size
  static constexpr int F2 = DIM == 3 ? L * L * Q : 0;         // forward pass-2 size
  // fields per backward-transform batch: one slot's fields in two batches
  // (at most 3 at a time) keep the transform scratch at the size the
  // per-component passes need
  static constexpr int NB1 = (EPB == 1 && NF > 3) ? 3 : NF;
  // ns_grad_kernel regions (per slot, doubles); the modal input A is dead
  // after the backward transform, so the primitive component Qc and its
  // gradient Gd live in it
  struct Grad {
    static constexpr int Qc = QD, Gd = DIM * QD;
    static constexpr int A = cmax(NF * LD, Qc + Gd), B = NF * QD, E = NFACE * NF * GF, E2 = NFACE * NF * GF;
    static constexpr int Fc = NFACE * DIM * GF, LFc = cmax(NFACE * DIM * QF, DIM * F2);
    static constexpr int S1 = cmax(cmax(NB1 * P1, DIM == 3 ? NFACE * DIM * Q * G : 0), DIM * F1);
    static constexpr int S2 = cmax(cmax(NB1 * P2, DIM * F2), DIM * LD);
    static constexpr int SLOT = A + B + E + E2 + Fc + LFc + S1 + S2;
    static constexpr size_t SMEM = (size_t)EPB * SLOT * 8 + (size_t)EPB * (sizeof(GeomClass) + NFACE * 16 + 16);
  };
  // ns_visc_kernel regions (per slot, doubles).  G holds the velocity
  // gradient, then in place the symmetric stress and the heat flux (NGS
  // slots: 6 + 3 in 3-D, 3 + 2 in 2-D; the modal input is parked there
  // first); the energy gradient goes to Dv, which then accumulates one
  // field's divergence at a time.  B holds the state until the stresses are
  // formed, then the face values FF and the divergence input Cv; X holds the
  // modal gradient components Gh in the first loop and the face-point
  // values Fg in the second.
  struct Visc {
    static constexpr int NGS = DIM == 3 ? 9 : 5;
    static constexpr int FF = cmax(NFACE * DIM * QF, F2), Cv = QD;
    static constexpr int B = cmax(NF * QD, FF + Cv);
    static constexpr int G = cmax(NGS * QD, NF * LD);
    static constexpr int X = cmax(DIM * LD, NFACE * DIM * GF);
    static constexpr int S1 = cmax(cmax(NB1 * P1, DIM * P1), cmax(DIM == 3 ? NFACE * DIM * C::G * Q : 0, F1));
    static constexpr int S2 = cmax(cmax(NB1 * P2, DIM * P2), LD);
    static constexpr int Dv = DIM * QD;
    static constexpr int SLOT = B + G + X + S1 + S2 + Dv;
    static constexpr size_t SMEM = (size_t)EPB * SLOT * 8 + (size_t)EPB * (sizeof(GeomClass) + NFACE * 16 + 16);
    static_assert(DIM * DIM <= NGS, "the velocity gradient fits the stress slots");
  };
  // slot of component d of the viscous flux vector g_n (n: momentum x, y,
  // [z], energy) in the symmetric stress / heat-flux layout
  static constexpr __host__ __device__ int gslot(int n, int d) {
    if (DIM == 3) {
      return n == 3 ? 6 + d : (n == 0 ? d : (n == 1 ? (d == 0 ? 1 : 2 + d) : (d == 0 ? 2 : (d == 1 ? 4 : 5))));
    }
    return n == 2 ? 3 + d : (n == 0 ? d : 1 + d);
  }
  // CTAs per SM for a viscous kernel of smem bytes: the tile's register cap
  // when it has one, else as many as shared memory holds while the register
  // budget stays at 64 or more per thread
  static constexpr int minb(size_t smem) {
    if (C::MINB_REQ > 0) return C::MINB_REQ;
    const int by_smem = (int)((228 * 1024) / (smem + 1024));
    const int by_regs = 65536 / (NT * 64);
    const int b = by_smem < by_regs ? by_smem : by_regs;
    return b < 1 ? 1 : (b > 8 ? 8 : b);
  }
  static constexpr int GRAD_MINB = minb(Grad::SMEM), VISC_MINB = minb(Visc::SMEM);
};

// Primitive variables of one conserved state (src/Euler3d.cpp:1170-1182):
// q = (u, v, [w], e) with e the internal energy.
template <int DIM>
__device__ __forceinline__ void primitive(const double *U, double *q) {
  const double r = U[0];
  double wk;
  if constexpr (DIM == 3) {
    const double u = U[1] / r, v = U[2] / r, w = U[3] / r;
    double e = U[4] / r;
    wk = u * u; wk = fma(v, v, wk); wk = fma(w, w, wk);
    e = fma(-0.5, wk, e);
    q[0] = u; q[1] = v; q[2] = w; q[3] = e;
  } else {
    const double u = U[1] / r, v = U[2] / r;
    double e = U[3] / r;
    wk = u * u; wk = fma(v, v, wk);
    e = fma(-0.5, wk, e);
    q[0] = u; q[1] = v; q[2] = e;
  }
}

// Gather the neighbour's state traces into face-major smem E2 in the own
// point order.  A boundary side's neighbour is its ghost state in the
// viscous BC database (Navier_Stokes3d::enforce_bc,
// src/Navier_Stokes3d.cpp:457-461; ghost_state) made from the own trace.
template <class C>
__device__ __forceinline__ void load_nbr_traces(double *E2, const double *T, const FaceLink *lnk, const int *eid,
                                                const GeomClass *geo, const StageArgs &a, int tid) {
  constexpr int NF = C::NF, GF = C::GF, NFACE = C::NFACE, EPB = C::EPB;
  for (int w = tid; w < NFACE * EPB * NF * GF; w += C::NT) {
    const int f = w / (EPB * NF * GF), rem = w - f * EPB * NF * GF;
    const int s = rem / (NF * GF), ng = rem - s * NF * GF, n = ng / GF, g = ng - n * GF;
    double v = n == 0 ? 1.0 : 0.0;
    if (eid[s] >= 0) {
      const FaceLink lk = lnk[s * NFACE + f];
      const int bt = (geo[s].bc >> (4 * f)) & 15;
      const double *t = T + ((size_t)(lk.elem * NFACE + lk.face) * NF) * GF + a.perm[lk.perm + g];
      if (bt) {
        double Uo[5], Un[5];
#pragma unroll
        for (int k = 0; k < NF; ++k) Uo[k] = t[k * GF];
        ghost_state<C::DIM, NF>(a.bckind[bt], a.bcpar[bt], Uo, geo[s].onrm[f], true, Un);
        v = Un[n];
      } else {
        v = t[n * GF];
      }
    }
    E2[w] = v;
  }
}

// G2GL of NB face-major arrays [f][slot][b][GF] and accumulation with the
// inverse end weights into dst [slot][b][QD] (faces in increasing order).
template <class C, int NB>
__device__ __forceinline__ void lift_batch(const double *Fg, double *LFc, double *S, double *dst, int tid) {
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q, G = C::G, EPB = C::EPB, QD = C::QD, QF = C::QF;
  constexpr int NBT = C::NFACE * EPB * NB;
  if constexpr (DIM == 3) {
    contract<G, G, 1, 0, G, Q, MatG2GL<L, Q>, false>(Fg, S, NBT, G * G, Q * G, tid, C::NT);
    __syncthreads();
    contract<Q, G, 1, 1, G, Q, MatG2GL<L, Q>, false>(S, LFc, NBT, Q * G, Q * Q, tid, C::NT);
  } else {
    contract<G, 1, 1, 0, G, Q, MatG2GL<L, Q>, false>(Fg, LFc, NBT, G, Q, tid, C::NT);
  }
  __syncthreads();
  const double w0 = 1.0 / cW<double, L, Q>[0], w1 = 1.0 / cW<double, L, Q>[Q - 1];
  for (int w = tid; w < EPB * NB * QD; w += C::NT) {
    const int slot = w / (NB * QD), rem = w - slot * NB * QD, b = rem / QD, p = rem - b * QD;
    double acc = dst[w];
    if constexpr (DIM == 3) {
      const int i = p / (Q * Q), j = (p / Q) % Q, k = p % Q;
      auto lf = [&](int f, int x, int y) { return LFc[((f * EPB + slot) * NB + b) * QF + x * Q + y]; };
      if (k == 0) acc = fma(w0, lf(0, i, j), acc);
      if (j == 0) acc = fma(w0, lf(1, i, k), acc);
      if (i == Q - 1) acc = fma(w1, lf(2, j, k), acc);
      if (j == Q - 1) acc = fma(w1, lf(3, i, k), acc);
      if (i == 0) acc = fma(w0, lf(4, j, k), acc);
      if (k == Q - 1) acc = fma(w1, lf(5, i, j), acc);
    } else {
      const int i = p / Q, j = p % Q;
      auto lf = [&](int f, int x) { return LFc[((f * EPB + slot) * NB + b) * QF + x]; };
      if (j == 0) acc = fma(w0, lf(0, i), acc);
      if (i == Q - 1) acc = fma(w1, lf(1, j), acc);
      if (j == Q - 1) acc = fma(w1, lf(2, i), acc);
      if (i == 0) acc = fma(w0, lf(3, j), acc);
    }
    dst[w] = acc;
  }
  __syncthreads();
}

// w-weighted projection of NB arrays [slot][b][QD] (weighted in place) to
// modal dst [slot][b][LD].
template <class C, int NB>
__device__ __forceinline__ void forward_batch(double *src, double *dst, double *S1, double *S2, int tid) {
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q, QD = C::QD, LD = C::LD, NBT = C::EPB * NB;
  for (int w = tid; w < NBT * QD; w += C::NT) {
    const int p = w % QD;
    double wq;
    if constexpr (DIM == 3) wq = cW<double, L, Q>[p / (Q * Q)] * cW<double, L, Q>[(p / Q) % Q] * cW<double, L, Q>[p % Q];
    else wq = cW<double, L, Q>[p / Q] * cW<double, L, Q>[p % Q];
    src[w] = wq * src[w];
  }
  __syncthreads();
  if constexpr (DIM == 3) {
    contract<Q, Q, Q, 0, Q, L, MatBt<L, Q>, false>(src, S1, NBT, QD, L * Q * Q, tid, C::NT);
    __syncthreads();
    contract<L, Q, Q, 1, Q, L, MatBt<L, Q>, false>(S1, S2, NBT, L * Q * Q, L * L * Q, tid, C::NT);
    __syncthreads();
    contract<L, L, Q, 2, Q, L, MatBt<L, Q>, false>(S2, dst, NBT, L * L * Q, LD, tid, C::NT);
  } else {
    contract<Q, Q, 1, 0, Q, L, MatBt<L, Q>, false>(src, S1, NBT, QD, L * Q, tid, C::NT);
    __syncthreads();
    contract<L, Q, 1, 1, Q, L, MatBt<L, Q>, false>(S1, dst, NBT, L * Q, LD, tid, C::NT);
  }
  __syncthreads();
}

// modal [slot][b][LD] -> GLL [slot][b][QD]
template <class C, int NB>
__device__ __forceinline__ void backward_batch(const double *src, double *dst, double *S1, double *S2, int tid) {
  constexpr int L = C::L, Q = C::Q, NBT = C::EPB * NB;
  if constexpr (C::DIM == 3) {
    contract<L, L, L, 0, L, Q, MatB<L, Q>, false>(src, S1, NBT, C::LD, Q * L * L, tid, C::NT);
    __syncthreads();
    contract<Q, L, L, 1, L, Q, MatB<L, Q>, false>(S1, S2, NBT, Q * L * L, Q * Q * L, tid, C::NT);
    __syncthreads();
    contract<Q, Q, L, 2, L, Q, MatB<L, Q>, false>(S2, dst, NBT, Q * Q * L, C::QD, tid, C::NT);
  } else {
    contract<L, L, 1, 0, L, Q, MatB<L, Q>, false>(src, S1, NBT, C::LD, Q * L, tid, C::NT);
    __syncthreads();
    contract<Q, L, 1, 1, L, Q, MatB<L, Q>, false>(S1, dst, NBT, Q * L, C::QD, tid, C::NT);
  }
  __syncthreads();
}

template <class C>
__device__ __forceinline__ void load_geo_slots(GeomClass *geo, FaceLink *lnk, int *eid, const StageArgs &a, int e0,
                                               int tid) {
  for (int s = tid; s < C::EPB; s += C::NT) {
    const int e = e0 + s;
    eid[s] = e < a.ne ? e : -1;
    geo[s] = a.classes[e < a.ne ? a.gclass[e] : 0];
  }
  for (int w = tid; w < C::EPB * C::NFACE; w += C::NT) {
    const int s = w / C::NFACE, f = w - s * C::NFACE, e = e0 + s;
    lnk[w] = e < a.ne ? a.links[(size_t)e * C::NFACE + f] : FaceLink{0, 0, 0, 0};
  }
}

// ---------------------------------------------------------------- gradients
template <class C, int PHYS, bool NODAL>
__global__ void __launch_bounds__(C::NT, NsCfg<C>::GRAD_MINB) ns_grad_kernel(StageArgs a) {
  using N = NsCfg<C>;
  using R = typename N::Grad;
  constexpr int DIM = C::DIM, NF = C::NF, Q = C::Q, L = C::L, EPB = C::EPB, QD = C::QD, GF = C::GF;
  constexpr int NFACE = C::NFACE, NVC = N::NVC, LD = C::LD;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  double *smem_raw = reinterpret_cast<double *>(smem_bytes);
  double *A = smem_raw, *B = A + EPB * R::A, *E = B + EPB * R::B, *E2 = E + EPB * R::E;
  double *Fc = E2 + EPB * R::E2, *LFc = Fc + EPB * R::Fc;
  double *S1 = LFc + EPB * R::LFc, *S2 = S1 + EPB * R::S1;
  double *Qc = A, *Gd = A + EPB * R::Qc;     // in the modal input, dead after the backward transform
  GeomClass *geo = reinterpret_cast<GeomClass *>(S2 + EPB * R::S2);
  FaceLink *lnk = reinterpret_cast<FaceLink *>(geo + EPB);
  int *eid = reinterpret_cast<int *>(lnk + EPB * NFACE);
  const int tid = threadIdx.x, e0 = blockIdx.x * EPB;
  load_geo_slots<C>(geo, lnk, eid, a, e0, tid);
  if constexpr (NODAL) {
    load_nodal<C>(B, a.Xn, e0, a.ne, tid);
  } else {
    load_modal<C>(A, a.X, e0, a.ne, tid);
  }
  load_own_traces<C, double, false>(E, a.Tin, e0, a.ne, tid);
  __syncthreads();
  load_nbr_traces<C>(E2, a.Tin, lnk, eid, geo, a, tid);
  if constexpr (!NODAL) {
    __syncthreads();
    if constexpr (N::NB1 == NF) {
      backward_batch<C, NF>(A, B, S1, S2, tid);
    } else {   // one slot: fields [0, NB1) then [NB1, NF)
      backward_batch<C, N::NB1>(A, B, S1, S2, tid);
      backward_batch<C, NF - N::NB1>(A + N::NB1 * LD, B + N::NB1 * QD, S1, S2, tid);
    }
  }
  __syncthreads();
  for (int c = 0; c < NVC; ++c) {
    // primitive component c at the GLL points
    for (int w = tid; w < EPB * QD; w += C::NT) {
      const int s = w / QD, p = w - s * QD;
      double U[5], q[4];
#pragma unroll
      for (int n = 0; n < NF; ++n) U[n] = B[(s * NF + n) * QD + p];
      primitive<DIM>(U, q);
      Qc[w] = q[c];
    }
    // lift inputs ({{q_c}} - q_c) J n_d per face point, master-frame average
    for (int w = tid; w < NFACE * EPB * GF; w += C::NT) {
      const int f = w / (EPB * GF), rem = w - f * EPB * GF, s = rem / GF, g = rem - s * GF;
      double Uo[5], Un[5], qo[4], qn[4];
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        Uo[n] = E[((f * EPB + s) * NF + n) * GF + g];
        Un[n] = E2[((f * EPB + s) * NF + n) * GF + g];
      }
      primitive<DIM>(Uo, qo);
      primitive<DIM>(Un, qn);
      const GeomClass &gc = geo[s];
      const bool master = (gc.master >> f) & 1;
      const double avg = master ? 0.5 * (qo[c] + qn[c]) : 0.5 * (qn[c] + qo[c]);
      const double d = (avg - qo[c]) * gc.jr[f];
#pragma unroll
      for (int k = 0; k < DIM; ++k) Fc[((f * EPB + s) * DIM + k) * GF + g] = gc.onrm[f][k] * d;
    }
    __syncthreads();
    // collocation derivatives along r, s, t
    using Sh = Sh3<DIM, Q>;
    contract<Sh::a, Sh::b, Sh::c, 0, Q, Q, MatD<L, Q>, false>(Qc, Gd, EPB, QD, DIM * QD, tid, C::NT);
    contract<Sh::a, Sh::b, Sh::c, 1, Q, Q, MatD<L, Q>, false>(Qc, Gd + QD, EPB, QD, DIM * QD, tid, C::NT);
    if constexpr (DIM == 3)
      contract<Sh::a, Sh::b, Sh::c, 2, Q, Q, MatD<L, Q>, false>(Qc, Gd + 2 * QD, EPB, QD, DIM * QD, tid, C::NT);
    __syncthreads();
    // chain rule (src/Hex.cpp:1994-2006): d/dx = rx d/dr + sx d/ds + tx d/dt
    for (int w = tid; w < EPB * QD; w += C::NT) {
      const int s = w / QD, p = w - s * QD;
      double *g = Gd + s * DIM * QD + p;
      const double *m = geo[s].metric;
      const double fr = g[0], fs = g[QD], ft = DIM == 3 ? g[2 * QD] : 0.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        double v = m[0 * 3 + k] * fr;
        v = fma(m[1 * 3 + k], fs, v);
        if (DIM == 3) v = fma(m[2 * 3 + k], ft, v);
        g[k * QD] = v;
      }
    }
    __syncthreads();
    lift_batch<C, DIM>(Fc, LFc, S1, Gd, tid);
    forward_batch<C, DIM>(Gd, S2, S1, LFc, tid);
    for (int w = tid; w < EPB * DIM * LD; w += C::NT) {
      const int s = w / (DIM * LD), rem = w - s * DIM * LD;
      const int e = e0 + s;
      if (e < a.ne) a.Ghat[((size_t)e * NVC + c) * DIM * LD + rem] = S2[w];
    }
    __syncthreads();
  }
}

// ----------------------------------------------- stresses, traces, divergence
template <class C, int PHYS, bool NODAL>
__global__ void __launch_bounds__(C::NT, NsCfg<C>::VISC_MINB) ns_visc_kernel(StageArgs a) {
  using N = NsCfg<C>;
  using R = typename N::Visc;
  constexpr int DIM = C::DIM, NF = C::NF, Q = C::Q, L = C::L, G = C::G, EPB = C::EPB, QD = C::QD;
  constexpr int GF = C::GF, QF = C::QF, NFACE = C::NFACE, NV = N::NV, NVC = N::NVC, LD = C::LD, NGS = R::NGS;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  double *smem_raw = reinterpret_cast<double *>(smem_bytes);
  double *B = smem_raw, *Gg = B + EPB * R::B, *X = Gg + EPB * R::G;
  double *S1 = X + EPB * R::X, *S2 = S1 + EPB * R::S1, *Dv = S2 + EPB * R::S2;
  double *Gh = X, *Fg = X;                    // first loop / second loop
  double *FF = B, *Cv = B + EPB * R::FF;      // after the stresses are formed
  GeomClass *geo = reinterpret_cast<GeomClass *>(Dv + EPB * R::Dv);
  FaceLink *lnk = reinterpret_cast<FaceLink *>(geo + EPB);
  int *eid = reinterpret_cast<int *>(lnk + EPB * NFACE);
  const int tid = threadIdx.x, e0 = blockIdx.x * EPB;
  load_geo_slots<C>(geo, lnk, eid, a, e0, tid);
  if constexpr (NODAL) {
    load_nodal<C>(B, a.Xn, e0, a.ne, tid);
  } else {
    load_modal<C>(Gg, a.X, e0, a.ne, tid);  // modal input parked in the gradient region
    __syncthreads();
    if constexpr (N::NB1 == NF) {
      backward_batch<C, NF>(Gg, B, S1, S2, tid);
    } else {   // one slot: fields [0, NB1) then [NB1, NF)
      backward_batch<C, N::NB1>(Gg, B, S1, S2, tid);
      backward_batch<C, NF - N::NB1>(Gg + N::NB1 * LD, B + N::NB1 * QD, S1, S2, tid);
    }
  }
  __syncthreads();
  // projected gradients at the GLL points: velocity components into Gg
  // (component c, direction d at slot c*DIM+d), the energy gradient into Dv
  for (int c = 0; c < NVC; ++c) {
    for (int w = tid; w < EPB * DIM * LD; w += C::NT) {
      const int s = w / (DIM * LD), rem = w - s * DIM * LD;
      const int e = e0 + s;
      Gh[w] = e < a.ne ? a.Ghat[((size_t)e * NVC + c) * DIM * LD + rem] : 0.0;
    }
    __syncthreads();
    backward_batch<C, DIM>(Gh, Dv, S1, S2, tid);
    if (c < DIM) {
      for (int w = tid; w < EPB * DIM * QD; w += C::NT) {
        const int s = w / (DIM * QD), rem = w - s * DIM * QD;
        Gg[(s * NGS + c * DIM) * QD + rem] = Dv[w];
      }
      __syncthreads();
    }
  }
  // stresses and heat flux, in place (slots gslot(n, d))
  const double mu = a.vis, gPr = a.gamma / a.Pr;
  for (int w = tid; w < EPB * QD; w += C::NT) {
    const int s = w / QD, p = w - s * QD;
    double *g = Gg + s * NGS * QD + p;
    const double *ge = Dv + s * DIM * QD + p;
    double U[5];
#pragma unroll
    for (int n = 0; n < NF; ++n) U[n] = B[(s * NF + n) * QD + p];
    const double r = U[0];
    if constexpr (DIM == 3) {
      const double u = U[1] / r, v = U[2] / r, ww = U[3] / r;
      const double ux = g[0 * QD], uy = g[1 * QD], uz = g[2 * QD];
      const double vx = g[3 * QD], vy = g[4 * QD], vz = g[5 * QD];
      const double wx = g[6 * QD], wy = g[7 * QD], wz = g[8 * QD];
      const double ex = ge[0], ey = ge[QD], ez = ge[2 * QD];
      double t12 = uy + vx; t12 = mu * t12;
      double t13 = uz + wx; t13 = mu * t13;
      double t23 = vz + wy; t23 = mu * t23;
      double wk = 2.0 * ux - vy;
      double t11 = 1.0 * wk - wz; t11 = (2.0 / 3.0) * t11; t11 = mu * t11;
      wk = 2.0 * vy - ux;
      double t22 = 1.0 * wk - wz; t22 = (2.0 / 3.0) * t22; t22 = mu * t22;
      wk = 2.0 * wz - ux;
      double t33 = 1.0 * wk - vy; t33 = (2.0 / 3.0) * t33; t33 = mu * t33;
      double qx = t11 * u; qx = fma(t12, v, qx); qx = fma(t13, ww, qx);
      double qy = t12 * u; qy = fma(t22, v, qy); qy = fma(t23, ww, qy);
      double qz = t13 * u; qz = fma(t23, v, qz); qz = fma(t33, ww, qz);
      qx = fma(gPr, mu * ex, qx); qy = fma(gPr, mu * ey, qy); qz = fma(gPr, mu * ez, qz);
      g[0 * QD] = t11; g[1 * QD] = t12; g[2 * QD] = t13;
      g[3 * QD] = t22; g[4 * QD] = t23; g[5 * QD] = t33;
      g[6 * QD] = qx; g[7 * QD] = qy; g[8 * QD] = qz;
    } else {
      const double u = U[1] / r, v = U[2] / r;
      const double ux = g[0 * QD], uy = g[1 * QD], vx = g[2 * QD], vy = g[3 * QD];
      const double ex = ge[0], ey = ge[QD];
      double t12 = uy + vx; t12 = mu * t12;
      double t11 = 2.0 * ux - vy; t11 = (2.0 / 3.0) * t11; t11 = mu * t11;
      double t22 = 2.0 * vy - ux; t22 = (2.0 / 3.0) * t22; t22 = mu * t22;
      double qx = t11 * u; qx = fma(t12, v, qx);
      double qy = t12 * u; qy = fma(t22, v, qy);
      qx = fma(gPr, mu * ex, qx); qy = fma(gPr, mu * ey, qy);
      g[0 * QD] = t11; g[1 * QD] = t12; g[2 * QD] = t22;
      g[3 * QD] = qx; g[4 * QD] = qy;
    }
  }
  __syncthreads();
  for (int n = 0; n < NV; ++n) {
    // face GLL values of g_n (DIM components), face-major [f][slot][d][QF]
    for (int w = tid; w < NFACE * EPB * DIM * QF; w += C::NT) {
      const int f = w / (EPB * DIM * QF), rem = w - f * EPB * DIM * QF;
      const int s = rem / (DIM * QF), rem2 = rem - s * DIM * QF, d = rem2 / QF, x = rem2 - d * QF;
      const double *src = Gg + (s * NGS + N::gslot(n, d)) * QD;
      int p;
      if constexpr (DIM == 3) {
        const int u = x / Q, v = x % Q;
        switch (f) {
          case 0: p = (u * Q + v) * Q + 0; break;
          case 1: p = (u * Q + 0) * Q + v; break;
          case 2: p = ((Q - 1) * Q + u) * Q + v; break;
          case 3: p = (u * Q + (Q - 1)) * Q + v; break;
          case 4: p = (0 * Q + u) * Q + v; break;
          default: p = (u * Q + v) * Q + (Q - 1); break;
        }
      } else {
        switch (f) {
          case 0: p = x * Q + 0; break;
          case 1: p = (Q - 1) * Q + x; break;
          case 2: p = x * Q + (Q - 1); break;
          default: p = 0 * Q + x; break;
        }
      }
      FF[w] = src[p];
    }
    __syncthreads();
    constexpr int NB = NFACE * EPB * DIM;
    if constexpr (DIM == 3) {
      contract<Q, Q, 1, 0, Q, G, MatGL2G<L, Q>, false>(FF, S1, NB, Q * Q, G * Q, tid, C::NT);
      __syncthreads();
      contract<G, Q, 1, 1, Q, G, MatGL2G<L, Q>, false>(S1, Fg, NB, G * Q, G * G, tid, C::NT);
    } else {
      contract<Q, 1, 1, 0, Q, G, MatGL2G<L, Q>, false>(FF, Fg, NB, Q, G, tid, C::NT);
    }
    __syncthreads();
    // g_n . n (own normals), the viscous trace of this side
    for (int w = tid; w < EPB * NFACE * GF; w += C::NT) {
      const int s = w / (NFACE * GF), rem = w - s * NFACE * GF, f = rem / GF, gq = rem - f * GF;
      const int e = e0 + s;
      if (e >= a.ne) continue;
      const double *nr = geo[s].onrm[f];
      double v = nr[0] * Fg[((f * EPB + s) * DIM + 0) * GF + gq];
      v = fma(nr[1], Fg[((f * EPB + s) * DIM + 1) * GF + gq], v);
      if (DIM == 3) v = fma(nr[2], Fg[((f * EPB + s) * DIM + 2) * GF + gq], v);
      a.V[(((size_t)e * NFACE + f) * NV + n) * GF + gq] = v;
    }
    // collocation divergence of g_n (contravariant form) into Dv [slot][QD]
    for (int r = 0; r < DIM; ++r) {
      for (int w = tid; w < EPB * QD; w += C::NT) {
        const int s = w / QD, p = w - s * QD;
        const double *m = geo[s].metric;
        const double *gs = Gg + s * NGS * QD + p;
        double v = m[3 * r + 0] * gs[N::gslot(n, 0) * QD];
        v = fma(m[3 * r + 1], gs[N::gslot(n, 1) * QD], v);
        if (DIM == 3) v = fma(m[3 * r + 2], gs[N::gslot(n, 2) * QD], v);
        Cv[w] = v;
      }
      __syncthreads();
      using Sh = Sh3<DIM, Q>;
      if (r == 0) contract<Sh::a, Sh::b, Sh::c, 0, Q, Q, MatD<L, Q>, false>(Cv, Dv, EPB, QD, QD, tid, C::NT);
      else if (r == 1) contract<Sh::a, Sh::b, Sh::c, 1, Q, Q, MatD<L, Q>, true>(Cv, Dv, EPB, QD, QD, tid, C::NT);
      else contract<Sh::a, Sh::b, Sh::c, 2, Q, Q, MatD<L, Q>, true>(Cv, Dv, EPB, QD, QD, tid, C::NT);
      __syncthreads();
    }
    // projected divergence of this field
    forward_batch<C, 1>(Dv, S2, S1, FF, tid);
    for (int w = tid; w < EPB * LD; w += C::NT) {
      const int s = w / LD, m = w - s * LD;
      const int e = e0 + s;
      if (e < a.ne) a.Pv[((size_t)e * NV + n) * LD + m] = S2[w];
    }
    __syncthreads();
  }
}

}  // namespace dgmx
