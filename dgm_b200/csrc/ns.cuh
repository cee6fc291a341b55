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

// A contraction of the viscous kernels: with TC, FP32 data and an operator
// of at least 5 x 5, on the tensor cores (contract_tc, 3xTF32); otherwise
// on the CUDA cores (contract).
template <bool TC, int I0, int I1, int I2, int AX, int K, int N, class M, bool ACC, class T, int IS0 = -1,
          int IS1 = -1, int OS0 = -1, int OS1 = -1>
__device__ __forceinline__ void vcontract(const T *in, T *out, int nbatch, int sin, int sout, int tid, int nthr) {
  if constexpr (TC && std::is_same<T, float>::value && K >= 5 && N >= 5)
    contract_tc<I0, I1, I2, AX, K, N, M, ACC, IS0, IS1, OS0, OS1>(in, out, nbatch, sin, sout, tid, nthr);
  else
    contract<I0, I1, I2, AX, K, N, M, ACC, T, IS0, IS1, OS0, OS1>(in, out, nbatch, sin, sout, tid, nthr);
}

// Bytes of a viscous kernel's value regions, rounded up to 8: the geometry
// slots that follow hold doubles, and an odd number of float values would
// leave them on a 4-byte boundary (a no-op for double values).
template <class V>
constexpr size_t ns_data_bytes(int values) { return ((size_t)values * sizeof(V) + 7) & ~(size_t)7; }

template <class C, class V = double>
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
  // ns_grad_kernel regions (per slot, counted in values of the working
  // type); the modal input A is dead after the backward transform, so the
  // primitive component Qc and its gradient Gd live in it.  The state
  // traces E, E2 are double in both forms (the BR1 lift inputs are formed
  // from them in double), and the FP32 form keeps each slot's density and
  // energy means in Rs (double): its GLL state holds rho - rho_mean and
  // E - E_mean, so the internal energy is formed without the cancellation
  // of E/rho (about 1/(gamma (gamma-1) Ma^2)) against |u|^2/2 in FP32.
  struct Grad {
    static constexpr bool F32 = std::is_same<V, float>::value;
    static constexpr int DW = (int)(sizeof(double) / sizeof(V));   // values per double
    static constexpr int pad(int n) { return (n + DW - 1) / DW * DW; }
    static constexpr int Qc = QD, Gd = DIM * QD;
    static constexpr int A = pad(cmax(NF * LD, Qc + Gd)), B = pad(NF * QD);
    // TRG: a tile with fewer threads than points (several CTAs per SM)
    // reads the own and neighbour traces from global memory in each
    // component's lift-input pass instead of staging them in E and E2
    static constexpr bool TRG = NT < QD;
    static constexpr int E = TRG ? 0 : NFACE * NF * GF * DW, E2 = E, Rs = F32 ? 2 * DW : 0;
    static constexpr int Fc = NFACE * DIM * GF, LFc = cmax(NFACE * DIM * QF, DIM * F2);
    static constexpr int S1 = cmax(cmax(NB1 * P1, DIM == 3 ? NFACE * DIM * Q * G : 0), DIM * F1);
    static constexpr int S2 = cmax(cmax(NB1 * P2, DIM * F2), DIM * LD);
    static constexpr int SLOT = A + B + E + E2 + Rs + Fc + LFc + S1 + S2;
    static constexpr size_t DATA = ns_data_bytes<V>(EPB * SLOT);
    static constexpr size_t SMEM = DATA + (size_t)EPB * (sizeof(GeomClass) + NFACE * 16 + 16);
  };
  // ns_visc_kernel regions (per slot, values of the working type).  G holds the velocity
  // gradient, then in place the symmetric stress and the heat flux (NGS
  // slots: 6 + 3 in 3-D, 3 + 2 in 2-D; the modal input is parked there
  // first); the energy gradient goes to Dv, which then accumulates one
  // field's divergence at a time.  B holds the state until the stresses are
  // formed, then the face values FF and the divergence input Cv; X holds the
  // modal gradient components Gh in the first loop and the face-point
  // values Fg in the second.
  struct Visc {
    // LEAN: a tile with fewer threads than points (several CTAs per SM).
    // It keeps only the density and momenta of the state (the stresses need
    // the velocity alone), transforms one field or gradient component at a
    // time, writes the velocity gradient straight into its stress slots,
    // forms the stresses before the energy gradient is brought into the
    // heat-flux slots, and keeps the divergence behind the face values in B.
    static constexpr bool LEAN = NT < QD && EPB == 1;
    static constexpr int NGS = DIM == 3 ? 9 : 5;
    static constexpr int FF = cmax(NFACE * DIM * QF, F2), Cv = QD;
    static constexpr int B = LEAN ? cmax((DIM + 1) * QD, FF + Cv + QD) : cmax(NF * QD, FF + Cv);
    static constexpr int G = cmax(NGS * QD, NF * LD);
    static constexpr int X = cmax(DIM * LD, NFACE * DIM * GF);
    static constexpr int S1 = LEAN ? cmax(P1, cmax(DIM == 3 ? NFACE * DIM * C::G * Q : 0, F1))
                                   : cmax(cmax(NB1 * P1, DIM * P1), cmax(DIM == 3 ? NFACE * DIM * C::G * Q : 0, F1));
    static constexpr int S2 = LEAN ? cmax(cmax(P2, LD), F2) : cmax(cmax(NB1 * P2, DIM * P2), LD);
    static constexpr int Dv = LEAN ? 0 : DIM * QD;
    static constexpr int SLOT = B + G + X + S1 + S2 + Dv;
    static constexpr size_t DATA = ns_data_bytes<V>(EPB * SLOT);
    static constexpr size_t SMEM = DATA + (size_t)EPB * (sizeof(GeomClass) + NFACE * 16 + 16);
    static_assert(DIM * DIM <= NGS, "the velocity gradient fits the stress slots");
    static_assert(DATA % 8 == 0 && DATA >= (size_t)EPB * SLOT * sizeof(V), "geometry slots 8-byte aligned");
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
template <int DIM, class V>
__device__ __forceinline__ void primitive(const V *U, V *q) {
  const V r = U[0];
  V wk;
  if constexpr (DIM == 3) {
    const V u = U[1] / r, v = U[2] / r, w = U[3] / r;
    V e = U[4] / r;
    wk = u * u; wk = fma(v, v, wk); wk = fma(w, w, wk);
    e = fma(V(-0.5), wk, e);
    q[0] = u; q[1] = v; q[2] = w; q[3] = e;
  } else {
    const V u = U[1] / r, v = U[2] / r;
    V e = U[3] / r;
    wk = u * u; wk = fma(v, v, wk);
    e = fma(V(-0.5), wk, e);
    q[0] = u; q[1] = v; q[2] = e;
  }
}

// Gather the neighbour's state traces into face-major smem E2 in the own
// point order.  A boundary side's neighbour is its ghost state in the
// viscous BC database (Navier_Stokes3d::enforce_bc,
// src/Navier_Stokes3d.cpp:457-461; ghost_state) made from the own trace.
template <class C, class V>
__device__ __forceinline__ void load_nbr_traces(V *E2, const double *T, const FaceLink *lnk, const int *eid,
                                                const GeomClass *geo, const StageArgs &a, int tid) {
  constexpr int NF = C::NF, GF = C::GF, NFACE = C::NFACE, EPB = C::EPB;
  for (int w = tid; w < NFACE * EPB * NF * GF; w += C::NT) {
    const int f = w / (EPB * NF * GF), rem = w - f * EPB * NF * GF;
    const int s = rem / (NF * GF), ng = rem - s * NF * GF, n = ng / GF, g = ng - n * GF;
    V v = V(n == 0 ? 1.0 : 0.0);
    if (eid[s] >= 0) {
      const FaceLink lk = lnk[s * NFACE + f];
      const int bt = (geo[s].bc >> (4 * f)) & 15;
      const double *t = T + ((size_t)(lk.elem * NFACE + lk.face) * NF) * GF + a.perm[lk.perm + g];
      if (bt) {
        double Uo[5], Un[5];
#pragma unroll
        for (int k = 0; k < NF; ++k) Uo[k] = t[k * GF];
        ghost_state<C::DIM, NF>(a.bckind[bt], a.bcpar[bt], Uo, geo[s].onrm[f], true, Un);
        v = V(Un[n]);
      } else {
        v = V(t[n * GF]);
      }
    }
    E2[w] = v;
  }
}

// G2GL of NB face-major arrays [f][slot][b][GF] and accumulation with the
// inverse end weights into dst [slot][b][QD] (faces in increasing order).
template <class C, int NB, class V, bool TC = false>
__device__ __forceinline__ void lift_batch(const V *Fg, V *LFc, V *S, V *dst, int tid) {
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q, G = C::G, EPB = C::EPB, QD = C::QD, QF = C::QF;
  constexpr int NBT = C::NFACE * EPB * NB;
  if constexpr (DIM == 3) {
    vcontract<TC, G, G, 1, 0, G, Q, MatG2GL<L, Q, V>, false>(Fg, S, NBT, G * G, Q * G, tid, C::NT);
    __syncthreads();
    vcontract<TC, Q, G, 1, 1, G, Q, MatG2GL<L, Q, V>, false>(S, LFc, NBT, Q * G, Q * Q, tid, C::NT);
  } else {
    vcontract<TC, G, 1, 1, 0, G, Q, MatG2GL<L, Q, V>, false>(Fg, LFc, NBT, G, Q, tid, C::NT);
  }
  __syncthreads();
  const V w0 = V(1.0) / cW<V, L, Q>[0], w1 = V(1.0) / cW<V, L, Q>[Q - 1];
  for (int w = tid; w < EPB * NB * QD; w += C::NT) {
    const int slot = w / (NB * QD), rem = w - slot * NB * QD, b = rem / QD, p = rem - b * QD;
    V acc = dst[w];
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
template <class C, int NB, class V, bool TC = false>
__device__ __forceinline__ void forward_batch(V *src, V *dst, V *S1, V *S2, int tid) {
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q, QD = C::QD, LD = C::LD, NBT = C::EPB * NB;
  for (int w = tid; w < NBT * QD; w += C::NT) {
    const int p = w % QD;
    V wq;
    if constexpr (DIM == 3) wq = cW<V, L, Q>[p / (Q * Q)] * cW<V, L, Q>[(p / Q) % Q] * cW<V, L, Q>[p % Q];
    else wq = cW<V, L, Q>[p / Q] * cW<V, L, Q>[p % Q];
    src[w] = wq * src[w];
  }
  __syncthreads();
  if constexpr (DIM == 3) {
    vcontract<TC, Q, Q, Q, 0, Q, L, MatBt<L, Q, V>, false>(src, S1, NBT, QD, L * Q * Q, tid, C::NT);
    __syncthreads();
    vcontract<TC, L, Q, Q, 1, Q, L, MatBt<L, Q, V>, false>(S1, S2, NBT, L * Q * Q, L * L * Q, tid, C::NT);
    __syncthreads();
    vcontract<TC, L, L, Q, 2, Q, L, MatBt<L, Q, V>, false>(S2, dst, NBT, L * L * Q, LD, tid, C::NT);
  } else {
    vcontract<TC, Q, Q, 1, 0, Q, L, MatBt<L, Q, V>, false>(src, S1, NBT, QD, L * Q, tid, C::NT);
    __syncthreads();
    vcontract<TC, L, Q, 1, 1, Q, L, MatBt<L, Q, V>, false>(S1, dst, NBT, L * Q, LD, tid, C::NT);
  }
  __syncthreads();
}

// modal [slot][b][LD] -> GLL [slot][b][QD]
template <class C, int NB, class V, bool TC = false>
__device__ __forceinline__ void backward_batch(const V *src, V *dst, V *S1, V *S2, int tid) {
  constexpr int L = C::L, Q = C::Q, NBT = C::EPB * NB;
  if constexpr (C::DIM == 3) {
    vcontract<TC, L, L, L, 0, L, Q, MatB<L, Q, V>, false>(src, S1, NBT, C::LD, Q * L * L, tid, C::NT);
    __syncthreads();
    vcontract<TC, Q, L, L, 1, L, Q, MatB<L, Q, V>, false>(S1, S2, NBT, Q * L * L, Q * Q * L, tid, C::NT);
    __syncthreads();
    vcontract<TC, Q, Q, L, 2, L, Q, MatB<L, Q, V>, false>(S2, dst, NBT, Q * Q * L, C::QD, tid, C::NT);
  } else {
    vcontract<TC, L, L, 1, 0, L, Q, MatB<L, Q, V>, false>(src, S1, NBT, C::LD, Q * L, tid, C::NT);
    __syncthreads();
    vcontract<TC, Q, L, 1, 1, L, Q, MatB<L, Q, V>, false>(S1, dst, NBT, Q * L, C::QD, tid, C::NT);
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

// Element-major modal registers, GLL values and own traces of the slot's
// elements in the working type V (elements past the end read a unit
// density and zero otherwise).
template <class C, class V>
__device__ __forceinline__ void load_modal_v(V *dst, const double *src, int e0, int ne, int tid) {
  constexpr int BLK = C::NF * C::LD;
  for (int w = tid; w < C::EPB * BLK; w += C::NT) {
    const int e = e0 + w / BLK;
    dst[w] = e < ne ? V(src[(size_t)e0 * BLK + w]) : V(w % C::LD == 0 ? 1.0 : 0.0);
  }
}

template <class C, class V>
__device__ __forceinline__ void load_nodal_v(V *B, const double *Xn, int e0, int ne, int tid) {
  constexpr int NF = C::NF, QD = C::QD;
  for (int w = tid; w < C::EPB * NF * QD; w += C::NT) {
    const int s = w / (NF * QD), rem = w - s * NF * QD, n = rem / QD, p = rem - n * QD;
    const int e = e0 + s;
    B[w] = e < ne ? V(Xn[((size_t)n * ne + e) * QD + p]) : V(n == 0 ? 1.0 : 0.0);
  }
}

template <class C, class V>
__device__ __forceinline__ void load_own_traces_v(V *E, const double *T, int e0, int ne, int tid) {
  constexpr int NF = C::NF, GF = C::GF, NFACE = C::NFACE, EPB = C::EPB;
  for (int w = tid; w < EPB * NFACE * NF * GF; w += C::NT) {
    const int s = w / (NFACE * NF * GF), rem = w - s * NFACE * NF * GF;
    const int f = rem / (NF * GF), ng = rem - f * NF * GF;
    const int e = e0 + s;
    E[(f * EPB + s) * NF * GF + ng] = e < ne ? V(T[(size_t)e * NFACE * NF * GF + rem]) : V(ng < GF ? 1.0 : 0.0);
  }
}

// The FP32 gradient kernel's state: the slot's modal registers (or, NODAL,
// GLL values) with the density and energy means taken out in double before
// rounding.  Modal: the constant coefficients c0 of density and energy go to
// Rs as means c0 phi0 (phi0 = 2^(-DIM/2), the constant orthonormal mode) and
// are zeroed.  Nodal: each element's values at its first point are the
// reference values subtracted.  Elements past the end read a unit density.
template <class C>
__device__ __forceinline__ void load_state_shifted(float *dst, double *Rs, const double *src, bool nodal, int e0,
                                                   int ne, int tid) {
  constexpr int NF = C::NF, LD = C::LD, QD = C::QD, EPB = C::EPB;
  const double phi0 = C::DIM == 3 ? 0.35355339059327373 : 0.5;
  if (nodal) {
    for (int w = tid; w < EPB * NF * QD; w += C::NT) {
      const int s = w / (NF * QD), rem = w - s * NF * QD, n = rem / QD, p = rem - n * QD;
      const int e = e0 + s;
      double x = e < ne ? src[((size_t)n * ne + e) * QD + p] : (n == 0 ? 1.0 : 0.0);
      if (n == 0 || n == NF - 1) {
        const double ref = e < ne ? src[((size_t)n * ne + e) * QD] : (n == 0 ? 1.0 : 0.0);
        if (p == 0) Rs[2 * s + (n == 0 ? 0 : 1)] = ref;
        x -= ref;
      }
      dst[w] = float(x);
    }
  } else {
    constexpr int BLK = NF * LD;
    for (int w = tid; w < EPB * BLK; w += C::NT) {
      const int s = w / BLK, k = w - s * BLK, n = k / LD, m = k - n * LD;
      const int e = e0 + s;
      double x = e < ne ? src[(size_t)e0 * BLK + w] : (m == 0 ? 1.0 : 0.0);
      if (m == 0 && (n == 0 || n == NF - 1)) {
        Rs[2 * s + (n == 0 ? 0 : 1)] = x * phi0;
        x = 0.0;
      }
      dst[w] = float(x);
    }
  }
}

// ---------------------------------------------------------------- gradients
// V: working type (double, or float for the FP32 viscous form); inputs and
// outputs in global memory stay double.
template <class C, int PHYS, bool NODAL, class V = double, bool TC = false>
__global__ void __launch_bounds__(C::NT, NsCfg<C, V>::GRAD_MINB) ns_grad_kernel(StageArgs a) {
  using N = NsCfg<C, V>;
  using R = typename N::Grad;
  constexpr int DIM = C::DIM, NF = C::NF, Q = C::Q, L = C::L, EPB = C::EPB, QD = C::QD, GF = C::GF;
  constexpr int NFACE = C::NFACE, NVC = N::NVC, LD = C::LD;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  V *smem_raw = reinterpret_cast<V *>(smem_bytes);
  V *A = smem_raw, *B = A + EPB * R::A;
  double *E = reinterpret_cast<double *>(B + EPB * R::B), *E2 = reinterpret_cast<double *>(B + EPB * (R::B + R::E));
  double *Rs = reinterpret_cast<double *>(B + EPB * (R::B + R::E + R::E2));
  V *Fc = B + EPB * (R::B + R::E + R::E2 + R::Rs), *LFc = Fc + EPB * R::Fc;
  V *S1 = LFc + EPB * R::LFc, *S2 = S1 + EPB * R::S1;
  V *Qc = A, *Gd = A + EPB * R::Qc;     // in the modal input, dead after the backward transform
  GeomClass *geo = reinterpret_cast<GeomClass *>(smem_bytes + R::DATA);
  FaceLink *lnk = reinterpret_cast<FaceLink *>(geo + EPB);
  int *eid = reinterpret_cast<int *>(lnk + EPB * NFACE);
  const int tid = threadIdx.x, e0 = blockIdx.x * EPB;
  load_geo_slots<C>(geo, lnk, eid, a, e0, tid);
  if constexpr (R::F32) {
    load_state_shifted<C>(NODAL ? B : A, Rs, NODAL ? a.Xn : a.X, NODAL, e0, a.ne, tid);
  } else if constexpr (NODAL) {
    load_nodal_v<C>(B, a.Xn, e0, a.ne, tid);
  } else {
    load_modal_v<C>(A, a.X, e0, a.ne, tid);
  }
  if constexpr (!R::TRG) load_own_traces_v<C>(E, a.Tin, e0, a.ne, tid);
  __syncthreads();
  if constexpr (!R::TRG) load_nbr_traces<C>(E2, a.Tin, lnk, eid, geo, a, tid);
  if constexpr (!NODAL) {
    __syncthreads();
    if constexpr (N::NB1 == NF) {
      backward_batch<C, NF, V, TC>(A, B, S1, S2, tid);
    } else {   // one slot: fields [0, NB1) then [NB1, NF)
      backward_batch<C, N::NB1, V, TC>(A, B, S1, S2, tid);
      backward_batch<C, NF - N::NB1, V, TC>(A + N::NB1 * LD, B + N::NB1 * QD, S1, S2, tid);
    }
  }
  __syncthreads();
  for (int c = 0; c < NVC; ++c) {
    // primitive component c at the GLL points
    for (int w = tid; w < EPB * QD; w += C::NT) {
      const int s = w / QD, p = w - s * QD;
      if constexpr (R::F32) {
        // B holds rho' = rho - rb, the momenta and E' = E - Eb; with
        // rho = rb + rho', E/rho - Eb/rb = (E' rb - Eb rho') / (rb rho), so
        // e - Eb/rb (a per-element constant shift, invisible to the gradient)
        // is formed from O(Ma^2) terms
        const V rb = V(Rs[2 * s]), Eb = V(Rs[2 * s + 1]);
        const V rp = B[(s * NF) * QD + p], r = rb + rp;
        if (c < DIM) {
          Qc[w] = B[(s * NF + 1 + c) * QD + p] / r;
        } else {
          V k = V(0.0);
#pragma unroll
          for (int d = 0; d < DIM; ++d) {
            const V u = B[(s * NF + 1 + d) * QD + p] / r;
            k = fma(u, u, k);
          }
          const V Ep = B[(s * NF + NF - 1) * QD + p];
          Qc[w] = fma(V(-0.5), k, (Ep * rb - Eb * rp) / (rb * r));
        }
      } else {
        V U[5], q[4];
#pragma unroll
        for (int n = 0; n < NF; ++n) U[n] = B[(s * NF + n) * QD + p];
        primitive<DIM>(U, q);
        Qc[w] = q[c];
      }
    }
    // lift inputs ({{q_c}} - q_c) J n_d per face point, master-frame average
    for (int w = tid; w < NFACE * EPB * GF; w += C::NT) {
      const int f = w / (EPB * GF), rem = w - f * EPB * GF, s = rem / GF, g = rem - s * GF;
      // formed in double in both forms, then rounded to the working type
      double Uo[5], Un[5], qo[4], qn[4];
      if constexpr (R::TRG) {
        // the values load_own_traces_v and load_nbr_traces would have staged
        const int e = eid[s];
        if (e >= 0) {
          const double *to = a.Tin + ((size_t)e * NFACE + f) * NF * GF + g;
          const FaceLink lk = lnk[s * NFACE + f];
          const double *t = a.Tin + ((size_t)(lk.elem * NFACE + lk.face) * NF) * GF + a.perm[lk.perm + g];
#pragma unroll
          for (int n = 0; n < NF; ++n) { Uo[n] = to[n * GF]; Un[n] = t[n * GF]; }
          const int bt = (geo[s].bc >> (4 * f)) & 15;
          if (bt) {
            double Ut[5];
#pragma unroll
            for (int n = 0; n < NF; ++n) Ut[n] = Un[n];
            ghost_state<C::DIM, NF>(a.bckind[bt], a.bcpar[bt], Ut, geo[s].onrm[f], true, Un);
          }
        } else {
#pragma unroll
          for (int n = 0; n < NF; ++n) Uo[n] = Un[n] = n == 0 ? 1.0 : 0.0;
        }
      } else {
#pragma unroll
        for (int n = 0; n < NF; ++n) {
          Uo[n] = E[((f * EPB + s) * NF + n) * GF + g];
          Un[n] = E2[((f * EPB + s) * NF + n) * GF + g];
        }
      }
      primitive<DIM>(Uo, qo);
      primitive<DIM>(Un, qn);
      const GeomClass &gc = geo[s];
      const bool master = (gc.master >> f) & 1;
      const double avg = master ? 0.5 * (qo[c] + qn[c]) : 0.5 * (qn[c] + qo[c]);
      const double d = (avg - qo[c]) * gc.jr[f];
#pragma unroll
      for (int k = 0; k < DIM; ++k) Fc[((f * EPB + s) * DIM + k) * GF + g] = V(gc.onrm[f][k] * d);
    }
    __syncthreads();
    // collocation derivatives along r, s, t
    using Sh = Sh3<DIM, Q>;
    vcontract<TC, Sh::a, Sh::b, Sh::c, 0, Q, Q, MatD<L, Q, V>, false>(Qc, Gd, EPB, QD, DIM * QD, tid, C::NT);
    vcontract<TC, Sh::a, Sh::b, Sh::c, 1, Q, Q, MatD<L, Q, V>, false>(Qc, Gd + QD, EPB, QD, DIM * QD, tid, C::NT);
    if constexpr (DIM == 3)
      vcontract<TC, Sh::a, Sh::b, Sh::c, 2, Q, Q, MatD<L, Q, V>, false>(Qc, Gd + 2 * QD, EPB, QD, DIM * QD, tid, C::NT);
    __syncthreads();
    // chain rule (src/Hex.cpp:1994-2006): d/dx = rx d/dr + sx d/ds + tx d/dt
    for (int w = tid; w < EPB * QD; w += C::NT) {
      const int s = w / QD, p = w - s * QD;
      V *g = Gd + s * DIM * QD + p;
      const double *m = geo[s].metric;
      const V fr = g[0], fs = g[QD], ft = DIM == 3 ? g[2 * QD] : V(0.0);
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        V v = V(m[0 * 3 + k]) * fr;
        v = fma(V(m[1 * 3 + k]), fs, v);
        if (DIM == 3) v = fma(V(m[2 * 3 + k]), ft, v);
        g[k * QD] = v;
      }
    }
    __syncthreads();
    lift_batch<C, DIM, V, TC>(Fc, LFc, S1, Gd, tid);
    forward_batch<C, DIM, V, TC>(Gd, S2, S1, LFc, tid);
    for (int w = tid; w < EPB * DIM * LD; w += C::NT) {
      const int s = w / (DIM * LD), rem = w - s * DIM * LD;
      const int e = e0 + s;
      if (e < a.ne) a.Ghat[((size_t)e * NVC + c) * DIM * LD + rem] = double(S2[w]);
    }
    __syncthreads();
  }
}

// ----------------------------------------------- stresses, traces, divergence
// The viscous stress (src/Navier_Stokes3d.cpp:305-344) from the velocity
// gradient at one point, g[k * stride] = (ux, uy, [uz,] vx, vy, [vz, wx, wy,
// wz]); t = (t11, t12, t13, t22, t23, t33) in 3-D, (t11, t12, t22) in 2-D.
template <int DIM, class V>
__device__ __forceinline__ void viscous_stress(const V *g, int stride, V mu, V *t) {
  if constexpr (DIM == 3) {
    const V ux = g[0 * stride], uy = g[1 * stride], uz = g[2 * stride];
    const V vx = g[3 * stride], vy = g[4 * stride], vz = g[5 * stride];
    const V wx = g[6 * stride], wy = g[7 * stride], wz = g[8 * stride];
    const V two = V(2.0), one = V(1.0), tt = V(2.0 / 3.0);
    V t12 = uy + vx; t12 = mu * t12;
    V t13 = uz + wx; t13 = mu * t13;
    V t23 = vz + wy; t23 = mu * t23;
    V wk = two * ux - vy;
    V t11 = one * wk - wz; t11 = tt * t11; t11 = mu * t11;
    wk = two * vy - ux;
    V t22 = one * wk - wz; t22 = tt * t22; t22 = mu * t22;
    wk = two * wz - ux;
    V t33 = one * wk - vy; t33 = tt * t33; t33 = mu * t33;
    t[0] = t11; t[1] = t12; t[2] = t13; t[3] = t22; t[4] = t23; t[5] = t33;
  } else {
    const V ux = g[0 * stride], uy = g[1 * stride], vx = g[2 * stride], vy = g[3 * stride];
    const V two = V(2.0), tt = V(2.0 / 3.0);
    V t12 = uy + vx; t12 = mu * t12;
    V t11 = two * ux - vy; t11 = tt * t11; t11 = mu * t11;
    V t22 = two * vy - ux; t22 = tt * t22; t22 = mu * t22;
    t[0] = t11; t[1] = t12; t[2] = t22;
  }
}

// The energy flux tau . u + (gamma mu / Pr) grad e at one point.
template <int DIM, class V>
__device__ __forceinline__ void heat_flux(const V *t, V u, V v, V w, V ex, V ey, V ez, V mu, V gPr, V *q) {
  if constexpr (DIM == 3) {
    V qx = t[0] * u; qx = fma(t[1], v, qx); qx = fma(t[2], w, qx);
    V qy = t[1] * u; qy = fma(t[3], v, qy); qy = fma(t[4], w, qy);
    V qz = t[2] * u; qz = fma(t[4], v, qz); qz = fma(t[5], w, qz);
    q[0] = fma(gPr, mu * ex, qx); q[1] = fma(gPr, mu * ey, qy); q[2] = fma(gPr, mu * ez, qz);
  } else {
    V qx = t[0] * u; qx = fma(t[1], v, qx);
    V qy = t[1] * u; qy = fma(t[2], v, qy);
    q[0] = fma(gPr, mu * ex, qx); q[1] = fma(gPr, mu * ey, qy);
  }
}

// The viscous kernel's first part for the lean tile (NsCfg::Visc::LEAN,
// one element per CTA): the density and momenta at the GLL points into B,
// the velocity gradient into the stress slots of Gg one component at a time
// (Gh = X holds one component's modal gradient), the stresses in place, the
// energy gradient into the heat-flux slots, then the heat flux in place.
// The arithmetic of every value is that of the staged path.
template <class C, bool NODAL, class V, bool TC>
__device__ __forceinline__ void ns_visc_lean_front(const StageArgs &a, V *B, V *Gg, V *X, V *S1, V *S2, int e0,
                                                   int tid) {
  using N = NsCfg<C, V>;
  constexpr int DIM = C::DIM, NF = C::NF, QD = C::QD, LD = C::LD, NVC = N::NVC, NGS = N::Visc::NGS;
  constexpr int NT6 = DIM == 3 ? 6 : 3;
  static_assert(C::EPB == 1, "the lean viscous tile holds one element");
  const int e = e0 < a.ne ? e0 : -1;
  // state: density and momenta (the stresses need the velocity only)
  if constexpr (NODAL) {
    for (int w = tid; w < (DIM + 1) * QD; w += C::NT) {
      const int n = w / QD, p = w - n * QD;
      B[w] = e >= 0 ? V(a.Xn[((size_t)n * a.ne + e) * QD + p]) : V(n == 0 ? 1.0 : 0.0);
    }
  } else {
    for (int w = tid; w < NF * LD; w += C::NT)
      Gg[w] = e >= 0 ? V(a.X[(size_t)e0 * NF * LD + w]) : V(w % LD == 0 ? 1.0 : 0.0);
    __syncthreads();
    for (int n = 0; n <= DIM; ++n) backward_batch<C, 1, V, TC>(Gg + n * LD, B + n * QD, S1, S2, tid);
  }
  __syncthreads();
  // velocity gradient: component c, direction d into slot c*DIM + d
  for (int c = 0; c < DIM; ++c) {
    for (int w = tid; w < DIM * LD; w += C::NT)
      X[w] = e >= 0 ? V(a.Ghat[((size_t)e * NVC + c) * DIM * LD + w]) : V(0.0);
    __syncthreads();
    for (int d = 0; d < DIM; ++d) backward_batch<C, 1, V, TC>(X + d * LD, Gg + (c * DIM + d) * QD, S1, S2, tid);
  }
  const V mu = V(a.vis), gPr = V(a.gamma / a.Pr);
  for (int p = tid; p < QD; p += C::NT) {
    V t[6];
    viscous_stress<DIM, V>(Gg + p, QD, mu, t);
#pragma unroll
    for (int k = 0; k < NT6; ++k) Gg[k * QD + p] = t[k];
  }
  __syncthreads();
  // energy gradient into the heat-flux slots (the velocity gradient's last
  // components, dead once the stresses are formed)
  for (int w = tid; w < DIM * LD; w += C::NT)
    X[w] = e >= 0 ? V(a.Ghat[((size_t)e * NVC + DIM) * DIM * LD + w]) : V(0.0);
  __syncthreads();
  for (int d = 0; d < DIM; ++d) backward_batch<C, 1, V, TC>(X + d * LD, Gg + (NT6 + d) * QD, S1, S2, tid);
  for (int p = tid; p < QD; p += C::NT) {
    V t[6], q[3];
#pragma unroll
    for (int k = 0; k < NT6; ++k) t[k] = Gg[k * QD + p];
    const V r = B[p];
    const V u = B[QD + p] / r, v = B[2 * QD + p] / r, w = DIM == 3 ? B[3 * QD + p] / r : V(0.0);
    const V *ge = Gg + NT6 * QD + p;
    heat_flux<DIM, V>(t, u, v, w, ge[0], ge[QD], DIM == 3 ? ge[2 * QD] : V(0.0), mu, gPr, q);
#pragma unroll
    for (int d = 0; d < DIM; ++d) Gg[(NT6 + d) * QD + p] = q[d];
  }
  static_assert(NGS == NT6 + DIM, "stress and heat-flux slots");
}

template <class C, int PHYS, bool NODAL, class V = double, bool TC = false>
__global__ void __launch_bounds__(C::NT, NsCfg<C, V>::VISC_MINB) ns_visc_kernel(StageArgs a) {
  using N = NsCfg<C, V>;
  using R = typename N::Visc;
  constexpr int DIM = C::DIM, NF = C::NF, Q = C::Q, L = C::L, G = C::G, EPB = C::EPB, QD = C::QD;
  constexpr int GF = C::GF, QF = C::QF, NFACE = C::NFACE, NV = N::NV, NVC = N::NVC, LD = C::LD, NGS = R::NGS;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  V *smem_raw = reinterpret_cast<V *>(smem_bytes);
  V *B = smem_raw, *Gg = B + EPB * R::B, *X = Gg + EPB * R::G;
  V *S1 = X + EPB * R::X, *S2 = S1 + EPB * R::S1, *Dv = S2 + EPB * R::S2;
  V *Gh = X, *Fg = X;                    // first loop / second loop
  V *FF = B, *Cv = B + EPB * R::FF;      // after the stresses are formed
  if constexpr (R::LEAN) Dv = Cv + EPB * R::Cv;   // the divergence behind the face values
  GeomClass *geo = reinterpret_cast<GeomClass *>(smem_bytes + R::DATA);
  FaceLink *lnk = reinterpret_cast<FaceLink *>(geo + EPB);
  int *eid = reinterpret_cast<int *>(lnk + EPB * NFACE);
  const int tid = threadIdx.x, e0 = (a.vtiles ? a.vtiles[blockIdx.x] : (int)blockIdx.x) * EPB;
  load_geo_slots<C>(geo, lnk, eid, a, e0, tid);
  if constexpr (R::LEAN) {
    ns_visc_lean_front<C, NODAL, V, TC>(a, B, Gg, X, S1, S2, e0, tid);
  } else if constexpr (NODAL) {
    load_nodal_v<C>(B, a.Xn, e0, a.ne, tid);
  } else {
    load_modal_v<C>(Gg, a.X, e0, a.ne, tid);  // modal input parked in the gradient region
    __syncthreads();
    if constexpr (N::NB1 == NF) {
      backward_batch<C, NF, V, TC>(Gg, B, S1, S2, tid);
    } else {   // one slot: fields [0, NB1) then [NB1, NF)
      backward_batch<C, N::NB1, V, TC>(Gg, B, S1, S2, tid);
      backward_batch<C, NF - N::NB1, V, TC>(Gg + N::NB1 * LD, B + N::NB1 * QD, S1, S2, tid);
    }
  }
  if constexpr (!R::LEAN) {
  __syncthreads();
  // projected gradients at the GLL points: velocity components into Gg
  // (component c, direction d at slot c*DIM+d), the energy gradient into Dv
  for (int c = 0; c < NVC; ++c) {
    for (int w = tid; w < EPB * DIM * LD; w += C::NT) {
      const int s = w / (DIM * LD), rem = w - s * DIM * LD;
      const int e = e0 + s;
      Gh[w] = e < a.ne ? V(a.Ghat[((size_t)e * NVC + c) * DIM * LD + rem]) : V(0.0);
    }
    __syncthreads();
    backward_batch<C, DIM, V, TC>(Gh, Dv, S1, S2, tid);
    if (c < DIM) {
      for (int w = tid; w < EPB * DIM * QD; w += C::NT) {
        const int s = w / (DIM * QD), rem = w - s * DIM * QD;
        Gg[(s * NGS + c * DIM) * QD + rem] = Dv[w];
      }
      __syncthreads();
    }
  }
  // stresses and heat flux, in place (slots gslot(n, d))
  const V mu = V(a.vis), gPr = V(a.gamma / a.Pr);
  for (int w = tid; w < EPB * QD; w += C::NT) {
    const int s = w / QD, p = w - s * QD;
    V *g = Gg + s * NGS * QD + p;
    const V *ge = Dv + s * DIM * QD + p;
    V U[5];
#pragma unroll
    for (int n = 0; n < NF; ++n) U[n] = B[(s * NF + n) * QD + p];
    const V r = U[0];
    V t[6], q[3];
    viscous_stress<DIM, V>(g, QD, mu, t);
    if constexpr (DIM == 3) {
      const V u = U[1] / r, v = U[2] / r, ww = U[3] / r;
      heat_flux<DIM, V>(t, u, v, ww, ge[0], ge[QD], ge[2 * QD], mu, gPr, q);
    } else {
      const V u = U[1] / r, v = U[2] / r;
      heat_flux<DIM, V>(t, u, v, V(0.0), ge[0], ge[QD], V(0.0), mu, gPr, q);
    }
    constexpr int NT6 = DIM == 3 ? 6 : 3;
#pragma unroll
    for (int k = 0; k < NT6; ++k) g[k * QD] = t[k];
#pragma unroll
    for (int d = 0; d < DIM; ++d) g[(NT6 + d) * QD] = q[d];
  }
  } // !LEAN
  __syncthreads();
  for (int n = 0; n < NV; ++n) {
    // face GLL values of g_n (DIM components), face-major [f][slot][d][QF]
    for (int w = tid; w < NFACE * EPB * DIM * QF; w += C::NT) {
      const int f = w / (EPB * DIM * QF), rem = w - f * EPB * DIM * QF;
      const int s = rem / (DIM * QF), rem2 = rem - s * DIM * QF, d = rem2 / QF, x = rem2 - d * QF;
      const V *src = Gg + (s * NGS + N::gslot(n, d)) * QD;
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
      vcontract<TC, Q, Q, 1, 0, Q, G, MatGL2G<L, Q, V>, false>(FF, S1, NB, Q * Q, G * Q, tid, C::NT);
      __syncthreads();
      vcontract<TC, G, Q, 1, 1, Q, G, MatGL2G<L, Q, V>, false>(S1, Fg, NB, G * Q, G * G, tid, C::NT);
    } else {
      vcontract<TC, Q, 1, 1, 0, Q, G, MatGL2G<L, Q, V>, false>(FF, Fg, NB, Q, G, tid, C::NT);
    }
    __syncthreads();
    // g_n . n (own normals), the viscous trace of this side
    for (int w = tid; w < EPB * NFACE * GF; w += C::NT) {
      const int s = w / (NFACE * GF), rem = w - s * NFACE * GF, f = rem / GF, gq = rem - f * GF;
      const int e = e0 + s;
      if (e >= a.ne) continue;
      const double *nr = geo[s].onrm[f];
      V v = V(nr[0]) * Fg[((f * EPB + s) * DIM + 0) * GF + gq];
      v = fma(V(nr[1]), Fg[((f * EPB + s) * DIM + 1) * GF + gq], v);
      if (DIM == 3) v = fma(V(nr[2]), Fg[((f * EPB + s) * DIM + 2) * GF + gq], v);
      a.V[(((size_t)e * NFACE + f) * NV + n) * GF + gq] = double(v);
    }
    // collocation divergence of g_n (contravariant form) into Dv [slot][QD]
    for (int r = 0; r < DIM; ++r) {
      for (int w = tid; w < EPB * QD; w += C::NT) {
        const int s = w / QD, p = w - s * QD;
        const double *m = geo[s].metric;
        const V *gs = Gg + s * NGS * QD + p;
        V v = V(m[3 * r + 0]) * gs[N::gslot(n, 0) * QD];
        v = fma(V(m[3 * r + 1]), gs[N::gslot(n, 1) * QD], v);
        if (DIM == 3) v = fma(V(m[3 * r + 2]), gs[N::gslot(n, 2) * QD], v);
        Cv[w] = v;
      }
      __syncthreads();
      using Sh = Sh3<DIM, Q>;
      if (r == 0) vcontract<TC, Sh::a, Sh::b, Sh::c, 0, Q, Q, MatD<L, Q, V>, false>(Cv, Dv, EPB, QD, QD, tid, C::NT);
      else if (r == 1) vcontract<TC, Sh::a, Sh::b, Sh::c, 1, Q, Q, MatD<L, Q, V>, true>(Cv, Dv, EPB, QD, QD, tid, C::NT);
      else vcontract<TC, Sh::a, Sh::b, Sh::c, 2, Q, Q, MatD<L, Q, V>, true>(Cv, Dv, EPB, QD, QD, tid, C::NT);
      __syncthreads();
    }
    // projected divergence of this field
    forward_batch<C, 1, V, TC>(Dv, S2, S1, FF, tid);
    for (int w = tid; w < EPB * LD; w += C::NT) {
      const int s = w / LD, m = w - s * LD;
      const int e = e0 + s;
      if (e < a.ne) a.Pv[((size_t)e * NV + n) * LD + m] = double(S2[w]);
    }
    __syncthreads();
  }
}

}  // namespace dgmx
