// Fused DG stage kernels for sm_100a (FP64, and FP32 with an FP64 solution
// register for the mixed-precision form).
//
// One launch evaluates Domain::time_derivative on a modal register and folds
// the RK stage update and the next stage's face traces into the same pass:
//   1. load the element's modal coefficients (element-major, one contiguous
//      block per element)
//   2. own face traces at the side Gauss points (modal -> Gauss, the
//      polynomial equivalent of fill_sides' GL2G interpolation,
//      src/Hex.cpp:933-947)
//   3. backward transform to the GLL points (src/Hex.cpp:795-812)
//   4. volume term: contravariant fluxes and collocation derivatives
//      (algebraically Sum_dir d/dx_dir F_dir, src/Euler3d.cpp:506-566)
//   5. numerical flux on every face point against the neighbour's traces
//      from the previous stage (src/Euler3d.cpp:584-817)
//   6. lift: G2GL interpolation and 1/w_end scaling onto the boundary GLL
//      points (src/Hex.cpp:1768-1952)
//   7. projection: w-weighted inner product with the orthonormal basis
//      (the J of wJ cancels the 1/J mass, src/Hex.cpp:200-205, :652-685)
//   8. RK stage update on the modal registers (src/TimeInt.cpp:266-302,
//      :826-860, :1989-2013)
//   9. traces of the updated register for the next stage
// Traces are double buffered, so an element may overwrite its own register
// in place: neighbours only ever read its traces.
#pragma once

#include <type_traits>

#include "kernels.cuh"

namespace dgmx {

constexpr int phys_dim(int p) { return (p == DGMX_EULER3D || p == DGMX_NS3D) ? 3 : 2; }
constexpr int phys_nf(int p) { return p == DGMX_SHALLOW ? 3 : (phys_dim(p) == 3 ? 5 : 4); }
constexpr int cmax(int a, int b) { return a > b ? a : b; }

// One kernel tile: PHYS physics, L modes and Q GLL points per direction,
// EPB elements per CTA, MINB CTAs per SM requested from the register
// allocator (__launch_bounds__ minimum blocks; 0 = no request).
// NT_ (nonzero) fixes the CTA's thread count, for kernels that run several
// tiles' bodies under one launch shape.
template <int PHYS, int L_, int Q_, int EPB_, int MINB_ = 0, bool MIXED_ = false, int NT_ = 0>
struct Cfg {
  // working precision: FP64, or FP32 for the mixed form (the solution
  // register U stays FP64 in global memory)
  static constexpr bool MIXED = MIXED_;
  static constexpr bool WARP = false;   // the helpers' team is the whole CTA
  static constexpr int FPT = 1;         // fields per contraction task (see contract)
  static constexpr int PHYSICS = PHYS;
  using R = std::conditional_t<MIXED_, float, double>;
  static constexpr int DIM = phys_dim(PHYS), NF = phys_nf(PHYS);
  static constexpr int L = L_, Q = Q_, G = Q_ - 1, EPB = EPB_, MINB = MINB_ > 0 ? MINB_ : 1;
  static constexpr int MINB_REQ = MINB_;   // 0: no register cap requested
  static constexpr int NFACE = 2 * DIM;
  static constexpr int LD = Pow<L, DIM>::v, QD = Pow<Q, DIM>::v;
  static constexpr int GF = Pow<G, DIM - 1>::v, QF = Pow<Q, DIM - 1>::v, LF = Pow<L, DIM - 1>::v;
  static constexpr int NT = NT_ > 0 ? NT_ : cmax(64, ((EPB * QD + 31) / 32) * 32 > 1024 ? 1024 : ((EPB * QD + 31) / 32) * 32);
  // per-slot region sizes (doubles)
  // Rows of an even number of values are stored at an odd pitch in shared
  // memory, so the pencils a warp reads (one per lane, K apart) fall on
  // distinct banks: modal rows of L (when L + 1 <= Q, so the padded
  // intermediates still fit their regions) and face-trace rows of G.
  static constexpr int PL = (L_ % 2 == 0 && L_ + 1 <= Q_) ? L_ + 1 : L_;
  static constexpr int PG = (G % 2 == 0) ? G + 1 : G;
  static constexpr int AB = DIM == 3 ? L_ * L_ * PL : L_ * PL;   // modal block (slot, field), padded
  static constexpr int EB = DIM == 3 ? G * PG : PG;              // face-trace block (face, slot, field)
  static constexpr int SZ_A = NF * AB;                 // modal register
  static constexpr int SZ_B = NF * QD;                 // GLL values
  static constexpr int SZ_C = NF * QD;                 // flux / scratch
  static constexpr int SZ_D = NF * QD;                 // divergence + lift
  static constexpr int SZ_E = NFACE * NF * EB;         // face traces / lift input
  // projected RHS (modal); shares the E region when it fits (E is dead
  // between the lift and the next-trace phase)
  static constexpr bool R_IN_E = NFACE * NF * EB >= NF * LD;
  static constexpr int SZ_R = R_IN_E ? 0 : NF * LD;
  static constexpr int SZ_S = cmax(cmax(NF * Q * (DIM == 3 ? LF : PL), NFACE * NF * (DIM == 3 ? LF : PL)),
                                   DIM == 3 ? NFACE * NF * Q * PG : 0);
  static constexpr int SZ_SLOT = SZ_A + SZ_B + SZ_C + SZ_D + SZ_E + SZ_R + SZ_S;
  static constexpr size_t DATA = ((size_t)EPB * SZ_SLOT * sizeof(R) + 15) / 16 * 16;
  static constexpr size_t SMEM = DATA + (size_t)EPB * (sizeof(GeomClass) + NFACE * sizeof(FaceLink) + 16 +
                                                     (MIXED_ ? sizeof(RefState<R>) : 0));
  static_assert(NFACE * QF <= 2 * QD, "lift face buffer must fit in the B+C regions");
  static_assert(DIM == 2 || NFACE * G * PL <= 2 * QD, "trace intermediate must fit in the B+C regions");
  static_assert(PL <= Q, "padded modal rows must fit the GLL-sized scratch");
  static_assert(SMEM <= 227 * 1024 || EPB > 1, "element slot does not fit in shared memory");
};



// Barrier of the helpers' team.
template <class C>
__device__ __forceinline__ void csync() {
  if constexpr (C::WARP) __syncwarp(); else __syncthreads();
}

// Trailing-1 shapes so one contraction routine serves 2-D and 3-D.
template <int DIM, int N> struct Sh3 { static constexpr int a = N, b = N, c = (DIM == 3 ? N : 1); };

template <class K>
struct Smem {
  using T = typename K::R;
  T *A, *B, *C, *D, *E, *R, *S;
  GeomClass *geo;
  FaceLink *lnk;
  int *eid;
  RefState<T> *ref;  // mixed form: the reference state of each slot's solve
  __device__ Smem(unsigned char *raw) {
    T *base = reinterpret_cast<T *>(raw);
    A = base;
    B = A + K::EPB * K::SZ_A;
    C = B + K::EPB * K::SZ_B;
    D = C + K::EPB * K::SZ_C;
    E = D + K::EPB * K::SZ_D;
    R = K::R_IN_E ? E : E + K::EPB * K::SZ_E;
    S = E + K::EPB * K::SZ_E + K::EPB * K::SZ_R;
    geo = reinterpret_cast<GeomClass *>(raw + K::DATA);
    lnk = reinterpret_cast<FaceLink *>(geo + K::EPB);
    eid = reinterpret_cast<int *>(lnk + K::EPB * K::NFACE);
    ref = reinterpret_cast<RefState<T> *>(eid + 4 * K::EPB);
  }
};

// ---- face-local helpers ----------------------------------------------------
// Face f: normal axis and end (0 = first GLL point, 1 = last).
// 3-D: 0 k=0, 1 j=0, 2 i=Q-1, 3 j=Q-1, 4 i=0, 5 k=Q-1 (src/Hex.cpp:815-865)
// 2-D: 0 j=0, 1 i=Q-1, 2 j=Q-1, 3 i=0 (src/Quad.cpp:767-790)
template <int DIM> __device__ __host__ constexpr int face_axis(int f) {
  return DIM == 3 ? (f == 0 || f == 5 ? 2 : (f == 1 || f == 3 ? 1 : 0)) : (f == 0 || f == 2 ? 1 : 0);
}
template <int DIM> __device__ __host__ constexpr int face_end(int f) {
  return DIM == 3 ? (f == 2 || f == 3 || f == 5) : (f == 1 || f == 2);
}

// Offset of face point g (0 .. GF-1) inside a padded trace block, and of
// modal entry m (row-major, rows of L) inside a padded modal block.
template <class C>
__device__ __forceinline__ int epos(int g) {
  if constexpr (C::DIM == 3) return (g / C::G) * C::PG + g % C::G;
  else return g;
}
template <class C>
__device__ __forceinline__ int apos(int m) { return (m / C::L) * C::PL + m % C::L; }


template <int L, int Q, class T>
struct MatEnd2 { static __device__ __forceinline__ T get(int a, int end) { return cEnd<T, L, Q>[end * L + a]; } };

// Endpoint reduction along axis AX of a batch of padded modal arrays: both
// end faces at once (FLO = the face at the first GLL point, FHI = the last),
// each into its face-local L^(DIM-1) array (planes, or padded 2-D lines).
template <class C, int AX, int FLO, int FHI>
__device__ __forceinline__ void face_reduce(const typename C::R *A, typename C::R *out, int tid, int nthr) {
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q;
  using Sh = Sh3<DIM, L>;
  constexpr int IS0 = DIM == 3 ? L * C::PL : C::PL, IS1 = DIM == 3 ? C::PL : 1;
  constexpr int OB = DIM == 3 ? C::LF : C::PL;   // output block: an L x L plane, or a padded line
  constexpr int FS = C::EPB * C::NF * OB;       // one face's blocks
  // plane strides of the outputs: (b, c) for AX 0, (a, c) for AX 1, (a, b) for AX 2
  constexpr int OS0 = DIM == 3 ? (AX == 1 ? L : (AX == 2 ? L : -1)) : (AX == 1 ? 1 : -1);
  constexpr int OS1 = DIM == 3 ? (AX == 0 ? L : (AX == 2 ? 1 : -1)) : (AX == 0 ? 1 : -1);
  contract<Sh::a, Sh::b, Sh::c, AX, L, 2, MatEnd2<L, Q, typename C::R>, false, typename C::R, IS0, IS1, OS0, OS1,
           C::FPT, (FHI - FLO) * FS>(A, out + FLO * FS, C::EPB * C::NF, C::AB, OB, tid, nthr);
}

// Traces at the side Gauss points of a modal register held in smem A.
// Result in E, face-major [f][slot][n][gf].  Uses S and B+C as scratch.
template <class C>
__device__ __forceinline__ void modal_traces(const typename C::R *A, typename C::R *E, typename C::R *S,
                                             typename C::R *Cs, int tid, int nthr) {
  using T = typename C::R;
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q, G = C::G;
  if constexpr (DIM == 3) {
    // faces: 0 k=0, 1 j=0, 2 i=Q-1, 3 j=Q-1, 4 i=0, 5 k=Q-1
    face_reduce<C, 0, 4, 2>(A, S, tid, nthr);
    face_reduce<C, 1, 1, 3>(A, S, tid, nthr);
    face_reduce<C, 2, 0, 5>(A, S, tid, nthr);
  } else {
    // faces: 0 j=0, 1 i=Q-1, 2 j=Q-1, 3 i=0
    face_reduce<C, 0, 3, 1>(A, S, tid, nthr);
    face_reduce<C, 1, 0, 2>(A, S, tid, nthr);
  }
  csync<C>();
  constexpr int NB = C::NFACE * C::EPB * C::NF, PL = C::PL, PG = C::PG;
  if constexpr (DIM == 3) {
    contract<L, L, 1, 0, L, G, MatBg<L, Q, T>, false, T, -1, -1, PL, 1, C::FPT>(S, Cs, NB, L * L, G * PL, tid, nthr);
    csync<C>();
    contract<G, L, 1, 1, L, G, MatBg<L, Q, T>, false, T, PL, 1, PG, 1, C::FPT>(Cs, E, NB, G * PL, C::EB, tid, nthr);
  } else {
    contract<L, 1, 1, 0, L, G, MatBg<L, Q, T>, false, typename C::R, -1, -1, -1, -1, C::FPT>(S, E, NB, PL, C::EB, tid, nthr);
  }
  csync<C>();
}

// Backward transform: modal A [slot][n][L^d] -> GLL B [slot][n][QD].  A is
// the padded modal block (PADDED) or a dense one.
template <class C, bool PADDED = true>
__device__ __forceinline__ void backward(const typename C::R *A, typename C::R *B, typename C::R *S,
                                         typename C::R *Cs, int tid, int nthr) {
  using T = typename C::R;
  constexpr int L = C::L, Q = C::Q, NB = C::EPB * C::NF, PL = C::PL;
  constexpr int AP = PADDED ? PL : L, ABLK = PADDED ? C::AB : C::LD;
  if constexpr (C::DIM == 3) {
    contract<L, L, L, 0, L, Q, MatB<L, Q, T>, false, T, L * AP, AP, -1, -1, C::FPT>(A, S, NB, ABLK, Q * L * L, tid, nthr);
    csync<C>();
    contract<Q, L, L, 1, L, Q, MatB<L, Q, T>, false, T, -1, -1, Q * PL, PL, C::FPT>(S, Cs, NB, Q * L * L, Q * Q * PL, tid,
                                                                            nthr);
    csync<C>();
    contract<Q, Q, L, 2, L, Q, MatB<L, Q, T>, false, T, Q * PL, PL, -1, -1, C::FPT>(Cs, B, NB, Q * Q * PL, C::QD, tid, nthr);
  } else {
    contract<L, L, 1, 0, L, Q, MatB<L, Q, T>, false, T, AP, 1, PL, 1, C::FPT>(A, S, NB, ABLK, Q * PL, tid, nthr);
    csync<C>();
    contract<Q, L, 1, 1, L, Q, MatB<L, Q, T>, false, T, PL, 1, -1, -1, C::FPT>(S, B, NB, Q * PL, C::QD, tid, nthr);
  }
  csync<C>();
}

// Forward projection: GLL D [slot][n][QD] -> modal R, the GLL quadrature
// weights applied by the weighted matrices (B w; the J of wJ cancels the
// 1/J mass of the orthonormal basis).
template <class C>
__device__ __forceinline__ void forward(const typename C::R *D, typename C::R *R, typename C::R *Cs,
                                        typename C::R *Bs, int tid, int nthr) {
  using T = typename C::R;
  constexpr int L = C::L, Q = C::Q, NB = C::EPB * C::NF, PL = C::PL;
  // the contiguous axis first, into rows of L at the odd pitch PL
  if constexpr (C::DIM == 3) {
    contract<Q, Q, Q, 2, Q, L, MatBtw<L, Q, T>, false, T, -1, -1, Q * PL, PL, C::FPT>(D, Cs, NB, C::QD, Q * Q * PL, tid, nthr);
    csync<C>();
    contract<Q, Q, L, 1, Q, L, MatBtw<L, Q, T>, false, T, Q * PL, PL, -1, -1, C::FPT>(Cs, Bs, NB, Q * Q * PL, Q * L * L, tid, nthr);
    csync<C>();
    contract<Q, L, L, 0, Q, L, MatBtw<L, Q, T>, false, typename C::R, -1, -1, -1, -1, C::FPT>(Bs, R, NB, Q * L * L, C::LD, tid, nthr);
  } else {
    contract<Q, Q, 1, 1, Q, L, MatBtw<L, Q, T>, false, T, -1, -1, PL, 1, C::FPT>(D, Cs, NB, C::QD, Q * PL, tid, nthr);
    csync<C>();
    contract<Q, L, 1, 0, Q, L, MatBtw<L, Q, T>, false, T, PL, 1, -1, -1, C::FPT>(Cs, R, NB, Q * PL, C::LD, tid, nthr);
  }
  csync<C>();
}

// Volume term: D = Sum_r d/dxi_r (metric_r . F(U)) for every field.
// With at most one point per thread the physical fluxes stay in registers
// across the DIM passes; otherwise they are re-evaluated per pass.
template <class C, int PHYS>
__device__ __forceinline__ void volume(const Smem<C> &sm, double gamma_, int tid) {
  using T = typename C::R;
  constexpr int DIM = C::DIM, NF = C::NF, Q = C::Q, QD = C::QD, NB = C::EPB * C::NF;
  constexpr bool ONE = C::EPB * QD <= C::NT;
  const T gamma = T(gamma_);
  T F[3][5];
  if constexpr (ONE) {
    if (tid < C::EPB * QD) {
      const int slot = tid / QD, p = tid - slot * QD;
      T U[5];
#pragma unroll
      for (int n = 0; n < NF; ++n) U[n] = sm.B[(slot * NF + n) * QD + p];
      if constexpr (C::MIXED) volume_flux_pert<PHYS, T>(sm.ref[slot], U, gamma, F);
      else volume_flux<PHYS, T>(U, gamma, F);
    }
  }
#pragma unroll
  for (int r = 0; r < DIM; ++r) {
    for (int w = tid; w < C::EPB * QD; w += C::NT) {
      const int slot = w / QD, p = w - slot * QD;
      if constexpr (!ONE) {
        T U[5];
#pragma unroll
        for (int n = 0; n < NF; ++n) U[n] = sm.B[(slot * NF + n) * QD + p];
        if constexpr (C::MIXED) volume_flux_pert<PHYS, T>(sm.ref[slot], U, gamma, F);
        else volume_flux<PHYS, T>(U, gamma, F);
      }
      const double *met = sm.geo[slot].metric;
#pragma unroll
      for (int n = 0; n < NF; ++n) {
        T g = T(met[3 * r + 0]) * F[0][n];
        g = fma(T(met[3 * r + 1]), F[1][n], g);
        if (DIM == 3) g = fma(T(met[3 * r + 2]), F[2][n], g);
        sm.C[(slot * NF + n) * QD + p] = g;
      }
    }
    csync<C>();
    using Sh = Sh3<DIM, Q>;
    if (r == 0) contract<Sh::a, Sh::b, Sh::c, 0, Q, Q, MatD<C::L, Q, T>, false, typename C::R, -1, -1, -1, -1, C::FPT>(sm.C, sm.D, NB, QD, QD, tid, C::NT);
    else if (r == 1) contract<Sh::a, Sh::b, Sh::c, 1, Q, Q, MatD<C::L, Q, T>, true, typename C::R, -1, -1, -1, -1, C::FPT>(sm.C, sm.D, NB, QD, QD, tid, C::NT);
    else contract<Sh::a, Sh::b, Sh::c, 2, Q, Q, MatD<C::L, Q, T>, true, typename C::R, -1, -1, -1, -1, C::FPT>(sm.C, sm.D, NB, QD, QD, tid, C::NT);
    csync<C>();
  }
}

// Trace buffers and the second register are FP32 in the mixed form.
template <class C>
__device__ __forceinline__ const typename C::R *trace_in(const StageArgs &a) {
  if constexpr (C::MIXED) return a.Tinf; else return a.Tin;
}
template <class C>
__device__ __forceinline__ typename C::R *trace_out(const StageArgs &a) {
  if constexpr (C::MIXED) return a.Toutf; else return a.Tout;
}

// Numerical flux on all face points; E holds own traces on entry and
// (F^ - F).J on exit.  Neighbour traces come from Tin.
// Ghost state of a boundary side from the side's own state Uo and outward
// unit normal n (Domain::enforce_bc looping BC::apply).  `viscous` selects
// the database: Navier_Stokes3d keeps its own beside the Domain's
// (src/Navier_Stokes3d.hpp:83) and Euler3d::convection reads the Domain's
// (src/Euler3d.cpp:476), where every "*wall*" code is Euler3d::WallBC; the
// 2-D inviscid flux calls the virtual enforce_bc (src/Euler.cpp:313-316) and
// sees the physics' own database.
//   slip wall          m -> m - (m.n) n, energy with the new kinetic energy
//                      (src/Euler3d.cpp:875-903, src/EulerBC.hpp:43-62)
//   isothermal wall    (r, 0, [0,] 0, (Eref - 1/2) r Tw), par = (Tw, Eref)
//                      (src/Navier_Stokes3d.cpp:472-494, src/Navier_StokesBC.hpp:47-65)
//   state              par (StateBC::apply, src/BC.cpp:17-28)
//   subsonic outflow   r, m kept, pressure of Mach par[0] (src/EulerBC.hpp:138-167)
//   supersonic outflow the own state (src/EulerBC.hpp:214-241)
template <int DIM, int NF>
__device__ __forceinline__ void ghost_state(int kind, const double *par, const double *Uo, const double *n,
                                            bool viscous, double *Un) {
  if constexpr (NF == 3) {   // shallow water: Shallow::WallBC (src/ShallowBC.hpp:45-61)
    Un[0] = Uo[0];
    Un[1] = (Uo[1] * n[1] - Uo[2] * n[0]) * n[1];
    Un[2] = (Uo[2] * n[0] - Uo[1] * n[1]) * n[0];
    return;
  }
  if (kind == DGMX_BC_STATE) {
#pragma unroll
    for (int k = 0; k < NF; ++k) Un[k] = par[k];
  } else if (kind == DGMX_BC_SUPERSONIC_OUTFLOW) {
#pragma unroll
    for (int k = 0; k < NF; ++k) Un[k] = Uo[k];
  } else if (kind == DGMX_BC_SUBSONIC_OUTFLOW && DIM == 2) {
    const double gam = 1.4, Mref = par[0];
    const double Eref = 1.0 / (gam * (gam - 1.0) * (Mref * Mref)) + 0.5;
    const double pref = (gam - 1.0) * (Eref - 0.5 * (1.0 - 0.0));
    const double rl = Uo[0], ml = Uo[1], nl = Uo[2];
    const double ul = ml / rl, vl = nl / rl;
    Un[0] = rl; Un[1] = ml; Un[2] = nl;
    Un[3] = pref / (gam - 1.0) + 0.5 * (ml * ul + nl * vl);
  } else if (kind == DGMX_BC_ISOTHERMAL_WALL && (viscous || DIM == 2)) {
    Un[0] = Uo[0];
#pragma unroll
    for (int k = 1; k < NF - 1; ++k) Un[k] = 0.0;
    Un[NF - 1] = (par[1] - 0.5) * Uo[0] * par[0];
  } else if constexpr (DIM == 3) {   // slip wall (and the 3-D isothermal wall's inviscid side)
    double up = Uo[1], vp = Uo[2], wp = Uo[3];
    const double dot = up * n[0] + vp * n[1] + wp * n[2];
    up = up - dot * n[0]; vp = vp - dot * n[1]; wp = wp - dot * n[2];
    Un[0] = Uo[0]; Un[1] = up; Un[2] = vp; Un[3] = wp;
    Un[4] = Uo[4] - 0.5 * (Uo[1] * Uo[1] + Uo[2] * Uo[2] + Uo[3] * Uo[3]) / Uo[0] +
            0.5 * (up * up + vp * vp + wp * wp) / Un[0];
  } else {
    Un[0] = Uo[0];
    Un[1] = (Uo[1] * n[1] - Uo[2] * n[0]) * n[1];
    Un[2] = (Uo[2] * n[0] - Uo[1] * n[1]) * n[0];
    Un[3] = Uo[3] - 0.5 * (Uo[1] * Uo[1] + Uo[2] * Uo[2]) / Uo[0] + 0.5 * (Un[1] * Un[1] + Un[2] * Un[2]) / Un[0];
  }
}

template <class C, int PHYS>
__device__ __forceinline__ void face_fluxes(const Smem<C> &sm, const StageArgs &a, int tid) {
  using T = typename C::R;
  constexpr int NF = C::NF, GF = C::GF, NFACE = C::NFACE, EPB = C::EPB;
  const T *Tin = trace_in<C>(a);
  for (int w = tid; w < NFACE * EPB * GF; w += C::NT) {
    const int f = w / (EPB * GF), rem = w - f * EPB * GF, slot = rem / GF, g = rem - slot * GF;
    const int e = sm.eid[slot];
    if (e < 0) continue;
    const FaceLink lk = sm.lnk[slot * NFACE + f];
    const GeomClass &gc = sm.geo[slot];
    const int gn = a.perm[lk.perm + g];
    T Uo[5], Un[5], Fh[5], FL[5], FR[5];
    constexpr int EB = C::EB;
    T *eo = sm.E + ((f * EPB + slot) * NF) * EB + epos<C>(g);
    const T *tn = Tin + ((size_t)(lk.elem * NFACE + lk.face) * NF) * GF + gn;
    const T nm[3] = {T(gc.nrm[f][0]), T(gc.nrm[f][1]), T(gc.nrm[f][2])};
#pragma unroll
    for (int n = 0; n < NF; ++n) { Uo[n] = eo[n * EB]; Un[n] = tn[n * GF]; }
    const int bt = (gc.bc >> (4 * f)) & 15;
    if constexpr (!C::MIXED) {
      // boundary side: the neighbour is the ghost state of the database the
      // inviscid flux reads (see ghost_state)
      if (bt) ghost_state<C::DIM, C::NF>(a.bckind[bt], a.bcpar[bt], Uo, nm, false, Un);
    }
    const bool master = (gc.master >> f) & 1;
    const T jr = T(gc.jr[f]);
    bool ok;
    if constexpr (C::MIXED) {
      // traces are perturbations about the solve's reference state
      // (Fh - FL = Dm, FR - Fh = DF - Dm)
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
    if constexpr (PHYS == DGMX_NS2D || PHYS == DGMX_NS3D) {
      // BR1 viscous lift: '-' average of the viscous normal-flux traces in
      // the master frame (src/Domain.cpp:1883-1937), subtracted like
      // scale(-1, Uv); Ur += Uv (src/Navier_Stokes3d.cpp:377-390)
      // a boundary side's ghost flux is -Vo (isothermal wall apply_flux,
      // src/Navier_Stokes3d.cpp:496-513), so the average is Vo and the
      // lift term vanishes
      const double *vo = a.V + ((size_t)(e * NFACE + f) * (NF - 1)) * GF + g;
      const double *vn = a.V + ((size_t)(lk.elem * NFACE + lk.face) * (NF - 1)) * GF + gn;
      if (!bt)
#pragma unroll
        for (int n = 1; n < NF; ++n) {
          const double Vo = vo[(n - 1) * GF], Vn = vn[(n - 1) * GF];
          const double fs = master ? 0.5 * (Vo - Vn) : -(0.5 * (Vn - Vo));
          eo[n * EB] = eo[n * EB] - (fs - Vo) * jr;
        }
    }
    if (!ok) {
      atomicOr(a.err, 1);
      atomicMin(a.err + 1, e);
    }
  }
  csync<C>();
}

// One face of the lift: G2GL (second pass in 3-D) straight into the face
// plane of D, scaled by 1/w_end (src/Hex.cpp:1942-1947).  Face plane (x, y)
// -> D offset OFF + x OX + y OY.
template <class C, int F>
__device__ __forceinline__ void lift_face(const Smem<C> &sm, int tid) {
  using T = typename C::R;
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q, G = C::G, FB = C::EPB * C::NF, QD = C::QD, PG = C::PG;
  constexpr int END = face_end<DIM>(F);
  if constexpr (DIM == 3) {
    // 0 k=0 (i,j), 1 j=0 (i,k), 2 i=Q-1 (j,k), 3 j=Q-1 (i,k), 4 i=0 (j,k), 5 k=Q-1 (i,j)
    constexpr int OX = (F == 2 || F == 4) ? Q : Q * Q;
    constexpr int OY = (F == 0 || F == 5) ? Q : 1;
    constexpr int OFF = F == 2 ? (Q - 1) * Q * Q : (F == 3 ? (Q - 1) * Q : (F == 5 ? Q - 1 : 0));
    contract<Q, G, 1, 1, G, Q, MatG2GLw<L, Q, END, T>, true, T, PG, 1, OX, OY, C::FPT>(
        sm.S + F * FB * Q * PG, sm.D + OFF, FB, Q * PG, QD, tid, C::NT);
  } else {
    // 0 j=0 (i), 1 i=Q-1 (j), 2 j=Q-1 (i), 3 i=0 (j)
    constexpr int OX = (F == 0 || F == 2) ? Q : 1;
    constexpr int OFF = F == 1 ? (Q - 1) * Q : (F == 2 ? Q - 1 : 0);
    contract<G, 1, 1, 0, G, Q, MatG2GLw<L, Q, END, T>, true, T, -1, -1, OX, 1, C::FPT>(
        sm.E + F * FB * C::EB, sm.D + OFF, FB, C::EB, QD, tid, C::NT);
  }
}

// Lift: the face terms E (Gauss points) are interpolated to the face GLL
// points and added to the boundary points of D (src/Hex.cpp:1768-1952,
// src/Quad.cpp:1971-2038).  The two faces normal to one axis touch disjoint
// points and go together; the axes follow one another.  The quadrature
// weights of the projection are in the forward transform.
template <class C>
__device__ __forceinline__ void lift(const Smem<C> &sm, int tid) {
  using T = typename C::R;
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q, G = C::G, PG = C::PG;
  constexpr int NB = C::NFACE * C::EPB * C::NF;
  if constexpr (DIM == 3) {
    contract<G, G, 1, 0, G, Q, MatG2GL<L, Q, T>, false, T, PG, 1, PG, 1, C::FPT>(sm.E, sm.S, NB, C::EB, Q * PG,
                                                                                tid, C::NT);
    csync<C>();
    lift_face<C, 2>(sm, tid);
    lift_face<C, 4>(sm, tid);
    csync<C>();
    lift_face<C, 1>(sm, tid);
    lift_face<C, 3>(sm, tid);
    csync<C>();
    lift_face<C, 0>(sm, tid);
    lift_face<C, 5>(sm, tid);
  } else {
    lift_face<C, 1>(sm, tid);
    lift_face<C, 3>(sm, tid);
    csync<C>();
    lift_face<C, 0>(sm, tid);
    lift_face<C, 2>(sm, tid);
  }
  csync<C>();
}

// Solve (reference-state row) of element e; 0 for a single-solve domain.
__device__ __forceinline__ int solve_of(const StageArgs &a, int e) {
  return (e >= 0 && a.esolve) ? a.esolve[e] : 0;
}

template <class C>
__device__ __forceinline__ void load_geometry(const Smem<C> &sm, const StageArgs &a, int e0, int tid) {
  // the geometry class is copied word by word by the whole team
  constexpr int GW = (int)(sizeof(GeomClass) / sizeof(double));
  static_assert(sizeof(GeomClass) % sizeof(double) == 0, "GeomClass is copied as doubles");
  for (int k = tid; k < C::EPB * GW; k += C::NT) {
    const int s = k / GW, j = k - s * GW, e = e0 + s;
    // elements past the end, and unallocated pool elements (class < 0),
    // are skipped
    const int gc = e < a.ne ? a.gclass[e] : -1;
    reinterpret_cast<double *>(sm.geo + s)[j] = reinterpret_cast<const double *>(a.classes + (gc >= 0 ? gc : 0))[j];
    if (j == 0) {
      sm.eid[s] = gc >= 0 ? e : -1;
      if constexpr (C::MIXED)
        sm.ref[s] = *reinterpret_cast<const RefState<float> *>(a.uref + kUrefStride * solve_of(a, gc >= 0 ? e : -1) + 10);
    }
  }
  for (int w = tid; w < C::EPB * C::NFACE; w += C::NT) {
    const int s = w / C::NFACE, f = w - s * C::NFACE, e = e0 + s;
    sm.lnk[w] = e < a.ne ? a.links[(size_t)e * C::NFACE + f] : FaceLink{0, 0, 0, 0};
  }
}

// Element-major modal register block of the slot's element: NF*LD doubles.
template <class C, class S>
__device__ __forceinline__ void load_modal(typename C::R *dst, const S *src, int e0, int ne, int tid) {
  using T = typename C::R;
  constexpr int BLK = C::NF * C::LD;
  for (int w = tid; w < C::EPB * BLK; w += C::NT) {
    const int s = w / BLK, e = e0 + s;
    dst[w] = e < ne ? T(src[(size_t)e0 * BLK + w]) : T(w % C::LD == 0 ? 1.0 : 0.0);
  }
}

// Row copies: N values of S between memory and registers, as 16-byte
// vectors when a row is a whole number of them (rows are then 16-byte
// aligned, as every row of these arrays starts at a multiple of its size).
template <int N, class S>
__device__ __forceinline__ void ld_row(const S *p, S (&v)[N]) {
  if constexpr ((N * sizeof(S)) % 16 == 0) {
    constexpr int V = 16 / (int)sizeof(S);
#pragma unroll
    for (int k = 0; k < N / V; ++k) {
      const uint4 q = reinterpret_cast<const uint4 *>(p)[k];
      S t[V];
      __builtin_memcpy(t, &q, 16);
#pragma unroll
      for (int j = 0; j < V; ++j) v[k * V + j] = t[j];
    }
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = p[k];
  }
}
template <int N, class S>
__device__ __forceinline__ void st_row(S *p, const S (&v)[N]) {
  if constexpr ((N * sizeof(S)) % 16 == 0) {
    constexpr int V = 16 / (int)sizeof(S);
#pragma unroll
    for (int k = 0; k < N / V; ++k) {
      S t[V];
#pragma unroll
      for (int j = 0; j < V; ++j) t[j] = v[k * V + j];
      uint4 q;
      __builtin_memcpy(&q, t, 16);
      reinterpret_cast<uint4 *>(p)[k] = q;
    }
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) p[k] = v[k];
  }
}

// The modal register into the padded modal block, a row of L values per
// thread (row r of the tile lands at r * PL).  Rows of elements past the end
// get the constant state 1 (their results are discarded).
template <class C, class S>
__device__ __forceinline__ void load_modal_pad(typename C::R *dst, const S *src, int e0, int ne, int tid) {
  using T = typename C::R;
  constexpr int L = C::L, RPF = C::LD / L, RPS = C::NF * RPF;
  for (int r = tid; r < C::EPB * RPS; r += C::NT) {
    const int e = e0 + r / RPS;
    S v[L];
    if (e < ne) {
      ld_row<L>(src + ((size_t)e0 * RPS + r) * L, v);
    } else {
#pragma unroll
      for (int k = 0; k < L; ++k) v[k] = S(k == 0 && r % RPF == 0 ? 1.0 : 0.0);
    }
#pragma unroll
    for (int k = 0; k < L; ++k) dst[r * C::PL + k] = T(v[k]);
  }
}

// Mixed form: the FP32 working copy of a modal register is the perturbation
// about the solve's reference state, formed in FP64 (only the constant mode
// carries the reference: row[5 + n] of the solve's reference row).
template <class C>
__device__ __forceinline__ void load_modal_pert(float *dst, const double *src, const StageArgs &a, int e0,
                                                int tid) {
  constexpr int L = C::L, RPF = C::LD / L, RPS = C::NF * RPF;
  for (int r = tid; r < C::EPB * RPS; r += C::NT) {
    const int s = r / RPS, e = e0 + s;
    double v[L];
    if (e < a.ne) {
      ld_row<L>(src + ((size_t)e0 * RPS + r) * L, v);
      if (r % RPF == 0) v[0] -= a.uref[kUrefStride * solve_of(a, e) + 5 + (r - s * RPS) / RPF];
    } else {
#pragma unroll
      for (int k = 0; k < L; ++k) v[k] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < L; ++k) dst[r * C::PL + k] = float(v[k]);
  }
}

// Traces: global [e][f][n][g] <-> shared face-major [f][slot][n][padded g],
// a row of G values per thread (a face block holds GF / G rows).
template <class C, class TT>
__device__ __forceinline__ void store_traces(const typename C::R *E, TT *T, int e0, int ne, int tid) {
  constexpr int NF = C::NF, GF = C::GF, G = C::G, NFACE = C::NFACE, EPB = C::EPB;
  constexpr int RPF = GF / G, RPS = NFACE * NF * RPF;
  for (int r = tid; r < EPB * RPS; r += C::NT) {
    const int s = r / RPS, rr = r - s * RPS, fn = rr / RPF, g1 = rr - fn * RPF, f = fn / NF, n = fn - f * NF;
    const int e = e0 + s;
    if (e >= ne) continue;
    const typename C::R *src = E + ((f * EPB + s) * NF + n) * C::EB + g1 * C::PG;
    TT v[G];
#pragma unroll
    for (int k = 0; k < G; ++k) v[k] = TT(src[k]);
    st_row<G>(T + (size_t)e * NFACE * NF * GF + rr * G, v);
  }
}

// The element's own traces, written by the previous stage (or the trace
// kernel), into padded blocks (PAD) or dense ones [f][slot][n][g].
template <class C, class TT, bool PAD = true>
__device__ __forceinline__ void load_own_traces(typename C::R *E, const TT *T, int e0, int ne, int tid) {
  using R = typename C::R;
  constexpr int NF = C::NF, GF = C::GF, G = C::G, NFACE = C::NFACE, EPB = C::EPB;
  if constexpr (PAD) {
    constexpr int RPF = GF / G, RPS = NFACE * NF * RPF;
    for (int r = tid; r < EPB * RPS; r += C::NT) {
      const int s = r / RPS, rr = r - s * RPS, fn = rr / RPF, g1 = rr - fn * RPF, f = fn / NF, n = fn - f * NF;
      const int e = e0 + s;
      TT v[G];
      if (e < ne) {
        ld_row<G>(T + (size_t)e * NFACE * NF * GF + rr * G, v);
      } else {
#pragma unroll
        for (int k = 0; k < G; ++k) v[k] = TT(n == 0 ? 1.0 : 0.0);
      }
      R *dst = E + ((f * EPB + s) * NF + n) * C::EB + g1 * C::PG;
#pragma unroll
      for (int k = 0; k < G; ++k) dst[k] = R(v[k]);
    }
  } else {
    for (int w = tid; w < EPB * NFACE * NF * GF; w += C::NT) {
      const int s = w / (NFACE * NF * GF), rem = w - s * NFACE * NF * GF;
      const int f = rem / (NF * GF), ng = rem - f * NF * GF;
      const int e = e0 + s;
      E[(f * EPB + s) * NF * GF + ng] = e < ne ? R(T[(size_t)e * NFACE * NF * GF + rem]) : R(ng < GF ? 1.0 : 0.0);
    }
  }
}

// ---------------------------------------------------------------- kernels
// One fused RK stage on the EPB elements from e0, run by the CTA.
template <class C, int PHYS>
__device__ __forceinline__ void stage_tile(const Smem<C> &sm, const StageArgs &a, int e0, int tid) {
  load_geometry<C>(sm, a, e0, tid);
  if constexpr (C::MIXED) load_modal_pert<C>(sm.A, a.X, a, e0, tid);
  else load_modal_pad<C>(sm.A, a.X, e0, a.ne, tid);
  load_own_traces<C>(sm.E, trace_in<C>(a), e0, a.ne, tid);
  csync<C>();
  backward<C>(sm.A, sm.B, sm.S, sm.C, tid, C::NT);
  volume<C, PHYS>(sm, a.gamma, tid);
  face_fluxes<C, PHYS>(sm, a, tid);
  lift<C>(sm, tid);
  forward<C>(sm.D, sm.R, sm.C, sm.B, tid, C::NT);
  // RK stage update on the modal registers, a row of L modes per thread
  constexpr int L = C::L, RPF = C::LD / L, RPS = C::NF * RPF;
  for (int r = tid; r < C::EPB * RPS; r += C::NT) {
    const int s = r / RPS, e = e0 + s;
    if (sm.eid[s] < 0) continue;
    const int n = (r - s * RPS) / RPF, m0 = (r % RPF) * L;   // field, first mode of the row
    const size_t gi = ((size_t)e0 * RPS + r) * L;
    const double dt = a.dts ? a.dts[solve_of(a, e)] : a.dt;   // per-solve step (pools)
    typename C::R *Ar = sm.A + r * C::PL;
    const typename C::R *Rr = sm.R + r * L;
    if constexpr (C::MIXED) {
      // FP32 right-hand side and second register, FP64 solution register:
      // Ut = A Ut - dt R in FP32; U = U + B Ut accumulated in FP64.
      float rr[L];
#pragma unroll
      for (int k = 0; k < L; ++k) rr[k] = Rr[k];
      if (a.Ssrc)
#pragma unroll
        for (int k = 0; k < L; ++k) rr[k] -= float(a.src_scale * a.Ssrc[gi + k]);
      if (a.Rsub)
#pragma unroll
        for (int k = 0; k < L; ++k) rr[k] -= float(a.Rsub[gi + k]);
      if (a.kind == kRHS) {
#pragma unroll
        for (int k = 0; k < L; ++k) a.A[gi + k] = rr[k];
        continue;
      }
      float ut[L];
      double u[L];
      ld_row<L>(a.Utf + gi, ut);
      ld_row<L>(a.U + gi, u);
      const float c0 = float(a.c0), mdt = -float(dt);
#pragma unroll
      for (int k = 0; k < L; ++k) {
        ut[k] = fmaf(mdt, rr[k], c0 * ut[k]);
        u[k] = fma(a.c1, double(ut[k]), u[k]);
      }
      st_row<L>(a.Utf + gi, ut);
      st_row<L>(a.U + gi, u);
      const double ref0 = m0 == 0 ? a.uref[kUrefStride * solve_of(a, e) + 5 + n] : 0.0;
#pragma unroll
      for (int k = 0; k < L; ++k) Ar[k] = float(k == 0 ? u[k] - ref0 : u[k]);
    } else {
      double rr[L];
#pragma unroll
      for (int k = 0; k < L; ++k) rr[k] = Rr[k];
      if (a.Ssrc)
#pragma unroll
        for (int k = 0; k < L; ++k) rr[k] -= a.src_scale * a.Ssrc[gi + k];
      if (a.Rcap)   // first RHS (shallow-water balance)
#pragma unroll
        for (int k = 0; k < L; ++k) a.Rcap[gi + k] = rr[k];
      if (a.Rsub)
#pragma unroll
        for (int k = 0; k < L; ++k) rr[k] -= a.Rsub[gi + k];
      if constexpr (PHYS == DGMX_NS2D || PHYS == DGMX_NS3D) {
        if (n >= 1)
#pragma unroll
          for (int k = 0; k < L; ++k) rr[k] -= a.Pv[((size_t)e * (C::NF - 1) + (n - 1)) * C::LD + m0 + k];
      }
      if (a.R0 && m0 == 0) a.R0[(size_t)e * C::NF + n] = rr[0];   // bulk-flow hold
      if (a.kind == kLSRK) {
        double ut[L], u[L];
        ld_row<L>(a.Ut + gi, ut);
#pragma unroll
        for (int k = 0; k < L; ++k) {
          ut[k] = fma(-dt, rr[k], a.c0 * ut[k]);
          u[k] = fma(a.c1, ut[k], Ar[k]);
          Ar[k] = u[k];
        }
        st_row<L>(a.Ut + gi, ut);
        st_row<L>(a.U + gi, u);
        continue;
      }
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const size_t g = gi + k;
        const double x = Ar[k], q = rr[k];
        double next;
        switch (a.kind) {
          case kTVD0: {
            const double ut = fma(-dt, q, x);
            a.Ut[g] = ut; next = ut;
            break;
          }
          case kTVD1: {
            const double t = fma(-dt, q, x);
            double ut = a.c1 * t;
            ut = fma(a.c0, a.U[g], ut);
            a.Ut[g] = ut; next = ut;
            break;
          }
          case kTVD2: {
            const double t = fma(-dt, q, x);
            double u = a.c0 * a.U[g];
            u = fma(a.c1, t, u);
            a.U[g] = u; next = u;
            break;
          }
          case kRK40: {
            const double ut = fma(a.c0, q, x);
            a.Ut[g] = ut; a.A[g] = a.c1 * q; next = ut;
            break;
          }
          case kRK41: {
            const double ut = fma(a.c0, q, a.U[g]);
            a.A[g] = fma(a.c1, q, a.A[g]);
            a.Ut[g] = ut; next = ut;
            break;
          }
          case kRHS: {
            a.A[g] = q; next = x;
            break;
          }
          default: {  // kRK43
            const double acc = fma(a.c1, q, a.A[g]);
            const double u = fma(a.c0, acc, a.U[g]);
            a.U[g] = u; next = u;
            break;
          }
        }
        Ar[k] = next;
      }
    }
  }
  csync<C>();
  modal_traces<C>(sm.A, sm.E, sm.S, sm.B, tid, C::NT);
  store_traces<C>(sm.E, trace_out<C>(a), e0, a.ne, tid);
}

// One tile per CTA, or, with a tile list (element pools), a persistent loop
// over the listed tiles; the count is read on the device so a captured
// graph stays valid while solves join and leave.
template <class C, int PHYS>
__global__ void __launch_bounds__(C::NT, C::MINB) stage_kernel(StageArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<C> sm(smem_raw);
  const int ntile = a.tiles ? *a.ntiles : (int)gridDim.x;
  for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
    if (t != (int)blockIdx.x) __syncthreads();
    stage_tile<C, PHYS>(sm, a, (a.tiles ? a.tiles[t] : t) * C::EPB, threadIdx.x);
  }
}


// Traces of a modal register (start of a run, after set_state).
template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB) traces_modal_kernel(StageArgs a, const double *Xm, typename C::R *T) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<C> sm(smem_raw);
  const int tid = threadIdx.x, e0 = blockIdx.x * C::EPB;
  if constexpr (C::MIXED) load_modal_pert<C>(sm.A, Xm, a, e0, tid);
  else load_modal_pad<C>(sm.A, Xm, e0, a.ne, tid);
  csync<C>();
  modal_traces<C>(sm.A, sm.E, sm.S, sm.B, tid, C::NT);
  store_traces<C>(sm.E, T, e0, a.ne, tid);
}

// Load GLL values from Field layout [n][e][QD] into B.
template <class C>
__device__ __forceinline__ void load_nodal(double *B, const double *Xn, int e0, int ne, int tid) {
  constexpr int NF = C::NF, QD = C::QD;
  for (int w = tid; w < C::EPB * NF * QD; w += C::NT) {
    const int s = w / (NF * QD), rem = w - s * NF * QD, n = rem / QD, p = rem - n * QD;
    const int e = e0 + s;
    B[w] = e < ne ? Xn[((size_t)n * ne + e) * QD + p] : (n == 0 ? 1.0 : 0.0);
  }
}

// GL2G traces of GLL values (fill_sides, src/Hex.cpp:933-947,
// src/Quad.cpp:884-905) for the Domain::time_derivative path.
template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB) traces_nodal_kernel(StageArgs a) {
  using T = typename C::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<C> sm(smem_raw);
  constexpr int DIM = C::DIM, L = C::L, Q = C::Q, G = C::G, NF = C::NF, EPB = C::EPB, QD = C::QD, QF = C::QF;
  const int tid = threadIdx.x, e0 = blockIdx.x * EPB;
  load_nodal<C>(sm.B, a.Xn, e0, a.ne, tid);
  csync<C>();
  // gather face GLL values, face-major [f][slot][n][QF]
  for (int w = tid; w < C::NFACE * EPB * NF * QF; w += C::NT) {
    const int f = w / (EPB * NF * QF), rem = w - f * EPB * NF * QF;
    const int sn = rem / QF, x = rem - sn * QF;
    const double *src = sm.B + sn * QD;
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
    sm.C[w] = src[p];
  }
  csync<C>();
  constexpr int NB = C::NFACE * EPB * NF;
  if constexpr (DIM == 3) {
    contract<Q, Q, 1, 0, Q, G, MatGL2G<L, Q, T>, false, typename C::R, -1, -1, -1, -1, C::FPT>(sm.C, sm.S, NB, Q * Q, G * Q, tid, C::NT);
    csync<C>();
    contract<G, Q, 1, 1, Q, G, MatGL2G<L, Q, T>, false, T, -1, -1, C::PG, 1, C::FPT>(sm.S, sm.E, NB, G * Q, C::EB, tid,
                                                                             C::NT);
  } else {
    contract<Q, 1, 1, 0, Q, G, MatGL2G<L, Q, T>, false, typename C::R, -1, -1, -1, -1, C::FPT>(sm.C, sm.E, NB, Q, C::EB, tid, C::NT);
  }
  csync<C>();
  store_traces<C>(sm.E, a.Tout, e0, a.ne, tid);
}

// Domain::time_derivative on GLL values: F = -dU/dt at GLL points (projected).
template <class C, int PHYS>
__global__ void __launch_bounds__(C::NT, C::MINB) rhs_nodal_kernel(StageArgs a) {
  using T = typename C::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<C> sm(smem_raw);
  constexpr int NF = C::NF, QD = C::QD, GF = C::GF, NFACE = C::NFACE, EPB = C::EPB;
  const int tid = threadIdx.x, e0 = blockIdx.x * EPB;
  load_geometry<C>(sm, a, e0, tid);
  load_nodal<C>(sm.B, a.Xn, e0, a.ne, tid);
  // own traces from Tin (written by traces_nodal_kernel)
  load_own_traces<C>(sm.E, a.Tin, e0, a.ne, tid);
  csync<C>();
  volume<C, PHYS>(sm, a.gamma, tid);
  face_fluxes<C, PHYS>(sm, a, tid);
  lift<C>(sm, tid);
  forward<C>(sm.D, sm.R, sm.C, sm.B, tid, C::NT);
  if constexpr (PHYS == DGMX_NS2D || PHYS == DGMX_NS3D) {
    constexpr int BLK = NF * C::LD;
    for (int w = tid; w < EPB * BLK; w += C::NT) {
      const int e = e0 + w / BLK, n = (w % BLK) / C::LD, m = w % C::LD;
      if (e < a.ne && n >= 1) sm.R[w] = sm.R[w] - a.Pv[((size_t)e * (NF - 1) + (n - 1)) * C::LD + m];
    }
    csync<C>();
  }
  if (a.Ssrc || a.Rcap || a.Rsub) {
    constexpr int BLK = NF * C::LD;
    for (int w = tid; w < EPB * BLK; w += C::NT) {
      const int e = e0 + w / BLK;
      if (e >= a.ne) continue;
      const size_t gi = (size_t)e0 * BLK + w;
      if (a.Ssrc) sm.R[w] = sm.R[w] - a.src_scale * a.Ssrc[gi];
      if (a.Rcap) a.Rcap[gi] = sm.R[w];
      if (a.Rsub) sm.R[w] = sm.R[w] - a.Rsub[gi];
    }
    csync<C>();
  }
  if (a.R0) {   // bulk-flow hold: constant coefficients of the projected RHS
    for (int w = tid; w < EPB * NF; w += C::NT) {
      const int e = e0 + w / NF;
      if (e < a.ne) a.R0[(size_t)e * NF + w % NF] = sm.R[(w / NF) * NF * C::LD + (w % NF) * C::LD];
    }
    csync<C>();
  }
  backward<C, false>(sm.R, sm.B, sm.S, sm.C, tid, C::NT);
  for (int w = tid; w < EPB * NF * QD; w += C::NT) {
    const int s = w / (NF * QD), rem = w - s * NF * QD, n = rem / QD, p = rem - n * QD;
    const int e = e0 + s;
    if (e < a.ne) a.Fn[((size_t)n * a.ne + e) * QD + p] = sm.B[w];
  }
}

// GLL values (Field layout) -> projected modal register (element-major).
template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB) forward_kernel(StageArgs a, const double *Un, double *Um) {
  using T = typename C::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<C> sm(smem_raw);
  constexpr int L = C::L, Q = C::Q, NF = C::NF, QD = C::QD, EPB = C::EPB;
  const int tid = threadIdx.x, e0 = blockIdx.x * EPB;
  load_nodal<C>(sm.D, Un, e0, a.ne, tid);
  csync<C>();
  forward<C>(sm.D, sm.R, sm.C, sm.B, tid, C::NT);
  constexpr int BLK = NF * C::LD;
  for (int w = tid; w < EPB * BLK; w += C::NT) {
    const int e = e0 + w / BLK;
    if (e < a.ne) Um[(size_t)e0 * BLK + w] = sm.R[w];
  }
}

// Modal register -> GLL values (Field layout).
template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB) backward_kernel(StageArgs a, const double *Um, double *Un) {
  using T = typename C::R;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem<C> sm(smem_raw);
  constexpr int NF = C::NF, QD = C::QD, EPB = C::EPB;
  const int tid = threadIdx.x, e0 = blockIdx.x * EPB;
  load_modal<C>(sm.A, Um, e0, a.ne, tid);
  csync<C>();
  backward<C, false>(sm.A, sm.B, sm.S, sm.C, tid, C::NT);
  for (int w = tid; w < EPB * NF * QD; w += C::NT) {
    const int s = w / (NF * QD), rem = w - s * NF * QD, n = rem / QD, p = rem - n * QD;
    const int e = e0 + s;
    if (e < a.ne) Un[((size_t)n * a.ne + e) * QD + p] = sm.B[w];
  }
}

}  // namespace dgmx
