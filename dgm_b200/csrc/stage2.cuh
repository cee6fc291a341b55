// Fused DG stage kernel, second form (3-D hexahedra, sm_100a), FP64 and the
// mixed FP32 form.
//
// Same arithmetic contract as stage_tile (stage.cuh): one launch evaluates
// Domain::time_derivative on the modal register, applies the LSRK stage
// update (or stores the right-hand side) and writes the next stage's face
// traces.  What differs is how the element's operators are ordered, so that
// every 1-D contraction reads and writes shared memory once and the number
// of passes (and barriers) per element is small:
//
//  * the projected volume term of the reference, forward(sum_r D_r G_r) with
//    G_r the contravariant flux (src/Euler3d.cpp:506-566 differentiated by
//    src/Hex.cpp:2030-2071 and projected by src/Hex.cpp:703-812), is one
//    sum-factorised operator: along its own axis r the weighted derivative
//    E = B W D (L x Q), along the other two the weighted basis P = B W, and
//    the three directions share passes:
//        R = P_k P_j (E_i G_0) + P_k E_j (P_i G_1) + E_k P_j (P_i G_2);
//    the i-axis pass runs in registers right after the pointwise fluxes
//    (one thread per (j, k) column and direction r);
//  * the lift of a face (G2GL interpolation, 1/w_end and the projection,
//    src/Hex.cpp:1768-1952) is the 2-D projection BwG x BwG of the face
//    term times the end value of the normal-axis basis, BwG = B W G2GL, and
//    is added to the projected right-hand side in the last pass;
//  * the update writes each modal row from registers and the next traces
//    (modal -> face Gauss points, src/Hex.cpp:933-947) start from the same
//    registers (end reduction along the contiguous axis);
//  * what only one thread consumes is read from global memory by that
//    thread (the face traces by the face-point threads, the modal rows by
//    the first backward pass), so shared memory carries only the
//    intermediates that change hands -- its bandwidth, not the FP64 pipe,
//    bounded the first version of this kernel;
//  * independent passes share a barrier interval (nine per element).
// Every (L, Q) works; the element's shared-memory regions are laid out by
// barrier interval (offsets below) with odd pitches on the rows that a warp
// reads along, so pencils fall on distinct banks.
//
// Scope: Euler 3-D, no boundary sides, LSRK and right-hand-side stages (the
// other stage kinds run the plain kernel of the same (L, Q)).
#pragma once

#include "stage.cuh"

namespace dgmx {

// Tables of the second form (constant memory, per working type and (L, Q)).
template <class T, int L, int Q> __constant__ T cE2[L * Q];          // E[a][j] = sum_i B[a][i] w_i D[i][j]
template <class T, int L, int Q> __constant__ T cBwG[L * (Q - 1)];   // BwG[a][g] = sum_i B[a][i] w_i G2GL[i][g]

template <int PHYS, int L_, int Q_, int EPB_, int NT_, int MINB_, bool MIXED_, int VDIRS_ = 0>
struct Cfg2 {
  static constexpr bool MIXED = MIXED_;
  // directions of the volume pass per thread: 1 spreads a column's three
  // directions over three warps, 3 keeps them in one thread (default: FP64
  // 1, FP32 3)
  static constexpr int VDIRS = VDIRS_ > 0 ? VDIRS_ : (MIXED_ ? 3 : 1);
  static_assert(VDIRS == 1 || VDIRS == 3, "the volume pass takes one or all three directions per thread");
  static constexpr int PHYSICS = PHYS;
  using R = std::conditional_t<MIXED_, float, double>;
  static constexpr int NF = phys_nf(PHYS), L = L_, Q = Q_, G = Q_ - 1, EPB = EPB_, NT = NT_;
  static constexpr int MINB = MINB_ > 0 ? MINB_ : 1, MINB_REQ = MINB_;
  static constexpr int NFACE = 6, GF = G * G, LD = L * L * L, QD = Q * Q * Q;
  // odd pitches for rows of an even length
  static constexpr int PL = L % 2 == 0 ? L + 1 : L;   // modal rows (and face-plane rows of L)
  static constexpr int PE = GF % 2 == 0 ? GF + 1 : GF;   // one (face, field) block of face terms
  // block pitches chosen for the passes that read or write across blocks:
  // XLS (one (face, field) block of lifted terms, odd: the lift writes one
  // value per block), FPS (one face plane, = L (mod 16) for L = 4: the
  // trace pass reads column b' of a block, L per block), XJ (one j-plane of
  // X and T2, [n a][k], = Q (mod 16): a pass over (j, k) columns writes or
  // reads Q consecutive k per j)
  static constexpr int XLS = (L * PL) % 2 == 0 ? L * PL + 1 : L * PL;
  static constexpr int FPS = L * PL;
  static constexpr int XJ = NF * L * Q + ((Q - NF * L * Q) % 16 + 16) % 16;
  // region sizes (values of R)
  static constexpr int S_EF = NFACE * NF * PE;          // face terms [f][n][g h], padded blocks
  static constexpr int S_XL = NFACE * NF * XLS;         // lifted-projected face terms [f][n][a'][b'] padded
  static constexpr int S_T1 = NF * L * L * Q;           // [b][n a][k]
  static constexpr int S_T2 = Q * XJ;                   // [j][n a][k], planes of XJ
  static constexpr int S_UN = NF * Q * Q * Q;           // nodal values [n][i][j][k]
  static constexpr int S_X1 = Q * XJ;                   // one of X0, X1, X2: [j][n a][k], planes of XJ
  static constexpr int S_X = 3 * S_X1 + 2;              // (+1 between arrays: they start on different banks)
  static constexpr int S_Y1 = NF * L * L * Q;           // Y0 or Y2: [b][n a][k]
  static constexpr int S_Y = 2 * S_Y1 + 1;
  static constexpr int S_UB = NF * L * L * PL;          // updated modal block, padded rows
  static constexpr int S_FP = NFACE * NF * FPS;         // end-reduced face planes [f][n][a'][b'], blocks of FPS
  static constexpr int S_W1 = NFACE * NF * G * PL;      // trace pass 1 [f][n][g][b'] padded
  // Barrier intervals: 1 face fluxes -> EF, backward k-pass -> T1;
  // 2 lift EF -> XL, j-pass T1 -> T2; 3 i-pass T2 -> UN; 4 volume UN -> X;
  // 5 j-pass X -> Y; 6 k-pass, lift, update Y, XL -> UB, FP; 7 ends UB -> FP;
  // 8 traces FP -> W1; 9 traces W1 -> global.  A region written in one
  // interval may share memory only with regions that no thread touches in
  // that interval.
  static constexpr int O_EF = 0, O_T1 = O_EF + S_EF, O_T2 = O_T1 + S_T1;   // intervals 1-2
  static constexpr int O_UN = 0;                                           // 3-4 (T2 is above it)
  static constexpr int O_Y = 0;                                            // 5-6
  static constexpr int O_X = cmax(S_UN, S_Y);                              // 4-5
  static constexpr int O_UB = O_X, O_FP = O_UB + S_UB, O_W1 = O_FP + S_FP;  // 6-9 (X is dead)
  static constexpr int O_XL = cmax(cmax(O_T2 + S_T2, O_X + S_X), O_W1 + S_W1);   // 2-6
  static_assert(O_T2 >= S_UN, "T2 (read in interval 3) must not overlap UN (written in interval 3)");
  static constexpr int SZ_SLOT = O_XL + S_XL;
  static constexpr size_t DATA = ((size_t)EPB * SZ_SLOT * sizeof(R) + 15) / 16 * 16;
  static constexpr size_t SMEM = DATA + (size_t)EPB * (NFACE * sizeof(FaceLink) + 16 + (MIXED_ ? sizeof(RefState<R>) : 0));
};

template <class C>
struct Smem2 {
  using T = typename C::R;
  T *base;
  FaceLink *lnk;
  int *eid, *cls;
  RefState<T> *ref;
  __device__ Smem2(unsigned char *raw) {
    base = reinterpret_cast<T *>(raw);
    lnk = reinterpret_cast<FaceLink *>(raw + C::DATA);
    eid = reinterpret_cast<int *>(lnk + C::EPB * C::NFACE);
    cls = eid + C::EPB;
    ref = reinterpret_cast<RefState<T> *>(reinterpret_cast<unsigned char *>(eid) + 16 * C::EPB);
  }
  __device__ T *slot(int s) const { return base + (size_t)s * C::SZ_SLOT; }
};

// End value B[m][end] of basis function m for a thread-varying m, by selects
// over compile-time constant-bank operands (no divergent constant loads).
template <class T, int L, int Q>
__device__ __forceinline__ T end_value(int end, int m) {
  T v = cEnd<T, L, Q>[end * L];
#pragma unroll
  for (int k = 1; k < L; ++k) v = (m == k) ? cEnd<T, L, Q>[end * L + k] : v;
  return v;
}


// ---- the tile's links, class and (mixed form) reference state ----------------
template <class C>
__device__ __forceinline__ void s2_load(const Smem2<C> &sm, const StageArgs &a, int e0, int tid) {
  constexpr int NFACE = C::NFACE, EPB = C::EPB;
  for (int w = tid; w < EPB * NFACE; w += C::NT) {
    const int s = w / NFACE, f = w - s * NFACE, e = e0 + s;
    const FaceLink lk = e < a.ne ? a.links[(size_t)e * NFACE + f] : FaceLink{0, 0, 0, -1};
    sm.lnk[w] = lk;
    if (f == 0) {
      const int gc = e < a.ne ? a.gclass[e] : -1;
      sm.cls[s] = gc >= 0 ? gc : 0;
      sm.eid[s] = gc >= 0 ? e : -1;
      if constexpr (C::MIXED)
        sm.ref[s] = *reinterpret_cast<const RefState<float> *>(a.uref + kUrefStride * solve_of(a, gc >= 0 ? e : -1) + 10);
    }
  }
}

// ---- interval 1a: numerical flux at every face point --------------------------
// The 3-D Euler flux of face_flux (kernels.cuh) written without the face
// frame: for an orthonormal frame (n, s, t) the rotation and its inverse
// cancel, so F(U).n = (m.n, m (u.n) + p n, (E + p) u.n), and the Roe
// dissipation's two tangential waves become one tangential vector
//   a_sh = (dm - (dm.n) n) - (u~ - (u~.n) n) drho,
// with G_n, G_0 and G_E as in the frame and G_t = u~_t G_0 + min(u~.n, 0) a_sh.
// Lax-Friedrichs (src/Euler3d.cpp:601-816) uses max(|u.n| + c) over both
// sides, which is the reference's max(|u.n - c|, |u.n|, |u.n + c|).  Same
// algebra as the frame form; only the rounding differs.
// What a side needs is the jump F^ - F(U_own).n: the master side (UL) gets
// the flux's dissipation part G = F^ - F(UL).n, the slave side (UR)
// D - G with D = F(UR).n - F(UL).n, so F^ itself is never formed (and the
// two sides' fluxes, F(UL).n + G, agree as before).
template <class T>
__device__ __forceinline__ bool face_jump_vec3(const T *UL, const T *UR, const T *n, T gamma, int flux, bool master,
                                               T *out) {
  const T gm1 = gamma - T(1.0);
  const T n0 = n[0], n1 = n[1], n2 = n[2];
  const T rl = UL[0], irl = T(1.0) / rl;
  const T uxl = UL[1] * irl, uyl = UL[2] * irl, uzl = UL[3] * irl;
  const T unl = fma(uzl, n2, fma(uyl, n1, uxl * n0));
  const T pl = gm1 * fma(T(-0.5), fma(UL[3], uzl, fma(UL[2], uyl, UL[1] * uxl)), UL[4]);
  const T rr = UR[0], irr = T(1.0) / rr;
  const T uxr = UR[1] * irr, uyr = UR[2] * irr, uzr = UR[3] * irr;
  const T unr = fma(uzr, n2, fma(uyr, n1, uxr * n0));
  const T pr = gm1 * fma(T(-0.5), fma(UR[3], uzr, fma(UR[2], uyr, UR[1] * uxr)), UR[4]);
  const bool ok = rl >= T(kAeps) && pl >= T(kAeps) && rr >= T(kAeps) && pr >= T(kAeps);
  // D = F(UR).n - F(UL).n, needed by the slave side only
  const T dp = pr - pl;
  T D[5];
  D[0] = fma(rr, unr, -rl * unl);
  D[1] = fma(UR[1], unr, fma(-UL[1], unl, dp * n0));
  D[2] = fma(UR[2], unr, fma(-UL[2], unl, dp * n1));
  D[3] = fma(UR[3], unr, fma(-UL[3], unl, dp * n2));
  D[4] = fma(UR[4] + pr, unr, -(UL[4] + pl) * unl);
  const T Hl = (UL[4] + pl) * irl, Hr = (UR[4] + pr) * irr;
  T Gv[5];   // F^ - F(UL).n
  if (flux == DGMX_FLUX_ROE) {
    const T R = sqrt(rr * irl), iRp1 = T(1.0) / (T(1.0) + R);
    const T ux = fma(R, uxr, uxl) * iRp1, uy = fma(R, uyr, uyl) * iRp1, uz = fma(R, uzr, uzl) * iRp1;
    const T H = fma(R, Hr, Hl) * iRp1;
    const T q2 = fma(uz, uz, fma(uy, uy, ux * ux));
    const T a2 = gm1 * fma(T(-0.5), q2, H);
    const T ainv = rsqrt(a2), a = a2 * ainv;
    const T un = fma(uz, n2, fma(uy, n1, ux * n0));
    const T dr = rr - rl, dmx = UR[1] - UL[1], dmy = UR[2] - UL[2], dmz = UR[3] - UL[3], dE = UR[4] - UL[4];
    const T dmn = fma(dmz, n2, fma(dmy, n1, dmx * n0));
    const T utx = fma(-un, n0, ux), uty = fma(-un, n1, uy), utz = fma(-un, n2, uz);
    const T shx = fma(-utx, dr, fma(-dmn, n0, dmx)), shy = fma(-uty, dr, fma(-dmn, n1, dmy)),
            shz = fma(-utz, dr, fma(-dmn, n2, dmz));
    const T shu = fma(shz, utz, fma(shy, uty, shx * utx));
    const T a1 = gm1 * ainv * ainv * (fma(dr, fma(-un, un, H), un * dmn) - (dE - shu));
    const T a0 = T(0.5) * ainv * (fma(dr, un + a, -dmn) - a * a1);
    const T a4 = dr - (a0 + a1);
    const T l0 = fmin(un - a, T(0.0)), l1 = fmin(un, T(0.0)), l4 = fmin(un + a, T(0.0));
    const T w0 = l0 * a0, w1 = l1 * a1, w4 = l4 * a4;
    const T G0 = w0 + w1 + w4;
    const T Gn = fma(un + a, w4, fma(un, w1, (un - a) * w0));
    Gv[0] = G0;
    Gv[1] = fma(Gn, n0, fma(G0, utx, l1 * shx));
    Gv[2] = fma(Gn, n1, fma(G0, uty, l1 * shy));
    Gv[3] = fma(Gn, n2, fma(G0, utz, l1 * shz));
    Gv[4] = fma(fma(un, a, H), w4, fma(T(0.5) * q2, w1, fma(fma(-un, a, H), w0, l1 * shu)));
  } else {
    const T cl = sqrt(gm1 * fma(T(-0.5), fma(uzl, uzl, fma(uyl, uyl, uxl * uxl)), Hl));
    const T cr = sqrt(gm1 * fma(T(-0.5), fma(uzr, uzr, fma(uyr, uyr, uxr * uxr)), Hr));
    const T hl = T(0.5) * fmax(fabs(unl) + cl, fabs(unr) + cr);
#pragma unroll
    for (int k = 0; k < 5; ++k) Gv[k] = fma(T(0.5), D[k], hl * (UL[k] - UR[k]));
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) out[k] = master ? Gv[k] : D[k] - Gv[k];
  return ok;
}


// E = (F^ - F(U_own)).n J_side/J_el at face point g of face f, as
// face_fluxes (stage.cuh) computes it, from the own and neighbour traces in
// global memory (a warp's points are two faces' contiguous rows).  Both sides
// of a face evaluate the flux with the master's state first; the states are
// selected before one flux evaluation so that a warp holding master and
// slave points runs it once.
template <class C, int PHYS>
__device__ __forceinline__ void s2_face_point(const Smem2<C> &sm, const StageArgs &a, int e0, int w) {
  using T = typename C::R;
  constexpr int NF = C::NF, GF = C::GF, NFACE = C::NFACE, PE = C::PE;
  const int s = w / (NFACE * GF), rem = w - s * NFACE * GF, f = rem / GF, g = rem - f * GF;
  const int e = sm.eid[s];
  if (e < 0) return;
  const FaceLink lk = sm.lnk[s * NFACE + f];
  const GeomClass *gc = a.classes + sm.cls[s];
  const T *Tin = trace_in<C>(a);
  const int gn = __ldg(a.perm + lk.perm + g);
  const T *to = Tin + ((size_t)e * NFACE + f) * NF * GF + g;
  const T *tn = Tin + ((size_t)lk.elem * NFACE + lk.face) * NF * GF + gn;
  const int mbits = __ldg(&gc->master);
  const bool master = (mbits >> f) & 1;
  T UL[5], UR[5], Fh[5], FR[5];
#pragma unroll
  for (int k = 0; k < NF; ++k) {
    const T uo = to[k * GF], un = tn[k * GF];
    UL[k] = master ? uo : un;
    UR[k] = master ? un : uo;
  }
  const T nm[3] = {T(__ldg(&gc->nrm[f][0])), T(__ldg(&gc->nrm[f][1])), T(__ldg(&gc->nrm[f][2]))};
  const T jr = T(__ldg(&gc->jr[f]));
  T *eo = sm.slot(s) + C::O_EF + f * NF * PE + g;
  bool ok;
  if constexpr (C::MIXED) {
    ok = face_flux_pert<PHYS, T>(sm.ref[s], UL, UR, nm, T(a.gamma), a.flux, Fh, FR, gc->fr[f]);
#pragma unroll
    for (int k = 0; k < NF; ++k) eo[k * PE] = (master ? Fh[k] : FR[k] - Fh[k]) * jr;
  } else {
    ok = face_jump_vec3<T>(UL, UR, nm, T(a.gamma), a.flux, master, Fh);
#pragma unroll
    for (int k = 0; k < NF; ++k) eo[k * PE] = Fh[k] * jr;
  }
  if (!ok) {
    atomicOr(a.err, 1);
    atomicMin(a.err + 1, e);
  }
}

// ---- interval 1b: backward k-pass from the modal rows in global memory ----
// T1[b][n a][k] = sum_c B[c][k] u[n][a][b][c]; the mixed form takes the
// solve's reference state out of the constant mode in FP64 first.  Elements
// past the end get the constant state (their results are discarded).
template <class C>
__device__ __forceinline__ void s2_backward_k_row(const Smem2<C> &sm, const StageArgs &a, int e0, int w) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, RPS = NF * L * L;
  const int s = w / RPS, r = w - s * RPS, e = e0 + s;   // r = (n*L + a)*L + b
  double v[L];
  if (e < a.ne) {
    ld_row<L>(a.X + ((size_t)e * RPS + r) * L, v);
    if constexpr (C::MIXED)
      if (r % (L * L) == 0) v[0] -= a.uref[kUrefStride * solve_of(a, e) + 5 + r / (L * L)];
  } else {
#pragma unroll
    for (int k = 0; k < L; ++k) v[k] = (!C::MIXED && k == 0 && r % (L * L) == 0) ? 1.0 : 0.0;
  }
  // planes of NF L Q = 4 (mod 16) values at p = 3: this pass's (n a, b) rows
  // and the j pass's contiguous reads both fall on distinct banks
  T *dst = sm.slot(s) + C::O_T1 + (r % L) * (NF * L * Q) + (r / L) * Q;
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    T acc = T(0);
#pragma unroll
    for (int c = 0; c < L; ++c) acc = fma(cB<T, L, Q>[c * Q + k], T(v[c]), acc);
    dst[k] = acc;
  }
}

template <class C, int PHYS>
__device__ __forceinline__ void s2_interval1(const Smem2<C> &sm, const StageArgs &a, int e0, int tid) {
  constexpr int N1 = C::EPB * C::NFACE * C::GF, N2 = C::EPB * C::NF * C::L * C::L;
  // two loops: one body holding both tasks keeps both tasks' state live
  for (int w = tid; w < N1; w += C::NT) s2_face_point<C, PHYS>(sm, a, e0, w);
  for (int w = tid; w < N2; w += C::NT) s2_backward_k_row<C>(sm, a, e0, w);
}

// ---- interval 2a: lift and projection of one face's terms of one field ------
// XL[a'][b'] = sum_g BwG[a'][g] sum_h BwG[b'][h] E[g][h]; one column b' at a
// time keeps the registers to the 16 face terms and 8 partial sums.
template <class C>
__device__ __forceinline__ void s2_lift(const Smem2<C> &sm, int w) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, G = C::G, GF = C::GF, NFACE = C::NFACE, PE = C::PE, PL = C::PL;
  const int s = w / (NFACE * NF), fn = w - s * NFACE * NF;
  const T *src = sm.slot(s) + C::O_EF + fn * PE;
  T E[GF];
#pragma unroll
  for (int q = 0; q < GF; ++q) E[q] = src[q];
  T *dst = sm.slot(s) + C::O_XL + fn * C::XLS;
#pragma unroll
  for (int b = 0; b < L; ++b) {
    T z[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      T acc = T(0);
#pragma unroll
      for (int h = 0; h < G; ++h) acc = fma(cBwG<T, L, Q>[b * G + h], E[g * G + h], acc);
      z[g] = acc;
    }
#pragma unroll
    for (int aa = 0; aa < L; ++aa) {
      T acc = T(0);
#pragma unroll
      for (int g = 0; g < G; ++g) acc = fma(cBwG<T, L, Q>[aa * G + g], z[g], acc);
      dst[aa * PL + b] = acc;
    }
  }
}

// ---- interval 2b-3: modal -> GLL values (j and i passes) ---------------------
template <class C>
__device__ __forceinline__ void s2_backward_j_pencil(const Smem2<C> &sm, int w) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, N = NF * L * Q;
  const int s = w / N, r = w - s * N;   // r = (n*L + a)*Q + k
  const T *src = sm.slot(s) + C::O_T1 + r;
  T v[L];
#pragma unroll
  for (int b = 0; b < L; ++b) v[b] = src[b * N];
  T *dst = sm.slot(s) + C::O_T2 + r;
#pragma unroll
  for (int j = 0; j < Q; ++j) {
    T acc = T(0);
#pragma unroll
    for (int b = 0; b < L; ++b) acc = fma(cB<T, L, Q>[b * Q + j], v[b], acc);
    dst[j * C::XJ] = acc;
  }
}

template <class C>
__device__ __forceinline__ void s2_interval2(const Smem2<C> &sm, int tid) {
  constexpr int N1 = C::EPB * C::NFACE * C::NF, N2 = C::EPB * C::NF * C::L * C::Q;
  for (int w = tid; w < N2; w += C::NT) s2_backward_j_pencil<C>(sm, w);
  for (int w = tid; w < N1; w += C::NT) s2_lift<C>(sm, w);
}

template <class C>
__device__ __forceinline__ void s2_backward_i(const Smem2<C> &sm, int tid) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, EPB = C::EPB;
  constexpr int N = NF * Q * Q;
  for (int w = tid; w < EPB * N; w += C::NT) {
    const int s = w / N, r = w - s * N, n = r / (Q * Q), jk = r - n * Q * Q, j = jk / Q, k = jk - j * Q;
    const T *src = sm.slot(s) + C::O_T2 + j * C::XJ + n * L * Q + k;
    T v[L];
#pragma unroll
    for (int a = 0; a < L; ++a) v[a] = src[a * Q];
    T *dst = sm.slot(s) + C::O_UN + n * Q * Q * Q + jk;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      T acc = T(0);
#pragma unroll
      for (int a = 0; a < L; ++a) acc = fma(cB<T, L, Q>[a * Q + i], v[a], acc);
      dst[i * Q * Q] = acc;
    }
  }
}

// ---- interval 4: contravariant fluxes and the i-axis pass --------------------
// Column (j, k), directions [R0, R0 + NR): G_r = sum_d metric[r][d] F_d(U)
// at the Q points of the column, then X_r[n][a] = sum_i C_r[a][i] G_r[n][i]
// with C_0 = E (the derivative along i) and C_1 = C_2 = B W.  With the
// contravariant velocity V_r = metric[r] . u:  G_r[rho] = rho V_r,
// G_r[m_d] = m_d V_r + p metric[r][d], G_r[E] = (E + p) V_r.  The mixed form
// evaluates F(Ub + u') - F(Ub) (as volume_flux_pert, kernels.cuh) the same
// way.  One direction per thread (20 accumulators; the columns of a direction
// fill whole warps) or all three (60); Cfg2::VDIRS chooses.
template <class C, int NR, int R0>
__device__ __forceinline__ void s2_volume_column(const Smem2<C> &sm, const StageArgs &a, int s, int jk) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q;
  const T gm1 = T(a.gamma) - T(1.0);
  const GeomClass *gc = a.classes + sm.cls[s];
  T met[NR][3];
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int d = 0; d < 3; ++d) met[r][d] = T(__ldg(&gc->metric[3 * (R0 + r) + d]));
  const T *un = sm.slot(s) + C::O_UN + jk;
  T acc[NR][5][L];
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int n = 0; n < NF; ++n)
#pragma unroll
      for (int b = 0; b < L; ++b) acc[r][n][b] = T(0);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    T U[5];
#pragma unroll
    for (int n = 0; n < NF; ++n) U[n] = un[(n * Q + i) * Q * Q];
    if constexpr (C::MIXED) {
      const RefState<T> &b = sm.ref[s];
      const T rho = b.r + U[0], ir = p_rcp(rho);
      const T mx = b.m[0] + U[1], my = b.m[1] + U[2], mz = b.m[2] + U[3];
      const T upx = (U[1] - b.u[0] * U[0]) * ir, upy = (U[2] - b.u[1] * U[0]) * ir, upz = (U[3] - b.u[2] * U[0]) * ir;
      T sdot = T(0);
      sdot = fma(U[1], b.u[0], sdot); sdot = fma(mx, upx, sdot);
      sdot = fma(U[2], b.u[1], sdot); sdot = fma(my, upy, sdot);
      sdot = fma(U[3], b.u[2], sdot); sdot = fma(mz, upz, sdot);
      const T pp = gm1 * fma(T(-0.5), sdot, U[4]);
      const T Hp = U[4] + pp, H = b.H + Hp;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const T m0 = met[r][0], m1 = met[r][1], m2 = met[r][2];
        const T Vb = m0 * b.u[0] + m1 * b.u[1] + m2 * b.u[2];       // reference contravariant velocity
        const T Vp = m0 * upx + m1 * upy + m2 * upz;                 // its perturbation
        T Gr[5];
        Gr[0] = m0 * U[1] + m1 * U[2] + m2 * U[3];
        Gr[1] = fma(U[1], Vb, fma(mx, Vp, pp * m0));
        Gr[2] = fma(U[2], Vb, fma(my, Vp, pp * m1));
        Gr[3] = fma(U[3], Vb, fma(mz, Vp, pp * m2));
        Gr[4] = fma(Hp, Vb, H * Vp);
#pragma unroll
        for (int n = 0; n < NF; ++n)
#pragma unroll
          for (int bb = 0; bb < L; ++bb)
            acc[r][n][bb] = fma(R0 + r == 0 ? cE2<T, L, Q>[bb * Q + i] : cBw<T, L, Q>[bb * Q + i], Gr[n], acc[r][n][bb]);
      }
    } else {
      const T ir = T(1.0) / U[0];
      const T u = U[1] * ir, v = U[2] * ir, ww = U[3] * ir;
      T p = u * U[1];
      p = fma(v, U[2], p);
      p = fma(ww, U[3], p);
      p = T(-0.5) * gm1 * p;
      p = fma(gm1, U[4], p);
      const T Ep = U[4] + p;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const T m0 = met[r][0], m1 = met[r][1], m2 = met[r][2];
        const T V = fma(m2, ww, fma(m1, v, m0 * u));
        T Gr[5];
        Gr[0] = U[0] * V;
        Gr[1] = fma(U[1], V, p * m0);
        Gr[2] = fma(U[2], V, p * m1);
        Gr[3] = fma(U[3], V, p * m2);
        Gr[4] = Ep * V;
#pragma unroll
        for (int n = 0; n < NF; ++n)
#pragma unroll
          for (int bb = 0; bb < L; ++bb)
            acc[r][n][bb] = fma(R0 + r == 0 ? cE2<T, L, Q>[bb * Q + i] : cBw<T, L, Q>[bb * Q + i], Gr[n], acc[r][n][bb]);
      }
    }
  }
  const int j = jk / Q, k = jk - j * Q;
  T *dst = sm.slot(s) + C::O_X + j * C::XJ + k;
#pragma unroll
  for (int r = 0; r < NR; ++r)
#pragma unroll
    for (int n = 0; n < NF; ++n)
#pragma unroll
      for (int b = 0; b < L; ++b) dst[(R0 + r) * (C::S_X1 + 1) + (n * L + b) * Q] = acc[r][n][b];
}

template <class C, int PHYS>
__device__ __forceinline__ void s2_volume(const Smem2<C> &sm, const StageArgs &a, int tid) {
  constexpr int Q = C::Q, EPB = C::EPB;
  // one direction per thread: the columns of one direction fill whole warps
  // (warp-uniform r)
  constexpr int NDIR = 3 / C::VDIRS, RS = (Q * Q + 31) / 32 * 32, N = NDIR * RS;
  for (int w = tid; w < EPB * N; w += C::NT) {
    const int s = w / N, rem = w - s * N, r = rem / RS, jk = rem - r * RS;
    if (jk >= Q * Q) continue;
    // the direction is a template argument, so the coefficients stay
    // constant-bank operands of the FMAs
    if constexpr (C::VDIRS == 3) s2_volume_column<C, 3, 0>(sm, a, s, jk);
    else if (r == 0) s2_volume_column<C, 1, 0>(sm, a, s, jk);
    else if (r == 1) s2_volume_column<C, 1, 1>(sm, a, s, jk);
    else s2_volume_column<C, 1, 2>(sm, a, s, jk);
  }
}

// ---- interval 5: j-axis pass --------------------------------------------------
// Y0 = P_j X0 + E_j X1, Y2 = P_j X2   ([b][n a][k]: planes of NF L Q = 4 (mod
// 16) values at p = 3, so both this pass's writes and the update's reads of
// (n a, b) rows fall on distinct banks)
template <class C>
__device__ __forceinline__ void s2_pass_j(const Smem2<C> &sm, int tid) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, EPB = C::EPB;
  constexpr int N = NF * L * Q;
  for (int w = tid; w < EPB * N; w += C::NT) {
    const int s = w / N, r = w - s * N;   // r = (n*L + a)*Q + k
    const T *x = sm.slot(s) + C::O_X + r;   // a warp reads contiguous values
    T x0[Q], x1[Q], x2[Q];
#pragma unroll
    for (int j = 0; j < Q; ++j) {
      x0[j] = x[j * C::XJ];
      x1[j] = x[(C::S_X1 + 1) + j * C::XJ];
      x2[j] = x[2 * (C::S_X1 + 1) + j * C::XJ];
    }
    T *y = sm.slot(s) + C::O_Y + r;
#pragma unroll
    for (int b = 0; b < L; ++b) {
      T y0 = T(0), y2 = T(0);
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        y0 = fma(cBw<T, L, Q>[b * Q + j], x0[j], y0);
        y0 = fma(cE2<T, L, Q>[b * Q + j], x1[j], y0);
        y2 = fma(cBw<T, L, Q>[b * Q + j], x2[j], y2);
      }
      y[b * N] = y0;
      y[(C::S_Y1 + 1) + b * N] = y2;
    }
  }
}

// ---- interval 6: k-axis pass, face terms, update, next modal block ---------
template <class C, int PHYS>
__device__ __forceinline__ void s2_update(const Smem2<C> &sm, const StageArgs &a, int tid) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, EPB = C::EPB, PL = C::PL;
  constexpr int N = NF * L * L;
  for (int w = tid; w < EPB * N; w += C::NT) {
    const int s = w / N, r = w - s * N, n = r / (L * L), ab = r - n * L * L, aa = ab / L, bb = ab - aa * L;
    const int e = sm.eid[s];
    T *sl = sm.slot(s);
    // R[c] = sum_k P[c][k] Y0[k] + E[c][k] Y2[k]
    const T *y = sl + C::O_Y + bb * (NF * L * Q) + (n * L + aa) * Q;
    T y0[Q], y2[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) { y0[k] = y[k]; y2[k] = y[(C::S_Y1 + 1) + k]; }
    // face terms: k faces (0: k=0, 5: k=Q-1) plane (a, b); j faces (1: j=0,
    // 3: j=Q-1) plane (a, c); i faces (4: i=0, 2: i=Q-1) plane (b, c)
    const T *xl = sl + C::O_XL;
    constexpr int FB = NF * C::XLS;   // one face's block
    const T xk0 = xl[0 * FB + n * C::XLS + aa * PL + bb], xk1 = xl[5 * FB + n * C::XLS + aa * PL + bb];
    const T *xj0 = xl + 1 * FB + n * C::XLS + aa * PL, *xj1 = xl + 3 * FB + n * C::XLS + aa * PL;
    const T *xi0 = xl + 4 * FB + n * C::XLS + bb * PL, *xi1 = xl + 2 * FB + n * C::XLS + bb * PL;
    const T eb0 = end_value<T, L, Q>(0, bb), eb1 = end_value<T, L, Q>(1, bb);
    const T ea0 = end_value<T, L, Q>(0, aa), ea1 = end_value<T, L, Q>(1, aa);
    T R[L];
#pragma unroll
    for (int c = 0; c < L; ++c) {
      T acc = T(0);
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        acc = fma(cBw<T, L, Q>[c * Q + k], y0[k], acc);
        acc = fma(cE2<T, L, Q>[c * Q + k], y2[k], acc);
      }
      acc = fma(cEnd<T, L, Q>[c], xk0, acc);
      acc = fma(cEnd<T, L, Q>[L + c], xk1, acc);
      acc = fma(eb0, xj0[c], acc);
      acc = fma(eb1, xj1[c], acc);
      acc = fma(ea0, xi0[c], acc);
      acc = fma(ea1, xi1[c], acc);
      R[c] = acc;
    }
    // The state the right-hand side was evaluated on (X; X = U for LSRK)
    // is read back from global memory: its shared copy is dead by now.
    T *ub = sl + C::O_UB + r * PL;
    if (e < 0) {
#pragma unroll
      for (int c = 0; c < L; ++c) ub[c] = T(0);
    } else {
      const size_t gi = ((size_t)e * N + r) * L;
      const double dt = a.dts ? a.dts[solve_of(a, e)] : a.dt;
      double x[L];
      ld_row<L>(a.X + gi, x);
      if constexpr (C::MIXED) {
        const double ref0 = ab == 0 ? a.uref[kUrefStride * solve_of(a, e) + 5 + n] : 0.0;
        float q[L];
#pragma unroll
        for (int c = 0; c < L; ++c) q[c] = R[c];
        if (a.Ssrc)
#pragma unroll
          for (int c = 0; c < L; ++c) q[c] -= float(a.src_scale * a.Ssrc[gi + c]);
        if (a.Rsub)
#pragma unroll
          for (int c = 0; c < L; ++c) q[c] -= float(a.Rsub[gi + c]);
        if (a.kind == kRHS) {
#pragma unroll
          for (int c = 0; c < L; ++c) { a.A[gi + c] = q[c]; ub[c] = float(c == 0 ? x[c] - ref0 : x[c]); }
        } else {
          float ut[L];
          double u[L];
          ld_row<L>(a.Utf + gi, ut);
          const float c0 = float(a.c0), mdt = -float(dt);
#pragma unroll
          for (int c = 0; c < L; ++c) {
            ut[c] = fmaf(mdt, q[c], c0 * ut[c]);
            u[c] = fma(a.c1, double(ut[c]), x[c]);
          }
          st_row<L>(a.Utf + gi, ut);
          st_row<L>(a.U + gi, u);
#pragma unroll
          for (int c = 0; c < L; ++c) ub[c] = float(c == 0 ? u[c] - ref0 : u[c]);
        }
      } else {
        double q[L];
#pragma unroll
        for (int c = 0; c < L; ++c) q[c] = R[c];
        if (a.Ssrc)
#pragma unroll
          for (int c = 0; c < L; ++c) q[c] -= a.src_scale * a.Ssrc[gi + c];
        if (a.Rcap)
#pragma unroll
          for (int c = 0; c < L; ++c) a.Rcap[gi + c] = q[c];
        if (a.Rsub)
#pragma unroll
          for (int c = 0; c < L; ++c) q[c] -= a.Rsub[gi + c];
        if (a.kind == kRHS) {
#pragma unroll
          for (int c = 0; c < L; ++c) { a.A[gi + c] = q[c]; ub[c] = x[c]; }
        } else {
          double ut[L], u[L];
          ld_row<L>(a.Ut + gi, ut);
#pragma unroll
          for (int c = 0; c < L; ++c) {
            ut[c] = fma(-dt, q[c], a.c0 * ut[c]);
            u[c] = fma(a.c1, ut[c], x[c]);
            ub[c] = u[c];
          }
          st_row<L>(a.Ut + gi, ut);
          st_row<L>(a.U + gi, u);
        }
      }
    }
    // end values along c of the next modal block: faces 0 (k=0) and 5 (k=Q-1)
    T f0 = T(0), f5 = T(0);
#pragma unroll
    for (int c = 0; c < L; ++c) {
      const T xv = ub[c];
      f0 = fma(cEnd<T, L, Q>[c], xv, f0);
      f5 = fma(cEnd<T, L, Q>[L + c], xv, f5);
    }
    T *fp = sl + C::O_FP + n * C::FPS + ab;
    constexpr int PB = NF * C::FPS;   // one face's planes
    fp[0 * PB] = f0;
    fp[5 * PB] = f5;
  }
}

// ---- interval 7: end values along b (faces 1, 3) and a (faces 4, 2) ---------
template <class C>
__device__ __forceinline__ void s2_ends_ab(const Smem2<C> &sm, int tid) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, EPB = C::EPB, PL = C::PL;
  constexpr int N = NF * L * L, PB = NF * C::FPS;
  for (int w = tid; w < EPB * 2 * N; w += C::NT) {
    const int s = w / (2 * N), rem = w - s * 2 * N, ax = rem / N, r = rem - ax * N;
    const int n = r / (L * L), xy = r - n * L * L, x = xy / L, y = xy - x * L;
    const T *ub = sm.slot(s) + C::O_UB + n * L * L * PL;
    T lo = T(0), hi = T(0);
    T *fp = sm.slot(s) + C::O_FP + n * C::FPS + xy;
    if (ax == 0) {   // along b at (a = x, c = y): faces 1 (j=0) and 3 (j=Q-1), plane (a, c)
#pragma unroll
      for (int b = 0; b < L; ++b) {
        const T v = ub[(x * L + b) * PL + y];
        lo = fma(cEnd<T, L, Q>[b], v, lo);
        hi = fma(cEnd<T, L, Q>[L + b], v, hi);
      }
      fp[1 * PB] = lo;
      fp[3 * PB] = hi;
    } else {         // along a at (b = x, c = y): faces 4 (i=0) and 2 (i=Q-1), plane (b, c)
#pragma unroll
      for (int aa = 0; aa < L; ++aa) {
        const T v = ub[(aa * L + x) * PL + y];
        lo = fma(cEnd<T, L, Q>[aa], v, lo);
        hi = fma(cEnd<T, L, Q>[L + aa], v, hi);
      }
      fp[4 * PB] = lo;
      fp[2 * PB] = hi;
    }
  }
}

// ---- intervals 8-9: face planes -> Gauss points, stored as the next traces --
// pass a: W1[f][n][g][b'] = sum_a' Bg[a'][g] FP[f][n][a'][b']
template <class C>
__device__ __forceinline__ void s2_traces_a(const Smem2<C> &sm, int tid) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, G = C::G, NFACE = C::NFACE, EPB = C::EPB, PL = C::PL;
  constexpr int N = NFACE * NF * L;
  for (int w = tid; w < EPB * N; w += C::NT) {
    const int s = w / N, r = w - s * N, fn = r / L, b = r - fn * L;
    const T *src = sm.slot(s) + C::O_FP + fn * C::FPS + b;
    T v[L];
#pragma unroll
    for (int aa = 0; aa < L; ++aa) v[aa] = src[aa * L];
    T *dst = sm.slot(s) + C::O_W1 + fn * G * PL + b;
#pragma unroll
    for (int g = 0; g < G; ++g) {
      T acc = T(0);
#pragma unroll
      for (int aa = 0; aa < L; ++aa) acc = fma(cBg<T, L, Q>[aa * G + g], v[aa], acc);
      dst[g * PL] = acc;
    }
  }
}
// pass b: trace[f][n][g][h] = sum_b' Bg[b'][h] W1[f][n][g][b'], a row of G
// per thread straight to global memory
template <class C, class TT>
__device__ __forceinline__ void s2_traces_b(const Smem2<C> &sm, TT *Tout, int e0, int ne, int tid) {
  using T = typename C::R;
  constexpr int NF = C::NF, L = C::L, Q = C::Q, G = C::G, NFACE = C::NFACE, EPB = C::EPB, PL = C::PL, GF = C::GF;
  constexpr int N = NFACE * NF * G;
  for (int w = tid; w < EPB * N; w += C::NT) {
    const int s = w / N, r = w - s * N, e = e0 + s;   // r = (f*NF + n)*G + g
    if (e >= ne) continue;
    const T *src = sm.slot(s) + C::O_W1 + r * PL;
    T v[L];
#pragma unroll
    for (int b = 0; b < L; ++b) v[b] = src[b];
    TT out[G];
#pragma unroll
    for (int h = 0; h < G; ++h) {
      T acc = T(0);
#pragma unroll
      for (int b = 0; b < L; ++b) acc = fma(cBg<T, L, Q>[b * G + h], v[b], acc);
      out[h] = TT(acc);
    }
    st_row<G>(Tout + (size_t)e * NFACE * NF * GF + r * G, out);
  }
}

// L2 prefetch hints (no data is moved into the SM, nothing waits): the
// second register of tile `tile` (read by its update, six intervals later),
// and the face traces, modal rows and second register of tile `next` (-1:
// none).  Only addresses of elements that exist are named.
__device__ __forceinline__ void prefetch_l2_lines(const void *base, int bytes, int line) {
  if (line * 128 < bytes) asm volatile("prefetch.global.L2 [%0];" ::"l"(static_cast<const char *>(base) + line * 128));
}

template <class C>
__device__ __forceinline__ void s2_prefetch(const StageArgs &a, int tile, int next, int tid) {
  using T = typename C::R;
  constexpr int TB = C::NFACE * C::NF * C::GF * (int)sizeof(T), XB = C::NF * C::LD * (int)sizeof(double);
  constexpr int UB = C::NF * C::LD * (int)sizeof(T);
  constexpr int LT = (TB + 127) / 128, LX = (XB + 127) / 128, LU = (UB + 127) / 128;
  const bool lsrk = a.kind == kLSRK;
  const T *ut = nullptr;
  if (lsrk) {
    if constexpr (C::MIXED) ut = a.Utf; else ut = a.Ut;
  }
  for (int w = tid; w < C::EPB * (LT + LX + 2 * LU); w += C::NT) {
    const int s = w / (LT + LX + 2 * LU), l = w - s * (LT + LX + 2 * LU);
    const int e = tile * C::EPB + s, en = next * C::EPB + s;
    if (l < LU) {
      if (lsrk && e < a.ne) prefetch_l2_lines(ut + (size_t)e * C::NF * C::LD, UB, l);
    } else if (next >= 0 && en < a.ne) {
      const int m = l - LU;
      if (m < LT) prefetch_l2_lines(trace_in<C>(a) + (size_t)en * C::NFACE * C::NF * C::GF, TB, m);
      else if (m < LT + LX) prefetch_l2_lines(a.X + (size_t)en * C::NF * C::LD, XB, m - LT);
      else if (lsrk) prefetch_l2_lines(ut + (size_t)en * C::NF * C::LD, UB, m - LT - LX);
    }
  }
}

template <class C, int PHYS>
__device__ __forceinline__ void stage2_tile(const Smem2<C> &sm, const StageArgs &a, int e0, int tid) {
  s2_load<C>(sm, a, e0, tid);
  __syncthreads();
  s2_interval1<C, PHYS>(sm, a, e0, tid);
  __syncthreads();
  s2_interval2<C>(sm, tid);
  __syncthreads();
  s2_backward_i<C>(sm, tid);
  __syncthreads();
  s2_volume<C, PHYS>(sm, a, tid);
  __syncthreads();
  s2_pass_j<C>(sm, tid);
  __syncthreads();
  s2_update<C, PHYS>(sm, a, tid);
  __syncthreads();
  s2_ends_ab<C>(sm, tid);
  __syncthreads();
  s2_traces_a<C>(sm, tid);
  __syncthreads();
  s2_traces_b<C>(sm, trace_out<C>(a), e0, a.ne, tid);
}

// One tile (EPB elements) per CTA, or with a tile list a persistent loop over
// the listed tiles (element pools).
template <class C, int PHYS>
__global__ void __launch_bounds__(C::NT, C::MINB) stage2_kernel(StageArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem2<C> sm(smem_raw);
  const int ntile = a.tiles ? *a.ntiles : (int)gridDim.x;
  // One tile per CTA: the CTAs resident at once are about (SMs x CTAs per SM)
  // and start in block order, so the tile that many blocks ahead starts
  // about when this one ends.  Persistent over a tile list: this CTA's next
  // tile.  Its inputs are asked into L2 now, and this tile's second
  // register, which only the update reads, too.
  unsigned nsm;
  asm("mov.u32 %0, %%nsmid;" : "=r"(nsm));
  const int ahead = (int)nsm * (C::MINB_REQ > 8 ? C::MINB_REQ : 8);
  for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
    if (t != (int)blockIdx.x) __syncthreads();
    const int tile = a.tiles ? a.tiles[t] : t;
    const int next = a.tiles ? (t + (int)gridDim.x < ntile ? a.tiles[t + gridDim.x] : -1) : t + ahead;
    // FP64 only: measured on 32^3, p = 3, the hints take an LSRK stage from
    // 292 to 279 us in FP64 and from 233 to 238 us in the FP32 form
    if constexpr (!C::MIXED) s2_prefetch<C>(a, tile, next, threadIdx.x);
    stage2_tile<C, PHYS>(sm, a, tile * C::EPB, threadIdx.x);
  }
}

}  // namespace dgmx
