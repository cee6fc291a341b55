// Device building blocks of the B200 DG engine: constant tables, the
// sum-factorised axis contraction, and the pointwise physics (volume fluxes
// and numerical face fluxes).  Included by the per-physics kernel units.
#pragma once

#include <cuda_runtime.h>

#include "dgmx_internal.hpp"

namespace dgmx {

template <int B, int E>
struct Pow { static constexpr int v = B * Pow<B, E - 1>::v; };
template <int B>
struct Pow<B, 0> { static constexpr int v = 1; };

// 1-D tables for one (L, Q) pair in constant memory, in the working
// precision T of the kernels that use them.  With the contraction loops
// fully unrolled the indices are compile-time constants, so the
// coefficients become constant-bank operands of the FMAs.
template <class T, int L, int Q> __constant__ T cB[L * Q];          // B[a*Q+i]
template <class T, int L, int Q> __constant__ T cBg[L * (Q - 1)];   // Bg[a*G+g]
template <class T, int L, int Q> __constant__ T cD[Q * Q];          // D[i*Q+m]
template <class T, int L, int Q> __constant__ T cG2GL[Q * (Q - 1)]; // [i*G+g]
template <class T, int L, int Q> __constant__ T cGL2G[(Q - 1) * Q]; // [g*Q+i]
template <class T, int L, int Q> __constant__ T cW[Q];              // GLL weights
template <class T, int L, int Q> __constant__ T cEnd[2 * L];        // B[a][0], B[a][Q-1]
template <class T, int L, int Q> __constant__ T cBw[L * Q];         // B[a][i] w[i] (weighted projection)
template <class T, int L, int Q> __constant__ T cG2GLw[2 * Q * (Q - 1)];  // G2GL / w_end, ends 0 and 1

// Matrix accessors: M::get(in_index, out_index)
template <int L, int Q, class T = double> struct MatB   { static __device__ __forceinline__ T get(int a, int i) { return cB<T, L, Q>[a * Q + i]; } };
template <int L, int Q, class T = double> struct MatBt  { static __device__ __forceinline__ T get(int i, int a) { return cB<T, L, Q>[a * Q + i]; } };
template <int L, int Q, class T = double> struct MatBg  { static __device__ __forceinline__ T get(int a, int g) { return cBg<T, L, Q>[a * (Q - 1) + g]; } };
template <int L, int Q, class T = double> struct MatD   { static __device__ __forceinline__ T get(int m, int i) { return cD<T, L, Q>[i * Q + m]; } };
template <int L, int Q, class T = double> struct MatG2GL{ static __device__ __forceinline__ T get(int g, int i) { return cG2GL<T, L, Q>[i * (Q - 1) + g]; } };
template <int L, int Q, class T = double> struct MatBtw { static __device__ __forceinline__ T get(int i, int a) { return cBw<T, L, Q>[a * Q + i]; } };
template <int L, int Q, int END, class T = double> struct MatG2GLw { static __device__ __forceinline__ T get(int g, int i) { return cG2GLw<T, L, Q>[END * Q * (Q - 1) + i * (Q - 1) + g]; } };
template <int L, int Q, class T = double> struct MatGL2G{ static __device__ __forceinline__ T get(int i, int g) { return cGL2G<T, L, Q>[g * Q + i]; } };

// Contraction along axis AX of a batch of 3-D arrays (I0, I1, I2) with
// I_AX = K: out[...n...] = sum_k M(k, n) in[...k...], N outputs per pencil.
// Each thread owns one pencil: K loads, K*N FMAs with uniform coefficients.
// Batch b reads in + b*sin and writes out + b*sout.  Axis 2 is contiguous;
// the strides of axes 0 and 1 default to the dense layout and may be given
// (IS0, IS1 input; OS0, OS1 output) to address rows padded to an odd pitch,
// which keeps a warp's pencils on distinct shared-memory banks.
//
// OSA (nonzero) overrides the output stride along AX (outputs of one pencil
// scattered to separate arrays, e.g. the two end faces of an axis).
// FPT > 1 gives each thread the same pencil of FPT consecutive batches (the
// fields of one element): one index computation serves FPT pencils and the
// thread has FPT independent FMA chains (the one-element-per-warp tiles).
template <int I0, int I1, int I2, int AX, int K, int N, class M, bool ACC, class T, int IS0 = -1, int IS1 = -1,
          int OS0 = -1, int OS1 = -1, int FPT = 1, int OSA = 0>
__device__ __forceinline__ void contract(const T *__restrict__ in, T *__restrict__ out, int nbatch,
                                         int sin, int sout, int tid, int nthr) {
  constexpr int O1 = AX == 1 ? N : I1, O2 = AX == 2 ? N : I2;
  constexpr int P0 = AX == 0 ? I1 : I0;
  constexpr int P1 = AX == 2 ? I1 : I2;
  constexpr int NP = P0 * P1;
  constexpr int is1 = IS1 >= 0 ? IS1 : I2, is0 = IS0 >= 0 ? IS0 : I1 * is1;
  constexpr int os1 = OS1 >= 0 ? OS1 : O2, os0 = OS0 >= 0 ? OS0 : O1 * os1;
  constexpr int isA = AX == 0 ? is0 : (AX == 1 ? is1 : 1);
  constexpr int osA = OSA != 0 ? OSA : (AX == 0 ? os0 : (AX == 1 ? os1 : 1));
  for (int w = tid; w < (nbatch / FPT) * NP; w += nthr) {
    const int b = (w / NP) * FPT, p = w - (w / NP) * NP;
    const int pa = p / P1, pb = p - pa * P1;
    int io, oo;
    if (AX == 0) { io = pa * is1 + pb; oo = pa * os1 + pb; }
    else if (AX == 1) { io = pa * is0 + pb; oo = pa * os0 + pb; }
    else { io = pa * is0 + pb * is1; oo = pa * os0 + pb * os1; }
#pragma unroll
    for (int f = 0; f < FPT; ++f) {
      const T *src = in + (size_t)(b + f) * sin + io;
      T *dst = out + (size_t)(b + f) * sout + oo;
      T v[K];
#pragma unroll
      for (int k = 0; k < K; ++k) v[k] = src[k * isA];
#pragma unroll
      for (int n = 0; n < N; ++n) {
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < K; ++k) acc = fma(M::get(k, n), v[k], acc);
        if (ACC) dst[n * osA] += acc; else dst[n * osA] = acc;
      }
    }
  }
}

// ------------------------------------------------- tensor-core contraction
// The same contraction as `contract` (FP32 data) on the tensor cores:
// rows = pencils of all batches, one 16-pencil tile per warp at a time,
// out[16 x N] = in[16 x K] M[K x N] as mma.sync m16n8k8 TF32 products with
// FP32 accumulation, K and N padded to multiples of 8 with zeros.  Each
// operand is split into a TF32 part and the TF32 rounding of its remainder
// (3xTF32: a b ~ a_s b_b + a_b b_s + a_b b_b, the small products first), so
// the products keep about FP32 accuracy.  Fragment layouts of m16n8k8.tf32
// (g = lane / 4, c = lane % 4): A (row g | g + 8, col c | c + 4), B (row c |
// c + 4, col g), D (row g | g + 8, col 2c, 2c + 1).
__device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void tf32_split(float x, unsigned &big, unsigned &small) {
  big = tf32_rna(x);
  small = tf32_rna(x - __uint_as_float(big));
}
__device__ __forceinline__ void mma_tf32_16x8x8(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int I0, int I1, int I2, int AX, int K, int N, class M, bool ACC, int IS0 = -1, int IS1 = -1,
          int OS0 = -1, int OS1 = -1>
__device__ __forceinline__ void contract_tc(const float *__restrict__ in, float *__restrict__ out, int nbatch,
                                            int sin, int sout, int tid, int nthr) {
  constexpr int O1 = AX == 1 ? N : I1, O2 = AX == 2 ? N : I2;
  constexpr int P0 = AX == 0 ? I1 : I0;
  constexpr int P1 = AX == 2 ? I1 : I2;
  constexpr int NP = P0 * P1;
  constexpr int is1 = IS1 >= 0 ? IS1 : I2, is0 = IS0 >= 0 ? IS0 : I1 * is1;
  constexpr int os1 = OS1 >= 0 ? OS1 : O2, os0 = OS0 >= 0 ? OS0 : O1 * os1;
  constexpr int isA = AX == 0 ? is0 : (AX == 1 ? is1 : 1);
  constexpr int osA = AX == 0 ? os0 : (AX == 1 ? os1 : 1);
  constexpr int KS = (K + 7) / 8, NS = (N + 7) / 8;
  const int lane = tid & 31, g = lane >> 2, c = lane & 3;
  // the operator's fragments, split once per call
  unsigned bb[KS][NS][2], bs[KS][NS][2];
#pragma unroll
  for (int ks = 0; ks < KS; ++ks)
#pragma unroll
    for (int ns = 0; ns < NS; ++ns)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int k = ks * 8 + c + 4 * h, n = ns * 8 + g;
        const float v = (k < K && n < N) ? M::get(k, n) : 0.0f;
        tf32_split(v, bb[ks][ns][h], bs[ks][ns][h]);
      }
  const int rows = nbatch * NP;
  for (int t0 = (tid >> 5) * 16; t0 < rows; t0 += (nthr >> 5) * 16) {
    int io[2], oo[2];
    size_t ib[2], ob[2];
    bool ok[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int w = t0 + g + 8 * h;
      ok[h] = w < rows;
      const int b = ok[h] ? w / NP : 0, p = ok[h] ? w - b * NP : 0;
      const int pa = p / P1, pb = p - pa * P1;
      if (AX == 0) { io[h] = pa * is1 + pb; oo[h] = pa * os1 + pb; }
      else if (AX == 1) { io[h] = pa * is0 + pb; oo[h] = pa * os0 + pb; }
      else { io[h] = pa * is0 + pb * is1; oo[h] = pa * os0 + pb * os1; }
      ib[h] = (size_t)b * sin; ob[h] = (size_t)b * sout;
    }
    float acc[NS][4];
#pragma unroll
    for (int ns = 0; ns < NS; ++ns)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[ns][q] = 0.0f;
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      unsigned ab[4], as[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int h = q & 1, k = ks * 8 + c + 4 * (q >> 1);
        const float v = (ok[h] && k < K) ? in[ib[h] + io[h] + k * isA] : 0.0f;
        tf32_split(v, ab[q], as[q]);
      }
#pragma unroll
      for (int ns = 0; ns < NS; ++ns) {
        mma_tf32_16x8x8(acc[ns], as, bb[ks][ns][0], bb[ks][ns][1]);
        mma_tf32_16x8x8(acc[ns], ab, bs[ks][ns][0], bs[ks][ns][1]);
        mma_tf32_16x8x8(acc[ns], ab, bb[ks][ns][0], bb[ks][ns][1]);
      }
    }
#pragma unroll
    for (int ns = 0; ns < NS; ++ns)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int h = q >> 1, n = ns * 8 + 2 * c + (q & 1);
        if (!ok[h] || n >= N) continue;
        float *dst = out + ob[h] + oo[h] + n * osA;
        if (ACC) *dst += acc[ns][q]; else *dst = acc[ns][q];
      }
  }
}

// ------------------------------------------------------------------ physics
// Positivity threshold aepsM = eps^(2/3) (src/Constants.hpp:43).
__device__ constexpr double kAeps = 4.8148248609680896e-11;

// Physical flux components for one point.  Operation order follows the
// reference volume loops (src/Euler.cpp:335-384, src/Euler3d.cpp:506-566,
// src/Shallow.cpp:305-339).  Fills F[d][n] for d < DIM.
template <int PHYS, class T>
__device__ __forceinline__ void volume_flux(const T *U, T gamma, T (*F)[5]) {
  if constexpr (PHYS == DGMX_EULER2D || PHYS == DGMX_NS2D) {
    const T gm1 = gamma - T(1.0), m5g = -T(0.5) * gm1;
    const T r = U[0], ru = U[1], rv = U[2], rE = U[3];
    const T ir = T(1.0) / r;
    const T u = ru * ir, v = rv * ir;
    T p = u * ru;
    p = v * rv + p;
    p = m5g * p;
    p = fma(gm1, rE, p);
    F[0][0] = ru;            F[1][0] = rv;
    F[0][1] = ru * u + p;    F[1][1] = ru * v;
    F[0][2] = rv * u;        F[1][2] = rv * v + p;
    const T e = rE + p;
    F[0][3] = u * e;         F[1][3] = v * e;
  } else if constexpr (PHYS == DGMX_EULER3D || PHYS == DGMX_NS3D) {
    const T gm1 = gamma - T(1.0), m5g = -T(0.5) * gm1;
    const T r = U[0], ru = U[1], rv = U[2], rw = U[3], rE = U[4];
    const T ir = T(1.0) / r;
    const T u = ru * ir, v = rv * ir, w = rw * ir;
    T p = u * ru;
    p = fma(v, rv, p);
    p = fma(w, rw, p);
    p = m5g * p;
    p = fma(gm1, rE, p);
    F[0][0] = ru; F[1][0] = rv; F[2][0] = rw;
    F[0][1] = fma(ru, u, p); F[1][1] = ru * v;        F[2][1] = ru * w;
    F[0][2] = rv * u;        F[1][2] = fma(rv, v, p); F[2][2] = rv * w;
    F[0][3] = rw * u;        F[1][3] = rw * v;        F[2][3] = fma(rw, w, p);
    const T e = rE + p;
    F[0][4] = u * e; F[1][4] = v * e; F[2][4] = w * e;
  } else {  // shallow water, geopotential form
    const T phi = U[0], uphi = U[1], vphi = U[2];
    const T iphi = T(1.0) / phi;
    const T u = uphi * iphi, v = vphi * iphi;
    const T p = T(0.5) * (phi * phi);
    F[0][0] = uphi;            F[1][0] = vphi;
    F[0][1] = fma(uphi, u, p); F[1][1] = uphi * v;
    F[0][2] = vphi * u;        F[1][2] = fma(vphi, v, p);
  }
}

// Flux-vector splittings of Euler::convective_flux (src/Euler.cpp:577-680)
// for one face-frame state (rho, u normal, v tangential, H): the positive
// part (plus) of the master state or the negative part of the slave state.
// Steger-Warming: eigenvalues u-a, u, u+a clipped at zero.
template <class T>
__device__ __forceinline__ void steger_warming_split(T r, T u, T v, T H, T gamma, bool plus, T *F) {
  const T gm1 = gamma - T(1.0);
  const T a = sqrt(gm1 * (H - T(0.5) * (u * u + v * v)));
  const T l0 = plus ? fmax(u - a, T(0.0)) : fmin(u - a, T(0.0));
  const T l1 = plus ? fmax(u, T(0.0)) : fmin(u, T(0.0));
  const T l3 = plus ? fmax(u + a, T(0.0)) : fmin(u + a, T(0.0));
  const T c1 = T(0.5) * r / gamma, c2 = T(2.0) * gm1;
  F[0] = c1 * (l0 + c2 * l1 + l3);
  F[1] = c1 * ((u - a) * l0 + c2 * u * l1 + (u + a) * l3);
  F[2] = c1 * (v * l0 + c2 * v * l1 + v * l3);
  F[3] = c1 * ((H - u * a) * l0 + gm1 * (u * u + v * v) * l1 + (H + u * a) * l3);
}
// van Leer: Mach-number polynomials (the subsonic branch, as the reference
// evaluates them at every Mach number).
template <class T>
__device__ __forceinline__ void van_leer_split(T r, T u, T v, T H, T gamma, bool plus, T *F) {
  const T gm1 = gamma - T(1.0);
  const T a = sqrt(gm1 * (H - T(0.5) * (u * u + v * v)));
  const T M = u / a;
  T c1, c2;
  if (plus) { c1 = T(0.25) * r * a * (T(1.0) + M) * (T(1.0) + M); c2 = T(0.5) * gm1 * M + T(1.0); }
  else { c1 = T(-0.25) * r * a * (T(1.0) - M) * (T(1.0) - M); c2 = T(0.5) * gm1 * M - T(1.0); }
  F[0] = c1;
  F[1] = plus ? c1 * T(2.0) * a * (T(1.0) / gamma) * c2 : c1 * T(2.0) * a / gamma * c2;
  F[2] = c1 * v;
  F[3] = c1 * (T(2.0) * a * a / (gamma * gamma - T(1.0)) * c2 * c2 + T(0.5) * v * v);
}

// Numerical flux on one face point in the frame of the master side:
// UL = master state, UR = slave state, n = master outward normal.
// Outputs Fh (numerical flux), FL = F(UL).n, FR = F(UR).n.
// Returns false if density or pressure is below aepsM.
// Euler 2-D: src/Euler.cpp:443-741 (LF and Roe); Euler 3-D:
// src/Euler3d.cpp:601-816 (LF) plus the rotated-frame Roe extension;
// shallow water: src/Shallow.cpp:380-510.
template <int PHYS, class T>
__device__ __forceinline__ bool face_flux(const T *UL, const T *UR, const T *n, T gamma,
                                          int flux, T *Fh, T *FL, T *FR, const double *frame = nullptr) {
  bool ok = true;
  if constexpr (PHYS == DGMX_EULER2D || PHYS == DGMX_NS2D) {
    const T gm1 = gamma - T(1.0);
    const T nx = n[0], ny = n[1];
    const T rl = UL[0], rul = UL[1] * nx + UL[2] * ny, rvl = UL[2] * nx - UL[1] * ny, rEl = UL[3];
    const T irl = T(1.0) / rl, ul = irl * rul, vl = irl * rvl;
    const T pl = gm1 * (rEl - T(0.5) * (rul * ul + rvl * vl));
    const T Hl = irl * (rEl + pl);
    ok = ok && rl >= T(kAeps) && pl >= T(kAeps);
    FL[0] = rul;
    FL[1] = (rul * ul + pl) * nx - (rvl * ul) * ny;
    FL[2] = (rul * ul + pl) * ny + (rvl * ul) * nx;
    FL[3] = ul * (rEl + pl);
    const T rr = UR[0], rur = UR[1] * nx + UR[2] * ny, rvr = UR[2] * nx - UR[1] * ny, rEr = UR[3];
    const T irr = T(1.0) / rr, ur = irr * rur, vr = irr * rvr;
    const T pr = gm1 * (rEr - T(0.5) * (rur * ur + rvr * vr));
    const T Hr = irr * (rEr + pr);
    ok = ok && rr >= T(kAeps) && pr >= T(kAeps);
    FR[0] = rr * ur;
    FR[1] = (rur * ur + pr) * nx - (rvr * ur) * ny;
    FR[2] = (rur * ur + pr) * ny + (rvr * ur) * nx;
    FR[3] = ur * (rEr + pr);
    if (flux == DGMX_FLUX_ROE) {
      const T R = sqrt(rr / rl), iRp1 = T(1.0) / (T(1.0) + R);
      const T u = (ul + R * ur) * iRp1, v = (vl + R * vr) * iRp1, H = (Hl + R * Hr) * iRp1;
      const T a = sqrt(gm1 * (H - T(0.5) * (u * u + v * v)));
      const T ainv = T(1.0) / a, c1inv = T(1.0) / (gm1 * ainv * ainv);
      T al[4], G[4];
      al[2] = (rvr - rvl) - v * (rr - rl);
      al[1] = gm1 * ainv * ainv * ((rr - rl) * (H - u * u) + u * (rur - rul) -
                                   ((rEr - rEl) - ((rvr - rvl) - v * (rr - rl)) * v));
      al[0] = T(0.5) * ainv * ((rr - rl) * (u + a) - (rur - rul) - a * al[1]);
      al[3] = (rr - rl) - (al[0] + al[1]);
      const T l0 = fmin(u - a, T(0.0)), l1 = fmin(u, T(0.0)), l3 = fmin(u + a, T(0.0));
      G[0] = l0 * al[0]; G[1] = l0 * (u - a) * al[0]; G[2] = l0 * v * al[0]; G[3] = l0 * (H - u * a) * al[0];
      G[0] += l1 * al[1]; G[1] += l1 * u * al[1]; G[2] += l1 * v * al[1]; G[3] += l1 * (H - c1inv) * al[1];
      G[2] += l1 * al[2]; G[3] += l1 * v * al[2];
      G[0] += l3 * al[3]; G[1] += l3 * (u + a) * al[3]; G[2] += l3 * v * al[3]; G[3] += l3 * (H + u * a) * al[3];
      Fh[0] = FL[0] + G[0];
      Fh[1] = FL[1] + G[1] * nx - G[2] * ny;
      Fh[2] = FL[2] + G[1] * ny + G[2] * nx;
      Fh[3] = FL[3] + G[3];
    } else if (flux == DGMX_FLUX_STEGER_WARMING || flux == DGMX_FLUX_VAN_LEER) {
      // flux-vector splitting in the face frame, F+(UL) + F-(UR), rotated back
      T P[4], M[4];
      if (flux == DGMX_FLUX_STEGER_WARMING) {
        steger_warming_split<T>(rl, ul, vl, Hl, gamma, true, P);
        steger_warming_split<T>(rr, ur, vr, Hr, gamma, false, M);
      } else {
        van_leer_split<T>(rl, ul, vl, Hl, gamma, true, P);
        van_leer_split<T>(rr, ur, vr, Hr, gamma, false, M);
      }
      const T G0 = P[0] + M[0], G1 = P[1] + M[1], G2 = P[2] + M[2], G3 = P[3] + M[3];
      Fh[0] = G0;
      Fh[1] = G1 * nx - G2 * ny;
      Fh[2] = G1 * ny + G2 * nx;
      Fh[3] = G3;
    } else {
      const T al = sqrt(gm1 * (Hl - T(0.5) * (ul * ul + vl * vl)));
      const T ar = sqrt(gm1 * (Hr - T(0.5) * (ur * ur + vr * vr)));
      T lmax = fmax(fabs(ul - al), fabs(ul));
      lmax = fmax(lmax, fabs(ul + al));
      lmax = fmax(lmax, fmax(fabs(ur - ar), fabs(ur)));
      lmax = fmax(lmax, fabs(ur + ar));
#pragma unroll
      for (int k = 0; k < 4; ++k) Fh[k] = T(0.5) * (FL[k] + FR[k] + lmax * (UL[k] - UR[k]));
    }
  } else if constexpr (PHYS == DGMX_EULER3D || PHYS == DGMX_NS3D) {
    const T gm1 = gamma - T(1.0);
    const T nx = n[0], ny = n[1], nz = n[2];
    // the face frame: precomputed per geometry class (face_frame), or here
    T sx, sy, sz, tx, ty, tz, xn, yn, zn, xs, ys, zs, xt, yt, zt;
    if (frame) {
      sx = T(frame[0]); sy = T(frame[1]); sz = T(frame[2]);
      tx = T(frame[3]); ty = T(frame[4]); tz = T(frame[5]);
      xn = T(frame[6]); yn = T(frame[7]); zn = T(frame[8]);
      xs = T(frame[9]); ys = T(frame[10]); zs = T(frame[11]);
      xt = T(frame[12]); yt = T(frame[13]); zt = T(frame[14]);
    } else {
      sx = ny; sy = nz; sz = nx;
      const T sdn = nx * sx + ny * sy + nz * sz;
      sx -= sdn * nx; sy -= sdn * ny; sz -= sdn * nz;
      const T sni = T(1.0) / sqrt(sx * sx + sy * sy + sz * sz);
      sx *= sni; sy *= sni; sz *= sni;
      tx = ny * sz - sy * nz; ty = nz * sx - sz * nx; tz = nx * sy - sx * ny;
      const T tni = T(1.0) / sqrt(tx * tx + ty * ty + tz * tz);
      tx *= tni; ty *= tni; tz *= tni;
      const T detA = (nx * sy * tz + sx * ty * nz + tx * sz * ny) - (nz * sy * tx + sz * ty * nx + tz * sx * ny);
      const T id = T(1.0) / detA;
      xn = (sy * tz - sz * ty) * id; yn = -(sx * tz - sz * tx) * id; zn = (sx * ty - sy * tx) * id;
      xs = -(ny * tz - nz * ty) * id; ys = (nx * tz - nz * tx) * id; zs = -(nx * ty - ny * tx) * id;
      xt = (ny * sz - nz * sy) * id; yt = -(nx * sz - nz * sx) * id; zt = (nx * sy - ny * sx) * id;
    }
    const T rl = UL[0];
    const T rul = UL[1] * nx + UL[2] * ny + UL[3] * nz;
    const T rvl = UL[1] * sx + UL[2] * sy + UL[3] * sz;
    const T rwl = UL[1] * tx + UL[2] * ty + UL[3] * tz;
    const T rEl = UL[4];
    const T irl = T(1.0) / rl, ul = irl * rul, vl = irl * rvl, wl = irl * rwl;
    const T pl = gm1 * (rEl - T(0.5) * (rul * ul + rvl * vl + rwl * wl));
    const T Hl = irl * (rEl + pl);
    ok = ok && rl >= T(kAeps) && pl >= T(kAeps);
    FL[0] = rl * ul;
    FL[1] = (rul * ul + pl) * xn + (rvl * ul) * xs + (rwl * ul) * xt;
    FL[2] = (rul * ul + pl) * yn + (rvl * ul) * ys + (rwl * ul) * yt;
    FL[3] = (rul * ul + pl) * zn + (rvl * ul) * zs + (rwl * ul) * zt;
    FL[4] = ul * (rEl + pl);
    const T rr = UR[0];
    const T rur = UR[1] * nx + UR[2] * ny + UR[3] * nz;
    const T rvr = UR[1] * sx + UR[2] * sy + UR[3] * sz;
    const T rwr = UR[1] * tx + UR[2] * ty + UR[3] * tz;
    const T rEr = UR[4];
    const T irr = T(1.0) / rr, ur = irr * rur, vr = irr * rvr, wr = irr * rwr;
    const T pr = gm1 * (rEr - T(0.5) * (rur * ur + rvr * vr + rwr * wr));
    const T Hr = irr * (rEr + pr);
    ok = ok && rr >= T(kAeps) && pr >= T(kAeps);
    FR[0] = rr * ur;
    FR[1] = (rur * ur + pr) * xn + (rvr * ur) * xs + (rwr * ur) * xt;
    FR[2] = (rur * ur + pr) * yn + (rvr * ur) * ys + (rwr * ur) * yt;
    FR[3] = (rur * ur + pr) * zn + (rvr * ur) * zs + (rwr * ur) * zt;
    FR[4] = ur * (rEr + pr);
    if (flux == DGMX_FLUX_ROE) {
      // Roe average in the (n, s, t) frame; the 2-D Roe of src/Euler.cpp
      // with a second tangential velocity carried like the first.
      const T R = sqrt(rr / rl), iRp1 = T(1.0) / (T(1.0) + R);
      const T u = (ul + R * ur) * iRp1, v = (vl + R * vr) * iRp1, w = (wl + R * wr) * iRp1;
      const T H = (Hl + R * Hr) * iRp1;
      const T a2 = gm1 * (H - T(0.5) * (u * u + v * v + w * w));
      const T a = sqrt(a2), ainv = T(1.0) / a, c1inv = a2 / gm1;
      const T dr = rr - rl, dru = rur - rul, drv = rvr - rvl, drw = rwr - rwl, drE = rEr - rEl;
      T al[5], G[5];
      al[2] = drv - v * dr;
      al[3] = drw - w * dr;
      al[1] = gm1 * ainv * ainv * (dr * (H - u * u) + u * dru - ((drE - al[2] * v - al[3] * w)));
      al[0] = T(0.5) * ainv * (dr * (u + a) - dru - a * al[1]);
      al[4] = dr - (al[0] + al[1]);
      const T l0 = fmin(u - a, T(0.0)), l1 = fmin(u, T(0.0)), l4 = fmin(u + a, T(0.0));
      G[0] = l0 * al[0]; G[1] = l0 * (u - a) * al[0]; G[2] = l0 * v * al[0]; G[3] = l0 * w * al[0];
      G[4] = l0 * (H - u * a) * al[0];
      G[0] += l1 * al[1]; G[1] += l1 * u * al[1]; G[2] += l1 * v * al[1]; G[3] += l1 * w * al[1];
      G[4] += l1 * (H - c1inv) * al[1];
      G[2] += l1 * al[2]; G[4] += l1 * v * al[2];
      G[3] += l1 * al[3]; G[4] += l1 * w * al[3];
      G[0] += l4 * al[4]; G[1] += l4 * (u + a) * al[4]; G[2] += l4 * v * al[4]; G[3] += l4 * w * al[4];
      G[4] += l4 * (H + u * a) * al[4];
      Fh[0] = FL[0] + G[0];
      Fh[1] = FL[1] + G[1] * xn + G[2] * xs + G[3] * xt;
      Fh[2] = FL[2] + G[1] * yn + G[2] * ys + G[3] * yt;
      Fh[3] = FL[3] + G[1] * zn + G[2] * zs + G[3] * zt;
      Fh[4] = FL[4] + G[4];
    } else {
      const T al = sqrt(gm1 * (Hl - T(0.5) * (ul * ul + vl * vl + wl * wl)));
      const T ar = sqrt(gm1 * (Hr - T(0.5) * (ur * ur + vr * vr + wr * wr)));
      T lmax = fmax(fabs(ul - al), fabs(ul));
      lmax = fmax(lmax, fabs(ul + al));
      lmax = fmax(lmax, fmax(fabs(ur - ar), fabs(ur)));
      lmax = fmax(lmax, fabs(ur + ar));
#pragma unroll
      for (int k = 0; k < 5; ++k) Fh[k] = T(0.5) * (FL[k] + FR[k] + lmax * (UL[k] - UR[k]));
    }
  } else {  // shallow water LF
    const T nx = n[0], ny = n[1];
    const T phil = UL[0], upl = UL[1] * nx + UL[2] * ny, vpl = UL[2] * nx - UL[1] * ny;
    const T ul = upl / phil, pl = T(0.5) * phil * phil;
    ok = ok && phil >= T(kAeps) && pl >= T(kAeps);
    FL[0] = upl;
    FL[1] = (upl * ul + pl) * nx - (vpl * ul) * ny;
    FL[2] = (upl * ul + pl) * ny + (vpl * ul) * nx;
    const T phir = UR[0], upr = UR[1] * nx + UR[2] * ny, vpr = UR[2] * nx - UR[1] * ny;
    const T ur = upr / phir, pr = T(0.5) * phir * phir;
    ok = ok && phir >= T(kAeps) && pr >= T(kAeps);
    FR[0] = upr;
    FR[1] = (upr * ur + pr) * nx - (vpr * ur) * ny;
    FR[2] = (upr * ur + pr) * ny + (vpr * ur) * nx;
    const T al = sqrt(phil), ar = sqrt(phir);
    T lmax = fmax(fabs(ul - al), fabs(ul));
    lmax = fmax(lmax, fabs(ul + al));
    lmax = fmax(lmax, fmax(fabs(ur - ar), fabs(ur)));
    lmax = fmax(lmax, fabs(ur + ar));
#pragma unroll
    for (int k = 0; k < 3; ++k) Fh[k] = T(0.5) * (FL[k] + FR[k] + lmax * (UL[k] - UR[k]));
  }
  return ok;
}

// ---- perturbation form (FP32 working precision) ----------------------------
// The mixed form splits every state as U = Ub + d, Ub a constant reference
// state of the solve, and evaluates F(Ub + d) - F(Ub).  The derivative of
// that difference equals the derivative of F, and its jump across a face
// equals the jump of F, so the scheme is unchanged algebraically; but it is
// formed from products that each carry a perturbation factor, so its FP32
// rounding error scales with |d| instead of |U| (at Mach 0.1 the pressure
// is ~70x the dynamic part).  Euler: with u' = (m' - ub rho')/rho,
//   p' = (g-1)(E' - (m'.ub + m.u')/2),  F'_rho = m',
//   F'_m = m' ub_d + m u'_d + p' e_d,   F'_E = H' ub_d + H u'_d  (H = E + p);
// shallow water: p' = phi'(phi_b + phi'/2) for the phi^2/2 pressure.
// Reciprocal, square root and reciprocal square root of the perturbation
// fluxes: the hardware approximations in FP32 (a few ulp, well inside the
// FP32 form's error, which its rounding of U sets), the correctly rounded
// operations in FP64.
template <class T> __device__ __forceinline__ T p_rcp(T x) { return T(1) / x; }
template <> __device__ __forceinline__ float p_rcp<float>(float x) { return __fdividef(1.0f, x); }
template <class T> __device__ __forceinline__ T p_sqrt(T x) { return sqrt(x); }
template <> __device__ __forceinline__ float p_sqrt<float>(float x) {
  float y;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
template <class T> __device__ __forceinline__ T p_rsqrt(T x) { return T(1) / sqrt(x); }
template <> __device__ __forceinline__ float p_rsqrt<float>(float x) { return rsqrtf(x); }

// F(Ub + d) - F(Ub) in every direction (volume term).
template <int PHYS, class T>
__device__ __forceinline__ void volume_flux_pert(const RefState<T> &b, const T *d, T gamma, T (*F)[5]) {
  constexpr bool SW = PHYS == DGMX_SHALLOW;
  constexpr int DIM = (PHYS == DGMX_EULER3D || PHYS == DGMX_NS3D) ? 3 : 2, NF = SW ? 3 : DIM + 2;
  const T rho = b.r + d[0], ir = p_rcp(rho);
  T m[3], up[3];
#pragma unroll
  for (int i = 0; i < DIM; ++i) { m[i] = b.m[i] + d[1 + i]; up[i] = (d[1 + i] - b.u[i] * d[0]) * ir; }
  T pp, Hp = T(0), H = T(0);
  if constexpr (SW) {
    pp = d[0] * fma(T(0.5), d[0], b.r);
  } else {
    T s = T(0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) { s = fma(d[1 + i], b.u[i], s); s = fma(m[i], up[i], s); }
    pp = (gamma - T(1.0)) * fma(T(-0.5), s, d[NF - 1]);
    Hp = d[NF - 1] + pp;
    H = b.H + Hp;
  }
#pragma unroll
  for (int k = 0; k < DIM; ++k) {
    F[k][0] = d[1 + k];
#pragma unroll
    for (int i = 0; i < DIM; ++i) F[k][1 + i] = fma(d[1 + i], b.u[k], m[i] * up[k]) + (i == k ? pp : T(0));
    if constexpr (!SW) F[k][NF - 1] = fma(Hp, b.u[k], H * up[k]);
  }
}

// Normal component of F(Ub + d) - F(Ub) plus the full state's normal
// velocity, sound speed (sqrt(phi) for shallow water) and realizability.
template <int PHYS, class T>
__device__ __forceinline__ bool normal_flux_pert(const RefState<T> &b, const T *d, const T *n, T gamma, T *Fn,
                                                 T &rho, T &un, T &c, T *vel, T &Hs) {
  constexpr bool SW = PHYS == DGMX_SHALLOW;
  constexpr int DIM = (PHYS == DGMX_EULER3D || PHYS == DGMX_NS3D) ? 3 : 2, NF = SW ? 3 : DIM + 2;
  rho = b.r + d[0];
  const T ir = p_rcp(rho);
  T m[3], up[3], ubn = T(0), upn = T(0), mpn = T(0);
#pragma unroll
  for (int i = 0; i < DIM; ++i) {
    m[i] = b.m[i] + d[1 + i];
    up[i] = (d[1 + i] - b.u[i] * d[0]) * ir;
    vel[i] = b.u[i] + up[i];
    ubn = fma(b.u[i], n[i], ubn);
    upn = fma(up[i], n[i], upn);
    mpn = fma(d[1 + i], n[i], mpn);
  }
  un = ubn + upn;
  T pp, p;
  if constexpr (SW) {
    pp = d[0] * fma(T(0.5), d[0], b.r);
    p = T(0.5) * rho * rho;
    c = p_sqrt(rho);
    Hs = T(0);
  } else {
    T s = T(0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) { s = fma(d[1 + i], b.u[i], s); s = fma(m[i], up[i], s); }
    pp = (gamma - T(1.0)) * fma(T(-0.5), s, d[NF - 1]);
    p = b.p + pp;
    const T Hp = d[NF - 1] + pp, H = b.H + Hp;
    Fn[NF - 1] = fma(Hp, ubn, H * upn);
    Hs = H * ir;                                   // total enthalpy per unit mass
    c = p_sqrt(gamma * fmax(p, T(0)) * ir);
  }
  Fn[0] = mpn;
#pragma unroll
  for (int i = 0; i < DIM; ++i) Fn[1 + i] = fma(d[1 + i], ubn, m[i] * upn) + pp * n[i];
  return rho >= T(kAeps) && p >= T(kAeps);
}

// Face flux in perturbation form, in the master's frame: dl = master-side
// perturbation, dr = slave side, n = master normal.  Returns
// Dm = F^ - F(UL).n and DF = F(UR).n - F(UL).n, which is all the lift needs
// (master: Dm, slave: DF - Dm).  Lax-Friedrichs as src/Euler3d.cpp:601-816
// and src/Shallow.cpp:380-510; Roe as src/Euler.cpp:682-741 (rotated to the
// face frame in 3-D), its upwind dissipation formed from the state jump.
template <int PHYS, class T>
__device__ __forceinline__ bool face_flux_pert(const RefState<T> &b, const T *dl, const T *dr, const T *n,
                                               T gamma, int flux, T *Dm, T *DF, const double *frame = nullptr) {
  constexpr bool SW = PHYS == DGMX_SHALLOW;
  constexpr int DIM = (PHYS == DGMX_EULER3D || PHYS == DGMX_NS3D) ? 3 : 2, NF = SW ? 3 : DIM + 2;
  T FL[5], FR[5], rl, rr, ul, ur, cl, cr, vl[3], vr[3], Hl, Hr;
  bool ok = normal_flux_pert<PHYS, T>(b, dl, n, gamma, FL, rl, ul, cl, vl, Hl);
  ok = normal_flux_pert<PHYS, T>(b, dr, n, gamma, FR, rr, ur, cr, vr, Hr) && ok;
  T dU[5];
#pragma unroll
  for (int k = 0; k < NF; ++k) { DF[k] = FR[k] - FL[k]; dU[k] = dr[k] - dl[k]; }
  if constexpr (!SW) {
    if (flux == DGMX_FLUX_ROE) {
      const T gm1 = gamma - T(1.0);
      // face frame: n, s (and t in 3-D)
      T s[3], t[3] = {T(0), T(0), T(0)};
      if constexpr (DIM == 2) {
        s[0] = -n[1]; s[1] = n[0]; s[2] = T(0);
      } else if (frame) {
        for (int k = 0; k < 3; ++k) { s[k] = T(frame[k]); t[k] = T(frame[3 + k]); }
      } else {
        s[0] = n[1]; s[1] = n[2]; s[2] = n[0];
        const T sdn = n[0] * s[0] + n[1] * s[1] + n[2] * s[2];
        s[0] -= sdn * n[0]; s[1] -= sdn * n[1]; s[2] -= sdn * n[2];
        const T sni = p_rsqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
        s[0] *= sni; s[1] *= sni; s[2] *= sni;
        t[0] = n[1] * s[2] - s[1] * n[2]; t[1] = n[2] * s[0] - s[2] * n[0]; t[2] = n[0] * s[1] - s[0] * n[1];
        const T tni = p_rsqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        t[0] *= tni; t[1] *= tni; t[2] *= tni;
      }
      T vsl = T(0), vsr = T(0), vtl = T(0), vtr = T(0), dms = T(0), dmt = T(0), dmn = T(0);
#pragma unroll
      for (int i = 0; i < DIM; ++i) {
        vsl = fma(vl[i], s[i], vsl); vsr = fma(vr[i], s[i], vsr);
        vtl = fma(vl[i], t[i], vtl); vtr = fma(vr[i], t[i], vtr);
        dmn = fma(dU[1 + i], n[i], dmn); dms = fma(dU[1 + i], s[i], dms); dmt = fma(dU[1 + i], t[i], dmt);
      }
      const T R = p_sqrt(rr * p_rcp(rl)), iRp1 = p_rcp(T(1.0) + R);
      const T u = (ul + R * ur) * iRp1, v = (vsl + R * vsr) * iRp1, w = (vtl + R * vtr) * iRp1;
      const T H = (Hl + R * Hr) * iRp1;
      const T a2 = gm1 * (H - T(0.5) * (u * u + v * v + w * w));
      const T ainv = p_rsqrt(a2), a = a2 * ainv, c1inv = a2 * p_rcp(gm1);
      const T d0 = dU[0], dE = dU[NF - 1];
      T al[5];
      al[2] = dms - v * d0;
      al[3] = dmt - w * d0;
      al[1] = gm1 * ainv * ainv * (d0 * (H - u * u) + u * dmn - (dE - al[2] * v - al[3] * w));
      al[0] = T(0.5) * ainv * (d0 * (u + a) - dmn - a * al[1]);
      al[4] = d0 - (al[0] + al[1]);
      const T l0 = fmin(u - a, T(0.0)), l1 = fmin(u, T(0.0)), l4 = fmin(u + a, T(0.0));
      T G0 = l0 * al[0], Gn = l0 * (u - a) * al[0], Gs = l0 * v * al[0], Gt = l0 * w * al[0];
      T GE = l0 * (H - u * a) * al[0];
      G0 += l1 * al[1]; Gn += l1 * u * al[1]; Gs += l1 * v * al[1]; Gt += l1 * w * al[1];
      GE += l1 * (H - c1inv) * al[1];
      Gs += l1 * al[2]; GE += l1 * v * al[2];
      Gt += l1 * al[3]; GE += l1 * w * al[3];
      G0 += l4 * al[4]; Gn += l4 * (u + a) * al[4]; Gs += l4 * v * al[4]; Gt += l4 * w * al[4];
      GE += l4 * (H + u * a) * al[4];
      Dm[0] = G0;
#pragma unroll
      for (int i = 0; i < DIM; ++i) Dm[1 + i] = Gn * n[i] + Gs * s[i] + Gt * t[i];
      Dm[NF - 1] = GE;
      return ok;
    }
  }
  const T lmax = fmax(fabs(ul) + cl, fabs(ur) + cr);
#pragma unroll
  for (int k = 0; k < NF; ++k) Dm[k] = T(0.5) * (DF[k] - lmax * dU[k]);
  return ok;
}

}  // namespace dgmx
