// Bulk-flow hold of the Navier-Stokes 3-D channel (Channel::holdBulkMassFlow,
// src/Channel.hpp:116-163): after the projected right-hand side F is formed,
// the volume means of its density, x-momentum and energy components are
// subtracted from every point (src/Navier_Stokes3d.cpp:160).
//
// In the orthonormal modal basis the mean of a projected field is carried by
// its constant mode alone: with phi0 = 2^(-3/2) the value of that mode,
//   mean(F_n) = phi0 * sum_e J_e c0_e(F_n) / sum_e J_e,
// and subtracting the mean from every point is subtracting cbar_n =
// sum_e J_e c0_e / sum_e J_e from every element's constant coefficient.
//
// The stage kernel updates its registers with the unheld F and writes each
// element's constant coefficients (StageArgs::R0); these two kernels then
// form cbar (one block, fixed summation order, so the result does not depend
// on scheduling) and apply the update's linear response to -cbar on the
// constant coefficients of the registers it wrote and on the traces of the
// next stage's state (a constant shift of every trace point).
#include "dgmx_internal.hpp"

namespace dgmx {
namespace {

constexpr int kHoldThreads = 256;

__device__ __forceinline__ bool held(int n, int nf) { return n == 0 || n == 1 || n == nf - 1; }

__global__ void __launch_bounds__(kHoldThreads) hold_reduce_kernel(HoldArgs h) {
  __shared__ double part[kHoldThreads][6];
  const int tid = threadIdx.x;
  double acc[5] = {0, 0, 0, 0, 0}, vol = 0.0;
  for (int e = tid; e < h.ne; e += kHoldThreads) {
    const double J = h.J[e];
    for (int n = 0; n < h.nf; ++n) acc[n] = fma(J, h.R0[(size_t)e * h.nf + n], acc[n]);
    vol += J;
  }
  for (int n = 0; n < 5; ++n) part[tid][n] = acc[n];
  part[tid][5] = vol;
  __syncthreads();
  for (int w = kHoldThreads / 2; w > 0; w >>= 1) {
    if (tid < w)
      for (int k = 0; k < 6; ++k) part[tid][k] += part[tid + w][k];
    __syncthreads();
  }
  if (tid < h.nf) h.cbar[tid] = held(tid, h.nf) ? part[0][tid] / part[0][5] : 0.0;
}

__global__ void __launch_bounds__(kHoldThreads) hold_apply_kernel(HoldArgs h) {
  const double phi0 = 0.35355339059327373;   // 2^(-3/2)
  const size_t per_e = (size_t)h.nf + (size_t)h.nfaces * h.nf * h.gf + (h.Fn ? (size_t)h.nf * h.qd : 0);
  const size_t total = (size_t)h.ne * per_e;
  for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (size_t)gridDim.x * blockDim.x) {
    const int e = (int)(w / per_e);
    size_t r = w - (size_t)e * per_e;
    if (r < (size_t)h.nf) {
      // constant coefficients of the registers the stage wrote
      const int n = (int)r;
      if (!held(n, h.nf)) continue;
      const double cb = h.cbar[n];
      const size_t g = ((size_t)e * h.nf + n) * h.ld;
      switch (h.kind) {
        case kLSRK: h.Ut[g] += h.dt * cb; h.U[g] += h.c1 * (h.dt * cb); break;
        case kTVD0: h.Ut[g] += h.dt * cb; break;
        case kTVD1: h.Ut[g] += h.c1 * (h.dt * cb); break;
        case kTVD2: h.U[g] += h.c1 * (h.dt * cb); break;
        case kRK40:
        case kRK41: h.Ut[g] -= h.c0 * cb; h.A[g] -= h.c1 * cb; break;
        case kRK43: h.A[g] -= h.c1 * cb; h.U[g] -= h.c0 * (h.c1 * cb); break;
        case kRHS: if (h.A) h.A[g] -= cb; break;
        default: break;
      }
      continue;
    }
    r -= h.nf;
    const size_t nt = (size_t)h.nfaces * h.nf * h.gf;
    if (r < nt) {
      // traces of the next stage's state
      if (!h.Tout) continue;
      const int n = (int)((r / h.gf) % h.nf);
      if (!held(n, h.nf)) continue;
      const double cb = h.cbar[n];
      double d;
      switch (h.kind) {
        case kLSRK: d = h.c1 * (h.dt * cb); break;
        case kTVD0: d = h.dt * cb; break;
        case kTVD1:
        case kTVD2: d = h.c1 * (h.dt * cb); break;
        case kRK40:
        case kRK41: d = -h.c0 * cb; break;
        case kRK43: d = -h.c0 * (h.c1 * cb); break;
        default: d = 0.0; break;
      }
      h.Tout[(size_t)e * nt + r] += d * phi0;
      continue;
    }
    r -= nt;
    // nodal right-hand side (Domain::time_derivative path), Field layout
    const int n = (int)(r / h.qd), p = (int)(r - (size_t)n * h.qd);
    if (held(n, h.nf)) h.Fn[((size_t)n * h.ne + e) * h.qd + p] -= h.cbar[n] * phi0;
  }
}

__global__ void scatter_rows_kernel(const double *__restrict__ src, const int *__restrict__ gid, int n, int nf,
                                    double *__restrict__ dst) {
  const long long total = (long long)n * nf;
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(w / nf), k = (int)(w - (long long)i * nf);
    const int g = gid[i];
    if (g >= 0) dst[(size_t)g * nf + k] = src[w];
  }
}

}  // namespace

cudaError_t launch_hold_reduce(const HoldArgs &h, cudaStream_t s) {
  hold_reduce_kernel<<<1, kHoldThreads, 0, s>>>(h);
  return cudaGetLastError();
}

cudaError_t launch_hold_apply(const HoldArgs &h, cudaStream_t s) {
  hold_apply_kernel<<<4 * 148, kHoldThreads, 0, s>>>(h);
  return cudaGetLastError();
}

cudaError_t launch_hold(const HoldArgs &h, cudaStream_t s) {
  cudaError_t e = launch_hold_reduce(h, s);
  return e == cudaSuccess ? launch_hold_apply(h, s) : e;
}

cudaError_t launch_scatter_rows(const double *src, const int *gid, int n, int nf, double *dst, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const long long b = ((long long)n * nf + 255) / 256;
  scatter_rows_kernel<<<(int)(b < 4 * 148 ? b : 4 * 148), 256, 0, s>>>(src, gid, n, nf, dst);
  return cudaGetLastError();
}

}  // namespace dgmx
