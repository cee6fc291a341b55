// One persistent stage kernel for every 2-D arena of an element pool.
//
// A pool keeps the solves of each (physics, p, q) in an arena of its own;
// the plain pool path launches one persistent stage kernel per arena and
// stage.  Here the 2-D arenas (Euler 2-D and shallow water, p = 1..7,
// q = p + 2) share ONE launch per LSRK stage: the kernel walks a device-side
// list of (arena, tile) work items and runs, for each, the fused stage body
// (stage_tile, stage.cuh) compiled for that arena's (physics, p, q) at a
// common launch shape of 128 threads per CTA.  The body of a work item is a
// CTA-uniform branch, so a launch mixes orders freely; per element the
// arithmetic is that of the body alone (each pencil's operations and their
// order do not depend on the thread count), so a solve's result is the same
// in either path.  Included by one compilation unit per working precision.
#pragma once

#include "dispatch.cuh"

namespace dgmx {

constexpr int kFusedBodies = 14;   // Euler 2-D p = 1..7, shallow water p = 1..7
constexpr int kFusedThreads = 128;
// CTAs per SM the register allocation is held to (the bodies of the largest
// orders spill a little at this cap; the small orders gain the occupancy)
constexpr int kFusedMinBlocks64 = 7, kFusedMinBlocksMixed = 8;

template <bool MIXED, int B>
struct FusedCfg {
  static constexpr int PHYS = B < 7 ? DGMX_EULER2D : DGMX_SHALLOW;
  static constexpr int P = B % 7 + 1, L = P + 1, Q = P + 2;
  static constexpr int EPB = default_epb(2, Q);
  using C = Cfg<PHYS, L, Q, EPB, 0, MIXED, kFusedThreads>;
};

template <bool MIXED, int B = 0>
constexpr size_t fused_smem() {
  if constexpr (B < kFusedBodies) {
    constexpr size_t here = FusedCfg<MIXED, B>::C::SMEM, rest = fused_smem<MIXED, B + 1>();
    return here > rest ? here : rest;
  } else {
    return 0;
  }
}

template <bool MIXED, int B = 0>
__device__ __forceinline__ void fused_dispatch(int body, unsigned char *raw, const StageArgs &a, int tile,
                                               int tid) {
  if constexpr (B < kFusedBodies) {
    if (body == B) {
      using F = FusedCfg<MIXED, B>;
      Smem<typename F::C> sm(raw);
      stage_tile<typename F::C, F::PHYS>(sm, a, tile * F::EPB, tid);
    } else {
      fused_dispatch<MIXED, B + 1>(body, raw, a, tile, tid);
    }
  }
}

// args: [stage][arena] stage arguments; bodies[arena]: body index;
// items[0 .. *nitems): (arena, tile) pairs.
template <bool MIXED>
__global__ void __launch_bounds__(kFusedThreads, MIXED ? kFusedMinBlocksMixed : kFusedMinBlocks64) fused_stage_kernel(const StageArgs *args, int narena,
                                                                       const int *bodies, const int2 *items,
                                                                       const int *nitems, int stage) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = *nitems;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    if (t != (int)blockIdx.x) __syncthreads();
    const int2 it = items[t];
    fused_dispatch<MIXED>(bodies[it.x], smem_raw, args[(size_t)stage * narena + it.x], it.y, threadIdx.x);
  }
}

// Constant tables of every body's (L, Q) in this compilation unit's module
// (the two physics share them).
template <bool MIXED, int B = 0>
static cudaError_t fused_upload() {
  if constexpr (B < 7) {
    using F = FusedCfg<MIXED, B>;
    const cudaError_t e = upload_tables_lq<F::L, F::Q, typename F::C::R>(make_tables(F::L, F::Q, F::Q - 1));
    if (e != cudaSuccess) return e;
    return fused_upload<MIXED, B + 1>();
  } else {
    return cudaSuccess;
  }
}

template <bool MIXED, int B = 0>
constexpr int fused_epb(int body) {
  if constexpr (B < kFusedBodies) return body == B ? FusedCfg<MIXED, B>::EPB : fused_epb<MIXED, B + 1>(body);
  else return 1;
}

template <bool MIXED>
struct FusedHost {
  static cudaError_t init() {
    cudaError_t e = fused_upload<MIXED>();
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(fused_stage_kernel<MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fused_smem<MIXED>());
  }
  static int blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fused_stage_kernel<MIXED>, kFusedThreads,
                                                      fused_smem<MIXED>()) != cudaSuccess) {
      cudaGetLastError();
      return 1;
    }
    return n > 0 ? n : 1;
  }
  static cudaError_t launch(const StageArgs *args, int narena, const int *bodies, const int2 *items,
                            const int *nitems, int stage, int grid, cudaStream_t s) {
    fused_stage_kernel<MIXED><<<grid, kFusedThreads, fused_smem<MIXED>(), s>>>(args, narena, bodies, items,
                                                                               nitems, stage);
    return cudaGetLastError();
  }
};

}  // namespace dgmx
