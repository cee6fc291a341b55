// Launchers for one kernel instantiation and the registry hook used by the
// per-physics compilation units (k_*.cu).
#pragma once

#include "ns.cuh"
#include "pipeline.cuh"
#include "stage2.cuh"

namespace dgmx {

// Every k_*.cu is its own device module with its own copy of the __constant__
// tables, whose host shadows have internal linkage.  The uploader must have
// internal linkage too: an ordinary (weak) template instantiation would be
// merged across compilation units by the linker and write only one module's
// tables.
template <int L, int Q, class T>
static cudaError_t upload_tables_lq(const Tables1D &t) {
  auto put = [](const auto &sym, const std::vector<double> &v, size_t n) {
    std::vector<T> c(n);
    for (size_t i = 0; i < n; ++i) c[i] = T(v[i]);
    return cudaMemcpyToSymbol(sym, c.data(), sizeof(T) * n);
  };
  cudaError_t e;
  if ((e = put(cB<T, L, Q>, t.B, (size_t)L * Q)) != cudaSuccess) return e;
  if ((e = put(cBg<T, L, Q>, t.Bg, (size_t)L * (Q - 1))) != cudaSuccess) return e;
  if ((e = put(cD<T, L, Q>, t.D, (size_t)Q * Q)) != cudaSuccess) return e;
  if ((e = put(cG2GL<T, L, Q>, t.g2gl, (size_t)Q * (Q - 1))) != cudaSuccess) return e;
  if ((e = put(cGL2G<T, L, Q>, t.gl2g, (size_t)(Q - 1) * Q)) != cudaSuccess) return e;
  if ((e = put(cW<T, L, Q>, t.w, (size_t)Q)) != cudaSuccess) return e;
  std::vector<double> end(2 * L);
  for (int a = 0; a < L; ++a) { end[a] = t.B[a * Q + 0]; end[L + a] = t.B[a * Q + Q - 1]; }
  if ((e = put(cEnd<T, L, Q>, end, (size_t)2 * L)) != cudaSuccess) return e;
  // projection with the GLL weights folded in, and lift with 1/w_end folded in
  std::vector<double> bw((size_t)L * Q), gw((size_t)2 * Q * (Q - 1));
  for (int a = 0; a < L; ++a)
    for (int i = 0; i < Q; ++i) bw[(size_t)a * Q + i] = t.B[(size_t)a * Q + i] * t.w[i];
  for (int end_ = 0; end_ < 2; ++end_)
    for (size_t k = 0; k < (size_t)Q * (Q - 1); ++k) gw[end_ * Q * (Q - 1) + k] = t.g2gl[k] / t.w[end_ ? Q - 1 : 0];
  if ((e = put(cBw<T, L, Q>, bw, (size_t)L * Q)) != cudaSuccess) return e;
  return put(cG2GLw<T, L, Q>, gw, (size_t)2 * Q * (Q - 1));
}

// Tables of the second-form stage kernel (only its compilation unit
// instantiates them: constant memory is 64 KB per module): the weighted
// derivative E = B W D and the lift-projection BwG = B W G2GL (L rows each).
template <int L, int Q, class T>
static cudaError_t upload_tables2_lq(const Tables1D &t) {
  std::vector<T> e2((size_t)L * Q), bwg((size_t)L * (Q - 1));
  for (int a = 0; a < L; ++a) {
    for (int j = 0; j < Q; ++j) {
      double acc = 0.0;
      for (int i = 0; i < Q; ++i) acc += t.B[(size_t)a * Q + i] * t.w[i] * t.D[(size_t)i * Q + j];
      e2[(size_t)a * Q + j] = T(acc);
    }
    for (int g = 0; g < Q - 1; ++g) {
      double acc = 0.0;
      for (int i = 0; i < Q; ++i) acc += t.B[(size_t)a * Q + i] * t.w[i] * t.g2gl[(size_t)i * (Q - 1) + g];
      bwg[(size_t)a * (Q - 1) + g] = T(acc);
    }
  }
  cudaError_t e = cudaMemcpyToSymbol(cE2<T, L, Q>, e2.data(), sizeof(T) * e2.size());
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(cBwG<T, L, Q>, bwg.data(), sizeof(T) * bwg.size());
}

// Whether CV::MINB CTAs of the FP32 viscous kernels' tile CV fit one SM's
// shared memory (Navier-Stokes only: other physics have no viscous kernels).
template <bool NS, class CV>
struct ViscPairFits {
  static constexpr bool value = false;
};
template <class CV>
struct ViscPairFits<true, CV> {
  static constexpr bool value = CV::MINB * (NsCfg<CV, float>::Grad::SMEM + 1024) <= 228 * 1024 &&
                                CV::MINB * (NsCfg<CV, float>::Visc::SMEM + 1024) <= 228 * 1024;
};

// Whether two CTAs of the FP64 gradient kernel's tile CG fit one SM.
template <bool NS, class CG>
struct GradPairFits {
  static constexpr bool value = false;
};
template <class CG>
struct GradPairFits<true, CG> {
  static constexpr bool value = 2 * (NsCfg<CG, double>::Grad::SMEM + 1024) <= 228 * 1024;
};

// Whether two CTAs of the lean FP64 viscous tile CW fit one SM.
template <bool NS, class CW>
struct ViscLeanFits {
  static constexpr bool value = false;
};
template <class CW>
struct ViscLeanFits<true, CW> {
  static constexpr bool value = NsCfg<CW, double>::Visc::LEAN && 2 * (NsCfg<CW, double>::Visc::SMEM + 1024) <= 228 * 1024;
};

template <int PHYS, int L, int Q, int EPB, int MINB, bool MIXED = false, int NT_ = 0>
struct Launch {
  using C = Cfg<PHYS, L, Q, EPB, MINB, MIXED, NT_>;
  // 3xTF32 tensor-core contractions in the FP32 viscous kernels: 3-D
  // Navier-Stokes at p >= 5 (1-D operators of at least 7 x 7)
  static constexpr bool kTensorViscous = PHYS == DGMX_NS3D && L >= 6;
  // The FP32 viscous kernels' tile.  Above 512 quadrature points one thread
  // per point (and its registers) leaves one CTA per SM, whose barriers then
  // idle the SM; 256 threads (about three points each) and four CTAs per SM
  // (the traces read from global memory and the lean viscous layout,
  // NsCfg::Grad::TRG and NsCfg::Visc::LEAN, ~50 KB each) let CTAs' barrier
  // waits overlap the others' work.  At p = 7, q = 9: as fast as 384 x 3 on
  // the CUDA cores, 15 % faster with the 3xTF32 contractions (64 registers).
  using CV2 = Cfg<PHYS, L, Q, EPB, 4, MIXED, 256>;
  static constexpr bool kViscPair = C::QD > 512 && EPB == 1 && ViscPairFits<is_ns(PHYS) && !MIXED, CV2>::value;
  using CV = std::conditional_t<kViscPair, CV2, C>;
  // The FP64 gradient kernel's tile, the same way: 512 threads and two CTAs
  // per SM (64 registers), where its shared memory without the staged traces
  // (read from global memory instead, NsCfg::Grad::TRG) fits twice.
  using CG2 = Cfg<PHYS, L, Q, EPB, 2, MIXED, 512>;
  static constexpr bool kGradPair = C::QD > 512 && EPB == 1 && GradPairFits<is_ns(PHYS) && !MIXED, CG2>::value;
  using CG = std::conditional_t<kGradPair, CG2, C>;
  // and the FP64 viscous kernel's, with its lean layout (NsCfg::Visc::LEAN)
  using CW2 = Cfg<PHYS, L, Q, EPB, 2, MIXED, 512>;
  static constexpr bool kViscLean = C::QD > 512 && EPB == 1 && ViscLeanFits<is_ns(PHYS) && !MIXED, CW2>::value;
  using CW = std::conditional_t<kViscLean, CW2, C>;
  static dim3 grid(int ne) { return dim3((unsigned)((ne + EPB - 1) / EPB)); }
  static dim3 vgrid(const StageArgs &a) { return a.vtiles ? dim3((unsigned)a.nvtiles) : grid(a.ne); }
  static cudaError_t init(const Tables1D &t) {
    cudaError_t e = upload_tables_lq<L, Q, typename C::R>(t);
    if (e != cudaSuccess) return e;
    const int sm = (int)C::SMEM;
    if ((e = cudaFuncSetAttribute(stage_kernel<C, PHYS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
    if ((e = cudaFuncSetAttribute(traces_modal_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
    if constexpr (!MIXED) {
      if ((e = cudaFuncSetAttribute(traces_nodal_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
      if ((e = cudaFuncSetAttribute(rhs_nodal_kernel<C, PHYS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
      if ((e = cudaFuncSetAttribute(forward_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
      if ((e = cudaFuncSetAttribute(backward_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm))) return e;
    }
    if constexpr (is_ns(PHYS) && !MIXED) {
      const int sg = (int)NsCfg<CG>::Grad::SMEM, sv = (int)NsCfg<CW>::Visc::SMEM;
      if ((e = cudaFuncSetAttribute(ns_grad_kernel<CG, PHYS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sg))) return e;
      if ((e = cudaFuncSetAttribute(ns_grad_kernel<CG, PHYS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sg))) return e;
      if ((e = cudaFuncSetAttribute(ns_visc_kernel<CW, PHYS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sv))) return e;
      if ((e = cudaFuncSetAttribute(ns_visc_kernel<CW, PHYS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sv))) return e;
    }
    if constexpr (is_ns(PHYS) && !MIXED && MINB == 0) {
      // the FP32 viscous kernels (one set per (physics, L, Q, EPB): the
      // uncapped tile carries them) and their FP32 tables
      using N = NsCfg<CV, float>;
      if ((e = upload_tables_lq<L, Q, float>(t)) != cudaSuccess) return e;
      const int sg = (int)N::Grad::SMEM, sv = (int)N::Visc::SMEM;
      if ((e = cudaFuncSetAttribute(ns_grad_kernel<CV, PHYS, false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sg))) return e;
      if ((e = cudaFuncSetAttribute(ns_grad_kernel<CV, PHYS, true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sg))) return e;
      if ((e = cudaFuncSetAttribute(ns_visc_kernel<CV, PHYS, false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sv))) return e;
      if ((e = cudaFuncSetAttribute(ns_visc_kernel<CV, PHYS, true, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sv))) return e;
      if constexpr (kTensorViscous) {
        if ((e = cudaFuncSetAttribute(ns_grad_kernel<CV, PHYS, false, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sg))) return e;
        if ((e = cudaFuncSetAttribute(ns_grad_kernel<CV, PHYS, true, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sg))) return e;
        if ((e = cudaFuncSetAttribute(ns_visc_kernel<CV, PHYS, false, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sv))) return e;
        if ((e = cudaFuncSetAttribute(ns_visc_kernel<CV, PHYS, true, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sv))) return e;
      }
    }
    return cudaSuccess;
  }
  static cudaError_t ns_grad32(const StageArgs &a, bool nodal, cudaStream_t s) {
    if constexpr (is_ns(PHYS) && !MIXED && MINB == 0) {
      using N = NsCfg<CV, float>;
      if (nodal) ns_grad_kernel<CV, PHYS, true, float><<<grid(a.ne), CV::NT, N::Grad::SMEM, s>>>(a);
      else ns_grad_kernel<CV, PHYS, false, float><<<grid(a.ne), CV::NT, N::Grad::SMEM, s>>>(a);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t ns_visc32(const StageArgs &a, bool nodal, cudaStream_t s) {
    if constexpr (is_ns(PHYS) && !MIXED && MINB == 0) {
      using N = NsCfg<CV, float>;
      if (nodal) ns_visc_kernel<CV, PHYS, true, float><<<vgrid(a), CV::NT, N::Visc::SMEM, s>>>(a);
      else ns_visc_kernel<CV, PHYS, false, float><<<vgrid(a), CV::NT, N::Visc::SMEM, s>>>(a);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t ns_grad32tc(const StageArgs &a, bool nodal, cudaStream_t s) {
    if constexpr (is_ns(PHYS) && !MIXED && MINB == 0 && kTensorViscous) {
      using N = NsCfg<CV, float>;
      if (nodal) ns_grad_kernel<CV, PHYS, true, float, true><<<grid(a.ne), CV::NT, N::Grad::SMEM, s>>>(a);
      else ns_grad_kernel<CV, PHYS, false, float, true><<<grid(a.ne), CV::NT, N::Grad::SMEM, s>>>(a);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t ns_visc32tc(const StageArgs &a, bool nodal, cudaStream_t s) {
    if constexpr (is_ns(PHYS) && !MIXED && MINB == 0 && kTensorViscous) {
      using N = NsCfg<CV, float>;
      if (nodal) ns_visc_kernel<CV, PHYS, true, float, true><<<vgrid(a), CV::NT, N::Visc::SMEM, s>>>(a);
      else ns_visc_kernel<CV, PHYS, false, float, true><<<vgrid(a), CV::NT, N::Visc::SMEM, s>>>(a);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t ns_grad(const StageArgs &a, bool nodal, cudaStream_t s) {
    if constexpr (is_ns(PHYS) && !MIXED) {
      using N = NsCfg<CG>;
      if (nodal) ns_grad_kernel<CG, PHYS, true><<<grid(a.ne), CG::NT, N::Grad::SMEM, s>>>(a);
      else ns_grad_kernel<CG, PHYS, false><<<grid(a.ne), CG::NT, N::Grad::SMEM, s>>>(a);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t ns_visc(const StageArgs &a, bool nodal, cudaStream_t s) {
    if constexpr (is_ns(PHYS) && !MIXED) {
      using N = NsCfg<CW>;
      if (nodal) ns_visc_kernel<CW, PHYS, true><<<vgrid(a), CW::NT, N::Visc::SMEM, s>>>(a);
      else ns_visc_kernel<CW, PHYS, false><<<vgrid(a), CW::NT, N::Visc::SMEM, s>>>(a);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t stage(const StageArgs &a, cudaStream_t s) {
    stage_kernel<C, PHYS><<<grid(a.ne), C::NT, C::SMEM, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t traces_modal(const StageArgs &a, const double *X, void *T, cudaStream_t s) {
    traces_modal_kernel<C><<<grid(a.ne), C::NT, C::SMEM, s>>>(a, X, static_cast<typename C::R *>(T));
    return cudaGetLastError();
  }
  static cudaError_t traces_nodal(const StageArgs &a, cudaStream_t s) {
    if constexpr (!MIXED) {
      traces_nodal_kernel<C><<<grid(a.ne), C::NT, C::SMEM, s>>>(a);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t rhs_nodal(const StageArgs &a, cudaStream_t s) {
    if constexpr (!MIXED) {
      rhs_nodal_kernel<C, PHYS><<<grid(a.ne), C::NT, C::SMEM, s>>>(a);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t forward(const StageArgs &a, const double *Un, double *Um, cudaStream_t s) {
    if constexpr (!MIXED) {
      forward_kernel<C><<<grid(a.ne), C::NT, C::SMEM, s>>>(a, Un, Um);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t backward(const StageArgs &a, const double *Um, double *Un, cudaStream_t s) {
    if constexpr (!MIXED) {
      backward_kernel<C><<<grid(a.ne), C::NT, C::SMEM, s>>>(a, Um, Un);
      return cudaGetLastError();
    } else {
      return cudaErrorNotSupported;
    }
  }
  static cudaError_t stage_grid(const StageArgs &a, int g, cudaStream_t s) {
    stage_kernel<C, PHYS><<<g, C::NT, C::SMEM, s>>>(a);
    return cudaGetLastError();
  }
  static int blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage_kernel<C, PHYS>, C::NT, C::SMEM) != cudaSuccess) {
      cudaGetLastError();
      return 1;
    }
    return n > 0 ? n : 1;
  }
  static KernelOps ops() {
    KernelOps o;
    o.stage_grid = stage_grid; o.blocks_per_sm = blocks_per_sm;
    o.epb = EPB; o.nt = C::NT; o.smem = C::SMEM; o.minb = MINB; o.mixed = MIXED;
    o.init = init; o.stage = stage; o.traces_modal = traces_modal; o.traces_nodal = traces_nodal;
    o.rhs_nodal = rhs_nodal; o.forward = forward; o.backward = backward;
    if constexpr (is_ns(PHYS) && !MIXED) { o.ns_grad = ns_grad; o.ns_visc = ns_visc; }
    if constexpr (is_ns(PHYS) && !MIXED && MINB == 0) { o.ns_grad32 = ns_grad32; o.ns_visc32 = ns_visc32; }
    if constexpr (is_ns(PHYS) && !MIXED && MINB == 0 && kTensorViscous) {
      o.ns_grad32tc = ns_grad32tc; o.ns_visc32tc = ns_visc32tc;
    }
    return o;
  }
};

// Elements per CTA: pack small elements so a CTA has >= ~128 threads.
constexpr int default_epb(int dim, int Q) {
  return dim == 3 ? (Q * Q * Q >= 100 ? 1 : (Q * Q * Q >= 50 ? 2 : 4))
                  : (Q * Q >= 100 ? 1 : (128 / (Q * Q) > 8 ? 8 : 128 / (Q * Q)));
}


// Streaming multiprocessors of the current device (cached per device).
inline int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
      cudaGetLastError();
      n = 148;
    }
    cached[dev] = n;
  }
  return cached[dev];
}

// The persistent pipelined stage kernel (stage_pipe_kernel) for LSRK and
// right-hand-side stages; other stage kinds run the plain kernel of the
// same tile.
template <int PHYS, int L, int Q, int EPB, int MINB, bool MIXED = false>
struct PLaunch {
  using Base = Launch<PHYS, L, Q, EPB, MINB, MIXED>;
  using C = typename Base::C;
  using P = Pipe<C>;
  static cudaError_t init(const Tables1D &t) {
    cudaError_t e = Base::init(t);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(stage_pipe_kernel<C, PHYS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)P::SMEM);
  }
  static int blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage_pipe_kernel<C, PHYS>, C::NT, P::SMEM) !=
        cudaSuccess) {
      cudaGetLastError();
      return 1;
    }
    return n > 0 ? n : 1;
  }
  static cudaError_t stage_grid(const StageArgs &a, int g, cudaStream_t s) {
    if (a.kind != kLSRK && a.kind != kRHS) return Base::stage(a, s);
    stage_pipe_kernel<C, PHYS><<<g, C::NT, P::SMEM, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t stage(const StageArgs &a, cudaStream_t s) {
    static int bps = 0;
    if (!bps) bps = blocks_per_sm();
    const int tiles = (a.ne + EPB - 1) / EPB;
    const int g = tiles < sm_count() * bps ? tiles : sm_count() * bps;
    return stage_grid(a, g, s);
  }
  static KernelOps ops() {
    KernelOps o = Base::ops();
    o.smem = P::SMEM; o.init = init; o.stage = stage; o.stage_grid = stage_grid; o.blocks_per_sm = blocks_per_sm;
    o.warp = 2;
    return o;
  }
};

// The second-form stage kernel (stage2.cuh) for LSRK and right-hand-side
// stages; other stage kinds, and every other kernel of the handle, come from
// the plain tile of the same (L, Q).
template <int PHYS, int L, int Q, int EPB, int NT, int MINB, bool MIXED = false, int VD = 0>
struct Launch2 {
  using Base = Launch<PHYS, L, Q, default_epb(3, Q), 0, MIXED>;
  using C = Cfg2<PHYS, L, Q, EPB, NT, MINB, MIXED, VD>;
  static cudaError_t init(const Tables1D &t) {
    cudaError_t e = Base::init(t);
    if (e != cudaSuccess) return e;
    if ((e = upload_tables2_lq<L, Q, typename C::R>(t)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(stage2_kernel<C, PHYS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  }
  static int blocks_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage2_kernel<C, PHYS>, NT, C::SMEM) != cudaSuccess) {
      cudaGetLastError();
      return 1;
    }
    return n > 0 ? n : 1;
  }
  static cudaError_t stage_grid(const StageArgs &a, int g, cudaStream_t s) {
    if (a.kind != kLSRK && a.kind != kRHS) return Base::stage_grid(a, g, s);
    stage2_kernel<C, PHYS><<<g, NT, C::SMEM, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t stage(const StageArgs &a, cudaStream_t s) {
    if (a.kind != kLSRK && a.kind != kRHS) return Base::stage(a, s);
    stage2_kernel<C, PHYS><<<(unsigned)((a.ne + EPB - 1) / EPB), NT, C::SMEM, s>>>(a);
    return cudaGetLastError();
  }
  static KernelOps ops() {
    KernelOps o = Base::ops();
    o.epb = EPB; o.nt = NT; o.minb = MINB; o.smem = C::SMEM;
    o.init = init; o.stage = stage; o.stage_grid = stage_grid; o.blocks_per_sm = blocks_per_sm;
    o.warp = 3;
    return o;
  }
};

template <int PHYS, int P, int Q, int EPB, int NT, int MINB, bool MIXED, int VD = 0>
void reg2_variant() {
  using C = Cfg2<PHYS, P + 1, Q, EPB, NT, MINB, MIXED, VD>;
  if constexpr (C::SMEM <= 227 * 1024 && (MINB == 0 || (65536 / (NT * MINB) >= 40 &&
                                                        (int)((228 * 1024) / (C::SMEM + 1024)) >= MINB)))
    register_ops(PHYS + (MIXED ? kMixedKey : 0), P + 1, Q, Launch2<PHYS, P + 1, Q, EPB, NT, MINB, MIXED, VD>::ops());
}

// CTAs per SM of NT threads that a cap of R registers per thread allows: a
// warp's registers come from one of the SM's four 16K-register scheduler
// partitions, so ceil(warps / 4) warps of 32 x R registers share 16K;
// clipped to what the tile's shared memory allows.
template <class C>
constexpr int blocks_for_regs(int nt, int r) {
  const int per_part = 16384 / (32 * r), warps = (nt + 31) / 32;
  const int by_regs = per_part * 4 / warps;
  const int by_smem = (int)((228 * 1024) / (C::SMEM + 1024));
  return by_regs < by_smem ? by_regs : by_smem;
}

// Second-form variants of a 3-D Euler (p, q): one element per CTA at two
// thread counts, uncapped and with the CTAs per SM that caps of 96 and 80
// (and for the FP32 form 64) registers per thread allow; for the FP32 form
// also the volume pass with one direction per thread (fewer registers) at
// caps of 80, 64 and 56.  Appended variants keep the earlier indices.
template <int PHYS, int P, int Q, bool MIXED = false>
void reg2() {
  constexpr int NTA = ((P + 1) * (P + 1) * 5 + 31) / 32 * 32;   // one thread per modal row
  constexpr int NTB = NTA + 32;
  using CA = Cfg2<PHYS, P + 1, Q, 1, NTA, 0, MIXED>;
  using CB = Cfg2<PHYS, P + 1, Q, 1, NTB, 0, MIXED>;
  constexpr int A96 = blocks_for_regs<CA>(NTA, 96), A80 = blocks_for_regs<CA>(NTA, 80);
  constexpr int B96 = blocks_for_regs<CB>(NTB, 96), B80 = blocks_for_regs<CB>(NTB, 80);
  constexpr int B64 = blocks_for_regs<CB>(NTB, 64), A64 = blocks_for_regs<CA>(NTA, 64);
  reg2_variant<PHYS, P, Q, 1, NTA, 0, MIXED>();
  reg2_variant<PHYS, P, Q, 1, NTB, 0, MIXED>();
  if constexpr (B96 >= 2) reg2_variant<PHYS, P, Q, 1, NTB, B96, MIXED>();
  if constexpr (A96 >= 2) reg2_variant<PHYS, P, Q, 1, NTA, A96, MIXED>();
  if constexpr (B80 >= 2 && B80 != B96) reg2_variant<PHYS, P, Q, 1, NTB, B80, MIXED>();
  if constexpr (A80 >= 2 && A80 != A96) reg2_variant<PHYS, P, Q, 1, NTA, A80, MIXED>();
  if constexpr (MIXED && B64 >= 2 && B64 != B80) reg2_variant<PHYS, P, Q, 1, NTB, B64, MIXED>();
  // FP32 with the volume's three directions spread over three warps
  if constexpr (MIXED && A80 >= 2) reg2_variant<PHYS, P, Q, 1, NTA, A80, MIXED, 1>();
  if constexpr (MIXED && B80 >= 2) reg2_variant<PHYS, P, Q, 1, NTB, B80, MIXED, 1>();
  if constexpr (MIXED && A64 >= 2 && A64 != A80) reg2_variant<PHYS, P, Q, 1, NTA, A64, MIXED, 1>();
  constexpr int A56 = blocks_for_regs<CA>(NTA, 56);
  if constexpr (MIXED && B64 >= 2 && B64 != B80) reg2_variant<PHYS, P, Q, 1, NTB, B64, MIXED, 1>();
  if constexpr (MIXED && A56 >= 2 && A56 != A64) reg2_variant<PHYS, P, Q, 1, NTA, A56, MIXED, 1>();
  // FP64 at 72 registers: one more CTA per SM for a few dozen bytes of spills
  constexpr int A72 = blocks_for_regs<CA>(NTA, 72), B72 = blocks_for_regs<CB>(NTB, 72);
  if constexpr (!MIXED && A72 >= 2 && A72 != A80) reg2_variant<PHYS, P, Q, 1, NTA, A72, MIXED>();
  if constexpr (!MIXED && B72 >= 2 && B72 != B80) reg2_variant<PHYS, P, Q, 1, NTB, B72, MIXED>();
}

template <int PHYS, int P, int Q, int EPB, int MINB, bool MIXED>
void reg_pipe() {
  using C = Cfg<PHYS, P + 1, Q, EPB, MINB, MIXED>;
  using PP = Pipe<C>;
  if constexpr (PP::OK && PP::SMEM <= 227 * 1024 && (MINB == 0 || 65536 / (C::NT * MINB) >= 48)) {
    if constexpr (MINB == 0 || (228 * 1024) / (PP::SMEM + 1024) >= MINB)
      register_ops(PHYS + (MIXED ? kMixedKey : 0), P + 1, Q, PLaunch<PHYS, P + 1, Q, EPB, MINB, MIXED>::ops());
  }
}




// CTAs per SM that the shared memory of one tile allows (228 KB per SM,
// 1 KB reserved per CTA).
template <class C>
constexpr int smem_blocks() { return (int)((228 * 1024) / (C::SMEM + 1024)); }

// Navier-Stokes tiles also need their viscous kernels to fit shared memory.
template <int PHYS, class C>
constexpr bool ns_fits() {
  if constexpr (is_ns(PHYS)) return NsCfg<C>::Grad::SMEM <= 227 * 1024 && NsCfg<C>::Visc::SMEM <= 227 * 1024;
  else return true;
}

// Register variant (EPB, MINB) when it is distinct and sensible: the
// register cap 64K/(NT*MINB) stays >= 48 and the tile fits shared memory.
template <int PHYS, int P, int Q, int EPB, int MINB, bool MIXED, int NT = 0>
void reg_variant() {
  using C = Cfg<PHYS, P + 1, Q, EPB, MINB, MIXED, NT>;
  if constexpr (ns_fits<PHYS, C>() && (MINB == 0 || (65536 / (C::NT * MINB) >= 48 && smem_blocks<C>() >= MINB))) {
    register_ops(PHYS + (MIXED ? kMixedKey : 0), P + 1, Q, Launch<PHYS, P + 1, Q, EPB, MINB, MIXED, NT>::ops());
  }
}


// Tile variants for (physics, p, q): the default packing without and with a
// register cap at the shared-memory occupancy, and twice the packing.  The
// first registered variant is the default; dgmx_autotune picks among all.
template <int PHYS, int P, int Q, bool MIXED = false>
void reg() {
  constexpr int E1 = default_epb(phys_dim(PHYS), Q);
  using C1 = Cfg<PHYS, P + 1, Q, E1, 0, MIXED>;
  constexpr int B1 = smem_blocks<C1>() > 8 ? 8 : smem_blocks<C1>();
  reg_variant<PHYS, P, Q, E1, 0, MIXED>();
  if constexpr (B1 >= 2) reg_variant<PHYS, P, Q, E1, B1, MIXED>();
  if constexpr (B1 >= 4) reg_variant<PHYS, P, Q, E1, (B1 * 3) / 4, MIXED>();
  constexpr int E2 = 2 * E1;
  if constexpr (Cfg<PHYS, P + 1, Q, E2, 0, MIXED>::NT <= 1024 && Cfg<PHYS, P + 1, Q, E2, 0, MIXED>::SMEM <= 200 * 1024) {
    using C2 = Cfg<PHYS, P + 1, Q, E2, 0, MIXED>;
    constexpr int B2 = smem_blocks<C2>() > 8 ? 8 : smem_blocks<C2>();
    if constexpr (B2 >= 2) reg_variant<PHYS, P, Q, E2, B2, MIXED>();
  }
  if constexpr (Pipe<C1>::OK) {
    constexpr int PB = (int)((228 * 1024) / (Pipe<C1>::SMEM + 1024)) > 8 ? 8 : (int)((228 * 1024) / (Pipe<C1>::SMEM + 1024));
    reg_pipe<PHYS, P, Q, E1, 0, MIXED>();
    if constexpr (PB >= 2) reg_pipe<PHYS, P, Q, E1, PB, MIXED>();
    if constexpr (PB >= 4) reg_pipe<PHYS, P, Q, E1, (PB * 3) / 4, MIXED>();
  }
}

}  // namespace dgmx
