// The pool's fused multi-order stage kernel, FP64 (fused.cuh).
#include "fused.cuh"

namespace dgmx {

const FusedOps &fused_ops_fp64() {
  static const FusedOps ops{FusedHost<false>::init, FusedHost<false>::blocks_per_sm, FusedHost<false>::launch,
                            [](int body) { return fused_epb<false>(body); }};
  return ops;
}

}  // namespace dgmx
