// The pool's fused multi-order stage kernel, mixed form (FP32 working precision) (fused.cuh).
#include "fused.cuh"

namespace dgmx {

const FusedOps &fused_ops_mixed() {
  static const FusedOps ops{FusedHost<true>::init, FusedHost<true>::blocks_per_sm, FusedHost<true>::launch,
                            [](int body) { return fused_epb<true>(body); }};
  return ops;
}

}  // namespace dgmx
