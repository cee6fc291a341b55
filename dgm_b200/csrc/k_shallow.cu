// Shallow-water kernel instantiations (Quad, FP64), p = 1..8, q = p+1, p+2.
#include "dispatch.cuh"

namespace dgmx {
namespace {
struct RegShallow {
  RegShallow() {
#define R(P) reg<DGMX_SHALLOW, P, P + 1>(); reg<DGMX_SHALLOW, P, P + 2>();
    R(1) R(2) R(3) R(4) R(5) R(6) R(7) R(8)
#undef R
  }
} reg_shallow;
}  // namespace
}  // namespace dgmx
