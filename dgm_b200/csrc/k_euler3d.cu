// Euler 3-D kernel instantiations (Hex, FP64), p = 1..7, q = p+2 (and p+1).
#include "dispatch.cuh"

namespace dgmx {
namespace {
struct RegEuler3D {
  RegEuler3D() {
    reg<DGMX_EULER3D, 1, 3>();
#define R(P) reg<DGMX_EULER3D, P, P + 1>(); reg<DGMX_EULER3D, P, P + 2>();
    R(2) R(3) R(4) R(5) R(6)
#undef R
    reg<DGMX_EULER3D, 7, 8>();
    // p = 7, q = 9: the one-thread-per-point tile (736 threads, one CTA per
    // SM by its shared memory) gets 80 registers and spills about 1.2 KB per
    // thread; 512 threads have 128 and no spills.  Registered first: the
    // default.
    reg_variant<DGMX_EULER3D, 7, 9, 1, 0, false, 512>();
    reg<DGMX_EULER3D, 7, 9>();
    // second-form stage kernels at q = p+2, after the plain tiles (every
    // template instantiation of a tile lives in one compilation unit: its
    // launchers and its constant tables must come from the same module)
#define R2(P) reg2<DGMX_EULER3D, P, P + 2>();
    R2(2) R2(3) R2(4) R2(5)
#undef R2
  }
} reg_euler3d;
}  // namespace
}  // namespace dgmx
