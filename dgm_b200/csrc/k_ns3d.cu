// Navier-Stokes 3-D kernel instantiations (Hex, FP64, BR1), p = 1..7, q = p+2 (and p+1 from p = 2).
#include "dispatch.cuh"

namespace dgmx {
namespace {
struct RegNS3D {
  RegNS3D() {
    reg<DGMX_NS3D, 1, 3>();
#define R(P) reg<DGMX_NS3D, P, P + 1>(); reg<DGMX_NS3D, P, P + 2>();
    R(2) R(3) R(4) R(5) R(6)
#undef R
    reg<DGMX_NS3D, 7, 8>();
    // p = 7, q = 9: 729 points leave the one-thread-per-point stage tile
    // (736 threads, one CTA per SM by its shared memory) 80 registers and
    // about 1 KB of spills per thread; with 512 threads (some take two
    // points) it has 128 and no spills.  Registered first: the default.
    reg_variant<DGMX_NS3D, 7, 9, 1, 0, false, 512>();
    reg<DGMX_NS3D, 7, 9>();
  }
} reg_ns3d;
}  // namespace
}  // namespace dgmx
