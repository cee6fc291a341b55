// A C++ caller of the engine's C ABI, compiled with g++ against
// include/dgmx.h and linked to dgm_b200/libdgmx.so: the shape of the DGM
// adapter (a Domain::time_derivative override and a TimeInt::advance
// override) reduced to the calls it makes.
//
//   abi_driver <case.bin> <out.bin>
//
// case.bin (little-endian): int32 dim, ne, ncon, physics, flux, inttype,
// nsteps; float64 dt; float64 verts[ne * 2^dim * 3]; int32 con[ncon * 4];
// int32 porder[ne]; int32 qorder[ne]; float64 U[nf * nq] (GLL values, Field
// layout).  out.bin: float64 F[nf * nq] = -dU/dt at U, then float64
// U_after[nf * nq] after nsteps steps from the projected U.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dgmx.h"

namespace {

template <class T>
bool read_n(std::FILE *f, T *p, size_t n) { return std::fread(p, sizeof(T), n, f) == n; }

int fail(const char *what, dgmx_domain *d) {
  std::fprintf(stderr, "abi_driver: %s failed: %s\n", what, dgmx_last_error(d));
  if (d) dgmx_destroy(d);
  return 2;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: abi_driver <case.bin> <out.bin>\n");
    return 1;
  }
  std::FILE *in = std::fopen(argv[1], "rb");
  if (!in) { std::perror(argv[1]); return 1; }
  int hdr[7];
  double dt = 0.0;
  if (!read_n(in, hdr, 7) || !read_n(in, &dt, 1)) { std::fprintf(stderr, "short header\n"); return 1; }
  const int dim = hdr[0], ne = hdr[1], ncon = hdr[2], nsteps = hdr[6];
  std::vector<double> verts((size_t)ne * (dim == 3 ? 8 : 4) * 3);
  std::vector<int> con((size_t)ncon * 4), porder(ne), qorder(ne);
  if (!read_n(in, verts.data(), verts.size()) || !read_n(in, con.data(), con.size()) ||
      !read_n(in, porder.data(), porder.size()) || !read_n(in, qorder.data(), qorder.size())) {
    std::fprintf(stderr, "short mesh\n");
    return 1;
  }
  dgmx_mesh mesh = {dim, ne, verts.data(), ncon, con.data(), porder.data(), qorder.data()};
  dgmx_params prm = {};
  prm.physics = hdr[3];
  prm.flux = hdr[4];
  prm.inttype = hdr[5];
  prm.precision = DGMX_FP64;
  prm.sw_balance = 1;
  prm.device = 0;
  prm.gamma = 1.4;
  prm.vis = 0.0;
  prm.Pr = 0.72;
  dgmx_domain *d = nullptr;
  if (dgmx_create(&mesh, &prm, &d) != DGMX_OK) return fail("dgmx_create", nullptr);
  long nf = 0, nq = 0, nm = 0;
  if (dgmx_sizes(d, &nf, &nq, &nm) != DGMX_OK) return fail("dgmx_sizes", d);
  std::vector<double> U((size_t)(nf * nq)), F(U.size());
  if (!read_n(in, U.data(), U.size())) { std::fprintf(stderr, "short state\n"); return 1; }
  std::fclose(in);
  // Domain::time_derivative(U, F)
  if (dgmx_time_derivative(d, U.data(), F.data()) != DGMX_OK) return fail("dgmx_time_derivative", d);
  // set_ic + project, then TimeInt::advance nsteps times
  if (dgmx_set_state(d, U.data()) != DGMX_OK) return fail("dgmx_set_state", d);
  if (dgmx_advance(d, dt, nsteps) != DGMX_OK) return fail("dgmx_advance", d);
  if (dgmx_get_state(d, U.data()) != DGMX_OK) return fail("dgmx_get_state", d);
  if (dgmx_destroy(d) != DGMX_OK) return 2;
  std::FILE *out = std::fopen(argv[2], "wb");
  if (!out) { std::perror(argv[2]); return 1; }
  const bool ok = std::fwrite(F.data(), sizeof(double), F.size(), out) == F.size() &&
                  std::fwrite(U.data(), sizeof(double), U.size(), out) == U.size();
  std::fclose(out);
  std::printf("abi_driver: %ld fields x %ld points, %d steps\n", nf, nq, nsteps);
  return ok ? 0 : 1;
}
