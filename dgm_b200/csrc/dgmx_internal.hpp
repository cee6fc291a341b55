// Internal declarations shared by the host setup (C++) and the kernels (CUDA).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/dgmx.h"

namespace dgmx {

// ------------------------------------------------------------------ tables
struct Tables1D {
  int L = 0, Q = 0, G = 0;
  std::vector<double> z, w, zg, wg;
  std::vector<double> D;      // Q x Q, D[i*Q+j] = l_j'(z_i)
  std::vector<double> B;      // L x Q orthonormal Legendre on GLL, B[a*Q+i]
  std::vector<double> Bg;     // L x G orthonormal Legendre on Gauss, Bg[a*G+g]
  std::vector<double> gl2g;   // G x Q
  std::vector<double> g2gl;   // Q x G
};
Tables1D make_tables(int L, int Q, int G);
void gll_points(int Q, double *z, double *w);
void gauss_points(int G, double *z, double *w);

// ------------------------------------------------------------ mesh / geometry
// Geometry shared by all elements of one class (affine elements with equal
// metrics, face normals, Jacobian ratios and master pattern).
struct GeomClass {
  double metric[9];     // rx ry rz sx sy sz tx ty tz (2-D: rx ry 0 sx sy 0 ...)
  double J;             // element Jacobian
  double nrm[6][3];     // unit normal of face f in the frame of its master side
  double onrm[6][3];    // this element's own outward unit normal of face f
  double jr[6];         // side Jacobian / element Jacobian on this element's side
  double fr[6][15];     // 3-D: face frame of nrm[f]: s (3), t (3), inverse rows (9)
  int master;           // bit f set: this element owns (is master of) face f
  int bc;               // bits 4f..4f+3: boundary type of face f (0: interior)
};

struct FaceLink {
  int elem;             // neighbour element
  int face;             // neighbour's face id
  int perm;             // offset of the point permutation in the perm table
  int cls;              // on face 0: the element's geometry class (-1: unallocated)
};

struct HostMesh {
  int dim = 0, ne = 0, p = 0, L = 0, Q = 0, G = 0, nfaces = 0, gf = 0;
  std::vector<double> cx, cy, cz;    // GLL coordinates, Field layout
  std::vector<double> J;             // per element Jacobian
  std::vector<int> gclass;           // per element geometry class
  std::vector<GeomClass> classes;
  std::vector<FaceLink> links;       // ne * nfaces
  std::vector<int> perm;             // concatenated permutations (gf each)
};

// The face frame of the 3-D fluxes for a unit normal n (src/Euler3d.cpp:
// 601-650): s from (ny, nz, nx) by Gram-Schmidt, t = n x s, both normalised,
// and the inverse of the rotation [n; s; t] by cofactors over its
// determinant.  out: s (3), t (3), then xn yn zn xs ys zs xt yt zt.
inline void face_frame(const double *n, double *out) {
  const double nx = n[0], ny = n[1], nz = n[2];
  double sx = ny, sy = nz, sz = nx;
  const double sdn = nx * sx + ny * sy + nz * sz;
  sx -= sdn * nx; sy -= sdn * ny; sz -= sdn * nz;
  const double sni = 1.0 / std::sqrt(sx * sx + sy * sy + sz * sz);
  sx *= sni; sy *= sni; sz *= sni;
  double tx = ny * sz - sy * nz, ty = nz * sx - sz * nx, tz = nx * sy - sx * ny;
  const double tni = 1.0 / std::sqrt(tx * tx + ty * ty + tz * tz);
  tx *= tni; ty *= tni; tz *= tni;
  const double detA = (nx * sy * tz + sx * ty * nz + tx * sz * ny) - (nz * sy * tx + sz * ty * nx + tz * sx * ny);
  const double id = 1.0 / detA;
  const double v[15] = {sx, sy, sz, tx, ty, tz,
                        (sy * tz - sz * ty) * id, -(sx * tz - sz * tx) * id, (sx * ty - sy * tx) * id,
                        -(ny * tz - nz * ty) * id, (nx * tz - nz * tx) * id, -(nx * ty - ny * tx) * id,
                        (ny * sz - nz * sy) * id, -(nx * sz - nz * sx) * id, (nx * sy - ny * sx) * id};
  for (int k = 0; k < 15; ++k) out[k] = v[k];
}

// Processes a DGM mesh: connectivity masters (src/Field.cpp:3478-3540),
// orientation flags (src/Field.cpp:416-680), affine geometry
// (src/Quad.cpp:1227-1285, src/Hex.cpp:1130-1280) and side geometry
// (src/Quad.cpp:1367-1455, src/Hex.cpp:1385-1497).
// A boundary side: element, face and its boundary type (1..kMaxBcTypes,
// an index into the domain's table of (kind, parameters)).
struct BoundarySide { int e, s, type; };
constexpr int kMaxBcTypes = 15;
bool build_mesh(const dgmx_mesh &m, const Tables1D &t, HostMesh &out, std::string &err,
                const std::vector<BoundarySide> *bcs = nullptr);

// Element partition of a processed mesh (the reference's root.part.N /
// Zoltan partitions, src/Field.cpp make_partition).  The local mesh holds the
// rank's elements in increasing global order; a face whose neighbour lives
// on another rank links to a ghost slot ne_local + g (ghosts in increasing
// global order) whose face trace the halo exchange fills.  For every peer
// q, send[q] lists the local (element * nfaces + face) blocks q needs and
// recv[q] the (slot * nfaces + face) blocks q sends here, both in the order
// of the global (element, face) they hold, so the two sides agree without
// exchanging metadata (src/vField.cpp:146-200 is the reference's exchange).
struct PartitionPlan {
  int nranks = 1, rank = 0, ne_local = 0, nghost = 0;
  std::vector<int> global_of_local, global_of_ghost;
  std::vector<std::vector<int>> send, recv;
};
bool partition_mesh(const HostMesh &g, const int *part, int nranks, int rank, HostMesh &local, PartitionPlan &plan,
                    std::string &err);
// Pack / unpack of blk-value blocks by index (exchange.cu); the FP32 forms
// place block i at buf + i * bs.
cudaError_t launch_pack(const double *T, const int *idx, int n, int blk, double *buf, cudaStream_t s);
cudaError_t launch_unpack(const double *buf, const int *idx, int n, int blk, double *T, cudaStream_t s);
cudaError_t launch_pack(const float *T, const int *idx, int n, int blk, int bs, float *buf, cudaStream_t s);
cudaError_t launch_unpack(const float *buf, const int *idx, int n, int blk, int bs, float *T, cudaStream_t s);

// DGM input files (.inp/.msh/.con/.ord)
struct FileCase {
  int dim = 0, ne = 0;
  std::vector<double> verts;
  std::vector<int> con, porder, qorder;
  int eqntype = -1, inttype = -1, p = -1, q = 0;
  double gamma = -1, vis = -1, Pr = -1;
  std::string flux;
  // root.bc records, root.bct blocks (code, values) by tag, root.chn present
  struct BcRecord { std::string tag; int e, s; };
  std::vector<BcRecord> bcs;
  std::map<std::string, std::pair<std::string, std::vector<double>>> bct;
  bool channel = false;
};
bool read_case_files(const std::string &root, FileCase &fc, std::string &err);

// LSRK14 coefficients A and B (src/TimeInt.cpp:1870-1917)
inline constexpr double kLsrkA[14] = {0.0, -0.7188012108672410, -0.7785331173421570, -0.0053282796654044,
                           -0.8552979934029281, -3.9564138245774565, -1.5780575380587385,
                           -2.0837094552574054, -0.7483334182761610, -0.7032861106563359,
                           0.0013917096117681, -0.0932075369637460, -0.9514200470875948,
                           -7.1151571693922548};
inline constexpr double kLsrkB[14] = {0.0367762454319673, 0.3136296607553959, 0.1531848691869027, 0.0030097086818182,
                           0.3326293790646110, 0.2440251405350864, 0.3718879239592277, 0.6204126221582444,
                           0.1524043173028741, 0.0760894927419266, 0.0077604214040978, 0.0024647284755382,
                           0.0780348340049386, 5.5059777270269628};
// LSRK14 stage times as fractions of the step (src/TimeInt.cpp:1903-1917)
inline constexpr double kLsrkC[14] = {0.0, 0.0367762454319673, 0.1249685262725025, 0.2446177702277698,
                                      0.2476149531070420, 0.2969311120382472, 0.3978149645802642,
                                      0.5270854589440328, 0.6981269994175695, 0.8190890835352128,
                                      0.8527059887098624, 0.8604711817462826, 0.8627060376969976,
                                      0.8734213127600976};

// ------------------------------------------------------------ mixed form
// Reference state of a solve (the working copies of the mixed form are
// perturbations about it): the conserved values, their velocity, E + p and
// pressure.  Built once per solve on the host.
template <class T>
struct RefState {
  T r, m[3], E;   // reference density (geopotential), momentum, energy
  T u[3], H, p;   // its velocity, E + p and pressure
  T pad[6];
};

// One row per solve in the reference-state array: [0, 5) the conserved
// reference values, [5, 10) their constant-mode coefficients, [10, 18) the
// FP32 RefState packed as doubles.
constexpr int kUrefStride = 24;

// Fills row[5..] from row[0..nf): phi0 is the constant basis function's
// value (the constant mode of a constant c is c / phi0).
__host__ __device__ inline void fill_reference_row(int physics, double gamma, double phi0, double *row) {
  const bool sw = physics == DGMX_SHALLOW;
  const int dim = (physics == DGMX_EULER3D || physics == DGMX_NS3D) ? 3 : 2, nf = sw ? 3 : dim + 2;
  for (int n = 0; n < nf; ++n) row[5 + n] = row[n] / phi0;
  RefState<float> rs{};
  const double r = row[0];
  double q = 0.0, u[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < dim; ++i) { u[i] = row[1 + i] / r; q += row[1 + i] * u[i]; }
  const double p = sw ? 0.5 * r * r : (gamma - 1.0) * (row[nf - 1] - 0.5 * q);
  rs.r = (float)r;
  for (int i = 0; i < dim; ++i) { rs.m[i] = (float)row[1 + i]; rs.u[i] = (float)u[i]; }
  rs.E = sw ? 0.0f : (float)row[nf - 1];
  rs.p = (float)p;
  rs.H = sw ? 0.0f : (float)(row[nf - 1] + p);
  static_assert(sizeof(RefState<float>) == 8 * sizeof(double), "RefState<float> packs into 8 doubles");
  __builtin_memcpy(row + 10, &rs, sizeof(rs));
}

// ------------------------------------------------------------------ kernels
// Integrator stage kinds.  X is the register the RHS is evaluated on.
enum StageKind : int {
  kLSRK = 0,      // X=U : Ut = A Ut - dt R; U = B Ut + U
  kTVD0 = 1,      // X=U : Ut = -dt R + U
  kTVD1 = 2,      // X=Ut: T = -dt R + Ut; Ut = b T; Ut = a U + Ut
  kTVD2 = 3,      // X=Ut: T = -dt R + Ut; U = a U; U = b T + U
  kRK40 = 4,      // X=U : Ut = c0 R + U; A = c1 R
  kRK41 = 5,      // X=Ut: Ut = c0 R + U; A = c1 R + A
  kRK43 = 6,      // X=Ut: A = c1 R + A; U = c0 A + U
  kRHS = 7,       // X   : A = R (no update)
};

struct StageArgs {
  // registers, element-major modal layout [e][field][L^d]
  const double *X;        // state the RHS is evaluated on
  double *U, *Ut, *A;     // solution, second register, RK4 accumulator
  const double *Tin;      // traces of X, [e][face][field][gf]
  double *Tout;           // traces of the next stage's X
  int kind;
  double c0, c1, c2;      // stage coefficients (see StageKind)
  double dt;
  // nodal I/O (Domain::time_derivative path), Field layout [field][e][Q^d]
  const double *Xn;
  double *Fn;
  // mesh
  const int *gclass;
  const GeomClass *classes;
  const FaceLink *links;
  const int *perm;
  int ne;
  double gamma, vis, Pr;
  int flux;
  int *err;               // err[0] bit 0: non-physical state; err[1]: min element
  // shallow-water balance (REO_SHALLOW_ENFORCE_BALANCE, src/Shallow.cpp:251-267)
  double *Rcap;           // if set, the projected RHS is stored here (modal)
  const double *Rsub;     // if set, subtracted from the projected RHS
  // if set, a source field of the 2-D physics projected once (modal,
  // register layout), subtracted from the projected RHS before the two
  // above: Source::apply's F -= S at the GLL points ahead of the projection
  // (src/Euler.cpp:282-287, src/Navier_Stokes.cpp:95-100,
  // src/Shallow.cpp:255-260), moved past it since projection is linear
  const double *Ssrc;
  // factor of Ssrc at this stage's time (1 for a source fixed in time)
  double src_scale;
  // mixed-precision form: FP32 second register and traces; the working
  // copies are perturbations about a reference state per solve:
  // uref[10 s + n] conserved values, uref[10 s + 5 + n] its constant-mode
  // coefficient; esolve[e] = solve of element e (null: solve 0)
  float *Utf;
  const float *Tinf;
  float *Toutf;
  const double *uref;
  const int *esolve;
  // element pools: persistent loop over tiles[0 .. *ntiles) (null: one
  // tile per CTA) and a step per solve, dts[esolve[e]] (null: dt)
  const int *tiles;
  const int *ntiles;
  const double *dts;
  // the viscous flux kernel over a tile list: CTA b takes tile vtiles[b]
  // (null: tile b), one CTA per listed tile (nvtiles)
  const int *vtiles;
  int nvtiles;
  // Navier-Stokes BR1 (src/Navier_Stokes3d.cpp:182-391)
  double *Ghat;           // projected primitive gradients, modal [e][comp][dir][L^d]
  double *V;              // viscous normal-flux traces [e][face][field-1][gf]
  double *Pv;             // projected viscous divergence, modal [e][field-1][L^d]
  // boundary types t = 1..15 (GeomClass::bc): kind (DGMX_BC_*) and parameters
  int bckind[kMaxBcTypes + 1];
  double bcpar[kMaxBcTypes + 1][5];
  // if set, the constant-mode coefficient of every field's final projected
  // RHS, [e][field] (bulk-flow hold)
  double *R0;
  // tries of the copy pipeline's wait for a tile's inputs before it gives
  // up (bit 1 of err[0]); kWaitTries unless a test lowers it
  int wait_tries;
};
constexpr int kWaitTries = 1 << 20;

// Bulk-flow hold (hold.cu): cbar[n] = sum_e J_e R0[e][n] / sum_e J_e for the
// held fields (density, x-momentum, energy), then the stage kind's linear
// response to -cbar on the constant coefficients of U / Ut / A, on the next
// state's traces Tout and, if Fn is set, on the nodal right-hand side.
struct HoldArgs {
  int ne, nf, ld, gf, qd, nfaces;
  const double *R0, *J;
  double *cbar;
  int kind;
  double c0, c1, dt;
  double *U, *Ut, *A, *Tout, *Fn;
};
cudaError_t launch_hold(const HoldArgs &h, cudaStream_t s);   // reduce, then apply
// The two halves: cbar from R0 / J over h.ne elements (one block, fixed
// order), and its application to the registers and traces of h.ne elements.
cudaError_t launch_hold_reduce(const HoldArgs &h, cudaStream_t s);
cudaError_t launch_hold_apply(const HoldArgs &h, cudaStream_t s);
// dst[gid[i]][0 .. nf) = src[i][0 .. nf) for the n rows with gid[i] >= 0
// (element partitions: a part's constant coefficients into the whole mesh's).
cudaError_t launch_scatter_rows(const double *src, const int *gid, int n, int nf, double *dst, cudaStream_t s);

// Registry key offset of the mixed-precision (FP32 working precision) tiles.
constexpr int kMixedKey = 1000;

// Launchers for one (physics, L, Q) instantiation; all enqueue on stream s.
struct KernelOps {
  int epb = 0, nt = 0, minb = 0, mixed = 0;
  int warp = 0;                                        // kind: 0 CTA tile, 2 prefetching persistent kernel
  size_t smem = 0;
  cudaError_t (*init)(const Tables1D &t) = nullptr;   // tables + smem attributes, current device
  cudaError_t (*stage)(const StageArgs &a, cudaStream_t s) = nullptr;
  // stage kernel on an explicit grid (persistent launch over a tile list)
  cudaError_t (*stage_grid)(const StageArgs &a, int grid, cudaStream_t s) = nullptr;
  int (*blocks_per_sm)() = nullptr;                    // resident stage CTAs per SM
  // T is double* (FP64 tiles) or float* (mixed tiles)
  cudaError_t (*traces_modal)(const StageArgs &a, const double *Xm, void *T, cudaStream_t s) = nullptr;
  cudaError_t (*traces_nodal)(const StageArgs &a, cudaStream_t s) = nullptr;
  cudaError_t (*rhs_nodal)(const StageArgs &a, cudaStream_t s) = nullptr;
  cudaError_t (*forward)(const StageArgs &a, const double *Un, double *Um, cudaStream_t s) = nullptr;
  cudaError_t (*backward)(const StageArgs &a, const double *Um, double *Un, cudaStream_t s) = nullptr;
  // Navier-Stokes only: lifted gradients, then viscous traces + divergence;
  // nodal = read GLL values from a.Xn instead of the modal register a.X
  cudaError_t (*ns_grad)(const StageArgs &a, bool nodal, cudaStream_t s) = nullptr;
  cudaError_t (*ns_visc)(const StageArgs &a, bool nodal, cudaStream_t s) = nullptr;
  // the same in FP32 (Navier-Stokes with precision = DGMX_MIXED); set on the
  // uncapped tile of each (physics, L, Q, EPB)
  cudaError_t (*ns_grad32)(const StageArgs &a, bool nodal, cudaStream_t s) = nullptr;
  cudaError_t (*ns_visc32)(const StageArgs &a, bool nodal, cudaStream_t s) = nullptr;
  // the FP32 viscous kernels with 3xTF32 tensor-core contractions (3-D,
  // p >= 5)
  cudaError_t (*ns_grad32tc)(const StageArgs &a, bool nodal, cudaStream_t s) = nullptr;
  cudaError_t (*ns_visc32tc)(const StageArgs &a, bool nodal, cudaStream_t s) = nullptr;
};
void register_ops(int physics, int L, int Q, const KernelOps &ops);
const KernelOps *find_ops(int physics, int L, int Q);            // default variant
const std::vector<KernelOps> *find_variants(int physics, int L, int Q);
void list_ops(std::vector<std::vector<int>> &out);

// Field integrals from modal register mode 0: out[n] = sum_e J_e c_d Um[e][n][0].
cudaError_t launch_integrals(int nf, int ne, int ld, double c_d, const double *Um, const double *J,
                             double *out, cudaStream_t s);
// The mixed form's reference integrals in a fixed order a host can repeat:
// field n's products J_e * Um[e][n][0], each rounded on its own, summed by
// lane l = e mod kRefLanes in increasing e, then lanes pairwise (halving
// strides), then times c_d.  Partitions gather the products
// (launch_element_integrands, [e][n]) and sum them in that order on the
// host (reference_sum), so every partition of a mesh gets the same row.
constexpr int kRefLanes = 256;
cudaError_t launch_reference_integrals(int nf, int ne, int ld, double c_d, const double *Um, const double *J,
                                       double *out, cudaStream_t s);
cudaError_t launch_element_integrands(int nf, int ne, int ld, const double *Um, const double *J, double *out,
                                      cudaStream_t s);
// The mixed form's reference row from those integrals, on the stream:
// uref[0 .. kUrefStride) = fill_reference_row(integ / vol).
cudaError_t launch_reference_row(int physics, int nf, double gamma, double phi0, double vol, const double *integ,
                                 double *uref, cudaStream_t s);

// The pools' multi-order stage kernel (fused.cuh): one launch per LSRK stage
// over (arena, tile) work items of every 2-D arena.
struct FusedOps {
  cudaError_t (*init)();                 // tables and attributes, current device
  int (*blocks_per_sm)();
  cudaError_t (*launch)(const StageArgs *args, int narena, const int *bodies, const int2 *items,
                        const int *nitems, int stage, int grid, cudaStream_t s);
  int (*epb)(int body);                  // elements per tile of a body
};
const FusedOps &fused_ops_fp64();
const FusedOps &fused_ops_mixed();
// Body of (physics, L, Q) in the fused kernel: Euler 2-D 0..6 and shallow
// water 7..13 for p = 1..7 at q = p + 2; -1 when it has none.
inline int fused_body(int physics, int L, int Q) {
  if ((physics != DGMX_EULER2D && physics != DGMX_SHALLOW) || Q != L + 1 || L < 2 || L > 8) return -1;
  return (physics == DGMX_SHALLOW ? 7 : 0) + (L - 2);
}

// What an entry point in another compilation unit needs from a handle.
struct DomainView {
  const KernelOps *ops;
  cudaStream_t stream;
  StageArgs base;           // mesh pointers and physics parameters
  size_t ntrace;            // doubles in one trace buffer
  int device;
  bool sw_balance;
  double *Rsw;
  bool *sw_captured;
  std::string *errmsg;
  long *launches;
};
// False for a null handle or a partitioned one (*partitioned tells which;
// the partitioned handle's error text is then reachable through *errmsg).
bool domain_view(dgmx_domain *d, DomainView *v, bool *partitioned = nullptr, std::string **errmsg = nullptr);

inline int nfields_of(int physics) {
  return physics == DGMX_SHALLOW ? 3 : (physics == DGMX_EULER3D || physics == DGMX_NS3D ? 5 : 4);
}
inline int dim_of(int physics) {
  return (physics == DGMX_EULER3D || physics == DGMX_NS3D) ? 3 : 2;
}

}  // namespace dgmx
