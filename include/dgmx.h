/*
 * dgmx.h -- C ABI of the B200 DG residual and RK-stage engine.
 *
 * One opaque handle (dgmx_domain) stands for one DGM Domain on one GPU: the
 * mesh, the discretisation tables, the conserved-variable state and the
 * integrator registers all live in device memory.  Every entry point returns
 * a dgmx_status; none throws, traps or aborts.  Calls on one handle are not
 * thread-safe; each handle owns one CUDA stream.
 *
 * Array layouts at this boundary are DGM's own (src/vField.cpp:88-111,
 * src/Field.cpp:3042-3123): a vField of nf Fields, each Field a contiguous
 * element-major array of element values, element e holding Q^d values at its
 * Gauss-Lobatto-Legendre points with the last direction fastest
 * (Quad: j + Q*i, src/Quad.cpp:772; Hex: k + Q*(j + Q*i), src/Hex.cpp:817).
 * Modal (restart) layouts follow src/vField.cpp:1102-1179: per field, per
 * element, L^d orthonormal-Legendre coefficients, index c + L*(b + L*a).
 */
#ifndef DGMX_H
#define DGMX_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dgmx_domain dgmx_domain;

typedef enum {
  DGMX_OK = 0,
  DGMX_ERR_ARGUMENT = 1,      /* bad pointer, size or parameter            */
  DGMX_ERR_UNSUPPORTED = 2,   /* order/physics/flux combination not built  */
  DGMX_ERR_CUDA = 3,          /* a CUDA runtime call failed                */
  DGMX_ERR_NONPHYSICAL = 4,   /* density or pressure below eps^(2/3) on a
                                 face point (src/Euler3d.cpp:706-762)      */
  DGMX_ERR_IO = 5,            /* input file missing or malformed           */
  DGMX_ERR_MEMORY = 6         /* device allocation failed                  */
} dgmx_status;

/* Physics codes are DGM's eqntype values (src/ReoProblem.cpp:75-156). */
enum { DGMX_EULER2D = 1, DGMX_NS2D = 2, DGMX_EULER3D = 8, DGMX_NS3D = 9, DGMX_SHALLOW = 30 };
/* Numerical flux (src/Euler.cpp:104-113).  Steger-Warming and van Leer:
 * Euler and Navier-Stokes 2-D in FP64 (Euler3d computes Lax-Friedrichs
 * only; Roe in 3-D is this library's extension). */
enum { DGMX_FLUX_LF = 0, DGMX_FLUX_ROE = 1, DGMX_FLUX_STEGER_WARMING = 2, DGMX_FLUX_VAN_LEER = 3 };
/* Integrators are DGM's inttype values (src/TimeInt.hpp:62-85). */
enum { DGMX_TVD3 = 3, DGMX_RK4 = 4, DGMX_LSRK14 = 14 };
/* Arithmetic of the stage kernels.  DGMX_MIXED: for Euler and shallow water
 * (LSRK14) FP32 states, fluxes, contractions and traces about an FP64 reference
 * state with the FP64 solution register; for Navier-Stokes the two BR1 viscous
 * kernels in FP32 (density and energy means taken out in FP64 first) while the
 * stage kernel, registers and traces stay FP64, with any integrator. */
enum { DGMX_FP64 = 0, DGMX_MIXED = 1 };
/* Boundary kinds (FP64).  DGMX_BC_SLIP_WALL: Euler and shallow-water solid
 * wall, Euler::WallBC / Euler3d::WallBC / Shallow::WallBC (src/EulerBC.hpp:43-62,
 * src/Euler3d.cpp:862-903, src/ShallowBC.hpp:45-61).  DGMX_BC_ISOTHERMAL_WALL: Navier-Stokes wall
 * with parameters (Tw, Eref), src/Navier_StokesBC.hpp:47-85,
 * src/Navier_Stokes3d.cpp:472-513.  In 3-D its inviscid flux sees the slip
 * wall of the Domain's BC database (Navier_Stokes3d keeps its own database
 * beside the Domain's, src/Navier_Stokes3d.hpp:83, and Euler3d::convection
 * calls Euler3d::enforce_bc); in 2-D the inviscid flux calls the virtual
 * enforce_bc (src/Euler.cpp:313-316) and sees the isothermal wall too. */
/* DGMX_BC_STATE: fixed conserved state (StateBC, src/BC.cpp:17-42), any
 * Euler/Navier-Stokes physics, parameters = the nf values.  2-D only:
 * DGMX_BC_SUBSONIC_OUTFLOW (density and momentum kept, pressure of Mach
 * parameter 0 with gamma 1.4, src/EulerBC.hpp:114-167) and
 * DGMX_BC_SUPERSONIC_OUTFLOW (the own state, src/EulerBC.hpp:199-241).
 * Every kind's viscous flux is the element's own (apply_flux: B = -S). */
enum { DGMX_BC_SLIP_WALL = 1, DGMX_BC_ISOTHERMAL_WALL = 2, DGMX_BC_STATE = 3, DGMX_BC_SUBSONIC_OUTFLOW = 4,
       DGMX_BC_SUPERSONIC_OUTFLOW = 5 };

typedef struct {
  int dim;               /* 2 (Quad) or 3 (Hex)                              */
  int ne;                /* number of elements                               */
  const double *verts;   /* ne * (4|8) * 3 vertex coordinates, DGM order     */
  int ncon;              /* number of connectivity records                   */
  const int *con;        /* ncon * 4: eid, side, link eid, link side (.con)  */
  const int *porder;     /* ne polynomial orders (p)                         */
  const int *qorder;     /* ne GLL point counts per direction (q, 0 = p+2)   */
} dgmx_mesh;

typedef struct {
  int physics;           /* DGMX_EULER2D ... DGMX_SHALLOW                    */
  int flux;              /* DGMX_FLUX_LF / DGMX_FLUX_ROE                     */
  int inttype;           /* DGMX_TVD3 / DGMX_RK4 / DGMX_LSRK14               */
  int precision;         /* DGMX_FP64 / DGMX_MIXED                           */
  int sw_balance;        /* shallow water: subtract the first RHS
                            (REO_SHALLOW_ENFORCE_BALANCE, src/Shallow.cpp:251) */
  int device;            /* CUDA device ordinal                              */
  double gamma;          /* ratio of specific heats (default 1.4)           */
  double vis;            /* dynamic viscosity mu ("vis" key)                 */
  double Pr;             /* Prandtl number (default 0.72)                    */
} dgmx_params;

/* Builds a Domain from an in-memory mesh.  Replaces the Field/Element
 * construction of Domain::Domain + Field::Field (src/Field.cpp:2257-2735)
 * and the physics constructors (src/Euler3d.cpp:47-142, src/Euler.cpp:80-180). */
dgmx_status dgmx_create(const dgmx_mesh *mesh, const dgmx_params *params, dgmx_domain **out);

/* Builds a Domain from DGM input files root.inp/.msh/.con/.ord (the same keys
 * and formats Reo::Problem::setup reads, src/ReoProblem.cpp:48-156).
 * Fields of *params that are not in root.inp keep the caller's values. */
dgmx_status dgmx_create_from_files(const char *root, const dgmx_params *params, dgmx_domain **out);

/* dgmx_create for a mesh with boundary sides (Field::initialize_bc,
 * src/Field.cpp:4426-4460, with the records of root.bc read by
 * src/Field.cpp:4469-4490).  bc_sides holds nbc records (element, side,
 * kind); bc_params five doubles per record (DGMX_BC_ISOTHERMAL_WALL: Tw,
 * Eref; DGMX_BC_STATE: the conserved values; DGMX_BC_SUBSONIC_OUTFLOW:
 * Mref; unused entries ignored).  A record replaces the side's
 * connectivity link; a linked partner side must be named too.  At most 15
 * distinct (kind, parameters) pairs; FP64 only.
 * dgmx_create_from_files reads root.bc and root.bct the same way when they
 * exist (codes state, *wall*, isothermal_wall, subsonicoutflow,
 * supersonicoutflow and the default tags S, W, O as each physics' databases
 * define them), and switches the bulk-flow hold on when root.chn exists. */
dgmx_status dgmx_create_with_boundaries(const dgmx_mesh *mesh, const dgmx_params *params, int nbc,
                                        const int *bc_sides, const double *bc_params, dgmx_domain **out);

/* ---- element partitions (the reference's MPI decomposition: root.part.N
 * partitions, side exchange in src/vField.cpp:146-200) ----
 * A partitioned handle owns the elements e with part[e] == rank (in
 * increasing global order: its Field-layout arrays are over those elements);
 * faces whose neighbour lives on another rank read ghost slots that a halo
 * exchange fills after every stage (and after the viscous flux kernel for
 * Navier-Stokes).  FP64 or DGMX_MIXED (FP32 trace blocks on the wire; the
 * reference state is the unpartitioned domain's, from every rank's element
 * integrals, so setting the state is collective).  Boundary sides as in
 * dgmx_create_with_boundaries (global element ids; each rank keeps its own).
 * The bulk-flow hold (dgmx_set_bulk_hold, Navier-Stokes 3-D) takes its means
 * over the whole mesh: after every stage each rank sends its elements'
 * constant coefficients to every peer, and the stage then runs without the
 * boundary / interior overlap. */
dgmx_status dgmx_create_partition(const dgmx_mesh *mesh, const dgmx_params *params, const int *part, int nranks,
                                  int rank, dgmx_domain **out);
dgmx_status dgmx_create_partition_with_boundaries(const dgmx_mesh *mesh, const dgmx_params *params, const int *part,
                                                  int nranks, int rank, int nbc, const int *bc_sides,
                                                  const double *bc_params, dgmx_domain **out);
/* NCCL transport for the multi-rank exchange: rank 0 makes the id, every
 * rank passes the same id (collective over the ranks).  One id per
 * communicator: each partitioned handle needs a fresh id.  Steps of such a
 * handle are enqueued directly, not replayed from a CUDA graph. */
#define DGMX_NCCL_ID_BYTES 128
dgmx_status dgmx_nccl_unique_id(unsigned char *id);
dgmx_status dgmx_set_exchange_nccl(dgmx_domain *d, const unsigned char *id);
/* Host-staged transport instead of NCCL (e.g. MPI, or gloo in tests): at
 * every exchange the packed face blocks are copied to pinned host memory
 * and fn is called with them: send holds, for every peer q in rank order,
 * counts[q] blocks of blk doubles at offsets[q] * blk; fn must fill recv the
 * same way with the blocks peer q sent here, and return 0.  Exchanges are
 * then synchronous and steps are not captured into graphs. */
typedef int (*dgmx_exchange_fn)(void *ctx, const double *send, double *recv, const int *counts,
                                const int *offsets, int blk, int nranks);
dgmx_status dgmx_set_exchange_host(dgmx_domain *d, dgmx_exchange_fn fn, void *ctx);
/* local element count, ghost slots and the global id of every local element */
dgmx_status dgmx_partition_info(const dgmx_domain *d, int *ne_local, int *nghost, int *global_of_local);
/* Host-only partition plan (see dgmx.cpp): sizes[3] = local elements, ghost
 * slots, exchanged face blocks; then the lists.  Any array may be NULL. */
dgmx_status dgmx_partition_plan(const dgmx_mesh *mesh, const int *part, int nranks, int rank, int *sizes,
                                int *global_of_local, int *global_of_ghost, int *peer_counts, int *send,
                                int *recv);

/* In-process partitions: every part as a handle on one device, stepped in
 * lockstep with the exchange done by device copies (runs the partitioned
 * path on one GPU).  State arrays are global, Field layout. */
typedef struct dgmx_group dgmx_group;
dgmx_status dgmx_group_create(const dgmx_mesh *mesh, const dgmx_params *params, const int *part, int nparts,
                              dgmx_group **out);
dgmx_status dgmx_group_create_with_boundaries(const dgmx_mesh *mesh, const dgmx_params *params, const int *part,
                                              int nparts, int nbc, const int *bc_sides, const double *bc_params,
                                              dgmx_group **out);
/* the bulk-flow hold on every part, means over the whole mesh */
dgmx_status dgmx_group_set_bulk_hold(dgmx_group *g, int on);
dgmx_status dgmx_group_destroy(dgmx_group *g);
dgmx_domain *dgmx_group_part(dgmx_group *g, int r);
dgmx_status dgmx_group_set_state(dgmx_group *g, const double *U);
dgmx_status dgmx_group_get_state(dgmx_group *g, double *U);
dgmx_status dgmx_group_advance(dgmx_group *g, double dt, int nsteps);
const char *dgmx_group_last_error(const dgmx_group *g);

/* Navier-Stokes 3-D channel forcing, Channel::holdBulkMassFlow
 * (src/Channel.hpp:116-163, called from src/Navier_Stokes3d.cpp:160): after
 * each projected right-hand side, its volume means of density, x-momentum
 * and energy are subtracted.  on = 0 switches it off. */
dgmx_status dgmx_set_bulk_hold(dgmx_domain *d, int on);

/* Source term of the 2-D physics, the Source database's apply (F -= S at
 * the GLL points before the projection) for a field that does not change
 * in time: FileSource (src/Source.hpp:150-180) with S the file's field,
 * ConstSource (src/Source.hpp:110-148) with S constant per field.  Called
 * from Euler::time_derivative (src/Euler.cpp:282-287),
 * Navier_Stokes::time_derivative (src/Navier_Stokes.cpp:95-100) and
 * Shallow::time_derivative (src/Shallow.cpp:255-260), where the
 * shallow-water balance's first right-hand side includes it.  S: GLL values
 * in the dgmx_set_state layout, projected once; NULL removes the source.
 * 3-D domains refuse (DGMX_ERR_UNSUPPORTED): Euler3d and Navier_Stokes3d
 * apply no source. */
dgmx_status dgmx_set_source(dgmx_domain *d, const double *S);

/* Domain::t: dgmx_advance[_async] adds dt per step (0 at creation). */
dgmx_status dgmx_set_time(dgmx_domain *d, double t);
dgmx_status dgmx_get_time(const dgmx_domain *d, double *t);

/* A time factor on the source: S(x, t) = S(x) exp(-(t - t0)^2 / (2 sigma_t^2)),
 * the form of Shallow::GaussianSource (src/Shallow.hpp:666-735), whose
 * spatial part hamp exp(-(x-x0)^2/(2 sx^2) - (y-y0)^2/(2 sy^2)) on the
 * height field is the S given to dgmx_set_source.  Each stage uses the time
 * the reference's integrator sets for it (Domain::t = tn + c_s dt,
 * src/TimeInt.cpp:266-302, :826-860, :1989-2013).  sigma_t <= 0 removes the
 * factor.  While it is on, steps run without a CUDA graph. */
dgmx_status dgmx_set_source_pulse(dgmx_domain *d, double t0, double sigma_t);

dgmx_status dgmx_destroy(dgmx_domain *d);

/* nf fields, nq = total GLL points per field, nm = total modes per field. */
dgmx_status dgmx_sizes(const dgmx_domain *d, long *nf, long *nq, long *nm);

/* GLL point coordinates in Field layout (z ignored in 2-D; may be NULL). */
dgmx_status dgmx_coordinates(const dgmx_domain *d, double *x, double *y, double *z);

/* Sets the solution from GLL values (host, Field layout) and projects it to
 * the polynomial space, as set_ic + project do (src/Euler3d.cpp:1040-1047).
 * Resets the integrator registers. */
dgmx_status dgmx_set_state(dgmx_domain *d, const double *U);
/* Same with device-resident input. */
dgmx_status dgmx_set_state_device(dgmx_domain *d, const double *U_dev);
/* Current solution at GLL points (host, Field layout). */
dgmx_status dgmx_get_state(dgmx_domain *d, double *U);
dgmx_status dgmx_get_state_device(dgmx_domain *d, double *U_dev);
/* Current solution as restart modal coefficients (host). */
dgmx_status dgmx_get_modes(dgmx_domain *d, double *Uh);

/* Sets the solution from restart-layout modal coefficients (the inverse of
 * dgmx_get_modes; no projection) and resets the integrator registers. */
dgmx_status dgmx_set_modes(dgmx_domain *d, const double *Uh);

/* Restart files in DGM's format (text header, src/Domain.cpp:1721-1785;
 * per-field mode counts, displacements and orthonormal coefficients,
 * src/vField.cpp:1082-1200).  Write the current state; read one back into
 * the state (the file's element count and order must match the domain). */
dgmx_status dgmx_write_restart(dgmx_domain *d, const char *path, int step, double t, double dt);
dgmx_status dgmx_read_restart(dgmx_domain *d, const char *path, int *step, double *t);

/* Host-only restart helpers (no CUDA calls).  dgmx_restart_write writes
 * modes in restart layout (nf x ne x nmodes) with a text header;
 * dgmx_restart_info reads the header; dgmx_restart_read reads nf fields
 * (per-element mode counts into nmodes[ne], coefficients into modes, at most
 * cap values). */
dgmx_status dgmx_restart_write(const char *path, int physics, int ne, int nmodes, int step, double t, double dt,
                               double vis, const double *modes);
dgmx_status dgmx_restart_info(const char *path, int *ne, int *nsd, int *lmax, int *step, double *t, double *dt,
                              double *vis);
dgmx_status dgmx_restart_read(const char *path, int nf, int ne, int *nmodes, double *modes, long long cap);

/* Domain::diff (src/Domain.cpp:1000-1066), host only: reads two restart
 * files on the given mesh, computes per field the Linf, L2 and H1 norms
 * (src/Field.cpp:4675-4697) of their difference and of the first, and sets
 * *status bits as the reference does: 1/2/4 absolute Linf/L2/H1 above aeps,
 * 8/16/32 relative Linf/L2/H1 above reps (where the first file's norm is above
 * sqrt(machine epsilon)); a negative tolerance skips its test.  norms
 * (optional) gets nf rows of (Linf, L2, H1 of the difference, Linf, L2, H1 of
 * the first file). */
dgmx_status dgmx_restart_diff(const dgmx_mesh *mesh, int physics, const char *rst1, const char *rst2, double aeps,
                              double reps, double *norms, int *status);
const char *dgmx_restart_last_error(void);

/* Domain::time_derivative(U, F) (src/Domain.hpp:243): F = -dU/dt at GLL
 * points, projected, for U given at GLL points.  Host buffers, Field layout. */
dgmx_status dgmx_time_derivative(dgmx_domain *d, const double *U, double *F);
/* Same with device buffers (Field layout), enqueued on the handle's stream. */
dgmx_status dgmx_time_derivative_device(dgmx_domain *d, const double *U_dev, double *F_dev);

/* TimeInt::advance repeated nsteps times with a fixed dt (TVD3:
 * src/TimeInt.cpp:826-860; RK4: :266-302; LSRK14: :1989-2013).  The state
 * stays on the device; the whole step is replayed from a CUDA graph.
 * Returns DGMX_ERR_NONPHYSICAL if a stage saw a non-realizable face state. */
dgmx_status dgmx_advance(dgmx_domain *d, double dt, int nsteps);

/* Same, but only enqueues the work on the handle's stream (no host sync,
 * no error readback); dgmx_sync collects the status. */
dgmx_status dgmx_advance_async(dgmx_domain *d, double dt, int nsteps);
/* dgmx_set_state / dgmx_get_state without the host wait, for pipelines that
 * keep several handles in flight (each handle's copies and kernels run in
 * order on its own stream, so one solve's transfers overlap another's
 * steps).  U must be page-locked host memory (cudaHostAlloc or a pinned
 * tensor); the caller leaves it untouched until dgmx_sync(d) returns, and
 * reads the result of dgmx_get_state_async only after that.  The mixed
 * form's reference state is formed on the device.  Not for partitioned
 * handles.  No counterpart call in the reference (its state lives on the
 * host). */
dgmx_status dgmx_set_state_async(dgmx_domain *d, const double *U);
dgmx_status dgmx_get_state_async(dgmx_domain *d, double *U);
dgmx_status dgmx_sync(dgmx_domain *d);

/* Conserved totals (integral of each field, FP64 device reduction). */
dgmx_status dgmx_integrals(dgmx_domain *d, double *totals);

/* Text of the last error on this handle (or of the last failed create when
 * d is NULL). */
const char *dgmx_last_error(const dgmx_domain *d);

/* Number of kernel launches the handle has issued since creation. */
long dgmx_launch_count(const dgmx_domain *d);

/* Measured fused multiply-add throughput of this GPU in TFLOP/s (fp64 = 1:
 * FP64, 0: FP32), best of `reps` timed launches of independent FMA chains
 * over a full grid; the denominator of the FP64/FP32 pipe fractions the
 * benchmark reports.  Allocates 16 bytes for the duration of the call.  No
 * counterpart in the reference. */
dgmx_status dgmx_measure_fma_peak(int device, int fp64, int reps, double *tflops);

/* The FP32 viscous form of Navier-Stokes 3-D at p >= 5 (precision
 * DGMX_MIXED): on = 1 runs the 1-D contractions of its two viscous kernels
 * on the tensor cores as 3xTF32 products (each operand split into a TF32
 * part and the TF32 rounding of its remainder, three mma.sync products
 * summed in FP32), on = 0 on the CUDA cores (the default).  No counterpart
 * in the reference, which contracts in FP64 (src/Hex.cpp:2030-2071). */
dgmx_status dgmx_set_tensor_contractions(dgmx_domain *d, int on);

/* Fault-injection hook for tests of failure detection (no counterpart in
 * the reference).  Bounds the number of tries of the prefetching stage
 * kernel's first wait for a tile's inputs; a wait that runs out sets bit 1
 * of the handle's device error word, the CTA waits (with the normal bound)
 * for its copies in flight and leaves, and the call returns DGMX_ERR_CUDA
 * with the context still usable.  0 makes every such wait run out at once;
 * a negative value restores the default (2^20 tries). */
dgmx_status dgmx_set_wait_limit(dgmx_domain *d, int tries);

/* Domain::time_derivative on device buffers for callers that cannot
 * allocate device memory when they need the RHS: a real-time loop that
 * forbids allocation on its call path, or a caller whose device memory is
 * owned by an arena sized once at start-up.  No counterpart in the
 * reference: the face-trace scratch lives in a fixed 8 MiB static device
 * array (at most 1,048,576 doubles = ne * faces * fields * side points)
 * instead of the handle's buffers; larger meshes return DGMX_ERR_ARGUMENT.
 * The array is shared by all calls on a device and keeps the last call's
 * contents, so calls that overlap on the GPU race.  It is called from an
 * ordinary host thread and does call the CUDA runtime (kernel launches; on
 * its first use on a device cudaGetSymbolAddress, which under lazy module
 * loading loads the module and reserves the array's 8 MiB on that device),
 * so it is not for host functions enqueued with cudaLaunchHostFunc; make
 * that first call at set-up time, before any stream capture.  Enqueued on
 * the handle's stream; no cudaMalloc, cudaFree or other allocation after
 * the first call.  Euler and shallow water on whole domains only
 * (Navier-Stokes and partitioned handles return DGMX_ERR_UNSUPPORTED). */
dgmx_status dgmx_time_derivative_static(dgmx_domain *d, const double *U_dev, double *F_dev);

/* The handle's CUDA stream (cudaStream_t), for callers that record events or
 * order their own work against the engine. */
void *dgmx_stream(const dgmx_domain *d);

/* Kernel instantiations in this library: rows of (physics, L, Q, elements
 * per CTA, threads per CTA, shared bytes, min CTAs per SM); returns the row
 * count and writes at most cap rows. */
int dgmx_kernel_list(int *rows, int cap);

/* Autotuner (no counterpart in the reference): times every compiled tile
 * variant for this handle's physics and order on its own mesh with
 * right-hand-side-only launches (the state is unchanged) and keeps the
 * fastest.  rows (optional): cap rows of (elements per CTA, min CTAs per SM,
 * threads per CTA, microseconds per launch). */
dgmx_status dgmx_autotune(dgmx_domain *d, int reps, double *rows, int cap, int *nvariants, int *chosen);

/* Selects compiled tile variant `index` (0 .. nvariants-1, the order of
 * dgmx_autotune's rows) for the stage kernel of this handle; *count gets the
 * number of variants and *warp the kind of the chosen one: 0 a CTA tile,
 * 2 the persistent kernel with a bulk-copy prefetch pipeline.  No
 * counterpart in the reference (tile choice is a GPU matter). */
dgmx_status dgmx_set_variant(dgmx_domain *d, int index, int *count, int *warp);

/* Host-only inspection, no CUDA calls.  1-D tables for L modes and Q GLL
 * points (G = Q-1 Gauss points): GLL z, w (Q); collocation D (QxQ,
 * src/Polylib.tpp:1008-1049); orthonormal Legendre on GLL B (LxQ) and on
 * Gauss Bg (LxG) (src/Basis.cpp:74-102); GL2G (GxQ) and G2GL (QxG)
 * interpolation (src/Hex.cpp:866-884). */
dgmx_status dgmx_tables(int L, int Q, double *z, double *w, double *D, double *B, double *Bg,
                        double *gl2g, double *g2gl);
/* Processed connectivity of a mesh: per element face (neighbour, neighbour
 * face, master flag, geometry class) and the neighbour's point index for
 * each own face point (src/Field.cpp:416-680, :3478-3540,
 * src/BaseHex.hpp:291-333). */
dgmx_status dgmx_mesh_links(const dgmx_mesh *mesh, int *links, int *perm_pairs);

#ifdef __cplusplus
}
#endif
#endif /* DGMX_H */
