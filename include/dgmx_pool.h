/*
 * dgmx_pool.h -- many independent solves on one GPU (batched ensembles and
 * a serving loop).
 *
 * DGM runs one Domain per process and advances it with TimeInt::advance
 * (src/Domain.cpp:935, src/TimeInt.cpp:1989-2013).  A pool holds many such
 * solves at once: each solve is a DGM Domain of its own (its own mesh,
 * order, physics, initial condition, step and end time), and one call
 * advances all of them by one LSRK14 step each.  There is no counterpart
 * of the pool itself in the reference; per solve the arithmetic is that of
 * dgmx_advance (dgmx.h) with inttype 14.
 *
 * Solves of equal (physics, p, q) share one set of device arrays (an
 * "arena").  The 2-D arenas (Euler 2-D and shallow water, p = 1..7,
 * q = p + 2) are stepped together: an RK stage is ONE persistent kernel
 * launch that walks a device-side list of (arena, tile) work items and runs
 * each with the stage body of its order, so a step of any mix of orders is
 * 14 launches replayed from one CUDA graph; other arenas launch their own
 * persistent stage kernel over their tile list.  Solves join and leave
 * between steps without re-capturing the graphs.  Solves never interact:
 * each result is the same alone and in any mix.
 *
 * Layouts are those of dgmx.h: initial values and states are GLL values in
 * DGM's Field layout (nf fields x ne elements x Q^d points).
 * Calls on one pool are not thread-safe.  Every entry point returns a
 * dgmx_status and never throws, traps or aborts.
 */
#ifndef DGMX_POOL_H
#define DGMX_POOL_H

#include <stddef.h>

#include "dgmx.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dgmx_pool dgmx_pool;

typedef struct {
  int precision;         /* DGMX_FP64 / DGMX_MIXED, for every solve         */
  int flux;              /* DGMX_FLUX_LF / DGMX_FLUX_ROE (shallow water: LF) */
  int device;            /* CUDA device ordinal                              */
  int autotune;          /* 1: time the tile variants of each new (physics,
                            p, q) once per process and keep the fastest     */
  double gamma;          /* ratio of specific heats (default 1.4)           */
  size_t budget_bytes;   /* device memory the pool may hold; 0 = no limit   */
} dgmx_pool_params;

dgmx_status dgmx_pool_create(const dgmx_pool_params *params, dgmx_pool **out);
dgmx_status dgmx_pool_destroy(dgmx_pool *p);

/* Prepares the arena of (physics, p, q) -- tables, tile choice, first
 * allocation of `elements` element slots -- so the first solve admitted
 * there does not pay for it.  q = 0 means p + 2. */
dgmx_status dgmx_pool_prepare(dgmx_pool *p, int physics, int porder, int qorder, int elements);

/* Admits one solve: physics DGMX_EULER2D / DGMX_EULER3D / DGMX_SHALLOW
 * (shallow water without the balance subtraction), a mesh with one order,
 * its initial GLL values U0 (projected like dgmx_set_state), its step dt
 * and end time t_end > 0.  The last step is shortened to land on t_end.
 * Returns DGMX_ERR_MEMORY, with nothing admitted, when the solve does not
 * fit the pool's budget now; it may fit after other solves are removed. */
dgmx_status dgmx_pool_add(dgmx_pool *p, const dgmx_mesh *mesh, int physics, const double *U0, double dt,
                          double t_end, int *id);

/* Advances every unfinished solve by up to nsteps steps and waits for the
 * GPU.  A solve that reaches t_end stops there and is reported once by
 * dgmx_pool_finished.  DGMX_ERR_NONPHYSICAL names the solve in
 * dgmx_pool_last_error; the other solves' steps are complete. */
dgmx_status dgmx_pool_step(dgmx_pool *p, int nsteps);

/* dgmx_pool_step without the wait: the steps are enqueued (one CUDA graph
 * per step) and the call returns, so the caller can admit new solves while
 * they run (admission into the fused 2-D arenas does not wait for a step in
 * flight unless an arena has to grow).  dgmx_pool_sync waits for them and
 * reports what dgmx_pool_step would have.  dgmx_pool_finished, get_state
 * and remove need the steps synced.  No counterpart in the reference. */
dgmx_status dgmx_pool_step_async(dgmx_pool *p, int nsteps);
dgmx_status dgmx_pool_sync(dgmx_pool *p);

/* Ids of solves that reached their end time since the previous call
 * (DGMX_ERR_ARGUMENT while steps enqueued by dgmx_pool_step_async are not
 * synced). */
dgmx_status dgmx_pool_finished(dgmx_pool *p, int *ids, int cap, int *n);

/* Current GLL values of a solve (Field layout), its time and step count. */
dgmx_status dgmx_pool_get_state(dgmx_pool *p, int id, double *U);
dgmx_status dgmx_pool_solve_info(dgmx_pool *p, int id, double *t, long *steps, int *finished);

/* Releases a solve's device slots (finished or not). */
dgmx_status dgmx_pool_remove(dgmx_pool *p, int id);

/* Device bytes held, solves resident, unfinished solves, and the modal
 * degrees of freedom (fields x elements x (p+1)^d) of the unfinished ones. */
dgmx_status dgmx_pool_stats(dgmx_pool *p, size_t *bytes, int *resident, int *active, long long *dof_active);

/* The stepping path of the 2-D arenas: 1 (default) one fused launch per
 * stage across orders, 0 one launch per arena per stage.  Only before the
 * first solve or prepare (DGMX_ERR_ARGUMENT afterwards).  No counterpart in
 * the reference. */
dgmx_status dgmx_pool_set_fused(dgmx_pool *p, int on);

/* Stage-kernel launches issued so far (14 per step for the fused 2-D arenas
 * together, plus 14 per other arena). */
long dgmx_pool_launch_count(const dgmx_pool *p);

const char *dgmx_pool_last_error(const dgmx_pool *p);

#ifdef __cplusplus
}
#endif

#endif
